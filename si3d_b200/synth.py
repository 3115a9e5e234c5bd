"""Seeded synthetic basins written in the reference's own input-file formats.

The reference ships no benchmark data, so every workload is generated here and written as the
files the reference reads: si3d_inp.txt (si3d_utils.f90:21-315 record layout), si3d_bathy
(depths in decimetres, header '(37X,I5,6X,I5,8X,I5//)', rows '(5X,ncolsG5.0)', si3d_utils.f90:
624-682) and si3d_init.txt (six header records + km1 rows '(10X,G11.5)', si3d_procedures.f90:
303-318).  Spatially varying wind stress, which the reference's ifsurfbc = 0 forcing cannot express,
goes into si3d_wind_override.bin (int32 im1, int32 jm1, float64 uair[im1*jm1], float64
vair[im1*jm1], i outer / j inner), read by the host as an overlay on surfbc CASE(0).

Workloads (all closed basins, constant eddy coefficients, active temperature, trapezoidal
iterations):
  c0  100 x 50 cells, dx = 100 m, parabolic bowl 20 m deep, 20 layers of 1 m, uniform 0.1 Pa wind,
      dt = 60 s;
  c1  1000 x 500, dx = 50 m, 40 layers (1.5 m), Gaussian-random-field bathymetry (correlation
      length 20 cells, 2-60 m, 30 % land), wind stress field 0.1 Pa +- 50 %, dt = 30 s;
  c2  2000 x 1000, 60 layers (1 m), the c1 generators with new seeds, dt = 30 s.
"""
from __future__ import annotations

import dataclasses
import math
import os
import struct
from typing import Optional

import numpy as np

RHOAIR = 1.3


@dataclasses.dataclass
class Basin:
    name: str
    nx: int
    ny: int
    dx: float
    dy: float
    depth: np.ndarray            # (nx, ny) metres; <= 0 is land
    nlayers: int
    ddz: float
    dt: float
    nsteps: int
    dzmin: float = 0.1
    wa: float = 0.0              # uniform wind speed (surfbc CASE 0)
    phi: float = 270.0
    uair: Optional[np.ndarray] = None   # (nx, ny) per-cell wind override
    vair: Optional[np.ndarray] = None
    t_top: float = 20.0
    t_bottom: float = 10.0
    cw: float = 1.2e-3
    cd: float = 0.0025
    Av0: float = 1e-3
    Dv0: float = 1e-3
    Ax0: float = 1.0
    Ay0: float = 1.0
    f: float = 1e-4
    niter: int = 2
    ibc: int = 1                 # baroclinic pressure term on/off
    ntr: int = 0                 # non-active (conservative) tracers, ecomod = 0
    iturb: int = 0               # 0 constant eddy coefficients, 1 Mellor-Yamada 2.5
    # binary outputs: H-planes every iop steps from itspfh (outh), tracers every iotr steps (outz),
    # the 3-D ptrack file every ipxml steps from itspf (outp); 0 = off
    iop: int = 0
    itspfh: int = 0
    planes: tuple = ()
    ipxml: int = 0
    itspf: int = 0
    iotr: int = 0
    itspftr: int = 0
    seeds: dict = dataclasses.field(default_factory=dict)
    # open boundaries with a specified water-surface elevation (itype 1): (iside, isbc, jsbc, iebc,
    # jebc) each, 1-based grid indices (the real cells are 2 .. nx + 1, 2 .. ny + 1), and the series
    # written to openbcNN.txt every obc_dtsec seconds: elevation (m) and temperature (deg C)
    obc: tuple = ()
    obc_dtsec: float = 600.0
    obc_wse: tuple = ()
    obc_temp: tuple = ()

    @property
    def zl(self) -> float:
        return self.nlayers * self.ddz


def wind_speed_for_stress(tau: np.ndarray | float, cw: float = 1.2e-3) -> np.ndarray | float:
    """U with rho_air * cw * U^2 = tau (the drag law of matmom, si3d_procedures.f90:1348-1360)."""
    return np.sqrt(np.asarray(tau) / (cw * RHOAIR))


def gaussian_field(shape, corr_cells: float, rng: np.random.Generator) -> np.ndarray:
    """White noise smoothed by a Gaussian of standard deviation `corr_cells` (periodic FFT
    filter), standardised to zero mean and unit variance."""
    noise = rng.standard_normal(shape)
    kx = np.fft.fftfreq(shape[0])[:, None]
    ky = np.fft.rfftfreq(shape[1])[None, :]
    filt = np.exp(-2.0 * (math.pi * corr_cells) ** 2 * (kx ** 2 + ky ** 2))
    f = np.fft.irfft2(np.fft.rfft2(noise) * filt, s=shape)
    return (f - f.mean()) / f.std()


def random_bathymetry(nx, ny, seed, corr=20.0, land=0.30, dmin=2.0, dmax=60.0) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    f = gaussian_field((nx, ny), corr, rng)
    f30 = np.quantile(f, land)
    depth = dmin + (dmax - dmin) * (f - f30) / (f.max() - f30)
    depth = np.round(depth * 10.0) / 10.0
    depth[f <= f30] = -9.9
    return depth


def stress_field(nx, ny, seed, mean=0.1, rel=0.5, corr=20.0) -> np.ndarray:
    rng = np.random.Generator(np.random.PCG64(seed))
    g = gaussian_field((nx, ny), corr, rng)
    return mean * (1.0 + rel * g / np.abs(g).max())


def bowl_bathymetry(nx, ny, dx, dy, hmax=20.0) -> np.ndarray:
    x = (np.arange(nx) + 0.5) * dx - nx * dx / 2.0
    y = (np.arange(ny) + 0.5) * dy - ny * dy / 2.0
    a, b = nx * dx / 2.0, ny * dy / 2.0
    h = hmax * (1.0 - (x[:, None] / a) ** 2 - (y[None, :] / b) ** 2)
    h = np.round(h * 10.0) / 10.0
    h[h <= 0.0] = -9.9
    return h


def config(name: str, nsteps: Optional[int] = None, seed_offset: int = 0) -> Basin:
    """The benchmark/parity workloads by name: c0, c1, c2, the small test basins t0/t1, and the
    profiler cases m1 (600 x 300 x 60 with c2's generators) and p2 (c2's 2000 x 1000 grid with 6
    layers of 10 m: a zeta system of c2's size with a ~3 GB 3-D state)."""
    if name == "c0":
        nx, ny, dx = 100, 50, 100.0
        return Basin("c0", nx, ny, dx, dx, bowl_bathymetry(nx, ny, dx, dx), 20, 1.0, 60.0, nsteps or 1000,
                     dzmin=0.05, wa=float(wind_speed_for_stress(0.1)), phi=270.0)
    if name in ("c1", "c2", "t1", "m1", "p2"):
        if name == "c1":
            nx, ny, dx, nl, ddz, steps, sb, sw = 1000, 500, 50.0, 40, 1.5, 1000, 1001, 1002
        elif name == "c2":
            nx, ny, dx, nl, ddz, steps, sb, sw = 2000, 1000, 50.0, 60, 1.0, 500, 2001, 2002
        elif name == "m1":  # medium basin for profiler captures (c2 generators, ~1.5 GB state)
            nx, ny, dx, nl, ddz, steps, sb, sw = 600, 300, 50.0, 60, 1.0, 50, 2001, 2002
        elif name == "p2":  # zeta-solve captures: c2's grid, seeds and wet mask, 6 layers of 10 m
            nx, ny, dx, nl, ddz, steps, sb, sw = 2000, 1000, 50.0, 6, 10.0, 50, 2001, 2002
        else:  # small random basin for fast parity tests
            nx, ny, dx, nl, ddz, steps, sb, sw = 96, 64, 50.0, 12, 5.0, 50, 3001, 3002
        sb += seed_offset
        sw += seed_offset
        corr = 20.0 if name != "t1" else 6.0
        depth = random_bathymetry(nx, ny, sb, corr=corr)
        tau = stress_field(nx, ny, sw, corr=corr)
        u = wind_speed_for_stress(tau)
        return Basin(name, nx, ny, dx, dx, depth, nl, ddz, 30.0, nsteps or steps, dzmin=0.1,
                     uair=u, vair=np.zeros_like(u), seeds={"bathymetry": sb, "wind": sw})
    if name in ("t2", "t3"):
        # open-boundary basins: a channel forced by a tide through its west end (t2), and a basin
        # with open east, north and south sides (t3); smooth bottom 3-9 m, 10 layers of 1 m
        nx, ny = (40, 16) if name == "t2" else (32, 24)
        x = (np.arange(nx) + 0.5) / nx
        y = (np.arange(ny) + 0.5) / ny
        depth = 6.0 + 2.5 * np.cos(2.0 * math.pi * x)[:, None] * np.sin(math.pi * y)[None, :] - 0.5 * x[:, None]
        depth = np.round(depth * 10.0) / 10.0
        if name == "t2":
            obc = ((1, 2, 2, 2, ny + 1),)
        else:
            obc = ((3, nx + 1, 4, nx + 1, ny - 3), (2, 6, ny + 1, nx - 5, ny + 1), (4, 6, 2, nx - 5, 2))
        dts = 600.0
        npts = 40
        t = np.arange(npts) * dts
        wse, temp = [], []
        for q in range(len(obc)):
            amp, period = 0.05 + 0.02 * q, 7200.0 + 1800.0 * q
            wse.append(tuple(np.round(amp * np.sin(2.0 * math.pi * t / period), 6)))
            temp.append(tuple(np.round(15.0 + 1.0 * np.cos(2.0 * math.pi * t / 5400.0) + q, 5)))
        return Basin(name, nx, ny, 100.0, 100.0, depth, 10, 1.0, 60.0, nsteps or 30, dzmin=0.05,
                     wa=float(wind_speed_for_stress(0.05)), phi=270.0, obc=obc, obc_dtsec=dts,
                     obc_wse=tuple(wse), obc_temp=tuple(temp))
    if name == "t0":  # tiny bowl
        nx, ny, dx = 24, 16, 100.0
        return Basin("t0", nx, ny, dx, dx, bowl_bathymetry(nx, ny, dx, dx, hmax=8.0), 8, 1.0, 60.0,
                     nsteps or 20, dzmin=0.05, wa=float(wind_speed_for_stress(0.1)), phi=270.0)
    raise ValueError(f"unknown workload {name}")


def _rec(label: str, value) -> str:
    if isinstance(value, float):
        v = repr(value) if abs(value) >= 1e-3 or value == 0.0 else f"{value:.6E}"
    else:
        v = str(value)
    return f" {label:<12}! {v:>18} !"


def write_inp(b: Basin, path: str) -> None:
    L = []
    sep = "-" * 55
    L += ["*" * 55, f"SYNTHETIC {b.name} {b.nx}x{b.ny}x{b.nlayers}", "=" * 55, "Start date and time", sep]
    L += [_rec("year", 2024), _rec("month", 1), _rec("day", 1), _rec("hour", 0)]
    L += [sep, "Space-time domains, cell size & time steps", sep]
    for lab, val in [("xl", b.nx * b.dx), ("yl", b.ny * b.dy), ("zl", b.zl), ("tl", b.nsteps * b.dt),
                     ("idx", b.dx), ("idy", b.dy), ("idz", b.ddz), ("dzmin", b.dzmin), ("datadj", 0.0),
                     ("zeta0", 0.0), ("idt", b.dt), ("ibathf", 0)]:
        L.append(_rec(lab, float(val) if lab != "ibathf" else val))
    L += [sep, "Parameters controlling solution algorithm", sep]
    for lab, val in [("itrap", 1), ("niter", b.niter), ("smooth", 0), ("beta", 0.05), ("iturb", b.iturb),
                     ("az0", b.Av0), ("dz0", b.Dv0), ("iadv", 1), ("itrmom", 1), ("ihd", 1), ("ax0", b.Ax0),
                     ("ay0", b.Ay0), ("f", b.f), ("theta", 1.0), ("ibc", b.ibc), ("isal", 1), ("itrsch", 4),
                     ("cd", b.cd), ("ifsbc", 0), ("dtsbc", 3600.0), ("icw", 0), ("cw", b.cw), ("ws", b.wa),
                     ("phi", b.phi), ("idbg", 0), ("nth", 1)]:
        L.append(_rec(lab, val))
    L += [sep, "Output specifications for time files", sep, _rec("ipt", 0), _rec("nnodes", 0),
          _rec("inodes", 0), _rec("jnodes", 0)]
    L += [sep, "Output specifications for H-plane files", sep, _rec("iop", b.iop), _rec("itspfh", b.itspfh),
          _rec("nplanes", len(b.planes)), _rec("planes", " ".join(str(k) for k in b.planes) or 0)]
    L += [sep, "Output specifications for X-section files", sep, _rec("ixt", 0)]
    L += [sep, "Output specifications for 3D space files", sep, _rec("ipxml", b.ipxml), _rec("itspf", b.itspf),
          _rec("iTurbVars", 0)]
    L += [sep, "Open boundary conditions specifications", sep, _rec("nopen", len(b.obc))]
    if b.obc:
        L += [_rec("dtopenbc", float(b.obc_dtsec))]
        cols = list(zip(*[(ob[0], 1, ob[1], ob[2], ob[3], ob[4]) for ob in b.obc]))
        L += [_rec(x, " ".join(str(v) for v in c)) for x, c in zip(("iside", "itype", "isbc", "jsbc", "iebc", "jebc"), cols)]
    else:
        L += [_rec("dtopenbc", 360.0)]
        L += [_rec(x, 0) for x in ("iside", "itype", "isbc", "jsbc", "iebc", "jebc")]
    L += [sep, "Open boundary conditions for nesting procedures", sep, _rec("nxBDO", 0)]
    L += [_rec(x, 0) for x in ("iob", "xxb", "iside", "isbc", "jsbc", "iebc", "jebc")]
    L += [sep, "Specification for tracer simulation", sep, _rec("ntr", b.ntr)]
    L += [_rec("ecomod", 0), _rec("iotr", b.iotr), _rec("itspftr", b.itspftr), _rec("ipwq", 0), _rec("nswq", 0)]
    L += [sep, "Specification for oxygenation system simulations", sep, _rec("iopts", 0)]
    L += [_rec(x, 0) for x in ("Nodev", "iodt", "ipss", "jpss", "iodev")]
    with open(path, "w") as fh:
        fh.write("\n".join(L) + "\n")


def write_bathy(b: Basin, path: str, ncols: int = 40) -> None:
    dm = np.where(b.depth > 0.0, np.round(b.depth * 10.0), -99).astype(np.int64)
    if dm.max() > 99999:
        raise ValueError("depth does not fit the I5/G5.0 field")
    head = f"{'Synthetic ' + b.name:<36} {b.nx:5d}{'':6}{b.ny:5d}{'':8}{ncols:5d}"
    lines = [head, "HV", " " * 5 + "".join(f"{i:5d}" for i in range(2, min(ncols, b.nx) + 2))]
    for ia in range(0, b.nx, ncols):
        ib = min(ia + ncols, b.nx)
        for j in range(b.ny - 1, -1, -1):   # rows j = jm .. 2
            lines.append(f"{j + 2:5d}" + "".join(f"{v:5d}" for v in dm[ia:ib, j]))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def layer_profile(b: Basin) -> np.ndarray:
    """Temperature at levels k = 1..km1: linear from t_top (first real layer) to t_bottom (last)."""
    km = int(math.ceil(b.zl / b.ddz)) + 1
    km1 = km + 1
    t = np.empty(km1)
    for k in range(1, km1 + 1):
        kk = min(max(k, 2), km)
        t[k - 1] = b.t_top + (b.t_bottom - b.t_top) * (kk - 2) / max(km - 2, 1)
    return t


def tracer_profiles(b: Basin) -> np.ndarray:
    """Initial tracer concentrations at levels k = 1..km1, shape (ntr, km1): tracer 1 is a step (1
    above mid-depth, 0 below: a sharp front for the flux limiter), with three or more tracers the
    last is uniform (0.5), and the others are Gaussian bands centred at evenly spaced depths."""
    km = int(math.ceil(b.zl / b.ddz)) + 1
    km1 = km + 1
    k = np.arange(1, km1 + 1, dtype=np.float64)
    out = np.zeros((b.ntr, km1))
    for t in range(b.ntr):
        if t == 0:
            out[t] = np.where(k <= (km + 2) / 2, 1.0, 0.0)
        elif t == b.ntr - 1 and b.ntr >= 3:
            out[t] = 0.5
        else:
            kc = 2 + t * (km - 2) / b.ntr
            w = max(1.0, (km - 2) / 8)
            out[t] = np.exp(-((k - kc) / w) ** 2)
    return np.round(out, 5)


def write_init(b: Basin, path: str) -> None:
    t = layer_profile(b)
    tr = tracer_profiles(b)
    head = "         z          T" + "".join(f"{'C' + str(i + 1):>11}" for i in range(b.ntr))
    lines = ["Initial condition file for si3d model", f"synthetic {b.name}", "synthetic profile",
             "Depths (m)   Temp (oC)", "Source: linear", head, "-" * 40]
    for k, tv in enumerate(t, start=1):
        z = -(k - 1.5) * b.ddz
        lines.append(f"{z:10.2f}{tv:11.5f}" + "".join(f"{tr[i, k - 1]:11.5f}" for i in range(b.ntr)))
    with open(path, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def write_wind(b: Basin, path: str) -> None:
    im1, jm1 = b.nx + 2, b.ny + 2
    u = np.zeros((im1, jm1))
    v = np.zeros((im1, jm1))
    u[1:-1, 1:-1] = b.uair
    v[1:-1, 1:-1] = b.vair
    with open(path, "wb") as fh:
        fh.write(struct.pack("<ii", im1, jm1))
        fh.write(np.ascontiguousarray(u, dtype="<f8").tobytes())
        fh.write(np.ascontiguousarray(v, dtype="<f8").tobytes())


def write_openbc(b: Basin, run_dir: str) -> None:
    """openbcNN.txt per open boundary (openbc0, si3d_boundaryconditions.f90:55-91): five header
    records, the record count in '(10X,I7)', then one record '(10X,(ntr+2)G11.2)' per time."""
    for nn, (wse, temp) in enumerate(zip(b.obc_wse, b.obc_temp), start=1):
        lines = [f"Open boundary {nn} of {b.name}", "water-surface elevation (m), temperature (deg C)",
                 f"every {b.obc_dtsec:g} s from t = 0", "synthetic", "-" * 40, f"{'npts':<10}{len(wse):7d}"]
        for w, t in zip(wse, temp):
            lines.append(f"{'':10}{w:11.6f}{t:11.5f}")
        with open(os.path.join(run_dir, f"openbc{nn:02d}.txt"), "w") as fh:
            fh.write("\n".join(lines) + "\n")


def write_run(b: Basin, run_dir: str) -> str:
    os.makedirs(run_dir, exist_ok=True)
    write_openbc(b, run_dir)
    write_inp(b, os.path.join(run_dir, "si3d_inp.txt"))
    write_bathy(b, os.path.join(run_dir, "si3d_bathy"))
    write_init(b, os.path.join(run_dir, "si3d_init.txt"))
    wp = os.path.join(run_dir, "si3d_wind_override.bin")
    if b.uair is not None:
        write_wind(b, wp)
    elif os.path.exists(wp):
        os.remove(wp)
    return run_dir


def make(name: str, run_dir: str, nsteps: Optional[int] = None, seed_offset: int = 0, ntr: int = 0,
         outputs: Optional[dict] = None, iturb: int = 0) -> Basin:
    """Write workload `name` into run_dir; `outputs` sets the output records (iop, itspfh, planes,
    ipxml, itspf, iotr, itspftr)."""
    b = config(name, nsteps, seed_offset)
    b.ntr = ntr
    b.iturb = iturb
    for k, v in (outputs or {}).items():
        setattr(b, k, v)
    write_run(b, run_dir)
    return b
