"""The N > 1 path on the CPU: two gloo ranks partition an ensemble of independent basins, each
advances only its own basins (here through the CPU oracle), and the results gathered from the
ranks equal a single-process run basin by basin.  The only collectives are the final gather and
the max-over-ranks timing reduction that bench.py uses."""
import dataclasses
import os
import socket
import tempfile

import numpy as np
import pytest

from si3d_b200 import replicas, synth


def _basins():
    out = []
    for k, (nx, ny, nl) in enumerate([(24, 16, 8), (30, 12, 6), (16, 16, 10), (20, 24, 8), (12, 10, 4)]):
        b = synth.config("t0", nsteps=10)
        b = dataclasses.replace(b, name=f"e{k}", nx=nx, ny=ny, nlayers=nl,
                                depth=synth.bowl_bathymetry(nx, ny, b.dx, b.dy, hmax=float(nl) - 0.5),
                                wa=float(synth.wind_speed_for_stress(0.05 + 0.03 * k)))
        out.append(b)
    return out


def _cost(b):
    return float((b.depth > 0).sum() * b.nlayers)


def _advance(b, root, steps=3):
    from oracle import pyoracle
    d = os.path.join(root, b.name)
    synth.write_run(b, d)
    o = pyoracle.OracleRun(d)
    o.run(steps)
    return o.get("s")[:o.lm].copy()


def _worker(rank, world, port, root, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        basins = _basins()
        mine = replicas.partition([_cost(b) for b in basins], world)[rank]
        res = {i: _advance(basins[i], os.path.join(root, f"r{rank}")) for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        tmax = replicas.max_over_ranks(float(rank + 1), dist)
        if rank == 0:
            merged = {}
            for g in gathered:
                assert not (set(g) & set(merged)), "a basin ran on two ranks"
                merged.update(g)
            np.savez(out, tmax=tmax, **{f"b{i}": v for i, v in merged.items()})
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_properties():
    costs = [9, 1, 4, 4, 7, 2, 2, 8]
    for world in (1, 2, 3, 8, 10):
        parts = replicas.partition(costs, world)
        assert len(parts) == world
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        assert parts == replicas.partition(costs, world)     # deterministic
    assert replicas.imbalance(costs, replicas.partition(costs, 2)) <= 1.03


def test_max_over_ranks_without_group():
    assert replicas.max_over_ranks(3.5) == 3.5


def test_two_gloo_ranks_match_one_process(oracle_lib, tmp_path):
    import torch.multiprocessing as mp
    out = str(tmp_path / "gathered.npz")
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path), out), nprocs=world, join=True,
                       start_method="spawn")
    got = np.load(out)
    assert float(got["tmax"]) == float(world)
    basins = _basins()
    serial_root = tempfile.mkdtemp(dir=str(tmp_path))
    for i, b in enumerate(basins):
        np.testing.assert_array_equal(got[f"b{i}"], _advance(b, serial_root))
