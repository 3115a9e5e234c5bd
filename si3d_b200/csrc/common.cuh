// Device-side layout of one basin's state and the helpers every kernel shares.
//
// HBM layout (B200-first): every 3-D field is stored LAYER-MAJOR, element (k, l) at
// (k-1)*P + (l-1) with the column index l fastest and the pitch P = lm1 rounded up to a multiple
// of 32 doubles (256 B), so a warp that walks 32 consecutive columns down the layers issues one
// fully-coalesced 256-byte access per field and layer.  (The reference stores (km1, lm1)
// column-major with k fastest; the C ABI transposes at the boundary.)  2-D fields are length P.
// Indices k and l are kept 1-based inside the kernels, and column lm1 keeps the reference's dry
// sentinel values, so every stencil below reads exactly the neighbours the Fortran reads.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

// Most levels per column (km1): the continuity kernels hold two planes of km1 + 1 levels x 32
// columns of FP64 terms in shared memory, 229,888 bytes at 448 (227 KB per block at most).
#define SI3D_MAXK 448

namespace si3d {

struct Fields3 {
  double *uh, *uhp, *uhpp, *up, *upp, *hu, *hup, *hupp, *agx, *arx;
  double *vh, *vhp, *vhpp, *vp, *vpp, *hv, *hvp, *hvpp, *agy, *ary;
  double *h, *hp, *hpp, *sal, *salp, *salpp, *rhop, *Av, *Dv, *wp, *HeatSource;
  double *Bth2, *Bth3, *Bth4;
  // Mellor-Yamada 2.5 (iturb = 1 only, else null): q2, q2l at three time levels, and u, v as save
  // leaves them
  double *q2, *q2p, *q2pp, *q2l, *q2lp, *q2lpp, *u, *v;
};

struct Fields2 {
  double *s, *sp, *spp, *eagx, *earx, *eagy, *eary, *sx, *sy, *dd, *qq, *rr, *uair, *vair, *cdw;
  int *k1z, *k1u, *k1v;
};

struct Grid {
  int lm, lm1, km1, km, k1, P;
  const int *lEC, *lWC, *lNC, *lSC, *kmz;   // [P], 1-based neighbour columns, lm1 = dry
  const double *hhs, *hhu, *hhv;            // [P]
  const double* zlevel;                     // [km1] (1-based via zl())
};

struct Params {
  double dt, dx, dy, twodt, dtdx, dtdy, gdtdx, gdtdy, gdt2dx2, gdt2dy2, twodx, twody, fourdx, fourdy, dxdx,
      dydy;
  // reciprocals of the grid constants: the momentum and scalar-transport kernels multiply by these
  // where the reference divides (a product is a few instructions, an FP64 division a long dependent
  // chain; the results differ from the quotients by at most an ulp)
  double rfourdx, rfourdy, rdxdx, rdydy, rdx, rdy;
  double Av0, Dv0, Ax0, Ay0, f, theta, cd, cw;
  int iadv, itrmom, ihd, ibc, isal;
};

// Everything a stage kernel needs, passed by value.
struct Dev {
  Grid g;
  Params p;
  Fields3 f;
  Fields2 s;
  double* scr;   // Thomas-sweep scratch (km1 x P)
  double tz;
};

// 32-bit element index: si3d_gpu_init rejects grids with km1 * P >= 2^31, so the product cannot
// overflow, and 32-bit address arithmetic costs half the instructions of 64-bit.
__device__ __forceinline__ int IX(const Dev& d, int k, int l) { return (k - 1) * d.g.P + (l - 1); }
__device__ __forceinline__ double zl(const Dev& d, int k) { return d.g.zlevel[k - 1]; }
__device__ __forceinline__ int NB(const int* a, int l) { return a[l - 1]; }

constexpr double ZERO = 0.0;
constexpr double HMIN = 0.0;
constexpr double G_GRAV = 9.806;
constexpr double RHOAIR = 1.3;

// densty_s (si3d_utils.f90:3863-3949), the same operation sequence as the oracle; salinity**(3/2)
// is salinity**1 in the reference (integer division) and is kept so.
__device__ __forceinline__ double densty_s(double t, double s, double z) {
  const double t2 = t * t, t3 = t2 * t, t4 = t3 * t, t5 = t4 * t;
  double densw = 999.842594 + 6.793952e-2 * t - 9.095290e-3 * t2 + 1.001685e-4 * t3 - 1.120083e-6 * t4 +
                 6.536332e-9 * t5;
  double densws = densw + s * (0.824493 - 4.0899e-3 * t + 7.6438e-5 * t2 - 8.2467e-7 * t3 + 5.3875e-9 * t4) +
                  s * (-5.72466e-3 + 1.0227e-4 * t - 1.6546e-6 * t2) + 4.8314e-4 * (s * s);
  double rhoguess = densws, delta = 1, rho = 0;
  int iter = 0;
  const double kw = 19652.21 + 148.4206 * t - 2.327105 * t2 + 1.360477e-2 * t3 - 5.155288e-5 * t4;
  const double ks = kw + s * (54.6746 - 0.603459 * t + 1.09987e-2 * t2 - 6.1670e-5 * t3) +
                    s * (7.944e-2 + 1.6483e-2 * t - 5.3009e-4 * t2);
  const double c1 = 3.239908 + 1.43713e-3 * t + 1.16092e-4 * t2 - 5.77905e-7 * t3;
  const double c2 = 2.2838e-3 - 1.0981e-5 * t - 1.6078e-6 * t2;
  const double c3 = 8.50935e-5 - 6.12293e-6 * t + 5.2787e-8 * t2;
  const double c4 = -9.9348e-7 + 2.0816e-8 * t + 9.1697e-10 * t2;
  while (delta > 1e-6 && iter < 10000) {
    double pressureh = rhoguess * 9.806 * z;
    double pressure = 1e-5 * pressureh;
    double k = ks + pressure * c1 + pressure * s * c2 + 1.91075e-4 * pressure * s + (pressure * pressure) * c3 +
               (pressure * pressure) * s * c4;
    rho = densws / (1 - pressure / k);
    delta = fabs(rho - rhoguess);
    rhoguess = rho;
    iter++;
  }
  return rho;
}

// 8-byte asynchronous global -> shared copy (cp.async, completion tracked per thread by commit
// groups).
__device__ __forceinline__ void cp_async8(double* smem, const double* gmem) {
  const unsigned int s = static_cast<unsigned int>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Roe's superbee limiter (the reference always uses it, si3d_procedures.f90:2931-2934 in exsal,
// :4186-4190 in exTracer); cf0 is the default C_f.
__device__ __forceinline__ double superbee(double s1, double s2, double s3, double s4, double vel, double cf0) {
  double C_f = cf0;
  if (s3 - s2 != 0) {
    const bool down = copysign(1.0, vel) > 0;  // gamma1 = -SIGN(1, vel)
    const double ratio = down ? (s2 - s1) / (s3 - s2) : (s4 - s3) / (s3 - s2);
    C_f = fmax(fmax(0., fmin(1., 2. * ratio)), fmin(2., ratio));
  }
  return C_f;
}

__device__ __forceinline__ double zmid(const Dev& d, int k, double hpk) {
  const double z = zl(d, k);
  return (z == -100.) ? 0.5 * hpk : z + 0.5 * hpk;
}

}  // namespace si3d
