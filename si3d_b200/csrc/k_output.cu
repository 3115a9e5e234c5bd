// Frames of the reference's binary output files packed on the device: outp (the ptrack file,
// si3d_utils.f90:2484-2602), outz (tracers, :2373-2481) and outh (horizontal planes, :2142-2334).
// A frame is the value list of one Fortran record in the reference's order, converted to 4-byte
// floats (round to nearest), so the host only frames and writes it.
//
// 3-D frames hold, for every wet column l = 1..lm (the reference's c loop visits the columns in l
// order) and layer k = k1..kmz(l) + 1, nv consecutive values; point p of column l, layer k is
// poff[l - 1] + k - k1.  Threads take 32 consecutive columns and walk the layers in lanes, so every
// field load of a layer is one coalesced access; each thread stores its point's nv values together.
#include "kernels.h"

namespace si3d {
namespace {

constexpr int OUT_LANES = 4;

struct Src3 {
  const double* f[5];
  int nf;
};

template <int CLN>
__global__ void __launch_bounds__(32 * CLN) k_pack_points(Dev d, Src3 S, const int* __restrict__ poff,
                                                       const int* __restrict__ l2i, const int* __restrict__ l2j,
                                                       int coords, float* __restrict__ out) {
  const int l = blockIdx.x * 32 + threadIdx.x + 1;
  if (l > d.g.lm) return;
  const int k1 = d.g.k1, kms = NB(d.g.kmz, l);
  const int nv = S.nf + (coords ? 3 : 0);
  const float fi = (float)l2i[l - 1], fj = (float)l2j[l - 1];
  const long long p0 = poff[l - 1];
  for (int k = k1 + threadIdx.y; k <= kms + 1; k += CLN) {
    const int ik = IX(d, k, l);
    float* o = out + (p0 + (k - k1)) * nv;
    int j = 0;
    if (coords) { o[0] = fi; o[1] = fj; o[2] = (float)k; j = 3; }
    for (int v = 0; v < S.nf; ++v) o[j + v] = (float)S.f[v][ik];
  }
}

// outh: one entry per column of the plane's list (the columns whose bottom layer reaches kp, or
// every column for the bottom plane kp > km).  First frame: i, j, up, vp, wp, salp, Av, s; later
// frames: u and v averaged over the cell's two faces, w over its two interfaces, salp, Av, s.
__global__ void k_pack_plane(Dev d, const int* __restrict__ cols, int n, int kp, int first,
                             const int* __restrict__ l2i, const int* __restrict__ l2j, float* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int l = cols[e];
  const int kb = kp > d.g.km ? NB(d.g.kmz, l) : kp;
  const int ik = IX(d, kb, l), P = d.g.P;
  const double* up = d.f.up;
  const double* vp = d.f.vp;
  const double* wp = d.f.wp;
  const double sal = (d.f.hp[ik] <= ZERO) ? -99. : d.f.salp[ik];
  const double av = 0.5 * (d.f.Av[ik] + d.f.Av[ik + P]);
  const double s = d.s.s[l - 1];
  if (first) {
    float* o = out + (long long)e * 8;
    o[0] = (float)l2i[l - 1]; o[1] = (float)l2j[l - 1];
    o[2] = (float)up[ik]; o[3] = (float)vp[ik]; o[4] = (float)wp[ik];
    o[5] = (float)sal; o[6] = (float)av; o[7] = (float)s;
  } else {
    const int lW = NB(d.g.lWC, l), lS = NB(d.g.lSC, l);
    float* o = out + (long long)e * 6;
    o[0] = (float)((up[ik] + up[ik + (lW - l)]) / 2.);
    o[1] = (float)((vp[ik] + vp[ik + (lS - l)]) / 2.);
    o[2] = (float)((wp[ik] + wp[ik + P]) / 2.);
    o[3] = (float)sal; o[4] = (float)av; o[5] = (float)s;
  }
}

}  // namespace

void launch_pack_points(const Dev& d, const double* const* fields, int nf, const int* poff, const int* l2i,
                        const int* l2j, bool coords, float* out, cudaStream_t st) {
  Src3 S{};
  S.nf = nf;
  for (int i = 0; i < nf; ++i) S.f[i] = fields[i];
  k_pack_points<OUT_LANES><<<(d.g.lm + 31) / 32, dim3(32, OUT_LANES), 0, st>>>(d, S, poff, l2i, l2j, coords ? 1 : 0, out);
}

void launch_pack_plane(const Dev& d, const int* cols, int n, int kp, bool first, const int* l2i, const int* l2j,
                       float* out, cudaStream_t st) {
  if (n > 0) k_pack_plane<<<(n + 255) / 256, 256, 0, st>>>(d, cols, n, kp, first ? 1 : 0, l2i, l2j, out);
}

}  // namespace si3d
