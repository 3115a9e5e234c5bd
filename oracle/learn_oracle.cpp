// CPU oracle of the learned initial guess network (test infrastructure only).
//
// The network and parameter layout are those of include/si3d_learn.h.  Every sum is accumulated in
// double.  With bf16 = 1 the values are rounded to BF16 exactly where the CUDA kernels round them
// (stem inputs and all weights; every activation image; the ReLU-masked gradient fed to the
// tensor-core data-gradient convolution), so GPU results can be compared with it; with bf16 = 0 the
// network is plain real arithmetic and its gradient can be checked by finite differences.
// There is no reference counterpart (the reference always starts the zeta solve from sp).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int C = 32, NIN = 4, NBLK = 4;
constexpr int OFF_STEM_B = 9 * NIN * C, OFF_BLK = OFF_STEM_B + C, BLK_SZ = 9 * C * C + C;
constexpr int OFF_HEAD_W = OFF_BLK + NBLK * BLK_SZ, OFF_HEAD_B = OFF_HEAD_W + 9 * C;
constexpr int NPARAM = OFF_HEAD_B + 1;

double bf16r(double x) {
  float f = (float)x;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  if ((u & 0x7f800000u) == 0x7f800000u) return f;   // inf / nan unchanged
  u += 0x7fffu + ((u >> 16) & 1u);
  u &= 0xffff0000u;
  std::memcpy(&f, &u, 4);
  return f;
}

struct Net {
  int B, H, W;
  bool rb;
  double R(double x) const { return rb ? bf16r(x) : x; }
  // neighbour (i + di, j + dj) of pixel p of image b, or -1 outside the image
  long nb(int b, int i, int j, int t) const {
    const int ii = i + t / 3 - 1, jj = j + t % 3 - 1;
    if (ii < 0 || ii >= H || jj < 0 || jj >= W) return -1;
    return ((long)b * H + ii) * W + jj;
  }
  long P() const { return (long)B * H * W; }
};

struct Acts {
  std::vector<double> fb;                 // rounded stem input [P][4]
  std::vector<double> x[NBLK + 1];        // layer inputs [P][C]
  std::vector<double> y[NBLK + 1];        // pre-activations [P][C]
  std::vector<double> out;                // [P]
};

void forward(const Net& n, const float* prm, const float* feat, Acts& A) {
  const long P = n.P();
  A.fb.assign(P * NIN, 0.0);
  for (long i = 0; i < P * NIN; ++i) A.fb[i] = n.R(feat[i]);
  // stem
  A.y[0].assign(P * C, 0.0);
  A.x[0].assign(P * C, 0.0);
  for (int b = 0; b < n.B; ++b)
    for (int i = 0; i < n.H; ++i)
      for (int j = 0; j < n.W; ++j) {
        const long p = ((long)b * n.H + i) * n.W + j;
        for (int co = 0; co < C; ++co) {
          double acc = 0.0;
          for (int t = 0; t < 9; ++t) {
            const long q = n.nb(b, i, j, t);
            if (q < 0) continue;
            for (int ci = 0; ci < NIN; ++ci) acc += A.fb[q * NIN + ci] * n.R(prm[(t * NIN + ci) * C + co]);
          }
          const double y = acc + prm[OFF_STEM_B + co];
          A.y[0][p * C + co] = y;
          A.x[0][p * C + co] = n.R(y > 0 ? y : 0.0);
        }
      }
  // residual blocks
  for (int k = 0; k < NBLK; ++k) {
    const float* Wk = prm + OFF_BLK + k * BLK_SZ;
    const float* bk = Wk + 9 * C * C;
    A.y[k + 1].assign(P * C, 0.0);
    A.x[k + 1].assign(P * C, 0.0);
    for (int b = 0; b < n.B; ++b)
      for (int i = 0; i < n.H; ++i)
        for (int j = 0; j < n.W; ++j) {
          const long p = ((long)b * n.H + i) * n.W + j;
          for (int co = 0; co < C; ++co) {
            double acc = 0.0;
            for (int t = 0; t < 9; ++t) {
              const long q = n.nb(b, i, j, t);
              if (q < 0) continue;
              for (int ci = 0; ci < C; ++ci) acc += A.x[k][q * C + ci] * n.R(Wk[(t * C + ci) * C + co]);
            }
            const double y = acc + bk[co];
            A.y[k + 1][p * C + co] = y;
            A.x[k + 1][p * C + co] = n.R(A.x[k][p * C + co] + (y > 0 ? y : 0.0));
          }
        }
  }
  // head
  A.out.assign(P, 0.0);
  for (int b = 0; b < n.B; ++b)
    for (int i = 0; i < n.H; ++i)
      for (int j = 0; j < n.W; ++j) {
        const long p = ((long)b * n.H + i) * n.W + j;
        double acc = 0.0;
        for (int t = 0; t < 9; ++t) {
          const long q = n.nb(b, i, j, t);
          if (q < 0) continue;
          for (int ci = 0; ci < C; ++ci) acc += A.x[NBLK][q * C + ci] * n.R(prm[OFF_HEAD_W + t * C + ci]);
        }
        A.out[p] = acc + prm[OFF_HEAD_B];
      }
}

// grad of loss = sum mask (out - t)^2 / sum mask
double backward(const Net& n, const float* prm, const Acts& A, const float* target, const float* mask,
                std::vector<double>& g) {
  const long P = n.P();
  g.assign(NPARAM, 0.0);
  double m = 0.0, l = 0.0;
  for (long p = 0; p < P; ++p)
    if (mask[p] > 0) { m += 1.0; l += (A.out[p] - target[p]) * (A.out[p] - target[p]); }
  if (m == 0.0) return 0.0;
  std::vector<double> gout(P, 0.0);
  for (long p = 0; p < P; ++p)
    if (mask[p] > 0) gout[p] = 2.0 * (A.out[p] - target[p]) / m;
  // head
  std::vector<double> G(P * C, 0.0);
  for (int b = 0; b < n.B; ++b)
    for (int i = 0; i < n.H; ++i)
      for (int j = 0; j < n.W; ++j) {
        const long p = ((long)b * n.H + i) * n.W + j;
        g[OFF_HEAD_B] += gout[p];
        for (int t = 0; t < 9; ++t) {
          const long q = n.nb(b, i, j, t);
          if (q < 0) continue;
          for (int ci = 0; ci < C; ++ci) {
            g[OFF_HEAD_W + t * C + ci] += A.x[NBLK][q * C + ci] * gout[p];
            G[q * C + ci] += gout[p] * n.R(prm[OFF_HEAD_W + t * C + ci]);
          }
        }
      }
  // blocks
  for (int k = NBLK - 1; k >= 0; --k) {
    const float* Wk = prm + OFF_BLK + k * BLK_SZ;
    double* gW = g.data() + OFF_BLK + k * BLK_SZ;
    std::vector<double> DY(P * C), DYb(P * C);
    for (long e = 0; e < P * C; ++e) {
      DY[e] = A.y[k + 1][e] > 0 ? G[e] : 0.0;
      DYb[e] = n.R(DY[e]);
    }
    std::vector<double> Gn = G;   // identity path of the residual
    for (int b = 0; b < n.B; ++b)
      for (int i = 0; i < n.H; ++i)
        for (int j = 0; j < n.W; ++j) {
          const long p = ((long)b * n.H + i) * n.W + j;
          for (int co = 0; co < C; ++co) gW[9 * C * C + co] += DY[p * C + co];
          for (int t = 0; t < 9; ++t) {
            const long q = n.nb(b, i, j, t);
            if (q < 0) continue;
            for (int ci = 0; ci < C; ++ci) {
              double s = 0.0;
              for (int co = 0; co < C; ++co) {
                gW[(t * C + ci) * C + co] += A.x[k][q * C + ci] * DY[p * C + co];
                s += DYb[p * C + co] * n.R(Wk[(t * C + ci) * C + co]);
              }
              Gn[q * C + ci] += s;
            }
          }
        }
    G.swap(Gn);
  }
  // stem
  for (int b = 0; b < n.B; ++b)
    for (int i = 0; i < n.H; ++i)
      for (int j = 0; j < n.W; ++j) {
        const long p = ((long)b * n.H + i) * n.W + j;
        for (int co = 0; co < C; ++co) {
          const double dy = A.y[0][p * C + co] > 0 ? G[p * C + co] : 0.0;
          g[OFF_STEM_B + co] += dy;
          for (int t = 0; t < 9; ++t) {
            const long q = n.nb(b, i, j, t);
            if (q < 0) continue;
            for (int ci = 0; ci < NIN; ++ci) g[(t * NIN + ci) * C + co] += A.fb[q * NIN + ci] * dy;
          }
        }
      }
  return l / m;
}

}  // namespace

extern "C" {

int orc_net_nparam() { return NPARAM; }

// out[B][H][W] = network(feat[B][H][W][4])
int orc_net_forward(const float* params, const float* feat, int B, int H, int W, int bf16, double* out) {
  if (B < 1 || H < 1 || W < 1) return -1;
  Net n{B, H, W, bf16 != 0};
  Acts A;
  forward(n, params, feat, A);
  std::memcpy(out, A.out.data(), sizeof(double) * A.out.size());
  return 0;
}

// loss and d loss / d params of the masked mean-square error against target.
int orc_net_grad(const float* params, const float* feat, const float* target, const float* mask, int B, int H, int W,
                 int bf16, double* grad, double* loss) {
  if (B < 1 || H < 1 || W < 1) return -1;
  Net n{B, H, W, bf16 != 0};
  Acts A;
  forward(n, params, feat, A);
  std::vector<double> g;
  *loss = backward(n, params, A, target, mask, g);
  std::memcpy(grad, g.data(), sizeof(double) * NPARAM);
  return 0;
}

}  // extern "C"
