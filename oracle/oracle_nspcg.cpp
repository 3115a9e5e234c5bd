// Oracle restatement of NSPCG's MIC-preconditioned conjugate gradient — TEST INFRASTRUCTURE ONLY
// (see oracle.hpp).
//
// Path restated (FP64, iparm/rparm as set by dfault + SolverSparse, si3d_procedures.f90:1986-1995):
//   nspcg (nspcg.f:7-138) -> echall (:17008) -> adjust (:14913) -> detsym (:16964)
//   -> [red-black only: prbndx colouring (:25337-25460) and the symmetric permutation of the
//       Purdue arrays that NSPCG applies with iperm = 1 (permut/permp :446-485, :837)]
//   -> mic1 (:1441-1479) -> move1 (:23287) -> pfact1 (:6583-6660) -> icfp MIC, property A
//      (:20724-20850) -> split/cg/cgw (:1256, :7791, :8328-8450) -> nmcalc (:24169)
//   -> itcg (:8967-9092) with suba8/mult1/vaddp (:3285, :23919, :32039, keygs = 1),
//      subq86/icsp/icfstp/icbsp (:5526, :21759, :22875, :22729), pstops (:25956-26100),
//      chgcon/eigvss/zbrent/determ (:16499, :17201, :32976, :16926).
//
// The red-black form keeps NSPCG's own algorithm (the natural-order routines applied to the
// colour-permuted matrix); the Purdue arrays are widened beyond mdim = 5 so that the red rows'
// four upper entries fit (the reference sizes coeffA with mdimA = 5, si3d_types.f90:156).
#include <algorithm>
#include <cmath>

#include "oracle.hpp"

namespace orc {

namespace {

struct Purdue {  // ndim x maxnz column-major, 1-based indices
  int n = 0, maxnz = 0;
  std::vector<real> c;
  std::vector<int> j;
  real& C(int i, int col) { return c[(size_t)(col - 1) * n + (i - 1)]; }
  int& J(int i, int col) { return j[(size_t)(col - 1) * n + (i - 1)]; }
};

// move1 (nspcg.f:23287-23380): upper-triangle columns first, then lower.
int move1(Purdue& A, int mdim, int& nt, int& nb) {
  const int n = A.n;
  int maxnz = A.maxnz, ntt = 0, nbb = 0;
  if (maxnz > 1) {
    for (int i = 1; i <= n; ++i) {
      int ntrow = 0, nbrow = 0;
      for (int jj = 2; jj <= maxnz; ++jj) {
        int d = A.J(i, jj) - i;
        if (d < 0) nbrow++;
        else if (d > 0) ntrow++;
      }
      ntt = std::max(ntt, ntrow);
      nbb = std::max(nbb, nbrow);
    }
    int ndtb = ntt + nbb + 1;
    if (ndtb > mdim) { nt = ntt; nb = nbb; return -9; }
    if (ntt * nbb != 0) {
      if (ndtb > maxnz) {
        A.c.resize((size_t)ndtb * n, 0.0);
        A.j.resize((size_t)ndtb * n, 0);
        for (int jj = maxnz + 1; jj <= ndtb; ++jj)
          for (int i = 1; i <= n; ++i) { A.C(i, jj) = 0.0; A.J(i, jj) = i; }
        maxnz = ndtb;
        A.maxnz = maxnz;
      }
      const int nt2 = ntt + 1, nb1 = nt2 + 1;
      for (int i = 1; i <= n; ++i) {
        int jbc = nt2;
        for (int jtc = 2; jtc <= nt2; ++jtc) {
          if (A.J(i, jtc) >= i) continue;
          do { jbc = jbc + 1; } while (A.J(i, jbc) < i);
          std::swap(A.J(i, jtc), A.J(i, jbc));
          std::swap(A.C(i, jtc), A.C(i, jbc));
        }
        int jtc = 1;
        for (jbc = nb1; jbc <= maxnz; ++jbc) {
          if (A.J(i, jbc) <= i) continue;
          do { jtc = jtc + 1; } while (A.J(i, jtc) > i);
          std::swap(A.J(i, jtc), A.J(i, jbc));
          std::swap(A.C(i, jtc), A.C(i, jbc));
        }
      }
    }
  }
  nt = ntt;
  nb = nbb;
  return 0;
}

// mult1 with keygs = 1 (explicit gathers): y = a x (nspcg.f:23919-23947, :32039-32115)
void mult1(Purdue& A, const std::vector<real>& x, std::vector<real>& y) {
  const int n = A.n;
  for (int i = 1; i <= n; ++i) y[i - 1] = A.C(i, 1) * x[i - 1];
  for (int jj = 2; jj <= A.maxnz; ++jj)
    for (int i = 1; i <= n; ++i) y[i - 1] = y[i - 1] + A.C(i, jj) * x[A.J(i, jj) - 1];
}

// icsp with ipropa = 1: (d + t^T) inv(d) (d + t) x = y, d holding reciprocal pivots
// (nspcg.f:21759-21805, icfstp :22875-22922, icbsp :22729-22777).
void icsp(Purdue& A, int maxt, const std::vector<real>& d, const std::vector<real>& y, std::vector<real>& x) {
  const int n = A.n;
  for (int i = 0; i < n; ++i) x[i] = y[i];
  for (int i = 1; i <= n; ++i) {
    x[i - 1] = x[i - 1] * d[i - 1];
    real term = x[i - 1];
    for (int jj = 1; jj <= maxt; ++jj) {
      int jt = A.J(i, jj + 1);
      x[jt - 1] = x[jt - 1] - A.C(i, jj + 1) * term;
    }
  }
  for (int i = 0; i < n; ++i) x[i] = x[i] / d[i];
  for (int i = n; i >= 1; --i) {
    real sum = x[i - 1];
    for (int jj = 1; jj <= maxt; ++jj) sum = sum - A.C(i, jj + 1) * x[A.J(i, jj + 1) - 1];
    sum = sum * d[i - 1];
    x[i - 1] = sum;
  }
}

real vdot(const std::vector<real>& a, const std::vector<real>& b) {
  real s = 0.0;
  for (size_t i = 0; i < a.size(); ++i) s = s + a[i] * b[i];
  return s;
}

// determ (nspcg.f:16926-16962)
real determ(int n, const std::vector<real>& tri, real x) {
  auto T = [&](int r, int c) { return tri[(size_t)(c - 1) * 2 + (r - 1)]; };
  int nm1 = n - 1;
  real d2 = T(1, n) - x;
  real d1 = d2 * (T(1, nm1) - x) - T(2, n);
  if (n != 2) {
    for (int l = nm1; l >= 2; --l) {
      real d3 = d2;
      d2 = d1;
      d1 = (T(1, l - 1) - x) * d2 - d3 * T(2, l);
    }
  }
  return d1;
}

// zbrent (nspcg.f:32976-33160)
void zbrent(int n, const std::vector<real>& tri, real eps, int nsig, real& aa, real& bb, int& maxfnn, int& ier) {
  real a = aa, b = bb;
  int maxfn = maxfnn;
  real t = std::pow(0.1, nsig);
  int ic = 2;
  real fa = determ(n, tri, a), fb = determ(n, tri, b), fc = 0, c = 0, d = 0, e = 0, s = b;
  real p, q, r, rone, tol, rm, temp;
  if (fa * fb > 0.0) { ier = 4; maxfn = ic; aa = a; bb = b; maxfnn = maxfn; return; }
L5:
  c = a; fc = fa; d = b - c; e = d;
L10:
  if (std::fabs(fc) < std::fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
  tol = t * std::max(std::fabs(b), 0.1);
  rm = (c - b) / 2.0;
  if (std::fabs(fb) <= eps) goto L40;
  if (std::fabs(c - b) <= tol) goto L40;
  if (ic >= maxfn) goto L45;
  if (std::fabs(e) < tol) goto L30;
  if (std::fabs(fa) <= std::fabs(fb)) goto L30;
  s = fb / fa;
  if (a != c) goto L20;
  p = (c - b) * s;
  q = 1.0 - s;
  goto L25;
L20:
  q = fa / fc;
  r = fb / fc;
  rone = r - 1.0;
  p = s * ((c - b) * q * (q - r) - (b - a) * rone);
  q = (q - 1.0) * rone * (s - 1.0);
L25:
  if (p > 0.0) q = -q;
  if (p < 0.0) p = -p;
  s = e;
  e = d;
  if (p + p >= 3.0 * rm * q) goto L30;
  if (p + p >= std::fabs(s * q)) goto L30;
  d = p / q;
  goto L35;
L30:
  e = rm;
  d = e;
L35:
  a = b;
  fa = fb;
  temp = d;
  if (std::fabs(temp) <= tol / 2.0) temp = std::copysign(tol / 2.0, rm);
  b = b + temp;
  s = b;
  fb = determ(n, tri, s);
  ic = ic + 1;
  if (fb * fc <= 0.0) goto L10;
  goto L5;
L40:
  a = c;
  maxfn = ic;
  aa = a; bb = b; maxfnn = maxfn;
  return;
L45:
  ier = 3;
  a = c;
  maxfn = ic;
  aa = a; bb = b; maxfnn = maxfn;
}

struct Itcom {
  real alpha = 0, beta = 0, zeta = 0, emax = 2.0, emin = 1.0, pap = 0, alphao = 0, stptst = 0, udnm = 1,
       bnorm = 0, rzdot = 0, dkm1 = 0, srelpr = 0;
  int in = 0, is = 0, itmax = 0, ntest = 5;
  bool halt = false, maxadp = true, minadp = true, q1 = false;
  real tl1 = 0, tl2 = 0, bl1 = 0, bl2 = 0;
  std::vector<real> tri;  // 2 x (itmax+2)
};

// eigvss (nspcg.f:17201-17240)
real eigvss(Itcom& I, int n, real start, real end, int icode, int& ier) {
  int itmp = (int)(-std::log10(std::fabs(I.zeta)));
  int nsig = std::max(itmp, 4);
  int maxfn = std::max(I.itmax, 50);
  real a = start, b = end;
  zbrent(n, I.tri, 0.0, nsig, a, b, maxfn, ier);
  if (icode == 1) return std::max(a, b);
  return std::min(a, b);
}

// chgcon (nspcg.f:16499-16620)
void chgcon(Itcom& I, int& ier) {
  auto T = [&](int r, int c) -> real& { return I.tri[(size_t)(c - 1) * 2 + (r - 1)]; };
  int ip = I.is;
  if (ip == 0) {
    real end = 1.0 / I.alpha;
    T(1, 1) = end; T(2, 1) = 0.0;
    if (I.maxadp) I.emax = end;
    if (I.minadp) I.emin = end;
    return;
  }
  if (ip == 1) {
    real t1 = 1.0 / I.alpha + I.beta / I.alphao;
    real t2 = I.beta / (I.alphao * I.alphao);
    T(1, 2) = t1; T(2, 2) = t2;
    real tsqr = std::sqrt(t2);
    I.tl1 = T(1, 1) + tsqr; I.tl2 = t1 + tsqr;
    I.bl1 = T(1, 1) - tsqr; I.bl2 = t1 - tsqr;
    real t3 = T(1, 1) + t1;
    real t4 = std::sqrt((t1 - T(1, 1)) * (t1 - T(1, 1)) + 4.0 * t2);
    if (I.maxadp) I.emax = (t3 + t4) / 2.0;
    if (I.minadp) I.emin = (t3 - t4) / 2.0;
    return;
  }
  real t1 = 1.0 / I.alpha + I.beta / I.alphao;
  real t2 = I.beta / (I.alphao * I.alphao);
  real tsqr = std::sqrt(t2);
  T(1, ip + 1) = t1; T(2, ip + 1) = t2;
  if (I.maxadp) {
    I.tl1 = std::max(I.tl1, I.tl2 + tsqr);
    I.tl2 = t1 + tsqr;
    real emaxo = I.emax;
    real end = std::max(I.tl1, I.tl2);
    real e1 = eigvss(I, ip + 1, emaxo, end, 2, ier);
    if (ier != 3 && ier != 4) {
      I.emax = e1;
      if (std::fabs(I.emax - emaxo) < I.emax * I.zeta) I.maxadp = false;
    } else I.maxadp = false;
  }
  if (!I.minadp) return;
  I.bl1 = std::min(I.bl1, I.bl2 - tsqr);
  I.bl2 = t1 - tsqr;
  real start = std::max(0.0, std::min(I.bl1, I.bl2));
  real emino = I.emin;
  real e1 = eigvss(I, ip + 1, start, emino, 1, ier);
  if (ier != 3 && ier != 4) {
    I.emin = e1;
    if (std::fabs(I.emin - emino) < I.emin * I.zeta) I.minadp = false;
  } else I.minadp = false;
}

// pstops tests 2 and 5 (nspcg.f:26034-26091)
void pstops(Itcom& I, const std::vector<real>& r, const std::vector<real>& z, const std::vector<real>& u) {
  I.halt = false;
  real tiny = 500.0 * I.srelpr;
  if (I.ntest == 2) {
    if (I.in < 1) {
      I.q1 = false;
      I.udnm = 1.0;
      I.stptst = std::sqrt(I.rzdot);
      if (I.stptst < tiny) I.halt = true;
      return;
    }
    if (!(I.q1) && !((I.in > 5) && (I.in % 5 != 0))) {
      real uold = I.udnm;
      I.udnm = std::sqrt(vdot(u, u));
      if (I.udnm < tiny) I.udnm = 1.0;
      if ((I.in > 5) && (std::fabs(I.udnm - uold) < I.udnm * I.zeta)) I.q1 = true;
    }
    real eminl = I.emin;
    if (eminl < tiny) eminl = tiny;
    real tl = std::sqrt(vdot(z, z));
    real tr = I.udnm * eminl;
    I.stptst = tl / tr;
    if (tl < tr * I.zeta) I.halt = true;
  } else {
    real tl = std::sqrt(vdot(r, r));
    real tr = I.bnorm;
    I.stptst = tl / tr;
    if (tl < tr * I.zeta) I.halt = true;
  }
}

}  // namespace

// prbndx-equivalent colouring: the first unlabelled node of each connected component is red,
// neighbours alternate; zero coefficients are not edges (nspcg.f:25337-25460).
std::vector<int> redblack_colors(int n, const std::vector<real>& coef, const std::vector<int>& jcoef) {
  std::vector<int> col(n, 0), stack;
  const int maxnz = (int)(coef.size() / (size_t)n);
  stack.reserve(n);
  for (int first = 1; first <= n; ++first) {
    if (col[first - 1] != 0) continue;
    col[first - 1] = 1;
    stack.clear();
    stack.push_back(first);
    for (size_t next = 0; next < stack.size(); ++next) {
      int k = stack[next];
      for (int jj = 1; jj <= maxnz; ++jj) {
        int jc = jcoef[(size_t)(jj - 1) * n + (k - 1)];
        if (jc < 1 || jc > n || jc == k) continue;
        if (coef[(size_t)(jj - 1) * n + (k - 1)] == 0.0) continue;
        int want = 3 - col[k - 1];
        if (col[jc - 1] == 0) { col[jc - 1] = want; stack.push_back(jc); }
        else if (col[jc - 1] != want) return {};
      }
    }
  }
  return col;
}

PcgResult nspcg_mic_cg(int n, const std::vector<real>& coef_in, const std::vector<int>& jcoef_in,
                       const std::vector<real>& rhs_in, std::vector<real>& u_io, const Opts& opt,
                       const std::vector<int>* color) {
  PcgResult res;
  Itcom I;
  I.srelpr = opt.srelpr;
  I.ntest = opt.pcg_test;
  I.itmax = opt.pcg_itmax;
  // echall (nspcg.f:17068-17120)
  I.zeta = opt.pcg_tol;
  int ier = 0;
  if (I.ntest != 2 && I.ntest != 5) { res.ier = -10; return res; }
  if (I.zeta < 500.0 * I.srelpr) { ier = 2; I.zeta = 500.0 * I.srelpr; }
  I.emax = 2.0; I.emin = 1.0;   // rparm(2), rparm(3) from dfault
  Purdue A;
  A.n = n;
  A.maxnz = 5;
  A.c = coef_in;
  A.j = jcoef_in;
  // adjust (nspcg.f:14913-14940)
  for (int jj = 2; jj <= A.maxnz; ++jj)
    for (int i = 1; i <= n; ++i) if (A.J(i, jj) <= 0) A.J(i, jj) = i;
  // detsym (nspcg.f:16964-17006): this restatement covers the symmetric branch only
  for (int i = 1; i <= n; ++i)
    for (int jj = 2; jj <= A.maxnz; ++jj) {
      int jc = A.J(i, jj);
      if (jc == i) continue;
      real val = A.C(i, jj);
      bool found = false;
      for (int j2 = 2; j2 <= A.maxnz; ++j2)
        if (A.J(jc, j2) == i) { found = true; if (A.C(jc, j2) != val) { res.ier = -10; return res; } break; }
      if (!found) { res.ier = -10; return res; }
    }
  std::vector<real> rhs = rhs_in, u = u_io;
  std::vector<int> perm, iperm;  // perm[new-1] = old, iperm[old-1] = new
  if (color) {
    for (int c = 1; c <= 2; ++c)
      for (int i = 1; i <= n; ++i) if ((*color)[i - 1] == c) perm.push_back(i);
    iperm.assign(n, 0);
    for (int k = 0; k < n; ++k) iperm[perm[k] - 1] = k + 1;
    Purdue B = A;
    for (int knew = 1; knew <= n; ++knew) {
      int iold = perm[knew - 1];
      for (int jj = 1; jj <= A.maxnz; ++jj) {
        B.C(knew, jj) = A.C(iold, jj);
        B.J(knew, jj) = iperm[A.J(iold, jj) - 1];
      }
      rhs[knew - 1] = rhs_in[iold - 1];
      u[knew - 1] = u_io[iold - 1];
    }
    A = B;
  }
  // mic1 -> move1 -> pfact1 (meth = 2, propa) -> icfp
  int nt = 0, nb = 0;
  if (move1(A, color ? 9 : 5, nt, nb) < 0) { res.ier = -9; return res; }
  std::vector<real> d(n);
  for (int i = 1; i <= n; ++i) d[i - 1] = A.C(i, 1);
  const int maxt = nt;
  const real omega = 1.0;
  if (maxt >= 1) {
    std::vector<real> wk(n, 0.0);
    for (int jj = 1; jj <= maxt; ++jj)
      for (int i = 1; i <= n; ++i) wk[i - 1] = wk[i - 1] + A.C(i, jj + 1);
    for (int k = 1; k <= n - 1; ++k) {
      real pivot = d[k - 1];
      if (pivot == 0.0) { res.ier = -12; return res; }
      for (int ii = 1; ii <= maxt; ++ii) {
        int jcol = A.J(k, ii + 1);
        if (jcol == k) continue;
        real term = A.C(k, ii + 1) / pivot;
        d[jcol - 1] = d[jcol - 1] - term * (omega * wk[k - 1] - (omega - 1.0) * A.C(k, ii + 1));
      }
    }
    if (d[n - 1] == 0.0) { res.ier = -12; return res; }
  }
  for (int i = 0; i < n; ++i) d[i] = 1.0 / d[i];
  for (int i = 0; i < n; ++i) if (d[i] < 0.0) { ier = 5; break; }

  // cgw (nspcg.f:8328-8450): nmcalc, then itcg
  if (I.ntest == 5) I.bnorm = std::max(std::sqrt(vdot(rhs, rhs)), I.srelpr);
  I.tri.assign((size_t)2 * (I.itmax + 2), 0.0);
  std::vector<real> r(n, 0.0), p(n, 0.0), z(n, 0.0);
  I.in = 0; I.is = 0; I.rzdot = 0.0; I.alpha = 0.0; I.beta = 0.0; I.alphao = 0.0;
  I.maxadp = true; I.minadp = true;
  mult1(A, u, r);
  for (int i = 0; i < n; ++i) r[i] = rhs[i] - r[i];
  bool first = true;
  for (;;) {
    if (!first)
      for (int i = 0; i < n; ++i) r[i] = r[i] - I.alpha * z[i];
    first = false;
    icsp(A, maxt, d, r, z);
    I.dkm1 = I.rzdot;
    I.rzdot = vdot(r, z);
    if (!(I.rzdot > 0.0)) { ier = -7; break; }
    pstops(I, r, z, u);
    if (I.halt || ier < 0) break;
    if (!(I.in < I.itmax)) { ier = 1; I.zeta = I.stptst; break; }
    if (I.in != 0) I.beta = I.rzdot / I.dkm1;
    for (int i = 0; i < n; ++i) p[i] = z[i] + I.beta * p[i];
    mult1(A, p, z);
    I.alphao = I.alpha;
    I.pap = vdot(p, z);
    I.alpha = I.rzdot / I.pap;
    if (!(I.pap > 0.0)) { ier = -6; break; }
    res.alphas.push_back(I.alpha);
    res.betas.push_back(I.beta);
    if (I.maxadp || I.minadp) chgcon(I, ier);
    for (int i = 0; i < n; ++i) u[i] = u[i] + I.alpha * p[i];
    I.in++;
    I.is++;
  }
  if (color) for (int knew = 1; knew <= n; ++knew) u_io[perm[knew - 1] - 1] = u[knew - 1];
  else u_io = u;
  res.iters = I.in;
  res.ier = ier;
  res.stptst = I.stptst;
  res.emin = I.emin;
  res.emax = I.emax;
  return res;
}

}  // namespace orc
