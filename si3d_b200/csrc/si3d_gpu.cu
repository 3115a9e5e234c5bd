// C-ABI implementation (include/si3d_gpu.h): handle management, device state, layout
// transposes at the boundary, and the stage sequence of fd / settrap / settrap2 / save.
#include <algorithm>
#include <functional>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/si3d_gpu.h"
#include "../../include/si3d_learn.h"
#include "common.cuh"
#include "kernels.h"
#include "learn.h"
#include "mg.h"

using namespace si3d;

namespace {

#define CK(x)                                                 \
  do {                                                        \
    cudaError_t e_ = (x);                                     \
    if (e_ != cudaSuccess) return cuda_fail(e_, #x, __LINE__); \
  } while (0)

thread_local std::string g_last_cuda;
int cuda_fail(cudaError_t e, const char* what = nullptr, int line = 0) {
  g_last_cuda = cudaGetErrorString(e);
  if (what) g_last_cuda += std::string(" [") + what + ", si3d_gpu.cu:" + std::to_string(line) + "]";
  return SI3D_ECUDA;
}

// ---------------------------------------------------------------------------- layout kernels
// (km1, lm1) column-major  <->  layer-major with pitch P
__global__ void k_colmajor_to_layer(const double* __restrict__ src, double* __restrict__ dst, int km1, int lm1, int P) {
  __shared__ double tile[32][33];
  const int l0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int l = l0 + r, k = k0 + threadIdx.x;
    if (l < lm1 && k < km1) tile[r][threadIdx.x] = src[(size_t)l * km1 + k];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int k = k0 + r, l = l0 + threadIdx.x;
    if (l < lm1 && k < km1) dst[(size_t)k * P + l] = tile[threadIdx.x][r];
  }
}

__global__ void k_layer_to_colmajor(const double* __restrict__ src, double* __restrict__ dst, int km1, int lm1, int P) {
  __shared__ double tile[32][33];
  const int l0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int k = k0 + r, l = l0 + threadIdx.x;
    if (l < lm1 && k < km1) tile[r][threadIdx.x] = src[(size_t)k * P + l];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += 8) {
    const int l = l0 + r, k = k0 + threadIdx.x;
    if (l < lm1 && k < km1) dst[(size_t)l * km1 + k] = tile[threadIdx.x][r];
  }
}

// ---------------------------------------------------------------------------- handle context
constexpr int kHistSlots = 4;   // leapfrog, trapezoidal 1, 2, and all later trapezoidal solves

struct Ctx {
  int device = 0;
  cudaStream_t st = nullptr;
  Dev d{};
  si3d_params prm{};
  int lm = 0, lm1 = 0, km1 = 0, P = 0;
  std::vector<void*> allocs;
  // face-column lists (id_columnCE / id_columnCN)
  int* ce = nullptr;
  int* cn = nullptr;
  int nce = 0, ncn = 0;
  FaceMeta* mce = nullptr;   // static indices of the u / v face columns (momentum stage)
  FaceMeta* mcn = nullptr;
  // red-black zeta system
  PcgDev pcg{};
  PcgDevF pcgf{};            // FP32 inner system of iterative refinement
  NatDev nat{};              // natural-order system (ordering SI3D_ORDER_NATURAL)
  bool natural = false;
  // host copies of the grid maps (1-based, lm entries) for set-ups that need (i, j) lookups
  std::vector<int> h_l2i, h_l2j, h_lEC, h_lWC, h_lNC, h_lSC;
  // open boundaries (si3d_gpu_set_open_boundaries): device cell lists, the series (host), their
  // spacing in seconds, and the time of the step in progress in hours (thrs of si3d.f90:327)
  std::vector<ObcDev> obc;
  std::vector<std::vector<double>> obc_wse, obc_tmp;
  double obc_dtsec = 0, thrs = 0;
  MgDev mg{};                // aggregation hierarchy of the MG inner solves (precision SI3D_MIXED_MG)
  int mg_blocks = 0;
  PcgScal* h_scf = nullptr;  // pinned
  int last_inner = 8;
  long long ir_outer = 0;
  PcgScal* h_sc = nullptr;  // pinned
  double* h_hist = nullptr; // pinned, 2 x itmax
  int last_iters = 8;
  // whole-solve cooperative kernel (k_pcg_persistent.cu); false -> one launch per phase
  bool persistent = true;
  int loop_blocks = 0, loop_blocks_f = 0;   // FP64 / FP32 grids of the cooperative solve
  GridBar* bar = nullptr;
  // si3d_gpu_test_wait_limit: barrier record for the next cooperative solve launch only
  GridBar bar_test{};
  bool bar_test_armed = false;
  bool log_solves = false;   // SI3D_LOG_SOLVES=1: per-solve iteration counts on stderr
  int cur_istep = 1;         // istep of the fd call in progress (1 = leapfrog, 2 = trapezoidal)
  // solve slot within a step (0 = leapfrog, 1.. = trapezoidal iterations, clamped to kHistSlots - 1)
  // and per slot the correction of that solve one step earlier, in colour order
  int trap_solves = 0, hist_slot = 0;
  double* hist = nullptr;
  // instrumentation: kernel-launch count and (optionally) per-stage device time
  long long launches = 0;
  bool prof = false;
  double prof_ms[16] = {0};
  long long prof_n[16] = {0};
  cudaEvent_t pe0 = nullptr, pe1 = nullptr;
  double* dz = nullptr;     // learned warm-start increment (device, lm1)
  bool dz_set = false;
  // learned initial guess: pixel of every wet column in the (im1, jm1) image, network state,
  // features of the current solve, optional training record
  int im1 = 1, jm1 = 1;
  int* pix = nullptr;
  bool net_loaded = false;
  float* net_params = nullptr;
  void* net_mem = nullptr;
  learn::Workspace net_ws;
  float *feat = nullptr, *net_out = nullptr;
  double *r0 = nullptr, *fpart = nullptr, *sigma = nullptr;
  float* rec_buf = nullptr;
  int rec_slots = 0, rec_count = 0;
  // graph-capturable stepping (ensembles): no host synchronisation inside a step; every solve
  // writes (iterations, ier) and its stopping-test value into device slots
  Tune tune;                     // launch shapes of the column stages (autotuned)
  bool graph_mode = false;
  int solve_slot = 0;
  // batched ensemble capture: solve() stops after the set-up of its FP64 loop and leaves the loop
  // to the ensemble's one launch, then solve_graph_post finishes it (hist and ier kept here)
  bool ens_defer = false;
  double* def_hist = nullptr;
  int def_ier = 0;
  int* d_stats_ii = nullptr;     // [24][2]
  double* d_stats_rr = nullptr;  // [24]
  double* staging = nullptr;  // device staging for transposes (km1 * lm1)
  float* staging_f = nullptr; // FP32 staging of the single-precision field copies (allocated on first use)
  // non-active tracers: two pools of ntr layer-major fields; tr_buf[tr_cur] holds tracer, the other
  // tracerpp.  save makes tracerpp = tracer by swapping the pools; after it the tracer pool is not
  // read (tr_alias: "tracer" reads resolve to tracerpp) until the next ImTracer rewrites every
  // entry it may change.  Entries no routine writes (below kmz + 1, the dry column) are the same in
  // both pools once tr_synced; a host write clears it and the next save copies instead of swapping.
  double* tr_buf[2] = {nullptr, nullptr};
  int tr_cur = 0;
  bool tr_alias = true, tr_synced = true;
  long long tr_stride = 0;
  double* tr_scr = nullptr;   // elimination factors, one km1 x P field per tracer group
  double* tr_fx = nullptr;    // face fluxes of one flux group (the last tracer's go to Bth2/3/4)
  double* turb_scr = nullptr; // Mellor-Yamada 2.5: four km1 x P scratch fields
  // output frames: column coordinates, point offsets of the 3-D frames, a device frame buffer and
  // the column list of each output plane requested so far
  int *d_l2i = nullptr, *d_l2j = nullptr, *poff = nullptr;
  long long npoints = 0;
  float* out_buf[2] = {nullptr, nullptr};   // device frames, used in turn
  long long out_cap = 0;
  int out_slot = 0;
  cudaStream_t cst = nullptr;                 // device-to-host copies of frames
  cudaEvent_t out_packed = nullptr, out_free[2] = {nullptr, nullptr};
  cudaEvent_t out_done[16] = {};              // one per copy in flight (tickets), used in turn
  int out_ev = 0;
  std::map<int, std::pair<int*, int>> planes;
  std::vector<int> h_kmz;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, evp0 = nullptr, evp1 = nullptr;
  // staged inputs and asynchronous field reads (si3d_gpu_stage_field, si3d_gpu_fetch_field): copy
  // streams for each direction, two staging slots used in turn, the committed groups oldest first
  struct Staged {
    std::map<std::string, double*> buf;
    std::vector<std::pair<double*, double*>> moves;   // (field, staged values)
    cudaEvent_t ready = nullptr, free = nullptr;
  };
  cudaStream_t ist = nullptr, fst = nullptr;
  Staged stg[2];
  int stg_fill = -1, stg_next = 0;
  std::deque<int> stg_queue;
  std::map<std::string, double*> snap;
  cudaEvent_t snap_ready = nullptr, fetch_done = nullptr;
  ~Ctx() {
    if (st) cudaStreamSynchronize(st);
    for (cudaStream_t x : {ist, fst}) if (x) { cudaStreamSynchronize(x); cudaStreamDestroy(x); }
    for (cudaEvent_t e : {stg[0].ready, stg[0].free, stg[1].ready, stg[1].free, snap_ready, fetch_done})
      if (e) cudaEventDestroy(e);
    for (void* p : allocs) cudaFree(p);
    if (h_sc) cudaFreeHost(h_sc);
    if (h_scf) cudaFreeHost(h_scf);
    if (h_hist) cudaFreeHost(h_hist);
    if (cst) cudaStreamSynchronize(cst);
    for (cudaEvent_t e : {ev0, ev1, evp0, evp1, pe0, pe1, out_packed, out_free[0], out_free[1]}) if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : out_done) if (e) cudaEventDestroy(e);
    if (cst) cudaStreamDestroy(cst);
    if (st) cudaStreamDestroy(st);
  }
  template <class T>
  int alloc(T** p, size_t n) {
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) { g_last_cuda = cudaGetErrorString(e); return SI3D_ENOMEM; }
    allocs.push_back(q);
    // the zero fill runs on the legacy default stream, which the handle's non-blocking streams do
    // not wait for: finish it before the buffer is handed out
    e = cudaMemset(q, 0, std::max<size_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) { g_last_cuda = cudaGetErrorString(e); return SI3D_ECUDA; }
    *p = static_cast<T*>(q);
    return 0;
  }
};

std::mutex g_mu;
std::vector<Ctx*> g_ctx;

// The barrier record armed by si3d_gpu_test_wait_limit, once (nullptr: the zeroed record).
const GridBar* take_bar_test(Ctx* c) {
  if (!c->bar_test_armed) return nullptr;
  c->bar_test_armed = false;
  return &c->bar_test;
}

Ctx* get(int h) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (h < 0 || h >= (int)g_ctx.size()) return nullptr;
  return g_ctx[h];
}

// Stage ids for the per-stage device timers.
enum { ST_MOMX, ST_MOMY, ST_MATCON, ST_PCG_SETUP, ST_PCG_ITER, ST_PCG_FINISH, ST_SLAYER, ST_VEL, ST_SCALAR, ST_VEL2,
       ST_SETTRAP, ST_SETTRAP2, ST_SAVE, ST_LEARN, ST_TRACER, ST_TURB, ST_COUNT };

// Run `f` (which enqueues `nk` kernels) as one timed stage.
template <class F>
int stage(Ctx* c, int id, int nk, F&& f) {
  if (c->prof) cudaEventRecord(c->pe0, c->st);
  f();
  c->launches += nk;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e);
  if (c->prof) {
    cudaEventRecord(c->pe1, c->st);
    e = cudaEventSynchronize(c->pe1);
    if (e != cudaSuccess) return cuda_fail(e);
    float ms = 0;
    cudaEventElapsedTime(&ms, c->pe0, c->pe1);
    c->prof_ms[id] += ms;
    c->prof_n[id] += 1;
  }
  return 0;
}

double* f3ptr(Ctx* c, const std::string& n) {
  Fields3& f = c->d.f;
  static const std::map<std::string, double* Fields3::*> t = {
      {"uh", &Fields3::uh},     {"uhp", &Fields3::uhp},   {"uhpp", &Fields3::uhpp}, {"up", &Fields3::up},
      {"upp", &Fields3::upp},   {"hu", &Fields3::hu},     {"hup", &Fields3::hup},   {"hupp", &Fields3::hupp},
      {"agx", &Fields3::agx},   {"arx", &Fields3::arx},   {"vh", &Fields3::vh},     {"vhp", &Fields3::vhp},
      {"vhpp", &Fields3::vhpp}, {"vp", &Fields3::vp},     {"vpp", &Fields3::vpp},   {"hv", &Fields3::hv},
      {"hvp", &Fields3::hvp},   {"hvpp", &Fields3::hvpp}, {"agy", &Fields3::agy},   {"ary", &Fields3::ary},
      {"h", &Fields3::h},       {"hp", &Fields3::hp},     {"hpp", &Fields3::hpp},   {"sal", &Fields3::sal},
      {"salp", &Fields3::salp}, {"salpp", &Fields3::salpp}, {"rhop", &Fields3::rhop}, {"Av", &Fields3::Av},
      {"Dv", &Fields3::Dv},     {"wp", &Fields3::wp},     {"HeatSource", &Fields3::HeatSource},
      {"Bth2", &Fields3::Bth2}, {"Bth3", &Fields3::Bth3}, {"Bth4", &Fields3::Bth4},
      {"q2", &Fields3::q2},     {"q2p", &Fields3::q2p},   {"q2pp", &Fields3::q2pp}, {"q2l", &Fields3::q2l},
      {"q2lp", &Fields3::q2lp}, {"q2lpp", &Fields3::q2lpp}, {"u", &Fields3::u},      {"v", &Fields3::v}};
  auto it = t.find(n);
  return it == t.end() ? nullptr : f.*(it->second);
}

// "tracer<nt>" / "tracerpp<nt>", nt = 1..ntr: sets *pp and returns nt, else 0.
int tracer_name(const Ctx* c, const std::string& n, bool* pp) {
  for (const char* pre : {"tracerpp", "tracer"}) {
    const size_t np = std::strlen(pre);
    if (n.size() > np && n.compare(0, np, pre) == 0 && n.find_first_not_of("0123456789", np) == std::string::npos) {
      const int nt = std::atoi(n.c_str() + np);
      *pp = np == 8;
      return (nt >= 1 && nt <= c->prm.ntr) ? nt : -1;
    }
  }
  return 0;
}

double* tracer_pool(Ctx* c, bool pp) { return c->tr_buf[pp ? 1 - c->tr_cur : c->tr_cur]; }

// Give the tracer pool its own copy of tracerpp before a host write to either field.
int tracer_materialise(Ctx* c) {
  if (!c->tr_alias) return 0;
  const size_t bytes = sizeof(double) * (size_t)c->tr_stride * c->prm.ntr;
  CK(cudaMemcpyAsync(tracer_pool(c, false), tracer_pool(c, true), bytes, cudaMemcpyDeviceToDevice, c->st));
  c->tr_alias = false;
  return 0;
}

// fd's tracer block (si3d_procedures.f90:520-544, ecomod = 0): every tracer's right-hand side and
// column solve; the persistent flux arrays end as the reference's last exTracer leaves them.
void tracer_stage(Ctx* c) {
  double* tr = tracer_pool(c, false);
  const double* trpp = tracer_pool(c, true);
  launch_tracers(c->d, trpp, tr, c->tr_alias, c->prm.ntr, c->tr_stride, c->tr_fx, c->tr_scr, c->st);
  c->tr_alias = false;
}

// save's tracerpp = tracer (:3771-3774, :3926-3929).
int tracer_save(Ctx* c) {
  if (c->prm.ntr == 0 || c->tr_alias) return 0;
  if (c->tr_synced) {
    c->tr_cur = 1 - c->tr_cur;
  } else {
    const size_t bytes = sizeof(double) * (size_t)c->tr_stride * c->prm.ntr;
    CK(cudaMemcpyAsync(tracer_pool(c, true), tracer_pool(c, false), bytes, cudaMemcpyDeviceToDevice, c->st));
    c->tr_synced = true;
  }
  c->tr_alias = true;
  return 0;
}

// settrap / settrap2 / save with the turbulence time levels (si3d_procedures.f90:3612, :4085,
// :3769, :3924) and save's tracer hand-over.
void obc_continuity(Ctx* c);
void settrap_all(Ctx* c) {
  launch_settrap(c->d, c->st);
  obc_continuity(c);
  if (c->prm.iturb == 1) launch_turb_half(c->d, 1, c->st);
}
void settrap2_all(Ctx* c) {
  launch_settrap2(c->d, c->st);
  obc_continuity(c);
  if (c->prm.iturb == 1) launch_turb_half(c->d, 2, c->st);
}
int save_all(Ctx* c, int istep) {
  launch_save(c->d, istep, c->st);
  obc_continuity(c);
  if (c->prm.iturb == 1) launch_turb_save(c->d, istep, c->st);
  return tracer_save(c);
}

double* f2ptr(Ctx* c, const std::string& n) {
  Fields2& s = c->d.s;
  static const std::map<std::string, double* Fields2::*> t = {
      {"s", &Fields2::s},       {"sp", &Fields2::sp},     {"spp", &Fields2::spp},   {"eagx", &Fields2::eagx},
      {"earx", &Fields2::earx}, {"eagy", &Fields2::eagy}, {"eary", &Fields2::eary}, {"sx", &Fields2::sx},
      {"sy", &Fields2::sy},     {"dd", &Fields2::dd},     {"qq", &Fields2::qq},     {"rr", &Fields2::rr},
      {"uair", &Fields2::uair}, {"vair", &Fields2::vair}, {"cdw", &Fields2::cdw}};
  auto it = t.find(n);
  return it == t.end() ? nullptr : s.*(it->second);
}

int* iptr(Ctx* c, const std::string& n) {
  if (n == "k1z") return c->d.s.k1z;
  if (n == "k1u") return c->d.s.k1u;
  if (n == "k1v") return c->d.s.k1v;
  return nullptr;
}

// Red-black colouring of the wet-column graph, as prbndx does it (nspcg.f:25337-25460): the
// lowest unlabelled column of each connected component is red and colours alternate.
void colour_columns(int lm, const int* lEC, const int* lWC, const int* lNC, const int* lSC, std::vector<int>& col) {
  const int lm1 = lm + 1;
  col.assign(lm, 0);
  std::vector<int> stack;
  stack.reserve(lm);
  for (int first = 1; first <= lm; ++first) {
    if (col[first - 1]) continue;
    col[first - 1] = 1;
    stack.clear();
    stack.push_back(first);
    for (size_t nx = 0; nx < stack.size(); ++nx) {
      const int k = stack[nx];
      const int nb[4] = {lWC[k - 1], lSC[k - 1], lNC[k - 1], lEC[k - 1]};
      for (int m : nb) {
        if (m == lm1) continue;
        if (!col[m - 1]) { col[m - 1] = 3 - col[k - 1]; stack.push_back(m); }
      }
    }
  }
}

// Aggregation hierarchy of the MG inner solves.  Level 0 is the (im1, jm1) image of the wet
// columns, so the grid maps must describe that image: every neighbour one row (east / west) or one
// column (north / south) away.  Levels halve both sides until one block can sweep the coarsest
// and the coarsest is mass-dominated (kMgMinLevels).
int build_mg(Ctx* c, const si3d_grid* g) {
  const int lm = g->lm, lm1 = lm + 1;
  if (!g->l2i || !g->l2j) return SI3D_EDIMS;
  MgDev& M = c->mg;
  int rows = c->im1, cols = c->jm1, rc = 0;
  M.nlev = 0;
  for (;;) {
    MgLevel& L = M.lv[M.nlev++];
    L.rows = rows;
    L.cols = cols;
    L.pitch = mg_pitch(cols);
    L.nq = (cols + 3) / 4;
    L.div_cols = fast_div(cols);
    L.div_q = fast_div(L.nq);
    const size_t ne = mg_level_elems(rows, cols);
    for (float** q : {&L.z, &L.b, &L.fc, &L.fr, &L.mass, &L.dinv}) rc |= c->alloc(q, ne);
    if (rc) return rc;
    if ((M.nlev >= kMgMinLevels && (long long)rows * cols <= kMgCoarsest) || M.nlev == kMgMaxLevels ||
        (rows == 1 && cols == 1))
      break;
    rows = (rows + 1) / 2;
    cols = (cols + 1) / 2;
  }
  const size_t n0 = mg_level_elems(c->im1, c->jm1);
  for (float** q : {&M.u, &M.p0, &M.p1, &M.q}) rc |= c->alloc(q, n0);
  for (double** q : {&M.u64, &M.b64, &M.fc64, &M.fr64, &M.dg64}) rc |= c->alloc(q, n0);
  if (rc) return rc;
  const int pitch = M.lv[0].pitch;
  std::vector<int> off(lm + 2, -1);
  for (int l = 1; l <= lm; ++l) {
    const int i = g->l2i[l - 1] - 1, j = g->l2j[l - 1] - 1;
    if (i < 0 || i >= c->im1 || j < 0 || j >= c->jm1) return SI3D_EDIMS;
    off[l] = (i + 1) * pitch + j + kMgColOff;
  }
  for (int l = 1; l <= lm; ++l) {
    const int e = g->lEC[l - 1], w = g->lWC[l - 1], n = g->lNC[l - 1], s = g->lSC[l - 1];
    if ((e != lm1 && off[e] != off[l] + pitch) || (w != lm1 && off[w] != off[l] - pitch) ||
        (n != lm1 && off[n] != off[l] + 1) || (s != lm1 && off[s] != off[l] - 1))
      return SI3D_EDIMS;
  }
  int* dl = nullptr;
  rc |= c->alloc(&dl, lm);
  if (rc) return rc;
  CK(cudaMemcpy(dl, off.data() + 1, lm * sizeof(int), cudaMemcpyHostToDevice));
  M.pixL = dl;
  // SI3D_MG_BLOCKS_PER_SM caps the resident blocks per SM of the MG solve (tuning)
  const char* bps = std::getenv("SI3D_MG_BLOCKS_PER_SM");
  c->mg_blocks = mg_loop_blocks(c->device, c->im1 * c->jm1, bps ? std::atoi(bps) : 0);
  rc |= c->alloc(&M.part, 6 * (size_t)c->mg_blocks);
  PcgScal* sc = nullptr;
  rc |= c->alloc(&sc, 1);
  M.sc = sc;
  return rc;
}

// The natural-order system of ordering SI3D_ORDER_NATURAL: rows are the wet columns in l order.
// Lower neighbours must precede a row and upper ones follow it (the reference's i-outer, j-inner
// numbering guarantees it).  Per row: the level of the triangular sweeps (one more than its lower
// neighbours') and the order in which NSPCG's move1 (nspcg.f:23287-23380) leaves the row's
// off-diagonal columns - upper columns first - which fixes the order of every row sum.
int build_natural(Ctx* c, const si3d_grid* g) {
  const int lm = g->lm, lm1 = lm + 1;
  NatDev& N = c->nat;
  N.n = lm;
  std::vector<int4> nb(lm);
  std::vector<int> level(lm, 0), order(lm, 0);
  int nt = 0, nbm = 0, nlev = 0;
  for (int i = 0; i < lm; ++i) {
    auto row = [&](const int* m) { const int v = m[i]; return v == lm1 ? lm : v - 1; };
    nb[i] = make_int4(row(g->lWC), row(g->lSC), row(g->lNC), row(g->lEC));
    const int cand[4] = {nb[i].x, nb[i].y, nb[i].z, nb[i].w};
    int up = 0, lo = 0, lev = 0;
    for (int m : cand) {
      if (m == lm) continue;
      if (m == i) return SI3D_EDIMS;
      if (m < i) { ++lo; lev = std::max(lev, level[m] + 1); }
      else ++up;
    }
    // the reference's numbering: W and S precede the row, N and E follow it
    if ((nb[i].x != lm && nb[i].x > i) || (nb[i].y != lm && nb[i].y > i) || (nb[i].z != lm && nb[i].z < i) ||
        (nb[i].w != lm && nb[i].w < i))
      return SI3D_EDIMS;
    level[i] = lev;
    nlev = std::max(nlev, lev + 1);
    nt = std::max(nt, up);
    nbm = std::max(nbm, lo);
  }
  N.nt = nt;
  N.nlev = nlev;
  // move1 on each row's column indices (absent neighbours are the row itself after adjust)
  for (int i = 0; i < lm; ++i) {
    const int cand[4] = {nb[i].x, nb[i].y, nb[i].z, nb[i].w};
    int J[6], code[6];
    J[1] = i; code[1] = 4;
    for (int q = 0; q < 4; ++q) { J[q + 2] = cand[q] == lm ? i : cand[q]; code[q + 2] = cand[q] == lm ? 4 : q; }
    const int maxnz = 5, nt2 = nt + 1, nb1 = nt2 + 1;
    if (nt * nbm != 0) {
      int jbc = nt2;
      for (int jtc = 2; jtc <= nt2; ++jtc) {
        if (J[jtc] >= i) continue;
        do { ++jbc; } while (jbc <= maxnz && J[jbc] < i);
        if (jbc > maxnz) return SI3D_EDIMS;
        std::swap(J[jtc], J[jbc]);
        std::swap(code[jtc], code[jbc]);
      }
      int jtc = 1;
      for (jbc = nb1; jbc <= maxnz; ++jbc) {
        if (J[jbc] <= i) continue;
        do { ++jtc; } while (jtc <= maxnz && J[jtc] > i);
        if (jtc > maxnz) return SI3D_EDIMS;
        std::swap(J[jtc], J[jbc]);
        std::swap(code[jtc], code[jbc]);
      }
    }
    int packed = 0;
    for (int q = 0; q < 4; ++q) packed |= code[q + 2] << (3 * q);
    order[i] = packed;
  }
  std::vector<int> off(nlev + 1, 0), rows(lm);
  for (int i = 0; i < lm; ++i) off[level[i] + 1]++;
  for (int L = 0; L < nlev; ++L) off[L + 1] += off[L];
  std::vector<int> fill(off.begin(), off.end() - 1);
  for (int i = 0; i < lm; ++i) rows[fill[level[i]]++] = i;
  int rc = 0;
  int *d_off = nullptr, *d_rows = nullptr, *d_order = nullptr;
  int4* d_nb = nullptr;
  rc |= c->alloc(&d_off, nlev + 1);
  rc |= c->alloc(&d_rows, lm);
  rc |= c->alloc(&d_order, lm);
  rc |= c->alloc(&d_nb, lm);
  for (double** q : {&N.cd, &N.cW, &N.cS, &N.cN, &N.cE, &N.b, &N.u, &N.r, &N.z, &N.p, &N.q, &N.piv, &N.dinv})
    rc |= c->alloc(q, (size_t)lm + 1);
  if (rc) return rc;
  CK(cudaMemcpy(d_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_rows, rows.data(), rows.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(d_nb, nb.data(), nb.size() * sizeof(int4), cudaMemcpyHostToDevice));
  N.lvl_off = d_off; N.lvl_row = d_rows; N.order = d_order; N.nbr = d_nb;
  // scalars, alpha/beta record and Lanczos tridiagonal shared with the red-black system
  N.sc = c->pcg.sc; N.hist_alpha = c->pcg.hist_alpha; N.hist_beta = c->pcg.hist_beta; N.tri = c->pcg.tri;
  c->natural = true;
  return 0;
}

int build_pcg(Ctx* c, const si3d_grid* g) {
  const int lm = g->lm, lm1 = lm + 1;
  std::vector<int> col;
  colour_columns(lm, g->lEC, g->lWC, g->lNC, g->lSC, col);
  std::vector<int> idx(lm + 2, -1), lr, lb;
  for (int l = 1; l <= lm; ++l) {
    if (col[l - 1] == 1) { idx[l] = (int)lr.size(); lr.push_back(l); }
    else { idx[l] = (int)lb.size(); lb.push_back(l); }
  }
  const int nR = (int)lr.size(), nB = (int)lb.size();
  auto nbrs = [&](const std::vector<int>& L, int nother) {
    std::vector<int4> v(L.size());
    for (size_t i = 0; i < L.size(); ++i) {
      const int l = L[i];
      auto m = [&](int q) { return q == lm1 ? nother : idx[q]; };
      v[i] = make_int4(m(g->lWC[l - 1]), m(g->lSC[l - 1]), m(g->lNC[l - 1]), m(g->lEC[l - 1]));
    }
    return v;
  };
  std::vector<int4> nbR = nbrs(lr, nB), nbB = nbrs(lb, nR);
  // a neighbour must carry the other colour (5-point graphs are bipartite)
  for (int l = 1; l <= lm; ++l) {
    const int nb[4] = {g->lWC[l - 1], g->lSC[l - 1], g->lNC[l - 1], g->lEC[l - 1]};
    for (int m : nb) if (m != lm1 && col[m - 1] == col[l - 1]) return SI3D_EDIMS;
  }
  PcgDev& P = c->pcg;
  int rc = 0;
  for (int which = 0; which < 2 && !rc; ++which) {
    PcgColor& C = which ? P.B : P.R;
    const std::vector<int>& L = which ? lb : lr;
    const std::vector<int4>& NBv = which ? nbB : nbR;
    C.n = (int)L.size();
    int* dl = nullptr;
    int4* dn = nullptr;
    rc |= c->alloc(&dl, L.size());
    rc |= c->alloc(&dn, L.size());
    if (rc) break;
    if (!L.empty()) {
      CK(cudaMemcpy(dl, L.data(), L.size() * sizeof(int), cudaMemcpyHostToDevice));
      CK(cudaMemcpy(dn, NBv.data(), NBv.size() * sizeof(int4), cudaMemcpyHostToDevice));
    }
    C.l = dl;
    C.nbr = dn;
    const size_t n1 = L.size() + 1;
    for (double** p : {&C.sx, &C.sy, &C.rhs, &C.u, &C.r, &C.z, &C.p, &C.p2, &C.q, &C.dinv, &C.diag, &C.rs})
      rc |= c->alloc(p, n1);
  }
  if (rc) return rc;
  // SI3D_PCG_BLOCKS_PER_SM caps the resident blocks per SM of the cooperative solve (tuning)
  const char* bps = std::getenv("SI3D_PCG_BLOCKS_PER_SM");
  c->loop_blocks = pcg_loop_blocks(c->device, nR, nB, bps ? std::atoi(bps) : 0, false);
  c->loop_blocks_f = pcg_loop_blocks(c->device, nR, nB, bps ? std::atoi(bps) : 0, true);
  const char* pers = std::getenv("SI3D_PCG_PERSISTENT");
  c->persistent = !(pers && pers[0] == '0');
  const char* lg = std::getenv("SI3D_LOG_SOLVES");
  c->log_solves = lg && lg[0] == '1';
  const int nblk = std::max(pcg_max_blocks(nR, nB), 3 * std::max(c->loop_blocks, c->loop_blocks_f));
  double* parts = nullptr;
  rc |= c->alloc(&parts, 4 * (size_t)nblk);
  rc |= c->alloc(&c->bar, 1);
  if (rc) return rc;
  P.part0 = parts; P.part1 = parts + nblk; P.part2 = parts + 2 * nblk; P.part3 = parts + 3 * nblk;
  P.part_n = nblk;
  rc |= c->alloc(&P.sc, 1);
  const int cap = std::max(c->prm.pcg_itmax, 1) + 1;
  rc |= c->alloc(&P.hist_alpha, cap);
  rc |= c->alloc(&P.hist_beta, cap);
  rc |= c->alloc(&P.tri, 2 * (size_t)(cap + 1));
  if (rc) return rc;
  CK(cudaMallocHost(&c->h_sc, sizeof(PcgScal)));
  CK(cudaMallocHost(&c->h_hist, sizeof(double) * 2 * cap));
  // FP32 copy of the system for the inner solves of iterative refinement (shares the node lists,
  // neighbour indices and reduction buffers with the FP64 system)
  PcgDevF& F = c->pcgf;
  for (int which = 0; which < 2 && !rc; ++which) {
    PcgColorT<float>& G = which ? F.B : F.R;
    const PcgColor& C = which ? P.B : P.R;
    G.n = C.n; G.l = C.l; G.nbr = C.nbr;
    G.rhs = G.diag = G.rs = nullptr;
    for (float** q : {&G.sx, &G.sy, &G.u, &G.r, &G.z, &G.p, &G.p2, &G.q, &G.dinv}) rc |= c->alloc(q, (size_t)C.n + 1);
  }
  rc |= c->alloc(&F.sc, 1);
  if (rc) return rc;
  F.part0 = P.part0; F.part1 = P.part1; F.part2 = P.part2; F.part3 = P.part3; F.part_n = P.part_n;
  F.hist_alpha = P.hist_alpha; F.hist_beta = P.hist_beta; F.tri = nullptr;
  CK(cudaMallocHost(&c->h_scf, sizeof(PcgScal)));
  if (c->prm.precision == SI3D_MIXED_MG) return build_mg(c, g);
  if (c->prm.ordering == SI3D_ORDER_NATURAL) return build_natural(c, g);
  return 0;
}

// chgcon/eigvss/zbrent/determ (nspcg.f:16499-16620, :17201, :32976, :16926) evaluated after the
// solve from the recorded alpha/beta sequence: with stopping test 5 the estimates do not feed
// back into the iteration, so they are reported rather than computed on the critical path.
double determ(int n, const std::vector<double>& tri, double x) {
  auto T = [&](int r, int cc) { return tri[(size_t)(cc - 1) * 2 + (r - 1)]; };
  double d2 = T(1, n) - x;
  double d1 = d2 * (T(1, n - 1) - x) - T(2, n);
  for (int l = n - 1; l >= 2; --l) { const double d3 = d2; d2 = d1; d1 = (T(1, l - 1) - x) * d2 - d3 * T(2, l); }
  return d1;
}

void zbrent(int n, const std::vector<double>& tri, int nsig, double& aa, double& bb, int maxfn, int& ier) {
  double a = aa, b = bb, t = std::pow(0.1, nsig), fa = determ(n, tri, a), fb = determ(n, tri, b);
  double c = 0, fc = 0, d = 0, e = 0, s = b, p, q, r, rm, tol, temp;
  int ic = 2;
  if (fa * fb > 0.0) { ier = 4; return; }
  for (;;) {
    c = a; fc = fa; d = b - c; e = d;
    for (;;) {
      if (std::fabs(fc) < std::fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
      tol = t * std::max(std::fabs(b), 0.1);
      rm = (c - b) / 2.0;
      if (std::fabs(fb) <= 0.0 || std::fabs(c - b) <= tol) { aa = c; bb = b; return; }
      if (ic >= maxfn) { ier = 3; aa = c; bb = b; return; }
      bool bisect = std::fabs(e) < tol || std::fabs(fa) <= std::fabs(fb);
      if (!bisect) {
        s = fb / fa;
        if (a == c) { p = (c - b) * s; q = 1.0 - s; }
        else {
          q = fa / fc; r = fb / fc;
          const double rone = r - 1.0;
          p = s * ((c - b) * q * (q - r) - (b - a) * rone);
          q = (q - 1.0) * rone * (s - 1.0);
        }
        if (p > 0.0) q = -q;
        if (p < 0.0) p = -p;
        s = e; e = d;
        if (p + p >= 3.0 * rm * q || p + p >= std::fabs(s * q)) bisect = true;
        else d = p / q;
      }
      if (bisect) { e = rm; d = e; }
      a = b; fa = fb; temp = d;
      if (std::fabs(temp) <= tol / 2.0) temp = std::copysign(tol / 2.0, rm);
      b = b + temp; s = b; fb = determ(n, tri, s); ic = ic + 1;
      if (!(fb * fc <= 0.0)) break;
    }
  }
}

void eigen_estimates(const double* al, const double* be, int n, double zeta, int itmax, double& emin, double& emax) {
  emax = 2.0; emin = 1.0;
  bool maxadp = true, minadp = true;
  std::vector<double> tri((size_t)2 * (n + 2), 0.0);
  auto T = [&](int r, int cc) -> double& { return tri[(size_t)(cc - 1) * 2 + (r - 1)]; };
  double tl1 = 0, tl2 = 0, bl1 = 0, bl2 = 0, alphao = 0;
  int ier = 0;
  const int nsig = std::max((int)(-std::log10(std::fabs(zeta))), 4), maxfn = std::max(itmax, 50);
  for (int ip = 0; ip < n; ++ip) {
    const double alpha = al[ip], beta = be[ip];
    if (ip == 0) { T(1, 1) = 1.0 / alpha; T(2, 1) = 0.0; emax = emin = 1.0 / alpha; alphao = alpha; continue; }
    const double t1 = 1.0 / alpha + beta / alphao, t2 = beta / (alphao * alphao), tsqr = std::sqrt(t2);
    T(1, ip + 1) = t1; T(2, ip + 1) = t2;
    if (ip == 1) {
      tl1 = T(1, 1) + tsqr; tl2 = t1 + tsqr; bl1 = T(1, 1) - tsqr; bl2 = t1 - tsqr;
      const double t3 = T(1, 1) + t1, t4 = std::sqrt((t1 - T(1, 1)) * (t1 - T(1, 1)) + 4.0 * t2);
      if (maxadp) emax = (t3 + t4) / 2.0;
      if (minadp) emin = (t3 - t4) / 2.0;
      alphao = alpha;
      continue;
    }
    if (maxadp) {
      tl1 = std::max(tl1, tl2 + tsqr); tl2 = t1 + tsqr;
      double a = emax, b = std::max(tl1, tl2);
      const double emaxo = emax;
      zbrent(ip + 1, tri, nsig, a, b, maxfn, ier);
      if (ier != 3 && ier != 4) { emax = std::min(a, b); if (std::fabs(emax - emaxo) < emax * zeta) maxadp = false; }
      else maxadp = false;
    }
    if (minadp) {
      bl1 = std::min(bl1, bl2 - tsqr); bl2 = t1 - tsqr;
      double a = std::max(0.0, std::min(bl1, bl2)), b = emin;
      const double emino = emin;
      zbrent(ip + 1, tri, nsig, a, b, maxfn, ier);
      if (ier != 3 && ier != 4) { emin = std::max(a, b); if (std::fabs(emin - emino) < emin * zeta) minadp = false; }
      else minadp = false;
    }
    alphao = alpha;
    if (!maxadp && !minadp) break;
  }
}

// Runs CG iterations in batches until the device-side `done` flag is set.  Every kernel of an
// iteration returns at once after convergence, so a batch may overshoot without changing the
// result; the host reads the scalars back once per batch.
template <class F, class G>
int iterate(Ctx* c, PcgScal* dsc, PcgScal* hsc, int itmax, int predicted, F&& launch_one, G&& launch_loop) {
  if (c->persistent) {
    if (launch_loop() != 0) return cuda_fail(cudaGetLastError(), "pcg_loop", __LINE__);
    c->launches += 1;
    CK(cudaMemcpyAsync(hsc, dsc, sizeof(PcgScal), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return hsc->done ? 0 : SI3D_ETIMEOUT;
  }
  int batch = std::max(1, std::min(predicted - 1, 256));
  int launched = 0;
  for (;;) {
    for (int i = 0; i < batch; ++i) launch_one((launched + i) & 1);
    launched += batch;
    c->launches += 3LL * batch;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(hsc, dsc, sizeof(PcgScal), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    if (hsc->done) return 0;
    if (launched > itmax + 8) return SI3D_ETIMEOUT;  // cannot happen: itcg stops at itmax
    batch = 4;
  }
}

// Mixed precision: FP32 MIC-PCG corrections inside an FP64 iterative-refinement loop.  The
// residual r = b - A u, its norm, the stopping test (test 5 at the caller's tolerance) and the
// update u += e are FP64; each inner solve runs the red-black MIC-PCG on FP32 copies of the
// coefficients, pivots and residual (dot products still accumulate in FP64) until its own
// residual has dropped by max(1e-5, what the outer test still needs).  (Precision SI3D_MIXED_MG runs
// the same refinement around multigrid-preconditioned inner solves on the device: solve_mg.)
int refine(Ctx* c, int* total_inner) {
  const si3d_params& p = c->prm;
  const double zeta = std::max(p.pcg_tol, 500.0 * p.srelpr);
  PcgScal& H = *c->h_sc;
  int outer = 0, inner_total = 0;
  const int max_outer = 40;
  for (;;) {
    ir_residual(c->pcg, c->st);
    c->launches += 3;
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(c->h_sc, c->pcg.sc, sizeof(PcgScal), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    const double rn = std::sqrt(H.stptst), bn = H.bnorm;
    H.stptst = rn / bn;
    if (rn < bn * zeta) break;
    if (outer >= max_outer) { H.ier = 1; break; }
    ir_inner_setup(c->pcg, c->pcgf, c->st);
    c->launches += 2;
    PcgScal fi{};
    fi.zeta = std::max(1e-5, 0.5 * zeta * bn / rn);
    fi.srelpr = 2.220446049250313e-16;
    fi.itmax = p.pcg_itmax;
    fi.ntest = 5;
    fi.bnorm = rn;
    fi.emax = 2.0; fi.emin = 1.0; fi.udnm = 1.0;
    fi.hist_cap = 0;
    *c->h_scf = fi;
    CK(cudaMemcpyAsync(c->pcgf.sc, c->h_scf, sizeof(PcgScal), cudaMemcpyHostToDevice, c->st));
    int rci = iterate(c, c->pcgf.sc, c->h_scf, p.pcg_itmax, c->last_inner,
                      [&](int par) { pcg_iteration_f(c->pcgf, par, c->st); },
                      [&] { return pcg_loop_f(c->pcgf, c->bar, c->loop_blocks_f, c->st, take_bar_test(c)); });
    if (rci) return rci;
    if (c->h_scf->ier == SI3D_ETIMEOUT) return SI3D_ETIMEOUT;
    const int its = c->h_scf->in;
    if (c->log_solves) std::fprintf(stderr, "si3d: inner FP32 MIC solve %d: %d iterations\n", outer + 1, its);
    inner_total += its;
    c->last_inner = std::max(its, 1);
    ir_correct(c->pcg, c->pcgf, c->st);
    c->launches += 2;
    ++outer;
  }
  c->ir_outer += outer;
  *total_inner = inner_total;
  return 0;
}

// The zeta solve of precision SI3D_MIXED_MG: FP64 refinement around FP32 multigrid-preconditioned CG,
// all of it in one cooperative launch (k_mg.cu) on the grid image; the red-black system is not used.
// `hist` holds per column (index l - 1) the correction of this solve one step earlier.
int solve_mg(Ctx* c, const PcgScal& init, int x0, double* hist, int ier, int* iters, double* relres, int* ier_out) {
  PcgScal& H = *c->h_sc;
  H = PcgScal{};
  H.zeta = init.zeta;
  H.srelpr = init.srelpr;
  H.itmax = init.itmax;
  CK(cudaMemcpyAsync(c->mg.sc, c->h_sc, sizeof(PcgScal), cudaMemcpyHostToDevice, c->st));
  int rc = stage(c, ST_PCG_SETUP, c->mg.nlev, [&] { mg_setup(c->d, c->mg, x0, c->dz, hist, c->st); });
  if (rc) return rc;
  if (c->prof) CK(cudaEventRecord(c->pe0, c->st));
  if (mg_solve(c->mg, c->bar, c->mg_blocks, c->st, take_bar_test(c)) != 0) return cuda_fail(cudaGetLastError(), "mg_solve", __LINE__);
  c->launches += 1;
  CK(cudaMemcpyAsync(c->h_sc, c->mg.sc, sizeof(PcgScal), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (!H.done || H.ier == SI3D_ETIMEOUT) return SI3D_ETIMEOUT;
  if (c->prof) {
    CK(cudaEventRecord(c->pe1, c->st));
    CK(cudaEventSynchronize(c->pe1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->pe0, c->pe1);
    c->prof_ms[ST_PCG_ITER] += ms;
    c->prof_n[ST_PCG_ITER] += H.in;
  }
  c->ir_outer += H.q1;
  if (c->log_solves) std::fprintf(stderr, "si3d: MG solve: %d inner iterations in %d passes\n", H.in, H.q1);
  rc = stage(c, ST_PCG_FINISH, 1, [&] { mg_finish(c->d, c->mg, hist, c->st); });
  if (rc) return rc;
  if (c->rec_buf) {
    float* slot = c->rec_buf + (size_t)(c->rec_count % c->rec_slots) * c->im1 * c->jm1 * 5;
    learn::record(c->d, c->pix, c->feat, c->sigma, slot, c->st);
    CK(cudaGetLastError());
    c->rec_count++;
  }
  if (H.ier != 0) ier = H.ier;
  *iters = H.in;
  *relres = H.stptst;
  *ier_out = ier;
  return 0;
}

// One zeta solve on the device (SolverSparse's call of nspcg, si3d_procedures.f90:1986-2003).
// The zeta solve with the reference's own ordering: natural-order MIC-CG in one single-block launch.
int solve_natural(Ctx* c, int x0, int ier, int* iters, double* relres, int* ier_out) {
  int rc = stage(c, ST_PCG_SETUP, 1, [&] { nat_setup(c->d, c->nat, x0, c->dz, c->st); });
  if (rc) return rc;
  if (c->prof) CK(cudaEventRecord(c->pe0, c->st));
  if (nat_solve(c->nat, c->prm.pcg_test == 2, c->st) != 0) return cuda_fail(cudaGetLastError(), "nat_solve", __LINE__);
  c->launches += 1;
  CK(cudaMemcpyAsync(c->h_sc, c->nat.sc, sizeof(PcgScal), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const PcgScal& S = *c->h_sc;
  if (!S.done) return SI3D_ETIMEOUT;
  if (c->prof) {
    CK(cudaEventRecord(c->pe1, c->st));
    CK(cudaEventSynchronize(c->pe1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->pe0, c->pe1);
    c->prof_ms[ST_PCG_ITER] += ms;
    c->prof_n[ST_PCG_ITER] += S.in;
  }
  if (c->log_solves) std::fprintf(stderr, "si3d: natural-order solve: %d iterations\n", S.in);
  rc = stage(c, ST_PCG_FINISH, 1, [&] { nat_finish(c->d, c->nat, c->st); });
  if (rc) return rc;
  if (S.negpiv & 2) ier = -12;
  else if (S.ier != 0) ier = S.ier;
  else if ((S.negpiv & 1) && ier == 0) ier = 5;
  *iters = S.in;
  *relres = S.stptst;
  *ier_out = ier;
  return 0;
}

// After the cooperative loop of a graph-mode FP64 solve: zeta back to the columns, and the solve's
// statistics into its device slot.
int solve_graph_post(Ctx* c, double* hist, int ier) {
  const int rc = stage(c, ST_PCG_FINISH, 2, [&] { pcg_finish(c->d, c->pcg, hist, c->st); });
  if (rc) return rc;
  pcg_record_stats(c->pcg.sc, ier, c->d_stats_ii, c->d_stats_rr, std::min(c->solve_slot, 23), c->st);
  c->launches += 1;
  c->solve_slot++;
  return 0;
}

int solve(Ctx* c, int* iters, double* relres, int* ier_out) {
  const si3d_params& p = c->prm;
  PcgScal init{};
  init.zeta = p.pcg_tol;
  init.srelpr = p.srelpr;
  int ier = 0;
  if (init.zeta < 500.0 * init.srelpr) { ier = 2; init.zeta = 500.0 * init.srelpr; }  // echall clamp
  init.itmax = p.pcg_itmax;
  init.ntest = p.pcg_test;
  init.emax = 2.0; init.emin = 1.0; init.udnm = 1.0;
  init.maxadp = 1; init.minadp = 1;
  init.hist_cap = p.pcg_itmax + 1;
  if (c->graph_mode) {
    // the scalars are set by a kernel (a host copy would capture a host buffer that later solves reuse)
    if (p.precision != SI3D_FP64 || !c->persistent || c->rec_buf || c->natural) return SI3D_EDIMS;
    pcg_init_scalars(c->pcg.sc, init, c->st);
    c->launches += 1;
  } else {
    *c->h_sc = init;
    CK(cudaMemcpyAsync(c->pcg.sc, c->h_sc, sizeof(PcgScal), cudaMemcpyHostToDevice, c->st));
  }
  // The learned guess predicts the leapfrog solve (istep 1) of a step, the solve it was trained on
  // where sp is the current zeta; the trapezoidal solves that follow start from the latest solution.
  const bool learned_step = p.x0_mode == SI3D_X0_LEARNED && c->cur_istep == 1;
  const bool use_net = learned_step && c->net_loaded;
  if (use_net || c->rec_buf) {
    // features of this system; with the network loaded, the predicted increment into dz
    int rf = 0;
    int rcl = stage(c, ST_LEARN, use_net ? 9 : 3, [&] {
      learn::features(c->d, c->pix, c->r0, c->fpart, c->sigma, c->feat, c->st);
      if (use_net) {
        rf = learn::forward(c->net_ws, c->net_params, c->feat, 1, c->im1, c->jm1, c->net_out, c->st);
        if (!rf) learn::scatter(c->lm, c->pix, c->net_out, c->sigma, c->dz, c->st);
      }
    });
    if (!rcl) rcl = rf;
    if (rcl) return rcl;
    if (use_net) c->dz_set = true;
  }
  int x0 = p.x0_mode;
  if (p.x0_mode == SI3D_X0_LEARNED) {
    if (!learned_step && c->net_loaded) x0 = SI3D_X0_LAST;
    else if (!c->dz_set) x0 = SI3D_X0_PREV;
  }
  const bool use_hist = p.x0_mode == SI3D_X0_HIST;
  double* hist = use_hist ? c->hist + (size_t)c->hist_slot * (c->pcg.R.n + c->pcg.B.n + 2) : nullptr;
  if (p.precision == SI3D_MIXED_MG) return solve_mg(c, init, x0, hist, ier, iters, relres, ier_out);
  if (c->natural) return solve_natural(c, x0, ier, iters, relres, ier_out);
  int rc0 = stage(c, ST_PCG_SETUP, 7, [&] { pcg_setup(c->d, c->pcg, x0, c->dz, hist, &c->pcg.sc->negpiv, c->st); });
  if (rc0) return rc0;
  if (c->graph_mode) {
    *iters = 0;
    *relres = 0.0;
    *ier_out = 0;
    if (c->ens_defer) {   // the ensemble's batched launch runs the loop
      c->def_hist = hist;
      c->def_ier = ier;
      return 0;
    }
    if (pcg_loop(c->pcg, c->bar, c->loop_blocks, c->prm.pcg_test == 2, c->st) != 0) return cuda_fail(cudaGetLastError(), "pcg_loop", __LINE__);
    c->launches += 1;
    return solve_graph_post(c, hist, ier);
  }
  if (c->prof) CK(cudaEventRecord(c->pe0, c->st));
  int total_iters = 0;
  if (p.precision == SI3D_MIXED_IR) {
    int rcir = refine(c, &total_iters);
    if (rcir) return rcir;
  } else {
    // run iterations in batches; every kernel returns at once after convergence
    int rci = iterate(c, c->pcg.sc, c->h_sc, p.pcg_itmax, c->last_iters,
                      [&](int par) { pcg_iteration(c->pcg, par, c->st); },
                      [&] {
                        return pcg_loop(c->pcg, c->bar, c->loop_blocks, c->prm.pcg_test == 2, c->st, take_bar_test(c));
                      });
    if (rci) return rci;
    total_iters = c->h_sc->in;
    c->last_iters = std::max(total_iters, 1);
    if (c->log_solves) std::fprintf(stderr, "si3d: FP64 solve: %d iterations\n", total_iters);
  }
  if (c->prof) {
    CK(cudaEventRecord(c->pe1, c->st));
    CK(cudaEventSynchronize(c->pe1));
    float ms = 0;
    cudaEventElapsedTime(&ms, c->pe0, c->pe1);
    c->prof_ms[ST_PCG_ITER] += ms;
    c->prof_n[ST_PCG_ITER] += total_iters;
  }
  rc0 = stage(c, ST_PCG_FINISH, 2, [&] { pcg_finish(c->d, c->pcg, hist, c->st); });
  if (rc0) return rc0;
  if (c->rec_buf) {
    float* slot = c->rec_buf + (size_t)(c->rec_count % c->rec_slots) * c->im1 * c->jm1 * 5;
    learn::record(c->d, c->pix, c->feat, c->sigma, slot, c->st);
    CK(cudaGetLastError());
    c->rec_count++;
  }
  const PcgScal& S = *c->h_sc;
  if (S.negpiv & 2) ier = -12;
  else if (S.ier != 0) ier = S.ier;
  else if ((S.negpiv & 1) && ier == 0) ier = 5;
  *iters = total_iters;
  *relres = S.stptst;
  *ier_out = ier;
  return 0;
}

// Parabolic interpolation in a boundary series of spacing dx hours from time 0 (the reference's
// parab, si3d_utils.f90:895-920); NaN past the series' end.
double series_at(const std::vector<double>& fx, double x, double dx) {
  int m = (int)(x / dx);
  const double om = m;
  double theta = (x - om * dx) / dx;
  if (m == 0) { m = 2; theta = theta - 1.0; }
  else m = m + 1;
  if (m + 1 > (int)fx.size() || m < 2) return std::nan("");
  auto f = [&](int i) { return fx[(size_t)(i - 1)]; };
  return f(m) + 0.5 * theta * (f(m + 1) - f(m - 1) + theta * (f(m + 1) + f(m - 1) - 2.0 * f(m)));
}

// openbcUVH CASE(1): zeta of the boundary cells at the current time.
int obc_uvh(Ctx* c) {
  for (size_t b = 0; b < c->obc.size(); ++b) {
    const double v = series_at(c->obc_wse[b], c->thrs, c->obc_dtsec / 3600.);
    if (std::isnan(v)) return SI3D_EDIMS;   // the series ends before the run does
    obc_set_s(c->d, c->obc[b], v, c->st);
  }
  return 0;
}

// Stages with the open-boundary adjustments that follow their kernels.
void momentum_stage(Ctx* c, int ieq) {
  if (ieq == 1) launch_momentum(c->d, 1, c->mce, c->nce, c->tune, c->st, c->obc.data(), (int)c->obc.size());
  else launch_momentum(c->d, 2, c->mcn, c->ncn, c->tune, c->st, c->obc.data(), (int)c->obc.size());
}
void matcon_stage(Ctx* c) {
  launch_matcon(c->d, c->st);
  for (const ObcDev& b : c->obc) obc_qq(c->d, b, c->st);   // MODqqddrr4openBC (:1859)
}
void obc_continuity(Ctx* c) {
  for (const ObcDev& b : c->obc) obc_vel(c->d, b, c->st);   // MODvel4openBC (:2821)
}
void vel_stage(Ctx* c) {
  launch_vel(c->d, c->ce, c->nce, c->cn, c->ncn, c->st);
  obc_continuity(c);
}
int scalar_stage(Ctx* c) {
  launch_exsal_imsal(c->d, c->tune, c->st);
  for (size_t b = 0; b < c->obc.size(); ++b) {   // openbcSCA (:515)
    const double v = series_at(c->obc_tmp[b], c->thrs, c->obc_dtsec / 3600.);
    if (std::isnan(v)) return SI3D_EDIMS;
    obc_sca(c->d, c->obc[b], v, c->st);
  }
  return 0;
}
int obc_launches(const Ctx* c) { return (int)c->obc.size(); }

// One fd call is fd_pre, the zeta solve and fd_post (the batched ensemble capture runs the three
// parts of all its members in lock step).
// fd up to the zeta solve: time-level factor, openbcUVH, momentum, matcon.
int fd_pre(Ctx* c, int istep) {
  Dev& d = c->d;
  d.tz = 1.0 / istep;
  c->cur_istep = istep;
  if (istep == 1) c->trap_solves = 0;
  c->hist_slot = istep == 1 ? 0 : std::min(++c->trap_solves, kHistSlots - 1);
  // openbcUVH (:423)
  int rc = obc_uvh(c);
  if (rc) return rc;
  c->launches += obc_launches(c);
  // surfbc CASE(0) is a constant per-column wind set by the host (uair/vair/cdw fields)
  rc = stage(c, ST_MOMX, 2 + obc_launches(c), [&] { momentum_stage(c, 1); });
  if (!rc) rc = stage(c, ST_MOMY, 2 + obc_launches(c), [&] { momentum_stage(c, 2); });
  if (!rc) rc = stage(c, ST_MATCON, 1 + 2 * obc_launches(c), [&] { matcon_stage(c); });
  return rc;
}

// fd after the zeta solve: surface layer, openbcUVH, velocities, scalar, tracers, wetting, mixing.
int fd_post(Ctx* c, bool lastiter) {
  Dev& d = c->d;
  int rc = stage(c, ST_SLAYER, 1, [&] { launch_slayer_h(d, c->st); });
  if (!rc) rc = obc_uvh(c);   // openbcUVH after the solve (:482)
  if (!rc) c->launches += obc_launches(c);
  if (!rc) rc = stage(c, ST_VEL, 3 + obc_launches(c), [&] { vel_stage(c); });
  if (!rc && c->prm.isal != 0) {
    int rs = 0;
    rc = stage(c, ST_SCALAR, 3 + obc_launches(c), [&] { rs = scalar_stage(c); });
    if (!rc) rc = rs;
  }
  if (!rc && c->prm.ntr > 0 && c->prm.niter > 0 && lastiter)
    rc = stage(c, ST_TRACER, 2 * ((c->prm.ntr + kTracerFluxGroup - 1) / kTracerFluxGroup) + 1, [&] { tracer_stage(c); });
  if (!rc) rc = stage(c, ST_VEL2, 1, [&] { launch_vel2(d, c->st); });
  // UpdateMixingCoefficients (si3d_procedures.f90:571)
  if (!rc && c->prm.iturb == 1) rc = stage(c, ST_TURB, 2, [&] { launch_turbulence(d, c->turb_scr, c->st); });
  return rc;
}

int fd_impl(Ctx* c, int istep, bool lastiter, si3d_step_stats* st) {
  int rc = fd_pre(c, istep);
  if (rc) return rc;
  if (st) CK(cudaEventRecord(c->evp0, c->st));
  int iters = 0, ier = 0;
  double rr = 0;
  rc = solve(c, &iters, &rr, &ier);
  if (rc) return rc;
  if (st) CK(cudaEventRecord(c->evp1, c->st));
  if (st) {
    if (st->nsolves < 24) {
      st->iters[st->nsolves] = iters; st->relres[st->nsolves] = rr; st->ier[st->nsolves] = ier;
    }
    st->nsolves++;
    st->total_iters += iters;
  }
  if (ier < 0) return ier;
  rc = fd_post(c, lastiter);
  if (rc) return rc;
  if (st) {
    CK(cudaEventSynchronize(c->evp1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->evp0, c->evp1));
    st->ms_pcg += ms;
  }
  return 0;
}

}  // namespace

extern "C" {

const char* si3d_gpu_strerror(int code) {
  switch (code) {
    case SI3D_OK: return "ok";
    case 1: return "zeta solve: itmax reached";
    case 2: return "zeta solve: tolerance clamped to 500*srelpr";
    case 3: return "zeta solve: eigenvalue estimate did not converge";
    case 4: return "zeta solve: eigenvalue bracket failed";
    case 5: return "zeta solve: negative pivot in the MIC factorisation";
    case -6: return "zeta solve: (p, Ap) <= 0";
    case -7: return "zeta solve: (r, z) <= 0";
    case -12: return "zeta solve: zero pivot in the MIC factorisation";
    case SI3D_ECUDA: return g_last_cuda.empty() ? "CUDA error" : g_last_cuda.c_str();
    case SI3D_EDIMS: return "bad dimensions or arguments";
    case SI3D_EHANDLE: return "unknown handle";
    case SI3D_ENAME: return "unknown field name";
    case SI3D_ENAN: return "non-finite value";
    case SI3D_ETIMEOUT: return "bounded device wait gave up";
    case SI3D_ENOMEM: return "device allocation failed";
    case SI3D_ENODEV: return "no sm_100 CUDA device";
    case SI3D_ECAPACITY: return "problem exceeds the fixed scratch of the allocation-free entry point";
    default: return "unknown error";
  }
}

int si3d_gpu_init(const si3d_grid* g, const si3d_params* prm, int device, int* handle) {
  if (!g || !prm || !handle) return SI3D_EDIMS;
  if (g->lm < 1 || g->km1 < 3 || g->km1 > SI3D_MAXK || g->k1 != 2) return SI3D_EDIMS;
  if (prm->itrmom != 1 || prm->ihd > 1 || prm->pcg_itmax < 1 || (prm->pcg_test != 5 && prm->pcg_test != 2))
    return SI3D_EDIMS;
  if (prm->x0_mode < SI3D_X0_PREV || prm->x0_mode > SI3D_X0_HIST) return SI3D_EDIMS;
  // 0 is taken as the default red-black ordering; the natural ordering is the plain FP64 solve only
  if (prm->ordering != 0 && prm->ordering != SI3D_ORDER_REDBLACK && prm->ordering != SI3D_ORDER_NATURAL)
    return SI3D_EDIMS;
  if (prm->ordering == SI3D_ORDER_NATURAL && (prm->precision != SI3D_FP64 || prm->x0_mode == SI3D_X0_HIST))
    return SI3D_EDIMS;
  if (prm->ntr < 0 || prm->ntr > 30) return SI3D_EDIMS;   // ntrmax (si3d_types.f90:291)
  if (prm->iturb != 0 && prm->iturb != 1) return SI3D_EDIMS;
  // every kernel indexes neighbours through the maps and layers down to kmz + 1: both are checked
  // here once, so no device access can leave its field
  for (int l = 0; l < g->lm; ++l) {
    if (g->kmz[l] < g->k1 || g->kmz[l] > g->km1 - 1) return SI3D_EDIMS;
    for (const int* m : {g->lEC, g->lWC, g->lNC, g->lSC})
      if (m[l] < 1 || m[l] > g->lm + 1) return SI3D_EDIMS;
  }
  if (prm->precision != SI3D_FP64 && prm->precision != SI3D_MIXED_IR && prm->precision != SI3D_MIXED_MG)
    return SI3D_EDIMS;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device) return SI3D_ENODEV;
  cudaDeviceProp pr;
  CK(cudaGetDeviceProperties(&pr, device));
  if (pr.major < 10) return SI3D_ENODEV;
  CK(cudaSetDevice(device));
  Ctx* c = new Ctx();
  c->device = device;
  c->prm = *prm;
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) { delete c; return SI3D_ECUDA; }
  for (cudaEvent_t* e : {&c->ev0, &c->ev1, &c->evp0, &c->evp1, &c->pe0, &c->pe1}) cudaEventCreate(e);
  const int lm = g->lm, lm1 = lm + 1, km1 = g->km1;
  const int P = (lm1 + 31) / 32 * 32;
  if ((long long)km1 * P >= (1LL << 31)) { delete c; return SI3D_EDIMS; }   // 32-bit device indexing
  c->lm = lm; c->lm1 = lm1; c->km1 = km1; c->P = P;
  Dev& d = c->d;
  d.g.lm = lm; d.g.lm1 = lm1; d.g.km1 = km1; d.g.km = km1 - 1; d.g.k1 = g->k1; d.g.P = P;
  int rc = 0;
  // maps, padded to P; the sentinel column lm1 points to itself
  auto up_int = [&](const int* src, int nsrc, int fill) -> const int* {
    std::vector<int> v(P, fill);
    for (int i = 0; i < nsrc; ++i) v[i] = src[i];
    int* p = nullptr;
    rc |= c->alloc(&p, P);
    if (!rc) cudaMemcpy(p, v.data(), P * sizeof(int), cudaMemcpyHostToDevice);
    return p;
  };
  auto up_dbl = [&](const double* src, int nsrc) -> const double* {
    std::vector<double> v(P, 0.0);
    for (int i = 0; i < nsrc; ++i) v[i] = src[i];
    double* p = nullptr;
    rc |= c->alloc(&p, P);
    if (!rc) cudaMemcpy(p, v.data(), P * sizeof(double), cudaMemcpyHostToDevice);
    return p;
  };
  c->h_l2i.assign(g->l2i, g->l2i + lm); c->h_l2j.assign(g->l2j, g->l2j + lm);
  c->h_lEC.assign(g->lEC, g->lEC + lm); c->h_lWC.assign(g->lWC, g->lWC + lm);
  c->h_lNC.assign(g->lNC, g->lNC + lm); c->h_lSC.assign(g->lSC, g->lSC + lm);
  d.g.lEC = up_int(g->lEC, lm, lm1);
  d.g.lWC = up_int(g->lWC, lm, lm1);
  d.g.lNC = up_int(g->lNC, lm, lm1);
  d.g.lSC = up_int(g->lSC, lm, lm1);
  d.g.kmz = up_int(g->kmz, lm1, km1);
  d.g.hhs = up_dbl(g->hhs, lm1);
  d.g.hhu = up_dbl(g->hhu, lm1);
  d.g.hhv = up_dbl(g->hhv, lm1);
  {
    double* z = nullptr;
    rc |= c->alloc(&z, km1);
    if (!rc) cudaMemcpy(z, g->zlevel, km1 * sizeof(double), cudaMemcpyHostToDevice);
    d.g.zlevel = z;
  }
  // parameters (si3d_utils.f90:291-306)
  Params& p = d.p;
  p.dt = prm->dt; p.dx = prm->dx; p.dy = prm->dy; p.twodt = 2. * p.dt; p.dtdx = p.dt / p.dx; p.dtdy = p.dt / p.dy;
  p.gdtdx = G_GRAV * p.dtdx; p.gdtdy = G_GRAV * p.dtdy; p.gdt2dx2 = p.gdtdx * p.dtdx; p.gdt2dy2 = p.gdtdy * p.dtdy;
  p.twodx = 2. * p.dx; p.twody = 2. * p.dy; p.fourdx = 2. * p.twodx; p.fourdy = 2. * p.twody;
  p.dxdx = p.dx * p.dx; p.dydy = p.dy * p.dy;
  p.rfourdx = 1.0 / p.fourdx; p.rfourdy = 1.0 / p.fourdy; p.rdxdx = 1.0 / p.dxdx; p.rdydy = 1.0 / p.dydy;
  p.rdx = 1.0 / p.dx; p.rdy = 1.0 / p.dy;
  p.Av0 = prm->Av0; p.Dv0 = prm->Dv0; p.Ax0 = prm->Ax0; p.Ay0 = prm->Ay0; p.f = prm->f; p.theta = prm->theta;
  p.cd = prm->cd; p.cw = prm->cw;
  p.iadv = prm->iadv; p.itrmom = prm->itrmom; p.ihd = prm->ihd; p.ibc = prm->ibc; p.isal = prm->isal;
  // state
  const size_t n3 = (size_t)km1 * P;
  Fields3& f = d.f;
  for (double** q : {&f.uh, &f.uhp, &f.uhpp, &f.up, &f.upp, &f.hu, &f.hup, &f.hupp, &f.agx, &f.arx, &f.vh, &f.vhp,
                     &f.vhpp, &f.vp, &f.vpp, &f.hv, &f.hvp, &f.hvpp, &f.agy, &f.ary, &f.h, &f.hp, &f.hpp, &f.sal,
                     &f.salp, &f.salpp, &f.rhop, &f.Av, &f.Dv, &f.wp, &f.HeatSource, &f.Bth2, &f.Bth3, &f.Bth4})
    rc |= c->alloc(q, n3);
  Fields2& s = d.s;
  for (double** q : {&s.s, &s.sp, &s.spp, &s.eagx, &s.earx, &s.eagy, &s.eary, &s.sx, &s.sy, &s.dd, &s.qq, &s.rr,
                     &s.uair, &s.vair, &s.cdw})
    rc |= c->alloc(q, P);
  for (int** q : {&s.k1z, &s.k1u, &s.k1v}) rc |= c->alloc(q, P);
  rc |= c->alloc(&d.scr, n3);
  if (prm->iturb == 1) {
    for (double** q : {&f.q2, &f.q2p, &f.q2pp, &f.q2l, &f.q2lp, &f.q2lpp, &f.u, &f.v}) rc |= c->alloc(q, n3);
    rc |= c->alloc(&c->turb_scr, 4 * n3);
  }
  {   // output frames: coordinates and point offsets (k1 .. kmz + 1 per wet column)
    std::vector<int> off(lm + 1, 0);
    c->h_kmz.assign(g->kmz, g->kmz + lm);
    for (int l = 0; l < lm; ++l) off[l + 1] = off[l] + (g->kmz[l] + 2 - g->k1);
    c->npoints = off[lm];
    rc |= c->alloc(&c->poff, lm + 1);
    rc |= c->alloc(&c->d_l2i, lm);
    rc |= c->alloc(&c->d_l2j, lm);
    if (!rc) {
      cudaMemcpy(c->poff, off.data(), sizeof(int) * (lm + 1), cudaMemcpyHostToDevice);
      cudaMemcpy(c->d_l2i, g->l2i, sizeof(int) * lm, cudaMemcpyHostToDevice);
      cudaMemcpy(c->d_l2j, g->l2j, sizeof(int) * lm, cudaMemcpyHostToDevice);
    }
  }
  if (prm->ntr > 0) {
    c->tr_stride = (long long)n3;
    rc |= c->alloc(&c->tr_buf[0], n3 * prm->ntr);
    rc |= c->alloc(&c->tr_buf[1], n3 * prm->ntr);
    rc |= c->alloc(&c->tr_scr, n3 * ((prm->ntr + kTracerGroup - 1) / kTracerGroup));
    rc |= c->alloc(&c->tr_fx, n3 * 3 * std::min(std::max(prm->ntr - 1, 1), kTracerFluxGroup));
  }
  rc |= c->alloc(&c->staging, (size_t)km1 * lm1);
  rc |= c->alloc(&c->dz, P);
  rc |= c->alloc(&c->d_stats_ii, 48);
  rc |= c->alloc(&c->d_stats_rr, 24);
  if (!rc && momentum_init(km1) != 0) { g_last_cuda = "momentum kernel shared-memory attribute"; rc = SI3D_ECUDA; }
  if (!rc && transport_init(km1) != 0) { g_last_cuda = "continuity kernel shared-memory attribute"; rc = SI3D_ECUDA; }
  // pixel (i - 1) * jm1 + (j - 1) of every wet column in the (im1, jm1) image of the learned
  // initial guess (only when the maps describe a real grid)
  c->im1 = std::max(g->im1, 1);
  c->jm1 = std::max(g->jm1, 1);
  if (!rc && g->l2i && g->l2j) {
    std::vector<int> px(lm);
    bool ok = true;
    for (int l = 0; l < lm; ++l) {
      const int i = g->l2i[l] - 1, j = g->l2j[l] - 1;
      if (i < 0 || i >= c->im1 || j < 0 || j >= c->jm1) ok = false;
      px[l] = i * c->jm1 + j;
    }
    if (ok) {
      rc |= c->alloc(&c->pix, lm);
      if (!rc) cudaMemcpy(c->pix, px.data(), sizeof(int) * lm, cudaMemcpyHostToDevice);
    }
  }
  if (rc) { delete c; return rc; }
  // face-column lists
  std::vector<int> ce, cn;
  for (int l = 1; l <= lm; ++l) {
    if (g->lEC[l - 1] != lm1) ce.push_back(l);
    if (g->lNC[l - 1] != lm1) cn.push_back(l);
  }
  c->nce = (int)ce.size(); c->ncn = (int)cn.size();
  rc |= c->alloc(&c->ce, ce.size());
  rc |= c->alloc(&c->cn, cn.size());
  if (rc) { delete c; return rc; }
  if (!ce.empty()) cudaMemcpy(c->ce, ce.data(), ce.size() * sizeof(int), cudaMemcpyHostToDevice);
  if (!cn.empty()) cudaMemcpy(c->cn, cn.data(), cn.size() * sizeof(int), cudaMemcpyHostToDevice);
  {
    // static per-face indices of the momentum stage (exmom/matmom neighbours and layer bounds)
    auto kz = [&](int q) { return g->kmz[q - 1]; };
    auto nbE = [&](int q) { return q == lm1 ? lm1 : g->lEC[q - 1]; };
    auto nbW = [&](int q) { return q == lm1 ? lm1 : g->lWC[q - 1]; };
    auto nbN = [&](int q) { return q == lm1 ? lm1 : g->lNC[q - 1]; };
    auto nbS = [&](int q) { return q == lm1 ? lm1 : g->lSC[q - 1]; };
    auto meta_of = [&](int l, bool X) {
      const int lE = nbE(l), lW = nbW(l), lN = nbN(l), lS = nbS(l);
      const int lO = X ? lE : lN;
      const int lX2 = X ? nbS(lE) : nbW(lN);
      const int kmx = std::min(kz(lO), kz(l));
      int mW_last = -1, mS_last = -1;
      if (X) {
        if (lW != lm1) mW_last = std::min(kz(l), kz(lW));
        if (lS != lm1 && nbE(lS) != lm1) mS_last = std::min(kz(nbE(lS)), kz(lS));
      } else {
        if (lS != lm1) mS_last = std::min(kz(l), kz(lS));
        if (lW != lm1 && nbN(lW) != lm1) mW_last = std::min(kz(nbN(lW)), kz(lW));
      }
      FaceMeta m;
      m.a = make_int4(l, lE, lW, lN);
      m.b = make_int4(lS, lX2, kmx, mW_last);
      m.c = make_int4(mS_last, 0, 0, 0);
      return m;
    };
    std::vector<FaceMeta> me, mn;
    for (int l : ce) me.push_back(meta_of(l, true));
    for (int l : cn) mn.push_back(meta_of(l, false));
    rc |= c->alloc(&c->mce, me.size());
    rc |= c->alloc(&c->mcn, mn.size());
    if (rc) { delete c; return rc; }
    if (!me.empty()) cudaMemcpy(c->mce, me.data(), me.size() * sizeof(FaceMeta), cudaMemcpyHostToDevice);
    if (!mn.empty()) cudaMemcpy(c->mcn, mn.data(), mn.size() * sizeof(FaceMeta), cudaMemcpyHostToDevice);
  }
  rc = build_pcg(c, g);
  if (!rc) rc = c->alloc(&c->hist, (size_t)kHistSlots * (c->pcg.R.n + c->pcg.B.n + 2));
  if (rc) { delete c; return rc; }
  if (cudaDeviceSynchronize() != cudaSuccess) { delete c; return SI3D_ECUDA; }
  std::lock_guard<std::mutex> lk(g_mu);
  g_ctx.push_back(c);
  *handle = (int)g_ctx.size() - 1;
  return 0;
}

void si3d_gpu_finalize(int h) {
  Ctx* c = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (h < 0 || h >= (int)g_ctx.size()) return;
    c = g_ctx[h];
    g_ctx[h] = nullptr;
  }
  if (c) { cudaSetDevice(c->device); delete c; }
}

int si3d_gpu_set_field(int h, const char* name, const double* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!name || !host) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  bool pp = false;
  const int nt = tracer_name(c, name, &pp);
  if (nt < 0) return SI3D_ENAME;
  double* dst = nullptr;
  if (nt > 0) {
    if (int rc = tracer_materialise(c)) return rc;
    c->tr_synced = false;
    dst = tracer_pool(c, pp) + (nt - 1) * c->tr_stride;
  } else {
    dst = f3ptr(c, name);
  }
  if (dst) {
    CK(cudaMemcpyAsync(c->staging, host, sizeof(double) * c->km1 * c->lm1, cudaMemcpyHostToDevice, c->st));
    dim3 b(32, 8), gr((c->lm1 + 31) / 32, (c->km1 + 31) / 32);
    k_colmajor_to_layer<<<gr, b, 0, c->st>>>(c->staging, dst, c->km1, c->lm1, c->P);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(c->st));
    return 0;
  }
  if (double* dst = f2ptr(c, name)) {
    CK(cudaMemcpyAsync(dst, host, sizeof(double) * c->lm1, cudaMemcpyHostToDevice, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
  }
  return SI3D_ENAME;
}

int si3d_gpu_get_field(int h, const char* name, double* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!name || !host) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  bool pp = false;
  const int nt = tracer_name(c, name, &pp);
  if (nt < 0) return SI3D_ENAME;
  const double* src = nt > 0 ? tracer_pool(c, pp || c->tr_alias) + (nt - 1) * c->tr_stride : f3ptr(c, name);
  if (src) {
    dim3 b(32, 8), gr((c->lm1 + 31) / 32, (c->km1 + 31) / 32);
    k_layer_to_colmajor<<<gr, b, 0, c->st>>>(src, c->staging, c->km1, c->lm1, c->P);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(host, c->staging, sizeof(double) * c->km1 * c->lm1, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
  }
  if (double* src = f2ptr(c, name)) {
    CK(cudaMemcpyAsync(host, src, sizeof(double) * c->lm1, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return 0;
  }
  return SI3D_ENAME;
}

// Single-precision copies: the reference as shipped keeps its module arrays in default REAL (4 bytes,
// si3d_types.f90:26).  The values cross the bus as floats and are widened (or rounded to nearest)
// on the device.
namespace {
__global__ void k_f32_to_f64(const float* __restrict__ s, double* __restrict__ d, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = (double)s[i];
}
__global__ void k_f64_to_f32(const double* __restrict__ s, float* __restrict__ d, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) d[i] = (float)s[i];
}
int staging_f(Ctx* c) {
  if (!c->staging_f) return c->alloc(&c->staging_f, (size_t)c->km1 * c->lm1);
  return 0;
}
}  // namespace

int si3d_gpu_set_field_f32(int h, const char* name, const float* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!name || !host) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  bool pp = false;
  const int nt = tracer_name(c, name, &pp);
  if (nt < 0) return SI3D_ENAME;
  const bool is3 = nt > 0 || f3ptr(c, name);
  if (!is3 && !f2ptr(c, name)) return SI3D_ENAME;
  if (int rc = staging_f(c)) return rc;
  const long long n = is3 ? (long long)c->km1 * c->lm1 : c->lm1;
  CK(cudaMemcpyAsync(c->staging_f, host, sizeof(float) * n, cudaMemcpyHostToDevice, c->st));
  if (is3) {
    double* dst = nullptr;
    if (nt > 0) {
      if (int rc = tracer_materialise(c)) return rc;
      c->tr_synced = false;
      dst = tracer_pool(c, pp) + (nt - 1) * c->tr_stride;
    } else {
      dst = f3ptr(c, name);
    }
    k_f32_to_f64<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>(c->staging_f, c->staging, n);
    dim3 b(32, 8), gr((c->lm1 + 31) / 32, (c->km1 + 31) / 32);
    k_colmajor_to_layer<<<gr, b, 0, c->st>>>(c->staging, dst, c->km1, c->lm1, c->P);
  } else {
    k_f32_to_f64<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>(c->staging_f, f2ptr(c, name), n);
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_get_field_f32(int h, const char* name, float* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!name || !host) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  bool pp = false;
  const int nt = tracer_name(c, name, &pp);
  if (nt < 0) return SI3D_ENAME;
  const double* src3 = nt > 0 ? tracer_pool(c, pp || c->tr_alias) + (nt - 1) * c->tr_stride : f3ptr(c, name);
  const double* src2 = src3 ? nullptr : f2ptr(c, name);
  if (!src3 && !src2) return SI3D_ENAME;
  if (int rc = staging_f(c)) return rc;
  const long long n = src3 ? (long long)c->km1 * c->lm1 : c->lm1;
  if (src3) {
    dim3 b(32, 8), gr((c->lm1 + 31) / 32, (c->km1 + 31) / 32);
    k_layer_to_colmajor<<<gr, b, 0, c->st>>>(src3, c->staging, c->km1, c->lm1, c->P);
    k_f64_to_f32<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>(c->staging, c->staging_f, n);
  } else {
    k_f64_to_f32<<<(unsigned)((n + 255) / 256), 256, 0, c->st>>>(src2, c->staging_f, n);
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(host, c->staging_f, sizeof(float) * n, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_set_ifield(int h, const char* name, const int* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  int* dst = name ? iptr(c, name) : nullptr;
  if (!dst) return SI3D_ENAME;
  if (!host) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(dst, host, sizeof(int) * c->lm1, cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_get_ifield(int h, const char* name, int* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  int* src = name ? iptr(c, name) : nullptr;
  if (!src) return SI3D_ENAME;
  if (!host) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  CK(cudaMemcpyAsync(host, src, sizeof(int) * c->lm1, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_set_warmstart(int h, const double* dz, int on_device) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  CK(cudaSetDevice(c->device));
  if (!dz) { c->dz_set = false; return 0; }
  CK(cudaMemcpyAsync(c->dz, dz, sizeof(double) * c->lm1, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                     c->st));
  CK(cudaStreamSynchronize(c->st));
  c->dz_set = true;
  return 0;
}

// Buffers of the learned initial guess that both inference and recording use.
static int ensure_learn(Ctx* c) {
  if (c->feat) return 0;
  if (!c->pix) return SI3D_EDIMS;
  const size_t npx = (size_t)c->im1 * c->jm1;
  int rc = c->alloc(&c->feat, npx * 4);
  rc |= c->alloc(&c->net_out, npx);
  rc |= c->alloc(&c->r0, c->lm);
  rc |= c->alloc(&c->fpart, learn::feature_partials(c->lm));
  rc |= c->alloc(&c->sigma, 1);
  return rc;
}

int si3d_learn_set_params(int h, const float* params) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  CK(cudaSetDevice(c->device));
  if (!params) { c->net_loaded = false; c->dz_set = false; return 0; }
  int rc = ensure_learn(c);
  if (rc) return rc;
  if (!c->net_params) {
    const size_t wsb = learn::Workspace::bytes(1, c->im1, c->jm1, false);
    char* mem = nullptr;
    rc |= c->alloc(&c->net_params, SI3D_NET_NPARAM);
    rc |= c->alloc(&mem, wsb);
    if (rc) return rc;
    c->net_mem = mem;
    if (!c->net_ws.carve(mem, wsb, 1, c->im1, c->jm1, false)) return SI3D_EDIMS;
  }
  CK(cudaMemcpyAsync(c->net_params, params, sizeof(float) * SI3D_NET_NPARAM, cudaMemcpyHostToDevice, c->st));
  learn::prepare(c->net_ws, c->net_params, c->st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  c->net_loaded = true;
  return 0;
}

int si3d_learn_record(int h, float* dev_buf, int nslots, int* hh, int* ww) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (dev_buf && nslots < 1) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  const int rc = ensure_learn(c);
  if (rc) return rc;
  c->rec_buf = dev_buf;
  c->rec_slots = dev_buf ? nslots : 0;
  c->rec_count = 0;
  if (hh) *hh = c->im1;
  if (ww) *ww = c->jm1;
  return 0;
}

int si3d_learn_recorded(int h) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  return c->rec_count;
}

int si3d_gpu_fd(int h, int n, int istep, int lastiter, si3d_step_stats* st) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  c->thrs = (double)n * c->prm.dt / 3600.;   // its = n idt, thrs = its / 3600. (si3d.f90:326-327)
  if (istep != 1 && istep != 2) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  if (st) { std::memset(st, 0, sizeof(*st)); CK(cudaEventRecord(c->ev0, c->st)); }
  int rc = fd_impl(c, istep, lastiter != 0, st);
  if (rc) return rc;
  if (st) {
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    st->ms_total = ms;
  }
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_density(int h) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  CK(cudaSetDevice(c->device));
  launch_density_init(c->d, c->st);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_stage(int h, const char* stage, int istep, si3d_step_stats* st) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!stage || (istep != 1 && istep != 2)) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  if (st) std::memset(st, 0, sizeof(*st));
  const std::string s = stage;
  Dev& d = c->d;
  d.tz = 1.0 / istep;
  if (s == "momentum") { momentum_stage(c, 1); momentum_stage(c, 2); }
  else if (s == "matcon") matcon_stage(c);
  else if (s == "solve") {
    int it = 0, ier = 0;
    double rr = 0;
    const int rc = solve(c, &it, &rr, &ier);
    if (rc) return rc;
    if (st) { st->nsolves = 1; st->iters[0] = it; st->relres[0] = rr; st->ier[0] = ier; st->total_iters = it; }
    if (ier < 0) return ier;
    launch_slayer_h(d, c->st);
  } else if (s == "vel") vel_stage(c);
  else if (s == "scalar") { if (int rc = scalar_stage(c)) return rc; }
  else if (s == "tracer") { if (c->prm.ntr > 0) tracer_stage(c); }
  else if (s == "turbulence") { if (c->prm.iturb == 1) launch_turbulence(d, c->turb_scr, c->st); }
  else if (s == "vel2") launch_vel2(d, c->st);
  else if (s == "settrap") settrap_all(c);
  else if (s == "settrap2") settrap2_all(c);
  else if (s == "save") { if (int rc = save_all(c, istep)) return rc; }
  else return SI3D_ENAME;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_settrap(int h) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  CK(cudaSetDevice(c->device));
  settrap_all(c);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_settrap2(int h) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  CK(cudaSetDevice(c->device));
  settrap2_all(c);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_save(int h, int istep) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (istep != 1 && istep != 2) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  if (int rc = save_all(c, istep)) return rc;
  c->trap_solves = 0;
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// Loop body of si3d.f90:324-458 for step n (outputs omitted).
// The stage sequence of one time step n (si3d.f90:324-458): leapfrog fd, settrap, niter
// trapezoidal fd/settrap2 iterations, save.  Enqueues only; the caller synchronises.
static int step_impl(Ctx* c, int n, si3d_step_stats* st) {
  c->trap_solves = 0;
  c->thrs = (double)n * c->prm.dt / 3600.;   // its = n idt, thrs = its / 3600. (si3d.f90:326-327)
  if (st) { std::memset(st, 0, sizeof(*st)); CK(cudaEventRecord(c->ev0, c->st)); }
  const si3d_params& p = c->prm;
  int niter1 = p.niter;
  int rc = 0;
  if (n == 1) {
    niter1 = std::max(2, p.niter);
  } else {
    const bool leapfrog_only = p.itrap == 0 || (n % std::max(p.itrap, 1)) != 0;
    rc = fd_impl(c, 1, leapfrog_only, st);
    if (rc) return rc;
    if (leapfrog_only) {
      int rs = 0;
      rc = stage(c, ST_SAVE, 2, [&] { rs = save_all(c, 1); });
      if (!rc) rc = rs;
      if (rc) return rc;
      goto done;
    }
    rc = stage(c, ST_SETTRAP, 3, [&] { settrap_all(c); });
    if (rc) return rc;
  }
  for (int it = 1; it <= niter1; ++it) {
    rc = fd_impl(c, 2, it == niter1, st);
    if (rc) return rc;
    if (it < niter1) {
      rc = stage(c, ST_SETTRAP2, 3, [&] { settrap2_all(c); });
      if (rc) return rc;
    }
    if (it > 20) break;
  }
  {
    int rs = 0;
    rc = stage(c, ST_SAVE, 2, [&] { rs = save_all(c, 2); });
    if (!rc) rc = rs;
  }
  if (rc) return rc;
done:
  CK(cudaGetLastError());
  if (st) {
    CK(cudaEventRecord(c->ev1, c->st));
    CK(cudaEventSynchronize(c->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    st->ms_total = ms;
  }
  return 0;
}

// The oldest committed group of staged inputs into its fields, on the compute stream after the
// group's copies; the slot is free again once these moves have run.
static int take_staged(Ctx* c) {
  if (c->stg_queue.empty()) return 0;
  const int slot = c->stg_queue.front();
  c->stg_queue.pop_front();
  Ctx::Staged& S = c->stg[slot];
  CK(cudaStreamWaitEvent(c->st, S.ready, 0));
  for (const auto& mv : S.moves)
    CK(cudaMemcpyAsync(mv.first, mv.second, sizeof(double) * c->lm1, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaEventRecord(S.free, c->st));
  return 0;
}

static int copy_streams(Ctx* c) {
  if (c->ist) return 0;
  CK(cudaStreamCreateWithFlags(&c->ist, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->fst, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&c->stg[0].ready, &c->stg[0].free, &c->stg[1].ready, &c->stg[1].free, &c->snap_ready,
                         &c->fetch_done})
    CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  for (cudaEvent_t e : {c->stg[0].free, c->stg[1].free}) CK(cudaEventRecord(e, c->ist));
  CK(cudaEventRecord(c->fetch_done, c->fst));
  return 0;
}

int si3d_gpu_stage_field(int h, const char* name, const double* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!name || !host) return SI3D_EDIMS;
  double* field = f2ptr(c, name);
  if (!field) return SI3D_ENAME;
  CK(cudaSetDevice(c->device));
  if (int rc = copy_streams(c)) return rc;
  if (c->stg_fill < 0) {
    if (c->stg_queue.size() >= 2) return SI3D_EDIMS;   // both slots hold groups no step has taken yet
    const int slot = c->stg_next;
    c->stg_next ^= 1;
    c->stg_fill = slot;
    c->stg[slot].moves.clear();
    CK(cudaStreamWaitEvent(c->ist, c->stg[slot].free, 0));   // the slot's previous group has been moved
  }
  Ctx::Staged& S = c->stg[c->stg_fill];
  double*& buf = S.buf[name];
  if (!buf && c->alloc(&buf, c->lm1)) return SI3D_ENOMEM;
  CK(cudaMemcpyAsync(buf, host, sizeof(double) * c->lm1, cudaMemcpyHostToDevice, c->ist));
  S.moves.emplace_back(field, buf);
  return 0;
}

int si3d_gpu_stage_commit(int h) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (c->stg_fill < 0) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  CK(cudaEventRecord(c->stg[c->stg_fill].ready, c->ist));
  c->stg_queue.push_back(c->stg_fill);
  c->stg_fill = -1;
  return 0;
}

int si3d_gpu_fetch_field(int h, const char* name, double* host) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!name || !host) return SI3D_EDIMS;
  const double* field = f2ptr(c, name);
  if (!field) return SI3D_ENAME;
  CK(cudaSetDevice(c->device));
  if (int rc = copy_streams(c)) return rc;
  double*& snap = c->snap[name];
  if (!snap && c->alloc(&snap, c->lm1)) return SI3D_ENOMEM;
  CK(cudaStreamWaitEvent(c->st, c->fetch_done, 0));   // the previous read has left the snapshots
  CK(cudaMemcpyAsync(snap, field, sizeof(double) * c->lm1, cudaMemcpyDeviceToDevice, c->st));
  CK(cudaEventRecord(c->snap_ready, c->st));
  CK(cudaStreamWaitEvent(c->fst, c->snap_ready, 0));
  CK(cudaMemcpyAsync(host, snap, sizeof(double) * c->lm1, cudaMemcpyDeviceToHost, c->fst));
  CK(cudaEventRecord(c->fetch_done, c->fst));
  return 0;
}

int si3d_gpu_copies_wait(int h) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!c->ist) return 0;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->ist));
  CK(cudaStreamSynchronize(c->fst));
  return 0;
}

int si3d_gpu_step(int h, int n, si3d_step_stats* st) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  CK(cudaSetDevice(c->device));
  if (int rs = take_staged(c)) return rs;
  const int rc = step_impl(c, n, st);
  if (rc) return rc;
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

// ---------------------------------------------------------------------------- autotuner
// Picks the launch shapes of the momentum and scalar-transport stages for this handle's grid by
// timing every candidate on the handle's current state.  The fields those stages write are saved
// first (device copy when memory allows, else host) and restored afterwards, so the model state is
// bit-identical before and after; the shapes never change results.
static int time_stage(Ctx* c, int which, int reps, float* best) {
  Dev& d = c->d;
  auto run = [&] {
    if (which == 0) {
      momentum_stage(c, 1);
      momentum_stage(c, 2);
    } else {
      launch_exsal_imsal(d, c->tune, c->st);
    }
  };
  run();   // warm-up
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->pe0, c->st));
  for (int r = 0; r < reps; ++r) run();
  CK(cudaEventRecord(c->pe1, c->st));
  CK(cudaEventSynchronize(c->pe1));
  CK(cudaGetLastError());
  float ms = 0;
  CK(cudaEventElapsedTime(&ms, c->pe0, c->pe1));
  *best = ms / reps;
  return 0;
}

int si3d_gpu_autotune(int h, int reps, int* choice) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (reps < 1) reps = 3;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  Dev& d = c->d;
  const size_t n3 = (size_t)c->km1 * c->P, n2 = (size_t)c->P;
  std::vector<std::pair<double*, size_t>> keep = {
      {d.f.agx, n3}, {d.f.arx, n3}, {d.f.agy, n3}, {d.f.ary, n3}, {d.scr, n3}, {d.f.Bth2, n3},
      {d.f.Bth3, n3}, {d.f.Bth4, n3}, {d.f.sal, n3}, {d.s.eagx, n2}, {d.s.earx, n2}, {d.s.eagy, n2},
      {d.s.eary, n2}};
  size_t total = 0;
  for (auto& k : keep) total += k.second;
  size_t free_b = 0, tot_b = 0;
  CK(cudaMemGetInfo(&free_b, &tot_b));
  double* dev_copy = nullptr;
  std::vector<double> host_copy;
  if (free_b > total * sizeof(double) + (size_t(2) << 30) &&
      cudaMalloc(&dev_copy, total * sizeof(double)) == cudaSuccess) {
    size_t o = 0;
    for (auto& k : keep) { CK(cudaMemcpy(dev_copy + o, k.first, k.second * sizeof(double), cudaMemcpyDeviceToDevice)); o += k.second; }
  } else {
    cudaGetLastError();
    host_copy.resize(total);
    size_t o = 0;
    for (auto& k : keep) { CK(cudaMemcpy(host_copy.data() + o, k.first, k.second * sizeof(double), cudaMemcpyDeviceToHost)); o += k.second; }
  }
  int rc = 0;
  // every pair of the two knobs of a stage (the best lane count depends on the block size)
  auto pick2 = [&](int which, int* cl, int* nt, std::initializer_list<int> cls) {
    int best_cl = *cl, best_nt = *nt;
    float best_t = 1e30f;
    for (int a : cls)
      for (int b : {64, 128, 256}) {
        if (rc) return;
        *cl = a;
        *nt = b;
        float t = 0;
        rc = time_stage(c, which, reps, &t);
        if (!rc && t < best_t) { best_t = t; best_cl = a; best_nt = b; }
      }
    *cl = best_cl;
    *nt = best_nt;
  };
  Tune& tu = c->tune;
  pick2(0, &tu.mom_cl, &tu.mom_nt, {1, 2, 4, 8});   // lanes 1: the fused one-pass kernel
  if (c->prm.isal != 0) pick2(1, &tu.sal_cl, &tu.sal_nt, {2, 4, 8});
  // restore the state the timing runs overwrote
  size_t o = 0;
  for (auto& k : keep) {
    const cudaError_t e = dev_copy ? cudaMemcpy(k.first, dev_copy + o, k.second * sizeof(double), cudaMemcpyDeviceToDevice)
                                   : cudaMemcpy(k.first, host_copy.data() + o, k.second * sizeof(double),
                                                cudaMemcpyHostToDevice);
    if (e != cudaSuccess && !rc) rc = cuda_fail(e);
    o += k.second;
  }
  if (dev_copy) cudaFree(dev_copy);
  if (rc) return rc;
  if (choice) { choice[0] = tu.mom_cl; choice[1] = tu.mom_nt; choice[2] = tu.sal_cl; choice[3] = tu.sal_nt; }
  return 0;
}

int si3d_gpu_set_tune(int h, const int* choice) {
  Ctx* c = get(h);
  if (!c || !choice) return c ? SI3D_EDIMS : SI3D_EHANDLE;
  auto ok_cl = [](int v) { return v == 2 || v == 4 || v == 8; };
  auto ok_nt = [](int v) { return v == 64 || v == 128 || v == 256; };
  if (!(choice[0] == 1 || ok_cl(choice[0])) || !ok_nt(choice[1]) || !ok_cl(choice[2]) || !ok_nt(choice[3]))
    return SI3D_EDIMS;
  c->tune.mom_cl = choice[0]; c->tune.mom_nt = choice[1]; c->tune.sal_cl = choice[2]; c->tune.sal_nt = choice[3];
  return 0;
}

// ---------------------------------------------------------------------------- ensembles
struct Ens {
  int device = 0;
  std::vector<int> hs;
  std::vector<int> nsolves;          // solves per step of each member (from the capture)
  cudaStream_t master = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t nodes = 0;
  std::vector<cudaEvent_t> joins;
  cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr, solved = nullptr;
  // batched solves: every zeta solve of the step is one cooperative launch for all members
  int mode = SI3D_ENS_SOLVE_BATCHED;   // requested; the per-member form when a member does not qualify
  bool batched = false;                // the form of the captured graph
  int loop_blocks = 0;                 // blocks of the batched launch
  int slots = 0;                       // batched launches per step (zeta solves of a step)
  std::vector<double> nodes_of;        // nodes of each member's larger colour
  std::vector<int> caps;               // blocks of each member's own solve launch
  PcgEnsItem* d_items = nullptr;       // [slots][members] shares of the batched launches
  GridBar* d_bars = nullptr;
  ~Ens() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaEvent_t e : joins) cudaEventDestroy(e);
    for (cudaEvent_t e : {fork, t0, t1, solved}) if (e) cudaEventDestroy(e);
    if (master) cudaStreamDestroy(master);
    if (d_items) cudaFree(d_items);
    if (d_bars) cudaFree(d_bars);
  }
};
std::vector<Ens*> g_ens;

Ens* get_ens(int e) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (e < 0 || e >= (int)g_ens.size()) return nullptr;
  return g_ens[e];
}

int si3d_ens_create(const int* handles, int n, int* ens) {
  if (!handles || n < 1 || !ens) return SI3D_EDIMS;
  auto E = std::make_unique<Ens>();
  for (int i = 0; i < n; ++i) {
    Ctx* c = get(handles[i]);
    if (!c) return SI3D_EHANDLE;
    if (i == 0) E->device = c->device;
    if (c->device != E->device || c->prm.precision != SI3D_FP64 || !c->persistent || c->natural || !c->obc.empty())
      return SI3D_EDIMS;
    for (int j = 0; j < i; ++j)
      if (handles[j] == handles[i]) return SI3D_EDIMS;
    E->hs.push_back(handles[i]);
  }
  CK(cudaSetDevice(E->device));
  CK(cudaStreamCreateWithFlags(&E->master, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&E->fork, &E->t0, &E->t1}) CK(cudaEventCreate(e));
  CK(cudaEventCreateWithFlags(&E->solved, cudaEventDisableTiming));
  E->joins.resize(n);
  for (auto& e : E->joins) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  std::lock_guard<std::mutex> lk(g_mu);
  g_ens.push_back(E.release());
  *ens = (int)g_ens.size() - 1;
  return 0;
}

// Whether every member qualifies for the batched solves: stopping test 5, no stored diagonal, no
// recording, the same time-stepping options, and no more members than co-resident blocks.  Fixes
// the launch's grid (every co-resident block, or the sum of the members' own launch sizes if
// smaller) and the solves a step has.
static bool ens_batch_plan(Ens* E) {
  const int m = (int)E->hs.size();
  const si3d_params& p0 = get(E->hs[0])->prm;
  E->nodes_of.assign(m, 0.0);
  E->caps.assign(m, 1);
  long long own = 0;
  for (int i = 0; i < m; ++i) {
    const Ctx* c = get(E->hs[i]);
    if (c->prm.pcg_test != 5 || c->pcg.diag_stored || c->rec_buf || c->prm.itrap != p0.itrap ||
        c->prm.niter != p0.niter || c->loop_blocks < 1)
      return false;
    E->nodes_of[i] = std::max(c->pcg.R.n, c->pcg.B.n);
    E->caps[i] = c->loop_blocks;
    own += c->loop_blocks;
  }
  const int nb = pcg_loop_ens_blocks(E->device);
  if (nb < m) return false;
  E->loop_blocks = (int)std::min<long long>(nb, own);
  const bool leapfrog_only = p0.itrap == 0 || (2 % std::max(p0.itrap, 1)) != 0;
  E->slots = leapfrog_only ? 1 : 1 + std::min(p0.niter, 21);
  return true;
}

// The members' shares of one batched launch, for solves that took its[i] iterations (all 1 before
// any step): one block each, then one more at a time to the member whose solve would take longest,
// its[i] x (a fixed cost per iteration + its nodes per block x a streaming cost per node), up to the
// blocks its own launch uses (its partial-sum arrays are sized for those).  Every block of the grid
// is given out.
static std::vector<int> ens_shares(const Ens* E, const std::vector<double>& its) {
  constexpr double kIterUs = 5.0;      // three grid barriers and the partial sums of an iteration
  constexpr double kNodeUs = 0.0066;   // both colours' streams of one node of the larger colour
  const int m = (int)E->hs.size();
  std::vector<int> b(m, 1);
  int left = E->loop_blocks - m;
  while (left > 0) {
    int best = -1;
    double bv = -1.0;
    for (int i = 0; i < m; ++i) {
      if (b[i] >= E->caps[i]) continue;
      const double t = its[i] * (kIterUs + kNodeUs * E->nodes_of[i] / b[i]);
      if (t > bv) { bv = t; best = i; }
    }
    if (best < 0) break;
    ++b[best];
    --left;
  }
  return b;
}

// Upload the shares of every solve slot of the step (its: [slot][member] iterations, or null for
// the first plan).
static int ens_upload_shares(Ens* E, const std::vector<std::vector<double>>* its) {
  const int m = (int)E->hs.size();
  std::vector<PcgEnsItem> items((size_t)m * E->slots);
  for (int k = 0; k < E->slots; ++k) {
    const std::vector<int> b = ens_shares(E, its ? (*its)[k] : std::vector<double>(m, 1.0));
    int first = 0;
    for (int i = 0; i < m; ++i) {
      PcgEnsItem& it = items[(size_t)k * m + i];
      it.P = get(E->hs[i])->pcg;
      it.bar = E->d_bars + i;
      it.first = first;
      it.nblk = b[i];
      first += b[i];
    }
  }
  CK(cudaMemcpy(E->d_items, items.data(), sizeof(PcgEnsItem) * items.size(), cudaMemcpyHostToDevice));
  return 0;
}

// Capture one step (n >= 2) with every zeta solve batched: the members advance in lock step on their
// own streams up to each solve's set-up, join the master stream for one cooperative launch that
// solves all of their systems (k_pcg_loop_ens, each member on its share of the blocks with its own
// barrier record), and fork again for the rest of the fd call.  The stage sequence is step_impl's
// for n >= 2.  The k-th launch reads its shares from slot k of the item array, which the steps
// refresh from each solve's last iteration counts without capturing again.
static int ens_capture_batched(Ens* E) {
  const int m = (int)E->hs.size();
  if (!E->d_items) {
    CK(cudaMalloc(&E->d_bars, sizeof(GridBar) * (size_t)m));
    CK(cudaMalloc(&E->d_items, sizeof(PcgEnsItem) * (size_t)m * E->slots));
    const int rc = ens_upload_shares(E, nullptr);
    if (rc) return rc;
  }
  int slot = 0;
  std::vector<Ctx*> cs(m);
  std::vector<char> prof(m);
  CK(cudaStreamBeginCapture(E->master, cudaStreamCaptureModeThreadLocal));
  cudaError_t e = cudaEventRecord(E->fork, E->master);
  for (int i = 0; i < m; ++i) {
    Ctx* c = cs[i] = get(E->hs[i]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(c->st, E->fork, 0);
    c->graph_mode = true;
    c->ens_defer = true;
    c->solve_slot = 0;
    c->trap_solves = 0;
    c->thrs = 2.0 * c->prm.dt / 3600.;
    prof[i] = c->prof;
    c->prof = false;
  }
  // one fd call of every member around one batched solve launch
  auto fd_all = [&](int istep, bool last) -> int {
    for (int i = 0; i < m; ++i) {
      int it = 0, ie = 0;
      double rr = 0.0;
      int r = fd_pre(cs[i], istep);
      if (!r) r = solve(cs[i], &it, &rr, &ie);
      if (r) return r;
      if (cudaEventRecord(E->joins[i], cs[i]->st) != cudaSuccess ||
          cudaStreamWaitEvent(E->master, E->joins[i], 0) != cudaSuccess)
        return cuda_fail(cudaGetLastError());
    }
    if (slot >= E->slots) return SI3D_EDIMS;
    if (pcg_loop_ens(E->d_items + (size_t)slot * m, m, E->loop_blocks, E->d_bars, E->master) != 0)
      return cuda_fail(cudaGetLastError(), "pcg_loop_ens", __LINE__);
    ++slot;
    cs[0]->launches += 1;
    if (cudaEventRecord(E->solved, E->master) != cudaSuccess) return cuda_fail(cudaGetLastError());
    for (int i = 0; i < m; ++i) {
      if (cudaStreamWaitEvent(cs[i]->st, E->solved, 0) != cudaSuccess) return cuda_fail(cudaGetLastError());
      int r = solve_graph_post(cs[i], cs[i]->def_hist, cs[i]->def_ier);
      if (!r) r = fd_post(cs[i], last);
      if (r) return r;
    }
    return 0;
  };
  auto each = [&](const std::function<int(Ctx*)>& f) -> int {
    for (Ctx* c : cs) {
      const int r = f(c);
      if (r) return r;
    }
    return 0;
  };
  auto save = [](int istep) {
    return [istep](Ctx* c) {
      int rs = 0;
      const int r = stage(c, ST_SAVE, 2, [&] { rs = save_all(c, istep); });
      return r ? r : rs;
    };
  };
  int rc = e == cudaSuccess ? 0 : cuda_fail(e);
  if (!rc) {
    const si3d_params& p = cs[0]->prm;
    const bool leapfrog_only = p.itrap == 0 || (2 % std::max(p.itrap, 1)) != 0;
    rc = fd_all(1, leapfrog_only);
    if (!rc && leapfrog_only) {
      rc = each(save(1));
    } else if (!rc) {
      rc = each([](Ctx* c) { return stage(c, ST_SETTRAP, 3, [&] { settrap_all(c); }); });
      for (int it = 1; it <= p.niter && !rc; ++it) {
        rc = fd_all(2, it == p.niter);
        if (!rc && it < p.niter) rc = each([](Ctx* c) { return stage(c, ST_SETTRAP2, 3, [&] { settrap2_all(c); }); });
        if (it > 20) break;
      }
      if (!rc) rc = each(save(2));
    }
    for (int i = 0; i < m && !rc; ++i) {
      if (cudaEventRecord(E->joins[i], cs[i]->st) != cudaSuccess ||
          cudaStreamWaitEvent(E->master, E->joins[i], 0) != cudaSuccess)
        rc = cuda_fail(cudaGetLastError());
    }
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(E->master, &g);
  E->nsolves.assign(m, 0);
  for (int i = 0; i < m; ++i) {
    cs[i]->graph_mode = false;
    cs[i]->ens_defer = false;
    cs[i]->prof = prof[i] != 0;
    E->nsolves[i] = std::min(cs[i]->solve_slot, 24);
  }
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e2 != cudaSuccess) return cuda_fail(e2);
  E->graph = g;
  E->batched = true;
  CK(cudaGraphGetNodes(g, nullptr, &E->nodes));
  CK(cudaGraphInstantiate(&E->exec, g, 0));
  return 0;
}

// Capture one step (n >= 2) of every member into one graph: a fork on the master stream, each
// member's step on its own stream, a join back.
static int ens_capture(Ens* E) {
  // a captured step replays fixed pointers, while the two tracer pools change roles at every save
  for (int h : E->hs)
    if (get(h)->prm.ntr > 0) return SI3D_EDIMS;
  if (E->mode == SI3D_ENS_SOLVE_BATCHED && ens_batch_plan(E)) return ens_capture_batched(E);
  E->batched = false;
  CK(cudaStreamBeginCapture(E->master, cudaStreamCaptureModeThreadLocal));
  int rc = 0;
  cudaError_t e = cudaEventRecord(E->fork, E->master);
  E->nsolves.assign(E->hs.size(), 0);
  for (size_t i = 0; i < E->hs.size() && !rc && e == cudaSuccess; ++i) {
    Ctx* c = get(E->hs[i]);
    e = cudaStreamWaitEvent(c->st, E->fork, 0);
    if (e != cudaSuccess) break;
    c->graph_mode = true;
    c->solve_slot = 0;
    const bool prof = c->prof;
    c->prof = false;
    rc = step_impl(c, 2, nullptr);
    c->prof = prof;
    c->graph_mode = false;
    E->nsolves[i] = std::min(c->solve_slot, 24);
    if (!rc) e = cudaEventRecord(E->joins[i], c->st);
    if (!rc && e == cudaSuccess) e = cudaStreamWaitEvent(E->master, E->joins[i], 0);
  }
  cudaGraph_t g = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(E->master, &g);
  if (rc) { if (g) cudaGraphDestroy(g); return rc; }
  if (e != cudaSuccess) { if (g) cudaGraphDestroy(g); return cuda_fail(e); }
  if (e2 != cudaSuccess) return cuda_fail(e2);
  E->graph = g;
  CK(cudaGraphGetNodes(g, nullptr, &E->nodes));
  CK(cudaGraphInstantiate(&E->exec, g, 0));
  return 0;
}

int si3d_ens_step(int ens, int n0, int nsteps, int* iters, int* ier, double* ms) {
  Ens* E = get_ens(ens);
  if (!E) return SI3D_EHANDLE;
  if (n0 < 1 || nsteps < 0) return SI3D_EDIMS;
  CK(cudaSetDevice(E->device));
  const int m = (int)E->hs.size();
  for (int s = 0; s < nsteps; ++s) {
    const int n = n0 + s;
    if (iters) for (int i = 0; i < m * SI3D_ENS_MAXSOLVES; ++i) iters[(size_t)s * m * SI3D_ENS_MAXSOLVES + i] = -1;
    if (ier) for (int i = 0; i < m * SI3D_ENS_MAXSOLVES; ++i) ier[(size_t)s * m * SI3D_ENS_MAXSOLVES + i] = 0;
    if (n == 1) {   // the start-up step has its own sequence; run it member by member
      CK(cudaEventRecord(E->t0, E->master));
      for (int i = 0; i < m; ++i) {
        Ctx* c = get(E->hs[i]);
        CK(cudaStreamWaitEvent(c->st, E->t0, 0));
        const int rc = step_impl(c, 1, nullptr);
        if (rc) return rc;
        CK(cudaEventRecord(E->joins[i], c->st));
        CK(cudaStreamWaitEvent(E->master, E->joins[i], 0));
      }
      CK(cudaEventRecord(E->t1, E->master));
    } else {
      if (!E->exec) {
        const int rc = ens_capture(E);
        if (rc) return rc;
      }
      CK(cudaEventRecord(E->t0, E->master));
      CK(cudaGraphLaunch(E->exec, E->master));
      CK(cudaEventRecord(E->t1, E->master));
    }
    CK(cudaStreamSynchronize(E->master));
    if (ms) {
      float t = 0;
      CK(cudaEventElapsedTime(&t, E->t0, E->t1));
      ms[s] = t;
    }
    const bool batched = n > 1 && E->batched;
    if (n > 1 && (iters || ier || batched)) {
      // each solve slot's iteration counts weight the next step's shares of the batched launches
      std::vector<std::vector<double>> its(batched ? E->slots : 0, std::vector<double>(m, 1.0));
      for (int i = 0; i < m; ++i) {
        Ctx* c = get(E->hs[i]);
        int buf[48];
        CK(cudaMemcpy(buf, c->d_stats_ii, sizeof(buf), cudaMemcpyDeviceToHost));
        for (int k = 0; k < std::min(E->nsolves[i], SI3D_ENS_MAXSOLVES); ++k) {
          const size_t o = ((size_t)s * m + i) * SI3D_ENS_MAXSOLVES + k;
          if (iters) iters[o] = buf[2 * k];
          if (ier) ier[o] = buf[2 * k + 1];
        }
        for (int k = 0; k < E->nsolves[i]; ++k)
          if (buf[2 * k + 1] < 0) return buf[2 * k + 1];   // the reference stops on ier < 0
        for (int k = 0; k < std::min(E->nsolves[i], (int)its.size()); ++k) its[k][i] = std::max(buf[2 * k], 1);
      }
      if (batched) {
        const int rc = ens_upload_shares(E, &its);
        if (rc) return rc;
      }
    }
  }
  return 0;
}

int si3d_ens_nodes(int ens) {
  Ens* E = get_ens(ens);
  if (!E) return SI3D_EHANDLE;
  return (int)E->nodes;
}

int si3d_ens_solve_mode(int ens, int mode) {
  Ens* E = get_ens(ens);
  if (!E) return SI3D_EHANDLE;
  if (mode != SI3D_ENS_SOLVE_MEMBERS && mode != SI3D_ENS_SOLVE_BATCHED) return SI3D_EDIMS;
  if (mode != E->mode) {   // the next step n >= 2 captures the graph again
    CK(cudaSetDevice(E->device));
    CK(cudaStreamSynchronize(E->master));
    if (E->exec) { cudaGraphExecDestroy(E->exec); E->exec = nullptr; }
    if (E->graph) { cudaGraphDestroy(E->graph); E->graph = nullptr; }
    E->nodes = 0;
    E->mode = mode;
  }
  return 0;
}

int si3d_ens_solve_blocks(int ens) {
  Ens* E = get_ens(ens);
  if (!E) return SI3D_EHANDLE;
  return E->exec && E->batched ? E->loop_blocks : 0;
}

void si3d_ens_destroy(int ens) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (ens < 0 || ens >= (int)g_ens.size() || !g_ens[ens]) return;
  cudaSetDevice(g_ens[ens]->device);
  cudaStreamSynchronize(g_ens[ens]->master);
  delete g_ens[ens];
  g_ens[ens] = nullptr;
}

int si3d_gpu_profile(int h, int enable) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  c->prof = enable != 0;
  for (int i = 0; i < 16; ++i) { c->prof_ms[i] = 0; c->prof_n[i] = 0; }
  return 0;
}

}  // extern "C"

namespace {

// Pack one frame into the next device buffer (after its previous copy has left it) and copy it to
// `host` on the copy stream; the returned event marks the copy's end.
int output_frame_impl(int h, int kind, int arg, int first, float* host, long long capacity, long long* count,
                      cudaEvent_t* done) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!count) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  Dev& d = c->d;
  const double* fields[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  int nf = 0;
  std::pair<int*, int> plane{nullptr, 0};
  long long n = 0;
  switch (kind) {
    case SI3D_OUT_PTRACK:
      fields[0] = d.f.hp; fields[1] = d.f.up; fields[2] = d.f.vp; fields[3] = d.f.wp; fields[4] = d.f.salp;
      nf = 5;
      n = c->npoints * (nf + (first ? 3 : 0));
      break;
    case SI3D_OUT_TRACER:
      if (arg < 1 || arg > c->prm.ntr) return SI3D_EDIMS;
      fields[0] = tracer_pool(c, c->tr_alias) + (arg - 1) * c->tr_stride;
      nf = 1;
      n = c->npoints * (nf + (first ? 3 : 0));
      break;
    case SI3D_OUT_PLANE: {
      if (arg < d.g.k1) return SI3D_EDIMS;   // "Output plane is not in DOMAIN" (si3d_utils.f90:2165)
      auto it = c->planes.find(arg);
      if (it == c->planes.end()) {   // CountPlaneCells (:2337-2368): kmz >= kp, or every column
        std::vector<int> cols;
        for (int l = 1; l <= c->lm; ++l)
          if (arg > d.g.km || c->h_kmz[l - 1] >= arg) cols.push_back(l);
        int* dc = nullptr;
        if (c->alloc(&dc, cols.size())) return SI3D_ENOMEM;
        if (!cols.empty()) CK(cudaMemcpy(dc, cols.data(), sizeof(int) * cols.size(), cudaMemcpyHostToDevice));
        it = c->planes.emplace(arg, std::make_pair(dc, (int)cols.size())).first;
      }
      plane = it->second;
      n = (long long)plane.second * (first ? 8 : 6);
      break;
    }
    default: return SI3D_EDIMS;
  }
  *count = n;
  if (!host) return 0;   // size query
  if (capacity < n) return SI3D_EDIMS;
  if (!c->out_buf[0]) {   // the largest frame: the first ptrack frame, or a plane's
    c->out_cap = std::max(c->npoints * 8, (long long)c->lm * 8);
    if (c->alloc(&c->out_buf[0], c->out_cap) || c->alloc(&c->out_buf[1], c->out_cap)) return SI3D_ENOMEM;
    CK(cudaStreamCreateWithFlags(&c->cst, cudaStreamNonBlocking));
    CK(cudaEventCreateWithFlags(&c->out_packed, cudaEventDisableTiming));
    for (cudaEvent_t* e : {&c->out_free[0], &c->out_free[1]}) CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    for (cudaEvent_t& e : c->out_done) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaEventRecord(c->out_free[0], c->cst));
    CK(cudaEventRecord(c->out_free[1], c->cst));
  }
  if (n > c->out_cap) return SI3D_EDIMS;
  const int slot = c->out_slot;
  c->out_slot ^= 1;
  float* buf = c->out_buf[slot];
  CK(cudaStreamWaitEvent(c->st, c->out_free[slot], 0));
  if (kind == SI3D_OUT_PLANE)
    launch_pack_plane(d, plane.first, plane.second, arg, first != 0, c->d_l2i, c->d_l2j, buf, c->st);
  else
    launch_pack_points(d, fields, nf, c->poff, c->d_l2i, c->d_l2j, first != 0, buf, c->st);
  c->launches += 1;
  CK(cudaGetLastError());
  CK(cudaEventRecord(c->out_packed, c->st));
  CK(cudaStreamWaitEvent(c->cst, c->out_packed, 0));
  if (n > 0) CK(cudaMemcpyAsync(host, buf, sizeof(float) * n, cudaMemcpyDeviceToHost, c->cst));
  CK(cudaEventRecord(c->out_free[slot], c->cst));
  cudaEvent_t ev = c->out_done[c->out_ev];
  c->out_ev = (c->out_ev + 1) % 16;
  CK(cudaEventRecord(ev, c->cst));
  *done = ev;
  return 0;
}

}  // namespace

extern "C" {

int si3d_gpu_output_frame(int h, int kind, int arg, int first, float* host, long long capacity, long long* count) {
  cudaEvent_t done = nullptr;
  const int rc = output_frame_impl(h, kind, arg, first, host, capacity, count, &done);
  if (rc || !host) return rc;
  CK(cudaEventSynchronize(done));
  return 0;
}

int si3d_gpu_output_frame_async(int h, int kind, int arg, int first, float* host, long long capacity,
                                long long* count, unsigned long long* ticket) {
  if (!ticket) return SI3D_EDIMS;
  cudaEvent_t done = nullptr;
  const int rc = output_frame_impl(h, kind, arg, first, host, capacity, count, &done);
  *ticket = reinterpret_cast<unsigned long long>(done);
  return rc;
}

int si3d_gpu_output_wait(int h, unsigned long long ticket) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (!ticket) return 0;
  CK(cudaSetDevice(c->device));
  CK(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(ticket)));
  return 0;
}

int si3d_gpu_host_alloc(long long bytes, void** ptr) {
  if (!ptr || bytes <= 0) return SI3D_EDIMS;
  *ptr = nullptr;
  const cudaError_t e = cudaMallocHost(ptr, (size_t)bytes);
  if (e != cudaSuccess) { g_last_cuda = cudaGetErrorString(e); *ptr = nullptr; return SI3D_ENOMEM; }
  return 0;
}

int si3d_gpu_host_free(void* ptr) {
  if (ptr && cudaFreeHost(ptr) != cudaSuccess) return SI3D_ECUDA;
  return 0;
}

int si3d_gpu_counters(int h, long long* launches, double* stage_ms, long long* stage_n) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (launches) *launches = c->launches;
  for (int i = 0; i < ST_COUNT; ++i) {
    if (stage_ms) stage_ms[i] = c->prof_ms[i];
    if (stage_n) stage_n[i] = c->prof_n[i];
  }
  return ST_COUNT;
}

int si3d_gpu_set_open_boundaries(int h, int nopen, const int* iside, const int* itype, const int* isbc,
                                 const int* jsbc, const int* iebc, const int* jebc, double dtsec, int npts,
                                 const double* wse, const double* temp) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (nopen < 0) return SI3D_EDIMS;
  if (nopen > 0 && (!iside || !itype || !isbc || !jsbc || !iebc || !jebc || !wse || !temp || npts < 3 || !(dtsec > 0)))
    return SI3D_EDIMS;
  // tracers at open boundaries (openbcTracer) and the FP32 MIC inner solves are not built for them
  if (nopen > 0 && (c->prm.precision == SI3D_MIXED_IR || c->prm.ntr > 0 || c->graph_mode)) return SI3D_EDIMS;
  CK(cudaSetDevice(c->device));
  const int im1 = c->im1, jm1 = c->jm1, lm1 = c->lm1;
  std::vector<int> ij((size_t)im1 * jm1, 0);
  for (int l = 1; l <= c->lm; ++l) ij[(size_t)(c->h_l2i[l - 1] - 1) * jm1 + (c->h_l2j[l - 1] - 1)] = l;
  auto cell = [&](int i, int j) { return (i < 1 || j < 1 || i > im1 || j > jm1) ? 0 : ij[(size_t)(i - 1) * jm1 + (j - 1)]; };
  std::vector<ObcDev> obc;
  std::vector<std::vector<int>> keep;
  for (int nn = 0; nn < nopen; ++nn) {
    const int side = iside[nn];
    if (itype[nn] != 1 || side < 1 || side > 4) return SI3D_EDIMS;   // water-surface elevation only
    std::vector<int> cells, inner, face, mom;
    const bool x = side == 1 || side == 3;
    const int a = x ? jsbc[nn] : isbc[nn], e = x ? jebc[nn] : iebc[nn];
    if (e < a) return SI3D_EDIMS;
    for (int q = a; q <= e; ++q) {
      const int i = x ? isbc[nn] : q, j = x ? q : jsbc[nn];
      const int lb = cell(i, j);
      const int outer = side == 1 ? cell(i - 1, j) : side == 2 ? cell(i, j + 1) : side == 3 ? cell(i + 1, j) : cell(i, j - 1);
      if (!lb || outer) return SI3D_EDIMS;   // a wet cell with a dry cell outside it (openbc0's checks)
      const int li = side == 1 ? c->h_lEC[lb - 1] : side == 2 ? c->h_lSC[lb - 1] : side == 3 ? c->h_lWC[lb - 1] : c->h_lNC[lb - 1];
      if (li == lm1) return SI3D_EDIMS;     // the interior neighbour must be wet
      cells.push_back(lb);
      inner.push_back(li);
      face.push_back((side == 1 || side == 4) ? lb : li);
      mom.push_back((side == 1 || side == 4) ? lb : li);
    }
    ObcDev B;
    B.side = side;
    B.n = B.nface = (int)cells.size();
    int *dc = nullptr, *di = nullptr, *df = nullptr, *dm = nullptr;
    int rc = c->alloc(&dc, cells.size());
    rc |= c->alloc(&di, cells.size());
    rc |= c->alloc(&df, cells.size());
    rc |= c->alloc(&dm, cells.size());
    if (rc) return rc;
    CK(cudaMemcpy(dc, cells.data(), cells.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(di, inner.data(), inner.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(df, face.data(), face.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(dm, mom.data(), mom.size() * sizeof(int), cudaMemcpyHostToDevice));
    B.cells = dc; B.inner = di; B.face = df; B.mom = dm;
    obc.push_back(B);
  }
  c->obc = obc;
  c->obc_wse.assign(nopen, {});
  c->obc_tmp.assign(nopen, {});
  for (int nn = 0; nn < nopen; ++nn) {
    c->obc_wse[nn].assign(wse + (size_t)nn * npts, wse + (size_t)(nn + 1) * npts);
    c->obc_tmp[nn].assign(temp + (size_t)nn * npts, temp + (size_t)(nn + 1) * npts);
  }
  c->obc_dtsec = dtsec;
  // the cut faces leave matcon's rr above 1 + sx + sx(W) + sy + sy(S): the iteration reads rr
  c->pcg.diag_stored = nopen > 0;
  return 0;
}

int si3d_gpu_test_wait_limit(int h, long long polls, int absent_blocks) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  if (polls < 1 || polls > (1LL << 26) || absent_blocks < 0 || absent_blocks > 1024) return SI3D_EDIMS;
  if (!c->persistent || c->graph_mode) return SI3D_EDIMS;
  c->bar_test = GridBar{};
  c->bar_test.absent = (unsigned int)absent_blocks;
  c->bar_test.limit = (unsigned long long)polls;
  c->bar_test_armed = true;
  return 0;
}

int si3d_gpu_sync(int h) {
  Ctx* c = get(h);
  if (!c) return SI3D_EHANDLE;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  return 0;
}

int si3d_gpu_solve_zeta(int lm, const double* coef, const int* jcoef, const double* rhs, double* zeta, int pcg_test,
                        double pcg_tol, int pcg_itmax, double srelpr, int precision, int ordering, int* iters,
                        double* stptst, double* emin, double* emax) {
  if (lm < 1 || !coef || !jcoef || !rhs || !zeta || pcg_itmax < 1 || (pcg_test != 5 && pcg_test != 2))
    return SI3D_EDIMS;
  if (precision != SI3D_FP64 && precision != SI3D_MIXED_IR) return SI3D_EDIMS;
  if (ordering != 0 && ordering != SI3D_ORDER_REDBLACK && ordering != SI3D_ORDER_NATURAL) return SI3D_EDIMS;
  // Recover the grid graph and sx/sy from the SolverSparse structure:
  // coef = [rr, -sx(lW), -sy(lS), -sy(l), -sx(l)], jcoef = [l, lWC, lSC, lNC, lEC] (0 = dry).
  const int lm1 = lm + 1;
  std::vector<int> E(lm), W(lm), N(lm), S(lm);
  std::vector<double> sx(lm1, 0.0), sy(lm1, 0.0), qq(lm1, 0.0), sp(lm1, 0.0);
  for (int m = 0; m < lm; ++m) {
    auto J = [&](int cidx) { const int v = jcoef[(size_t)cidx * lm + m]; return v <= 0 ? lm1 : v; };
    if (jcoef[m] != m + 1) return SI3D_EDIMS;
    W[m] = J(1); S[m] = J(2); N[m] = J(3); E[m] = J(4);
    sx[m] = -coef[(size_t)4 * lm + m];
    sy[m] = -coef[(size_t)3 * lm + m];
    qq[m] = rhs[m];
    sp[m] = zeta[m];
  }
  // the diagonal is the caller's (SolverSparse's rr); when it differs from 1 + the face sum (open
  // boundaries cut faces after rr is formed) the iteration reads it instead of forming it
  std::vector<double> rrv(lm1, 1.0);
  bool diag_is_sum = true;
  for (int m = 0; m < lm; ++m) {
    const double sxw = W[m] == lm1 ? 0.0 : sx[W[m] - 1], sys = S[m] == lm1 ? 0.0 : sy[S[m] - 1];
    if (-coef[(size_t)1 * lm + m] != sxw || -coef[(size_t)2 * lm + m] != sys) return SI3D_EDIMS;
    rrv[m] = coef[m];
    if (coef[m] != 1 + sx[m] + sxw + sy[m] + sys) diag_is_sum = false;
    if (E[m] != lm1 && W[E[m] - 1] != m + 1) return SI3D_EDIMS;
    if (N[m] != lm1 && S[N[m] - 1] != m + 1) return SI3D_EDIMS;
  }
  if (!diag_is_sum && precision == SI3D_MIXED_IR) return SI3D_EDIMS;   // the FP32 inner rows form it
  si3d_grid g{};
  std::vector<int> kmz(lm1, 2), l2(lm, 1);   // one layer (k1 = 2) per column; the sentinel at km1
  kmz[lm] = 3;
  std::vector<double> hh(lm1, 1.0), zlv = {-100., -100., 1.0};
  g.im1 = 1; g.jm1 = 1; g.km1 = 3; g.k1 = 2; g.lm = lm;
  g.l2i = l2.data(); g.l2j = l2.data(); g.lEC = E.data(); g.lWC = W.data(); g.lNC = N.data(); g.lSC = S.data();
  g.kmz = kmz.data(); g.hhs = hh.data(); g.hhu = hh.data(); g.hhv = hh.data(); g.zlevel = zlv.data();
  si3d_params prm{};
  prm.dt = 1; prm.dx = 1; prm.dy = 1; prm.theta = 1; prm.itrmom = 1; prm.ihd = 1;
  prm.pcg_test = pcg_test; prm.pcg_tol = pcg_tol; prm.pcg_itmax = pcg_itmax; prm.srelpr = srelpr;
  prm.ordering = ordering == SI3D_ORDER_NATURAL ? SI3D_ORDER_NATURAL : SI3D_ORDER_REDBLACK;
  prm.x0_mode = SI3D_X0_PREV; prm.precision = precision;
  int hdl = -1;
  int rc = si3d_gpu_init(&g, &prm, 0, &hdl);
  if (rc) return rc;
  Ctx* c = get(hdl);
  int ier = 0, it = 0;
  double rr = 0;
  rc = si3d_gpu_set_field(hdl, "sx", sx.data());
  if (!rc) rc = si3d_gpu_set_field(hdl, "sy", sy.data());
  if (!rc) rc = si3d_gpu_set_field(hdl, "rr", rrv.data());
  c->pcg.diag_stored = !diag_is_sum;
  if (!rc) rc = si3d_gpu_set_field(hdl, "qq", qq.data());
  if (!rc) rc = si3d_gpu_set_field(hdl, "sp", sp.data());
  if (!rc) rc = solve(c, &it, &rr, &ier);
  std::vector<double> s(lm1);
  if (!rc) rc = si3d_gpu_get_field(hdl, "s", s.data());
  if (!rc) {
    for (int m = 0; m < lm; ++m) zeta[m] = s[m];
    *iters = it; *stptst = rr;
    std::vector<double> al(std::max(it, 1)), be(std::max(it, 1));
    if (it > 0) {
      cudaMemcpy(al.data(), c->pcg.hist_alpha, sizeof(double) * it, cudaMemcpyDeviceToHost);
      cudaMemcpy(be.data(), c->pcg.hist_beta, sizeof(double) * it, cudaMemcpyDeviceToHost);
    }
    double zt = pcg_tol < 500.0 * srelpr ? 500.0 * srelpr : pcg_tol;
    double e0 = 1.0, e1 = 2.0;
    if (pcg_test == 2) { e0 = c->h_sc->emin; e1 = c->h_sc->emax; }   // adapted on the device during the solve
    else if (it > 0) eigen_estimates(al.data(), be.data(), it, zt, pcg_itmax, e0, e1);
    if (emin) *emin = e0;
    if (emax) *emax = e1;
  }
  si3d_gpu_finalize(hdl);
  return rc ? rc : ier;
}

int si3d_gpu_column_tridiag(int n, int nsys, const double* a, const double* b, const double* c, const double* g,
                            const double* r, double* ag, double* ar) {
  if (n < 1 || nsys < 1 || !a || !b || !c || !g || !r || !ag || !ar) return SI3D_EDIMS;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return SI3D_ENODEV;
  const size_t N = (size_t)n * nsys;
  std::vector<double> host(N);
  double* dbuf = nullptr;
  CK(cudaMalloc(&dbuf, 8 * N * sizeof(double)));
  double* D[8];
  for (int i = 0; i < 8; ++i) D[i] = dbuf + i * N;
  // host blocks are n x nsys column-major (system-contiguous); the device wants k-major
  auto up = [&](const double* src, double* dst) {
    for (int s = 0; s < nsys; ++s)
      for (int k = 0; k < n; ++k) host[(size_t)k * nsys + s] = src[(size_t)s * n + k];
    return cudaMemcpy(dst, host.data(), N * sizeof(double), cudaMemcpyHostToDevice);
  };
  cudaError_t e = cudaSuccess;
  const double* srcs[5] = {a, b, c, g, r};
  for (int i = 0; i < 5 && e == cudaSuccess; ++i) e = up(srcs[i], D[i]);
  if (e == cudaSuccess) {
    launch_column_tridiag(n, nsys, D[0], D[1], D[2], D[3], D[4], D[5], D[6], D[7], 0);
    e = cudaGetLastError();
  }
  for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
    e = cudaMemcpy(host.data(), D[5 + i], N * sizeof(double), cudaMemcpyDeviceToHost);
    double* out = i ? ar : ag;
    for (int s = 0; s < nsys && e == cudaSuccess; ++s)
      for (int k = 0; k < n; ++k) out[(size_t)s * n + k] = host[(size_t)k * nsys + s];
  }
  cudaFree(dbuf);
  if (e != cudaSuccess) return cuda_fail(e);
  return 0;
}

}  // extern "C"
