/*
 * si3d_gpu.h — C ABI of the B200 (sm_100a) implementation of pSi3D's per-timestep
 * semi-implicit core: momentum explicit terms + per-column tridiagonals, free-surface (zeta)
 * assembly, the MIC-preconditioned conjugate-gradient zeta solve, velocities/continuity,
 * active-scalar transport and the leapfrog-trapezoidal bookkeeping.
 *
 * The reference calls these stages from Fortran (si3d.f90:324-458 -> fd,
 * si3d_procedures.f90:382-575).  A Fortran host binds this header through ISO_C_BINDING
 * (module si3d_gpu_iface in si3d_b200/fortran/); every scalar is passed by value or by
 * pointer, every array is a plain pointer to host memory laid out exactly as the reference's
 * arrays: 3-D fields (km1, lm1) column-major with k fastest, 2-D fields of length lm1, all
 * column indices 1-based with lm1 = lm + 1 the dry sentinel.
 *
 * Ownership: the caller owns every host array; the library copies what it needs and never
 * retains host pointers.  The library owns the device state of a handle (one CUDA stream,
 * device buffers, captured graphs).  Calls are synchronous: on return the device state is
 * updated (or the host outputs are valid).  Handles are independent; one handle must not be
 * used from two threads at once.
 *
 * Errors: every entry point returns an int.  0 = success.  The zeta solve reports NSPCG's own
 * codes (1 = itmax reached, 2 = tolerance clamped, 3/4 = eigenvalue estimate halted,
 * -6 = pAp <= 0, -7 = (r,z) <= 0); library errors are <= -100 (see SI3D_E*).  The library never
 * traps, never exits and never waits without a bound.
 */
#ifndef SI3D_GPU_H
#define SI3D_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* library error codes */
#define SI3D_OK 0
#define SI3D_ECUDA (-100)     /* a CUDA runtime call failed */
#define SI3D_EDIMS (-101)     /* bad dimensions or arguments */
#define SI3D_EHANDLE (-102)   /* unknown handle */
#define SI3D_ENAME (-103)     /* unknown field name */
#define SI3D_ENAN (-104)      /* non-finite value detected */
#define SI3D_ETIMEOUT (-105)  /* a bounded device wait gave up */
#define SI3D_ENOMEM (-106)    /* device allocation failed */
#define SI3D_ENODEV (-107)    /* no CUDA device / not sm_100 */
#define SI3D_ECAPACITY (-108) /* problem larger than the fixed scratch of an allocation-free call */

/* precision forms */
#define SI3D_FP64 0       /* plain FP64 everywhere */
#define SI3D_MIXED_IR 1   /* FP32 SpMV + MIC inside an FP64 iterative-refinement loop */
#define SI3D_MIXED_MG 2   /* FP32 SpMV + aggregation-multigrid V-cycle inside FP64 iterative
                             refinement (needs the l2i/l2j maps of a plain (im1, jm1) grid);
                             a project addition with no counterpart in the reference */

/* zeta-solve orderings */
#define SI3D_ORDER_REDBLACK 1   /* NSPCG iperm=1 red-black MIC (the GPU form; 0 means the same) */
#define SI3D_ORDER_NATURAL 2    /* the reference's own natural-order MIC (mic1, nspcg.f:21759-21805,
                                   :22875-22922, :22729-22777): its triangular sweeps are recurrences
                                   along l, run level by level by one thread block, so it is meant for
                                   small systems (iterate-level comparison with the reference's
                                   algorithm); plain FP64 only, not with SI3D_X0_HIST or ensembles */

/* initial guess for the zeta solve */
#define SI3D_X0_PREV 0      /* sp, as the reference (si3d_procedures.f90:1970) */
#define SI3D_X0_ZERO 1
#define SI3D_X0_LEARNED 2   /* with a network loaded (si3d_learn_set_params): sp + the predicted
                               increment for the leapfrog solve of a step, the latest solution for
                               the trapezoidal solves after it; otherwise sp + the increment set by
                               si3d_gpu_set_warmstart for every solve */
#define SI3D_X0_LAST 3      /* s, the latest accepted solution: within a step the trapezoidal solves
                               start from the previous solve's zeta(n+1) instead of the half level sp
                               (LAST and HIST are project additions, no counterpart in the reference) */
#define SI3D_X0_HIST 4      /* s + the same solve's correction one step earlier (solve k of step n
                               starts from s + (x_k(n-1) - s_k(n-1)), where s_k is the zeta solve k
                               started from); the first step starts from s */

/* Grid description produced by the host's `bathy` (si3d_utils.f90:595-892). */
typedef struct si3d_grid {
  int im1, jm1;            /* (i,j) extents including the fictitious border */
  int km1;                 /* number of levels incl. fictitious top and bottom layers (3 .. 448;
                              si3d_gpu_init returns SI3D_EDIMS outside) */
  int k1;                  /* first real layer (2) */
  int lm;                  /* number of wet columns */
  const int* l2i;          /* [lm]   i of column l (1-based) */
  const int* l2j;          /* [lm]   j of column l */
  const int* lEC;          /* [lm]   east / west / north / south neighbour, lm+1 if dry */
  const int* lWC;
  const int* lNC;
  const int* lSC;
  const int* kmz;          /* [lm+1] bottom layer index; kmz[lm] = km1 */
  const double* hhs;       /* [lm+1] depth at zeta points */
  const double* hhu;       /* [lm+1] depth at u points */
  const double* hhv;       /* [lm+1] depth at v points */
  const double* zlevel;    /* [km1]  depth of the top of each layer (-100 above the surface) */
} si3d_grid;

/* Run parameters read by the host's `input` (si3d_utils.f90:21-315) plus the solver overlay. */
typedef struct si3d_params {
  double dt, dx, dy;
  double Av0, Dv0, Ax0, Ay0, f, theta, cd, cw, beta;
  int iadv, itrmom, ihd, ibc, isal, itrap, niter, ismooth;
  /* zeta solve: NSPCG stopping test (2 or 5), tolerance, itmax, machine precision srelpr */
  int pcg_test;
  double pcg_tol;
  int pcg_itmax;
  double srelpr;
  int ordering;            /* SI3D_ORDER_REDBLACK or SI3D_ORDER_NATURAL */
  int x0_mode;             /* SI3D_X0_* */
  int precision;           /* SI3D_FP64, SI3D_MIXED_IR or SI3D_MIXED_MG */
  int ntr;                 /* non-active tracers, 0..30 (ntrmax, si3d_types.f90:291); conservative
                              tracers only (ecomod = 0, srcsnk00), advanced once per step by fd */
  int iturb;               /* 0 constant eddy coefficients, 1 Mellor-Yamada 2.5 (si3d_mixing.f90:33-551) */
} si3d_params;

/* Per-call statistics (one entry per zeta solve inside the call). */
typedef struct si3d_step_stats {
  int nsolves;             /* zeta solves performed by the call */
  int iters[24];           /* PCG iterations of each solve */
  double relres[24];       /* final stopping-test value of each solve */
  int ier[24];             /* NSPCG-style code of each solve */
  int total_iters;
  double ms_total;         /* device time of the call */
  double ms_pcg;           /* device time spent in the zeta solves */
} si3d_step_stats;

/* Replaces the reference's allocation + init hand-off: uploads maps and parameters and
 * allocates the device state (zero-initialised; the host then sets the initial fields).
 * Reference interface replaced: the state set-up done by bathy/init before the time loop
 * (si3d.f90:56-68) feeding fd (si3d_procedures.f90:382). */
int si3d_gpu_init(const si3d_grid* grid, const si3d_params* params, int device, int* handle);

/* Copy one reference array between host and device.  3-D names: uh uhp uhpp up upp hu hup hupp
 * agx arx vh vhp vhpp vp vpp hv hvp hvpp agy ary h hp hpp sal salp salpp rhop Av Dv wp
 * HeatSource Bth2 Bth3 Bth4 ((km1, lm1) column-major); with iturb = 1 also q2 q2p q2pp q2l q2lp
 * q2lpp u v; and per tracer nt = 1..ntr the names
 * "tracer<nt>" and "tracerpp<nt>" (tracer(:,:,nt), tracerpp(:,:,nt), si3d_utils.f90:571-574).
 * 2-D names: s sp spp eagx earx eagy eary sx sy dd qq rr uair vair cdw (lm1).  Replaces the
 * Fortran module arrays of si3d_types.f90:117-164. */
int si3d_gpu_set_field(int handle, const char* name, const double* host);
int si3d_gpu_get_field(int handle, const char* name, double* host);
/* The same copies for a host whose arrays are default REAL (4 bytes), as the reference is built
 * (si3d_types.f90:26-27, no -r8 in its makefile): values are widened to FP64 on the device, and
 * rounded to the nearest float on the way back.  Same names, layout and errors as above. */
int si3d_gpu_set_field_f32(int handle, const char* name, const float* host);
int si3d_gpu_get_field_f32(int handle, const char* name, float* host);
/* Integer column arrays k1z k1u k1v (lm1 entries). */
int si3d_gpu_set_ifield(int handle, const char* name, const int* host);
int si3d_gpu_get_ifield(int handle, const char* name, int* host);

/* Density anomaly rhop = densty_s(salp, 4e-5, z) - 1000 at every column (sentinel included) and
 * level k1..km1 from the uploaded salp and hp, as InitializeScalarFields does after reading the
 * initial profile (si3d_procedures.f90:363-373). */
int si3d_gpu_density(int handle);

/* One call of fd (si3d_procedures.f90:382-575): surfbc CASE 0, exmom+matmom (x, y), matcon,
 * SolverSparse (NSPCG mic1+cg replacement), vel + continuity(1), exsal + imsal, and with
 * ntr > 0, niter > 0 and lastiter = 1 exTracer + ImTracer for every tracer (:520-544), then vel2.
 * Replaces CALL fd(...) at si3d.f90:353 and si3d.f90:373. */
int si3d_gpu_fd(int handle, int n, int istep, int lastiter, si3d_step_stats* stats);
/* settrap (si3d_procedures.f90:3418), settrap2 (:3944), save (:3621, which also sets
 * tracerpp = tracer); replace the calls at si3d.f90:365, :383, :393. */
int si3d_gpu_settrap(int handle);
int si3d_gpu_settrap2(int handle);
int si3d_gpu_save(int handle, int istep);
/* One whole time step n of the loop body si3d.f90:324-458 (leapfrog, settrap, niter
 * trapezoidal iterations with settrap2, save); stats cover every solve of the step. */
int si3d_gpu_step(int handle, int n, si3d_step_stats* stats);

/* One routine of fd or of the step bookkeeping, for stage-by-stage unit tests: "momentum"
 * (exmom + matmom + trid, x then y), "matcon", "solve" (SolverSparse incl. slayer_h), "vel"
 * (vel + continuity(1)), "scalar" (exsal + imsal), "vel2", "settrap", "settrap2", "save". */
int si3d_gpu_stage(int handle, const char* stage, int istep, si3d_step_stats* stats);

/* Learned warm start: the increment added to sp for the next solve(s) when x0_mode is
 * SI3D_X0_LEARNED (lm1 entries, host or device pointer flagged by `on_device`). */
int si3d_gpu_set_warmstart(int handle, const double* dzeta, int on_device);

/* Standalone replacement of CALL nspcg(mic1, cg, ...) (si3d_procedures.f90:1999-2000) on
 * host Purdue arrays: coef (lm x 5, column-major: diagonal, W, S, N, E), jcoef (1-based,
 * 0 = no entry), rhs (lm), zeta (lm; in: x0, out: solution).  The matrix must have the
 * 5-point structure SolverSparse builds (jcoef columns = l, lWC, lSC, lNC, lEC).
 * ordering: SI3D_ORDER_REDBLACK (0 or 1) or SI3D_ORDER_NATURAL (NSPCG's default numbering, the
 * reference's; precision SI3D_FP64 only).
 * Outputs: iterations, final stopping-test value, emin/emax estimates. */
int si3d_gpu_solve_zeta(int lm, const double* coeffA, const int* jcoefA, const double* rhs, double* zeta,
                        int pcg_test, double pcg_tol, int pcg_itmax, double srelpr, int precision, int ordering,
                        int* iters, double* stptst, double* emin, double* emax);

/* Batched tridiagonal solves with two right-hand sides sharing one factorisation, as trid
 * (si3d_procedures.f90:3210-3289): for each of `nsys` systems of size `n` (column-major
 * blocks a/b/c/g/r/ag/ar of n x nsys) solve [a b c] ag = g and [a b c] ar = r.  Host arrays. */
int si3d_gpu_column_tridiag(int n, int nsys, const double* a, const double* b, const double* c,
                            const double* g, const double* r, double* ag, double* ar);

/* Output frames of the reference's binary writers, packed on the device in the order of the
 * record the reference writes and converted to 4-byte floats (the default-REAL build the readers
 * expect); the caller adds the record framing and the time stamp.  Replaces the array packing of
 * outp (si3d_utils.f90:2484-2602), outz (:2373-2481) and outh (:2142-2334).  kind:
 *   SI3D_OUT_PTRACK  hp up vp wp salp at every layer k1..kmz+1 of every wet column (first frame:
 *                    i j k before them)
 *   SI3D_OUT_TRACER  tracer `arg` (1..ntr) at the same points (first frame: i j k before it)
 *   SI3D_OUT_PLANE   layer `arg` of every column that reaches it (arg > km: each column's bottom
 *                    layer): first frame i j u v w salp Av s, later frames face-averaged u v w,
 *                    salp (-99 where dry), Av, s
 * first != 0 selects the first frame's layout.  *count receives the number of floats; with host ==
 * NULL the call only reports it.  SI3D_EDIMS when capacity < count or arg is out of range. */
#define SI3D_OUT_PTRACK 1
#define SI3D_OUT_TRACER 2
#define SI3D_OUT_PLANE 3
int si3d_gpu_output_frame(int handle, int kind, int arg, int first, float* host, long long capacity, long long* count);
/* The same without waiting: the frame is packed on the handle's stream (in order with the time
 * steps) and copied to `host` (page-locked) on a separate copy stream, overlapping the steps that
 * follow; *ticket identifies the copy, and si3d_gpu_output_wait(handle, ticket) returns once it has
 * landed.  At most 16 copies may be in flight per handle.  Project additions without a reference
 * counterpart. */
int si3d_gpu_output_frame_async(int handle, int kind, int arg, int first, float* host, long long capacity,
                                long long* count, unsigned long long* ticket);
int si3d_gpu_output_wait(int handle, unsigned long long ticket);
/* Page-locked host memory for output frames (the device-to-host copy then runs at full link
 * bandwidth).  Project additions without a reference counterpart. */
int si3d_gpu_host_alloc(long long bytes, void** ptr);
int si3d_gpu_host_free(void* ptr);

/* Instrumentation.  si3d_gpu_profile(h, 1) makes every stage record CUDA events on the handle's
 * stream and wait for them (stage boundaries become synchronisation points); counters returns the
 * number of kernels the handle has launched and, per stage, the accumulated device milliseconds
 * and call counts (the zeta-solve iteration stage counts iterations).  Stage order: momentum x,
 * momentum y, matcon, pcg setup, pcg iterations, pcg finish, slayer_h, vel, scalar, vel2,
 * settrap, settrap2, save, learned guess, tracers.  Returns the number of stages. */
int si3d_gpu_profile(int handle, int enable);
int si3d_gpu_counters(int handle, long long* launches, double* stage_ms, long long* stage_n);

/* Allocation-free form of si3d_gpu_column_tridiag, for callers that cannot call cudaMalloc (a
 * model coupled into a framework that owns the device allocator, or a loop that must not allocate
 * once running).  No counterpart in the reference.  Inputs and outputs are the caller's DEVICE
 * buffers in layer-major order (element k of system s at k*nsys + s); the sweep's scratch is a
 * fixed array inside the library, so n*nsys must not exceed SI3D_NOALLOC_MAX_ELEMS (larger
 * problems return SI3D_ECAPACITY without touching the GPU).  The library image keeps that 8 MiB
 * array on every GPU that loads it until the process exits.  Every call looks the array's address
 * up in the current context.  All calls share the array, so calls whose kernels overlap on one GPU
 * race: serialise them, for example on one stream.  Work is queued on `stream` (a cudaStream_t,
 * NULL = the default stream) and the call returns after that stream has finished it, so the call
 * cannot be made on a stream that is capturing a CUDA graph.  A CUDA error already pending when
 * the call starts is reported as SI3D_ECUDA (and left pending) without launching anything. */
#define SI3D_NOALLOC_MAX_ELEMS (1 << 20)
int si3d_gpu_column_tridiag_noalloc(int n, int nsys, const double* a, const double* b, const double* c,
                                   const double* g, const double* r, double* ag, double* ar, void* stream);

/* Autotuner (no reference counterpart): times every pair of launch-shape knobs of the momentum and
 * scalar-transport stages on this handle's current state and keeps the fastest - layer lanes per
 * column of the cell-parallel kernels (2, 4, 8; for momentum also 1, which selects the fused kernel
 * that forms the explicit terms and runs the column sweep in one pass down each face column) and
 * threads per block of the column-sequential kernels (64, 128, 256).  The fields those stages write are restored afterwards, so the state is
 * unchanged; shapes never change results.  `reps` timed launches per candidate; the choice
 * {mom_lanes, mom_threads, scalar_lanes, scalar_threads} is returned through `choice` (optional). */
int si3d_gpu_autotune(int handle, int reps, int* choice);
/* Apply a launch-shape choice (e.g. a cached autotuner result). */
int si3d_gpu_set_tune(int handle, const int* choice);

/* Open boundaries with a specified water-surface elevation (the reference's itype = 1), replacing
 * the boundary set-up of openbc0 (si3d_boundaryconditions.f90:23-897) and the per-stage
 * adjustments openbcUVH (:900), MODexmom4openBCX/Y (:1801, :2370), MODqqddrr4openBC (:1508),
 * MODvel4openBC (:2941) and openbcSCA (:3157), which the library then applies inside si3d_gpu_fd,
 * si3d_gpu_settrap, si3d_gpu_settrap2 and si3d_gpu_save.  Per boundary nn (0-based arrays of nopen):
 * side iside (1 W, 2 N, 3 E, 4 S), itype (must be 1), the cell range isbc/jsbc/iebc/jebc in the
 * reference's 1-based (i, j); every boundary cell must be wet with a dry cell outside it and a wet
 * one inside.  The series (elevation wse and temperature temp, [nopen][npts] row-major) hold one
 * value every dtsec seconds from t = 0 and are interpolated as parab does (si3d_utils.f90:895)
 * at the step's time n * dt; a step past their end returns SI3D_EDIMS.  The host sets sp of the
 * boundary cells to the first value at t = 0, as openbc0 does.  Not with SI3D_MIXED_IR, tracers or
 * ensembles (SI3D_EDIMS). */
int si3d_gpu_set_open_boundaries(int handle, int nopen, const int* iside, const int* itype, const int* isbc,
                                 const int* jsbc, const int* iebc, const int* jebc, double dtsec, int npts,
                                 const double* wse, const double* temp);

/* Wait for the handle's stream. */
int si3d_gpu_sync(int handle);
/* Test hook for the bounded device waits (no counterpart in the reference).  The next cooperative
 * zeta-solve launch of this handle (FP64 or FP32 MIC loop, or the multigrid solve) waits at each
 * grid barrier for `absent_blocks` blocks beyond its grid - blocks that do not exist - and gives up
 * after `polls` polls (1 .. 2^26) instead of the built-in limit.  That solve then ends with
 * SI3D_ETIMEOUT through the call that ran it, and the handle stays usable.  Applies once.
 * SI3D_EDIMS for out-of-range arguments or a handle whose steps are being captured in a graph. */
int si3d_gpu_test_wait_limit(int handle, long long polls, int absent_blocks);
/* Staged inputs and asynchronous reads, for a host loop that overlaps its transfers with the time
 * steps (no counterpart in the reference, whose fields live in host memory).  Work on 2-D fields
 * (lm1 values, e.g. uair, vair, cdw, s) and PINNED host memory (si3d_gpu_host_alloc).
 * si3d_gpu_stage_field queues a copy of the host values into a staging slot of the handle on a
 * host-to-device copy stream and returns at once; si3d_gpu_stage_commit closes the group staged
 * since the last commit.  Each si3d_gpu_step first takes the oldest committed group: it waits for
 * the group's copies and moves the values into their fields before its first kernel, so a loop can
 * stage step n + 1's inputs while step n runs.  Two groups at most may wait for a step
 * (SI3D_EDIMS otherwise); the host buffer must stay unchanged until the copy has run
 * (si3d_gpu_copies_wait).  si3d_gpu_fetch_field snapshots a 2-D field on the device after the work
 * queued so far and copies the snapshot to the host buffer on a device-to-host copy stream,
 * returning at once; the values are in the buffer after si3d_gpu_copies_wait, which waits for
 * every staged and fetched copy of the handle. */
int si3d_gpu_stage_field(int handle, const char* name, const double* host_pinned);
int si3d_gpu_stage_commit(int handle);
int si3d_gpu_fetch_field(int handle, const char* name, double* host_pinned);
int si3d_gpu_copies_wait(int handle);

/* Human-readable text for an error code. */
const char* si3d_gpu_strerror(int code);
/* Free the device state of a handle. */
void si3d_gpu_finalize(int handle);

/* ---------------------------------------------------------------- ensembles
 * No counterpart in the reference (one si3d process runs one basin).  Several handles (basins of
 * any size) advance in lock step: every member's time step is enqueued on its own stream without
 * host synchronisation (each zeta solve is one cooperative launch that iterates to convergence on the
 * device), and one ensemble step (n >= 2) is captured once into one CUDA graph - a fork on a master
 * stream, one branch per member, a join - then replayed, one graph launch per step.  Members must be
 * FP64 handles on one device with the cooperative solve enabled, and must outlive the ensemble. */
#define SI3D_ENS_MAXSOLVES 4
int si3d_ens_create(const int* handles, int n, int* ens);
/* Time steps n0 .. n0 + nsteps - 1 of every member.  Optional outputs per step: iters/ier
 * [nsteps][n][SI3D_ENS_MAXSOLVES] for each zeta solve (-1 / 0 past a member's solves and for the
 * start-up step n = 1, which runs member by member), ms[nsteps] device time of the whole ensemble step.
 * Returns the first negative solver ier met (the reference stops there). */
int si3d_ens_step(int ens, int n0, int nsteps, int* iters, int* ier, double* ms);
/* Nodes of the captured step graph (0 before the first step n >= 2). */
int si3d_ens_nodes(int ens);
/* How the captured step runs the members' zeta solves (no counterpart in the reference).
 * SI3D_ENS_SOLVE_BATCHED (the default): the members advance in lock step, and each of the step's
 * zeta solves is ONE cooperative launch for all members, each basin iterating to its own
 * convergence on its share of the SMs with its own barrier counter; it applies when every member
 * uses stopping test 5, the same itrap and niter, and no open boundary, and there are no more
 * members than co-resident blocks (otherwise the step falls back to the per-member form).
 * SI3D_ENS_SOLVE_MEMBERS: one cooperative solve launch per member, on the member's own stream.
 * A member that gets as many blocks in the batched launch as its own launch uses (the members'
 * needs fit the GPU together) sums its dot products in the same order, and both forms give
 * bit-identical states; when the members share fewer blocks, a basin's dot products are summed
 * over fewer partials and its state agrees with the other form to rounding, each solve still
 * iterating to the same tolerance.  Changing the mode re-captures at the next step. */
#define SI3D_ENS_SOLVE_MEMBERS 0
#define SI3D_ENS_SOLVE_BATCHED 1
int si3d_ens_solve_mode(int ens, int mode);
/* Blocks of the batched solve launch in the captured graph (0: per-member form, or not captured). */
int si3d_ens_solve_blocks(int ens);
void si3d_ens_destroy(int ens);

#ifdef __cplusplus
}
#endif
#endif /* SI3D_GPU_H */
