/*
 * si3d_host.h — C++ host side above the si3d_gpu C ABI.
 *
 * The reference's host is Fortran (si3d.f90 + si3d_utils.f90 + si3d_procedures.f90 set-up).  No
 * Fortran compiler is available to build it here, so this library restates the host duties the
 * GPU core needs: it reads the reference's own input files (si3d_inp.txt, si3d_bathy,
 * si3d_init.txt) with the reference's record formats, builds the grid maps as `bathy` does,
 * initialises the state as `init` does, hands everything to si3d_gpu_init/si3d_gpu_set_field and
 * runs the time loop of si3d.f90:324-458 through si3d_gpu_step.
 */
#ifndef SI3D_HOST_H
#define SI3D_HOST_H

#include "si3d_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Solver overlay applied on top of si3d_inp.txt (the reference hard-codes these in
 * SolverSparse, si3d_procedures.f90:1989-1995). */
typedef struct si3d_solver_opts {
  int pcg_test;      /* 2 or 5 */
  double pcg_tol;
  int pcg_itmax;
  double srelpr;
  int x0_mode;       /* SI3D_X0_* */
  int precision;     /* SI3D_FP64 / SI3D_MIXED_IR / SI3D_MIXED_MG */
  int ordering;      /* SI3D_ORDER_REDBLACK (0 or 1) or SI3D_ORDER_NATURAL */
} si3d_solver_opts;

/* Read the input files of a run directory and build grid + initial state on the host.
 * An optional si3d_wind_override.bin (int32 im1, int32 jm1, float64 uair[im1*jm1],
 * float64 vair[im1*jm1], i outer / j inner) replaces the uniform wind of surfbc CASE(0). */
int si3d_host_open(const char* run_dir, const si3d_solver_opts* opts, int* hm, char* err, int errlen);
/* im1, jm1, km1, lm, km, nts */
int si3d_host_dims(int hm, int* dims);
/* Host copy of a grid/map array: "l2i" "l2j" "lEC" "lWC" "lNC" "lSC" "kmz" (int, lm1 entries). */
int si3d_host_get_map(int hm, const char* name, int* out);
/* zlevel (km1 entries). */
int si3d_host_get_zlevel(int hm, double* out);
/* Create the GPU state (si3d_gpu_init), upload the initial fields and write the initial output
 * frames (si3d.f90:89-100). */
int si3d_host_attach_gpu(int hm, int device, int* gpu_handle);
/* Run `nsteps` time steps from the current step counter; per-step stats (optional, nsteps
 * entries).  The binary outputs the input file selects (outh planes, outz tracers, outp ptrack
 * file: si3d.f90:430-438) are written into the run directory: frames are packed on the device and
 * copied asynchronously, and a writer thread writes the records while the next steps run; every
 * record is in its file when the call returns. */
int si3d_host_run(int hm, int nsteps, si3d_step_stats* stats);
/* Current time-step counter n. */
int si3d_host_step_count(int hm);
void si3d_host_close(int hm);

#ifdef __cplusplus
}
#endif
#endif /* SI3D_HOST_H */
