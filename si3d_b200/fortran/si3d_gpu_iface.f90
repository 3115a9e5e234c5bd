!*************************************************************************
                          MODULE si3d_gpu_iface
!*************************************************************************
!
!  ISO_C_BINDING interface to the B200 semi-implicit core (include/si3d_gpu.h).
!  Every routine returns an INTEGER(C_INT) status: 0 = ok, NSPCG codes for the
!  zeta solve (1, 2, -6, -7, ...), <= -100 for library errors.
!  Arrays are passed as assumed-size (*) actual arguments with the layout the
!  si3d module arrays already have: (km1, lm1) column-major, lm1 sentinel.
!
!-------------------------------------------------------------------------
   USE ISO_C_BINDING
   IMPLICIT NONE

   TYPE, BIND(C) :: si3d_grid_t
      INTEGER(C_INT) :: im1, jm1, km1, k1, lm
      TYPE(C_PTR)    :: l2i, l2j, lEC, lWC, lNC, lSC, kmz
      TYPE(C_PTR)    :: hhs, hhu, hhv, zlevel
   END TYPE si3d_grid_t

   TYPE, BIND(C) :: si3d_params_t
      REAL(C_DOUBLE) :: dt, dx, dy
      REAL(C_DOUBLE) :: Av0, Dv0, Ax0, Ay0, f, theta, cd, cw, beta
      INTEGER(C_INT) :: iadv, itrmom, ihd, ibc, isal, itrap, niter, ismooth
      INTEGER(C_INT) :: pcg_test
      REAL(C_DOUBLE) :: pcg_tol
      INTEGER(C_INT) :: pcg_itmax
      REAL(C_DOUBLE) :: srelpr
      INTEGER(C_INT) :: ordering, x0_mode, precision
      INTEGER(C_INT) :: ntr, iturb
   END TYPE si3d_params_t

   TYPE, BIND(C) :: si3d_step_stats_t
      INTEGER(C_INT) :: nsolves
      INTEGER(C_INT) :: iters(24)
      REAL(C_DOUBLE) :: relres(24)
      INTEGER(C_INT) :: ier(24)
      INTEGER(C_INT) :: total_iters
      REAL(C_DOUBLE) :: ms_total, ms_pcg
   END TYPE si3d_step_stats_t

   INTERFACE
      INTEGER(C_INT) FUNCTION si3d_gpu_init(grid, params, device, handle) BIND(C, NAME="si3d_gpu_init")
         IMPORT :: C_INT, si3d_grid_t, si3d_params_t
         TYPE(si3d_grid_t), INTENT(IN)   :: grid
         TYPE(si3d_params_t), INTENT(IN) :: params
         INTEGER(C_INT), VALUE           :: device
         INTEGER(C_INT), INTENT(OUT)     :: handle
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_set_field(handle, name, host) BIND(C, NAME="si3d_gpu_set_field")
         IMPORT :: C_INT, C_CHAR, C_DOUBLE
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         REAL(C_DOUBLE), INTENT(IN)         :: host(*)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_get_field(handle, name, host) BIND(C, NAME="si3d_gpu_get_field")
         IMPORT :: C_INT, C_CHAR, C_DOUBLE
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         REAL(C_DOUBLE), INTENT(OUT)        :: host(*)
      END FUNCTION

      ! staged inputs / asynchronous reads of 2-D fields through pinned buffers (si3d_gpu_host_alloc)
      INTEGER(C_INT) FUNCTION si3d_gpu_stage_field(handle, name, host) BIND(C, NAME="si3d_gpu_stage_field")
         IMPORT :: C_INT, C_CHAR, C_PTR
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         TYPE(C_PTR), VALUE                 :: host
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_stage_commit(handle) BIND(C, NAME="si3d_gpu_stage_commit")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: handle
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_fetch_field(handle, name, host) BIND(C, NAME="si3d_gpu_fetch_field")
         IMPORT :: C_INT, C_CHAR, C_PTR
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         TYPE(C_PTR), VALUE                 :: host
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_copies_wait(handle) BIND(C, NAME="si3d_gpu_copies_wait")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: handle
      END FUNCTION

      ! the same for the reference's default-REAL (4-byte) module arrays, without -r8
      INTEGER(C_INT) FUNCTION si3d_gpu_set_field_f32(handle, name, host) BIND(C, NAME="si3d_gpu_set_field_f32")
         IMPORT :: C_INT, C_CHAR, C_FLOAT
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         REAL(C_FLOAT), INTENT(IN)          :: host(*)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_get_field_f32(handle, name, host) BIND(C, NAME="si3d_gpu_get_field_f32")
         IMPORT :: C_INT, C_CHAR, C_FLOAT
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         REAL(C_FLOAT), INTENT(OUT)         :: host(*)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_set_ifield(handle, name, host) BIND(C, NAME="si3d_gpu_set_ifield")
         IMPORT :: C_INT, C_CHAR
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         INTEGER(C_INT), INTENT(IN)         :: host(*)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_get_ifield(handle, name, host) BIND(C, NAME="si3d_gpu_get_ifield")
         IMPORT :: C_INT, C_CHAR
         INTEGER(C_INT), VALUE              :: handle
         CHARACTER(KIND=C_CHAR), INTENT(IN) :: name(*)
         INTEGER(C_INT), INTENT(OUT)        :: host(*)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_density(handle) BIND(C, NAME="si3d_gpu_density")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: handle
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_fd(handle, n, istep, lastiter, stats) BIND(C, NAME="si3d_gpu_fd")
         IMPORT :: C_INT, si3d_step_stats_t
         INTEGER(C_INT), VALUE                  :: handle, n, istep, lastiter
         TYPE(si3d_step_stats_t), INTENT(OUT)   :: stats
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_settrap(handle) BIND(C, NAME="si3d_gpu_settrap")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: handle
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_settrap2(handle) BIND(C, NAME="si3d_gpu_settrap2")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: handle
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_save(handle, istep) BIND(C, NAME="si3d_gpu_save")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: handle, istep
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_step(handle, n, stats) BIND(C, NAME="si3d_gpu_step")
         IMPORT :: C_INT, si3d_step_stats_t
         INTEGER(C_INT), VALUE                :: handle, n
         TYPE(si3d_step_stats_t), INTENT(OUT) :: stats
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_solve_zeta(lm, coeffA, jcoefA, rhs, zeta, pcg_test, pcg_tol, pcg_itmax, &
                                                  srelpr, precision, ordering, iters, stptst, emin, emax)  &
                                                  BIND(C, NAME="si3d_gpu_solve_zeta")
         IMPORT :: C_INT, C_DOUBLE
         INTEGER(C_INT), VALUE         :: lm, pcg_test, pcg_itmax, precision, ordering
         REAL(C_DOUBLE), VALUE         :: pcg_tol, srelpr
         REAL(C_DOUBLE), INTENT(IN)    :: coeffA(*), rhs(*)
         INTEGER(C_INT), INTENT(IN)    :: jcoefA(*)
         REAL(C_DOUBLE), INTENT(INOUT) :: zeta(*)
         INTEGER(C_INT), INTENT(OUT)   :: iters
         REAL(C_DOUBLE), INTENT(OUT)   :: stptst, emin, emax
      END FUNCTION

      ! open boundaries with a specified water-surface elevation (openbc0 and the stage adjustments
      ! of si3d_boundaryconditions.f90), the series varsOpenBC(nn,1,:) and (nn,2,:) as wse, temp
      INTEGER(C_INT) FUNCTION si3d_gpu_set_open_boundaries(handle, nopen, iside, itype, isbc, jsbc, iebc,  &
                                                           jebc, dtsec, npts, wse, temp)                 &
                                                           BIND(C, NAME="si3d_gpu_set_open_boundaries")
         IMPORT :: C_INT, C_DOUBLE
         INTEGER(C_INT), VALUE      :: handle, nopen, npts
         INTEGER(C_INT), INTENT(IN) :: iside(*), itype(*), isbc(*), jsbc(*), iebc(*), jebc(*)
         REAL(C_DOUBLE), VALUE      :: dtsec
         REAL(C_DOUBLE), INTENT(IN) :: wse(*), temp(*)
      END FUNCTION

      SUBROUTINE si3d_gpu_finalize(handle) BIND(C, NAME="si3d_gpu_finalize")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: handle
      END SUBROUTINE

      ! launch-shape autotuner: choice = (momentum lanes, momentum threads, scalar lanes, scalar threads)
      INTEGER(C_INT) FUNCTION si3d_gpu_autotune(handle, reps, choice) BIND(C, NAME="si3d_gpu_autotune")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE       :: handle, reps
         INTEGER(C_INT), INTENT(OUT) :: choice(4)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_set_tune(handle, choice) BIND(C, NAME="si3d_gpu_set_tune")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE      :: handle
         INTEGER(C_INT), INTENT(IN) :: choice(4)
      END FUNCTION

      ! ensembles: several handles advanced in lock step, one CUDA graph launch per step
      INTEGER(C_INT) FUNCTION si3d_ens_create(handles, n, ens) BIND(C, NAME="si3d_ens_create")
         IMPORT :: C_INT
         INTEGER(C_INT), INTENT(IN)  :: handles(*)
         INTEGER(C_INT), VALUE       :: n
         INTEGER(C_INT), INTENT(OUT) :: ens
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_ens_step(ens, n0, nsteps, iters, ier, ms) BIND(C, NAME="si3d_ens_step")
         IMPORT :: C_INT, C_DOUBLE
         INTEGER(C_INT), VALUE       :: ens, n0, nsteps
         INTEGER(C_INT), INTENT(OUT) :: iters(*), ier(*)
         REAL(C_DOUBLE), INTENT(OUT) :: ms(*)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_ens_solve_mode(ens, mode) BIND(C, NAME="si3d_ens_solve_mode")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: ens, mode
      END FUNCTION

      SUBROUTINE si3d_ens_destroy(ens) BIND(C, NAME="si3d_ens_destroy")
         IMPORT :: C_INT
         INTEGER(C_INT), VALUE :: ens
      END SUBROUTINE

      ! learned initial guess (include/si3d_learn.h): SI3D_NET_NPARAM FP32 parameters
      INTEGER(C_INT) FUNCTION si3d_learn_set_params(handle, params) BIND(C, NAME="si3d_learn_set_params")
         IMPORT :: C_INT, C_FLOAT
         INTEGER(C_INT), VALUE     :: handle
         REAL(C_FLOAT), INTENT(IN) :: params(*)
      END FUNCTION

      INTEGER(C_INT) FUNCTION si3d_gpu_output_frame(handle, kind, arg, first, host, capacity, count) &
            BIND(C, NAME="si3d_gpu_output_frame")
         IMPORT :: C_INT, C_FLOAT, C_LONG_LONG
         INTEGER(C_INT), VALUE            :: handle, kind, arg, first
         REAL(C_FLOAT), INTENT(OUT)       :: host(*)
         INTEGER(C_LONG_LONG), VALUE      :: capacity
         INTEGER(C_LONG_LONG), INTENT(OUT) :: count
      END FUNCTION
   END INTERFACE

END MODULE si3d_gpu_iface
