!-------------------------------------------------------------------------------
! cumc_gpu.f90 -- ISO_C_BINDING interface to libcumc3d_gpu.so (the B200 MHD
! stage engine, include/cumc3d_gpu.h) for the CUMC3D Fortran host code.
!
! With this module the reference's main loop (solver/mhd/main.f90:56-139)
! keeps its structure: GET_MODEL fills prim/epsilon on the host as before,
! then the device owns the state.  The routine names mirror the ones they
! replace: CUMC_INITIAL_UPDATE (INITIAL_UPDATE), CUMC_FINDDT (FINDDT),
! CUMC_RUNGEKUTTA (RUNGEKUTTA), CUMC_FIND_DIVB (FIND_DIVB).
!
! This file is not compiled in this repository (no Fortran compiler in the
! build image); the C entry points it binds are exercised by tests/.
!-------------------------------------------------------------------------------
MODULE CUMC_GPU
USE ISO_C_BINDING
IMPLICIT NONE

INTEGER(C_INT), PARAMETER :: CUMC_OK = 0
INTEGER(C_INT), PARAMETER :: CUMC_RECON_TVD_MM = 0, CUMC_RECON_TVD_VL = 1, CUMC_RECON_TVD_MC = 2
INTEGER(C_INT), PARAMETER :: CUMC_RECON_PPM = 3, CUMC_RECON_WENO = 4
INTEGER(C_INT), PARAMETER :: CUMC_RS_LF = 0, CUMC_RS_HLL = 1, CUMC_RS_HLLC = 2, CUMC_RS_HLLD = 3
INTEGER(C_INT), PARAMETER :: CUMC_FP64 = 0, CUMC_FP32 = 1
INTEGER(C_INT), PARAMETER :: CUMC_FLOOR_NONE = 0, CUMC_FLOOR_EPS = 1, CUMC_FLOOR_TORUS = 2, CUMC_FLOOR_COLLAPSAR = 3
INTEGER(C_INT), PARAMETER :: CUMC_SRC_NONE = 0, CUMC_SRC_CONST_GY = 1, CUMC_SRC_PM_CYL = 2, CUMC_SRC_PM_SPH = 3
INTEGER(C_INT), PARAMETER :: CUMC_SRC_COLLAPSAR = 4
INTEGER(C_INT), PARAMETER :: CUMC_BOUNDARY_EXCHANGE = 9
INTEGER(C_INT), PARAMETER :: CUMC_FILL_STATE = 0, CUMC_FILL_EMF = 1

! cumc_model (include/cumc3d_gpu.h)
TYPE, BIND(C) :: cumc_model
  REAL(C_DOUBLE) :: gamma
  INTEGER(C_INT) :: floor_kind
  REAL(C_DOUBLE) :: rho_floor, eps_floor, p_floor
  INTEGER(C_INT) :: source_kind
  REAL(C_DOUBLE) :: g_const, r_sh
  INTEGER(C_INT) :: bc_kind
END TYPE

! cumc_config (include/cumc3d_gpu.h)
TYPE, BIND(C) :: cumc_config
  INTEGER(C_INT) :: nx, ny, nz, n_dim, coordinate_flag
  INTEGER(C_INT) :: boundary_flag(6)
  TYPE(C_PTR) :: xF, yF, zF
  REAL(C_DOUBLE) :: cfl
  INTEGER(C_INT) :: recon, riemann, precision, learned, fixpole
  INTEGER(C_INT) :: fix_periodic_normal_faces, positivity_fallback
  TYPE(cumc_model) :: model
END TYPE

! cumc_batch_config (include/cumc3d_gpu.h): many 1D problems in one launch
TYPE, BIND(C) :: cumc_batch_config
  INTEGER(C_INT) :: n_problems
  TYPE(C_PTR) :: nx             ! INTEGER(C_INT) nx(n_problems)
  TYPE(C_PTR) :: xF             ! TYPE(C_PTR) xF(n_problems), each -3:nx+3 faces
  TYPE(C_PTR) :: t_end          ! REAL(C_DOUBLE) t_end(n_problems)
  REAL(C_DOUBLE) :: cfl, gamma
  INTEGER(C_INT) :: recon, riemann, precision, floor_kind, positivity_fallback
END TYPE

INTEGER(C_INT), PARAMETER :: CUMC_LEARN_NP = 2657

! cumc_train_config (include/cumc3d_gpu.h): Adam training of the flag network
TYPE, BIND(C) :: cumc_train_config
  INTEGER(C_INT) :: steps, batch
  REAL(C_FLOAT) :: lr, delta
  REAL(C_FLOAT) :: beta1, beta2, eps
  INTEGER(C_LONG_LONG) :: seed
END TYPE

INTERFACE
  INTEGER(C_INT) FUNCTION cumc_create(cfg, h) BIND(C, NAME='cumc_create')
    IMPORT :: C_INT, C_PTR, cumc_config
    TYPE(cumc_config), INTENT(IN) :: cfg
    TYPE(C_PTR), INTENT(OUT) :: h
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_destroy(h) BIND(C, NAME='cumc_destroy')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_set_state(h, prim, eps) BIND(C, NAME='cumc_set_state')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(IN) :: prim(*), eps(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_get_state(h, prim, eps) BIND(C, NAME='cumc_get_state')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: prim(*), eps(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_initial_update(h) BIND(C, NAME='cumc_initial_update')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_finddt(h, dt) BIND(C, NAME='cumc_finddt')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: dt
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_rk3_step(h, dt) BIND(C, NAME='cumc_rk3_step')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), VALUE :: dt
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_evolve(h, t_end, max_steps, t, steps) BIND(C, NAME='cumc_evolve')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), VALUE :: t_end
    INTEGER(C_INT), VALUE :: max_steps
    REAL(C_DOUBLE), INTENT(INOUT) :: t
    INTEGER(C_INT), INTENT(OUT) :: steps
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_max_divb(h, divb) BIND(C, NAME='cumc_max_divb')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: divb
  END FUNCTION
  TYPE(C_PTR) FUNCTION cumc_last_error(h) BIND(C, NAME='cumc_last_error')
    IMPORT :: C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  ! batched 1D problems (the n_dim = 1 build of main.f90, many at once)
  INTEGER(C_INT) FUNCTION cumc_batch_create(cfg, b) BIND(C, NAME='cumc_batch_create')
    IMPORT :: C_INT, C_PTR, cumc_batch_config
    TYPE(cumc_batch_config), INTENT(IN) :: cfg
    TYPE(C_PTR), INTENT(OUT) :: b
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_batch_set_state(b, p, prim, eps) BIND(C, NAME='cumc_batch_set_state')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: b
    INTEGER(C_INT), VALUE :: p
    REAL(C_DOUBLE), INTENT(IN) :: prim(*), eps(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_batch_run(b, max_steps, t, steps, status) BIND(C, NAME='cumc_batch_run')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: b
    INTEGER(C_INT), VALUE :: max_steps
    REAL(C_DOUBLE), INTENT(OUT) :: t(*)
    INTEGER(C_INT), INTENT(OUT) :: steps(*), status(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_batch_get_state(b, p, prim_row, eps_row) BIND(C, NAME='cumc_batch_get_state')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: b
    INTEGER(C_INT), VALUE :: p
    REAL(C_DOUBLE), INTENT(OUT) :: prim_row(*), eps_row(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_batch_destroy(b) BIND(C, NAME='cumc_batch_destroy')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: b
  END FUNCTION
  ! learned smooth-face flag (a handle created with cfg%learned = 1, WENO)
  INTEGER(C_INT) FUNCTION cumc_learn_set(h, params, threshold, flag_interval, audit_interval, audit_tol) &
      BIND(C, NAME='cumc_learn_set')
    IMPORT :: C_INT, C_PTR, C_FLOAT
    TYPE(C_PTR), VALUE :: h
    REAL(C_FLOAT), INTENT(IN) :: params(*)
    REAL(C_FLOAT), VALUE :: threshold, audit_tol
    INTEGER(C_INT), VALUE :: flag_interval, audit_interval
  END FUNCTION
  ! self-gravity potential of the collapsar model (spherical grids)
  INTEGER(C_INT) FUNCTION cumc_poisson_setup(h, rho_atm, omega) BIND(C, NAME='cumc_poisson_setup')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), VALUE :: rho_atm, omega
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_poisson_solve(h, max_iter, tol, iters, err, converged) &
      BIND(C, NAME='cumc_poisson_solve')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: max_iter
    REAL(C_DOUBLE), VALUE :: tol
    INTEGER(C_INT), INTENT(OUT) :: iters, converged
    REAL(C_DOUBLE), INTENT(OUT) :: err
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_poisson_get(h, phi) BIND(C, NAME='cumc_poisson_get')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: phi(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_poisson_set(h, phi) BIND(C, NAME='cumc_poisson_set')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(IN) :: phi(*)
  END FUNCTION
  ! z-slab groups (slabs: an array of handles in z order)
  INTEGER(C_INT) FUNCTION cumc_group_initial_update(slabs, n) BIND(C, NAME='cumc_group_initial_update')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: slabs
    INTEGER(C_INT), VALUE :: n
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_group_finddt(slabs, n, dt) BIND(C, NAME='cumc_group_finddt')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: slabs
    INTEGER(C_INT), VALUE :: n
    REAL(C_DOUBLE), INTENT(OUT) :: dt
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_group_step(slabs, n, dt) BIND(C, NAME='cumc_group_step')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: slabs
    INTEGER(C_INT), VALUE :: n
    REAL(C_DOUBLE), VALUE :: dt
  END FUNCTION
  ! one slab per MPI rank: the caller moves the packed device buffers
  ! (CUDA-aware MPI_Sendrecv, or NCCL) between neighbouring ranks
  INTEGER(C_INT) FUNCTION cumc_slab_seam(h, side) BIND(C, NAME='cumc_slab_seam')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: side
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_halo_bytes(h, fill, side, nbytes) BIND(C, NAME='cumc_slab_halo_bytes')
    IMPORT :: C_INT, C_PTR, C_SIZE_T
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: fill, side
    INTEGER(C_SIZE_T), INTENT(OUT) :: nbytes
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_halo_pack(h, fill, side, buf) BIND(C, NAME='cumc_slab_halo_pack')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h, buf
    INTEGER(C_INT), VALUE :: fill, side
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_halo_unpack(h, fill, side, buf) BIND(C, NAME='cumc_slab_halo_unpack')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h, buf
    INTEGER(C_INT), VALUE :: fill, side
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_initial_begin(h) BIND(C, NAME='cumc_slab_initial_begin')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_initial_end(h) BIND(C, NAME='cumc_slab_initial_end')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_step_begin(h, dt) BIND(C, NAME='cumc_slab_step_begin')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), VALUE :: dt
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_stage(h, stage, part) BIND(C, NAME='cumc_slab_stage')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: stage, part
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_slab_step_end(h) BIND(C, NAME='cumc_slab_step_end')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  ! output snapshots (the datasets of print_hydroprofile)
  INTEGER(C_INT) FUNCTION cumc_snapshot_start(h, primitive, epsilon, bfield) BIND(C, NAME='cumc_snapshot_start')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: primitive(*), epsilon(*), bfield(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_snapshot_wait(h) BIND(C, NAME='cumc_snapshot_wait')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  ! the collapsar model's black hole
  INTEGER(C_INT) FUNCTION cumc_collapsar_set(h, m_bh, c_code) BIND(C, NAME='cumc_collapsar_set')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), VALUE :: m_bh, c_code
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_collapsar_get(h, m_bh, r_sh) BIND(C, NAME='cumc_collapsar_get')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    REAL(C_DOUBLE), INTENT(OUT) :: m_bh, r_sh
  END FUNCTION
  ! arrays, synchronisation, stream, counters
  INTEGER(C_INT) FUNCTION cumc_get_array(h, which, out, n_doubles) BIND(C, NAME='cumc_get_array')
    IMPORT :: C_INT, C_PTR, C_DOUBLE, C_SIZE_T
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: which
    REAL(C_DOUBLE), INTENT(OUT) :: out(*)
    INTEGER(C_SIZE_T), VALUE :: n_doubles
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_sync(h) BIND(C, NAME='cumc_sync')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  INTEGER(C_INT64_T) FUNCTION cumc_launch_count(h) BIND(C, NAME='cumc_launch_count')
    IMPORT :: C_INT64_T, C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  TYPE(C_PTR) FUNCTION cumc_stream(h) BIND(C, NAME='cumc_stream')
    IMPORT :: C_PTR
    TYPE(C_PTR), VALUE :: h
  END FUNCTION
  ! diagnostics, autotuner, numerics self-checks
  INTEGER(C_INT) FUNCTION cumc_profile_step(h, nsteps, ms_out, n_out) BIND(C, NAME='cumc_profile_step')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: nsteps, n_out
    REAL(C_DOUBLE), INTENT(OUT) :: ms_out(*)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_autotune(h, choice_out, best_ms_out) BIND(C, NAME='cumc_autotune')
    IMPORT :: C_INT, C_PTR, C_DOUBLE
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), INTENT(OUT) :: choice_out(5)
    REAL(C_DOUBLE), INTENT(OUT) :: best_ms_out
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_set_tuning(h, choice) BIND(C, NAME='cumc_set_tuning')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), INTENT(IN) :: choice(5)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_set_concurrent_sweeps(h, on) BIND(C, NAME='cumc_set_concurrent_sweeps')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: on
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_fallback_count(h, enable, count_out) BIND(C, NAME='cumc_fallback_count')
    IMPORT :: C_INT, C_PTR, C_LONG_LONG
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: enable
    INTEGER(C_LONG_LONG), INTENT(OUT) :: count_out
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_check_dv(seed, n, mismatches, example) BIND(C, NAME='cumc_check_dv')
    IMPORT :: C_INT, C_LONG_LONG, C_DOUBLE
    INTEGER(C_LONG_LONG), VALUE :: seed, n
    INTEGER(C_LONG_LONG) :: mismatches
    REAL(C_DOUBLE) :: example(2)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_check_div3(seed, n, mismatches, example) BIND(C, NAME='cumc_check_div3')
    IMPORT :: C_INT, C_LONG_LONG, C_DOUBLE
    INTEGER(C_LONG_LONG), VALUE :: seed, n
    INTEGER(C_LONG_LONG), INTENT(OUT) :: mismatches
    REAL(C_DOUBLE), INTENT(OUT) :: example
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_fp64_peak(tflops) BIND(C, NAME='cumc_fp64_peak')
    IMPORT :: C_INT, C_DOUBLE
    REAL(C_DOUBLE), INTENT(OUT) :: tflops
  END FUNCTION
  ! batched 1D problems: synchronisation, stream, counter
  INTEGER(C_INT) FUNCTION cumc_batch_sync(b) BIND(C, NAME='cumc_batch_sync')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: b
  END FUNCTION
  TYPE(C_PTR) FUNCTION cumc_batch_last_error(b) BIND(C, NAME='cumc_batch_last_error')
    IMPORT :: C_PTR
    TYPE(C_PTR), VALUE :: b
  END FUNCTION
  TYPE(C_PTR) FUNCTION cumc_batch_stream(b) BIND(C, NAME='cumc_batch_stream')
    IMPORT :: C_PTR
    TYPE(C_PTR), VALUE :: b
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_batch_set_cluster(b, cluster_size, coop_min_n) BIND(C, NAME='cumc_batch_set_cluster')
    IMPORT :: C_INT, C_PTR
    TYPE(C_PTR), VALUE :: b
    INTEGER(C_INT), VALUE :: cluster_size, coop_min_n
  END FUNCTION
  INTEGER(C_INT64_T) FUNCTION cumc_batch_launch_count(b) BIND(C, NAME='cumc_batch_launch_count')
    IMPORT :: C_INT64_T, C_PTR
    TYPE(C_PTR), VALUE :: b
  END FUNCTION
  ! one 1D problem with no device allocation (hosts that own all device
  ! memory, e.g. an OpenACC code whose arrays are mapped once); err holds
  ! the message of a failed call
  INTEGER(C_INT) FUNCTION cumc_batch_run1_noalloc(cfg, prim, eps, max_steps, stream, prim_row, eps_row, &
      t_out, steps_out, status_out, err, err_len) BIND(C, NAME='cumc_batch_run1_noalloc')
    IMPORT :: C_INT, C_PTR, C_DOUBLE, C_CHAR, C_SIZE_T, cumc_batch_config
    TYPE(cumc_batch_config), INTENT(IN) :: cfg
    REAL(C_DOUBLE), INTENT(IN) :: prim(*), eps(*)
    INTEGER(C_INT), VALUE :: max_steps
    TYPE(C_PTR), VALUE :: stream
    REAL(C_DOUBLE), INTENT(OUT) :: prim_row(*), eps_row(*)
    REAL(C_DOUBLE), INTENT(OUT) :: t_out
    INTEGER(C_INT), INTENT(OUT) :: steps_out, status_out
    CHARACTER(KIND=C_CHAR), INTENT(OUT) :: err(*)
    INTEGER(C_SIZE_T), VALUE :: err_len
  END FUNCTION
  ! learned flag: counters, flag maps, sample harvest, network kernels
  INTEGER(C_INT) FUNCTION cumc_learn_stats(h, out4) BIND(C, NAME='cumc_learn_stats')
    IMPORT :: C_INT, C_PTR, C_LONG_LONG
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_LONG_LONG), INTENT(OUT) :: out4(4)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_learn_flags(h, dir, flags, warps, tiles, sizes_out) BIND(C, NAME='cumc_learn_flags')
    IMPORT :: C_INT, C_PTR, C_LONG_LONG
    TYPE(C_PTR), VALUE :: h, flags, warps, tiles
    INTEGER(C_INT), VALUE :: dir
    INTEGER(C_LONG_LONG), INTENT(OUT) :: sizes_out(3)
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_learn_harvest(h, dir, stride, out, cap, rows_out) BIND(C, NAME='cumc_learn_harvest')
    IMPORT :: C_INT, C_PTR, C_LONG_LONG, C_FLOAT
    TYPE(C_PTR), VALUE :: h
    INTEGER(C_INT), VALUE :: dir
    INTEGER(C_LONG_LONG), VALUE :: stride, cap
    REAL(C_FLOAT), INTENT(OUT) :: out(*)
    INTEGER(C_LONG_LONG), INTENT(OUT) :: rows_out
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_mlp_grad(params, samples, n, delta, grad_out, loss_out) BIND(C, NAME='cumc_mlp_grad')
    IMPORT :: C_INT, C_LONG_LONG, C_FLOAT
    REAL(C_FLOAT), INTENT(IN) :: params(*), samples(*)
    INTEGER(C_LONG_LONG), VALUE :: n
    REAL(C_FLOAT), VALUE :: delta
    REAL(C_FLOAT), INTENT(OUT) :: grad_out(*), loss_out
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_mlp_train(samples, n, tc, params_inout, loss_curve) BIND(C, NAME='cumc_mlp_train')
    IMPORT :: C_INT, C_LONG_LONG, C_FLOAT, C_PTR, cumc_train_config
    REAL(C_FLOAT), INTENT(IN) :: samples(*)
    INTEGER(C_LONG_LONG), VALUE :: n
    TYPE(cumc_train_config), INTENT(IN) :: tc
    REAL(C_FLOAT), INTENT(INOUT) :: params_inout(*)
    TYPE(C_PTR), VALUE :: loss_curve      ! REAL(C_FLOAT) per step, or C_NULL_PTR
  END FUNCTION
  INTEGER(C_INT) FUNCTION cumc_mlp_infer(params, features, ld, n, logits) BIND(C, NAME='cumc_mlp_infer')
    IMPORT :: C_INT, C_LONG_LONG, C_FLOAT
    REAL(C_FLOAT), INTENT(IN) :: params(*), features(*)
    INTEGER(C_INT), VALUE :: ld
    INTEGER(C_LONG_LONG), VALUE :: n
    REAL(C_FLOAT), INTENT(OUT) :: logits(*)
  END FUNCTION
  TYPE(C_PTR) FUNCTION cumc_mlp_last_error() BIND(C, NAME='cumc_mlp_last_error')
    IMPORT :: C_PTR
  END FUNCTION
END INTERFACE

TYPE(C_PTR), SAVE :: cumc_h = C_NULL_PTR

CONTAINS

  ! STOP with the engine's message, as the reference STOPs on bad setup
  SUBROUTINE CUMC_CHECK(rc)
    INTEGER(C_INT), INTENT(IN) :: rc
    CHARACTER(KIND=C_CHAR), POINTER :: msg(:)
    INTEGER :: n
    IF (rc /= CUMC_OK) THEN
      CALL C_F_POINTER(cumc_last_error(cumc_h), msg, [512])
      n = 0
      DO WHILE (n < 512)
        IF (msg(n + 1) == C_NULL_CHAR) EXIT
        n = n + 1
      END DO
      WRITE(*,*) 'cumc3d_gpu error ', rc, ': ', msg(1:n)
      STOP 'cumc3d_gpu'
    END IF
  END SUBROUTINE
END MODULE CUMC_GPU
