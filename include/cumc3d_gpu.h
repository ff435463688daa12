/*
 * cumc3d_gpu.h -- C-ABI of the B200 (sm_100a) finite-volume MHD stage engine.
 *
 * This is the drop-in boundary for the per-timestep update of CUMC3D
 * (leon-astrophy/cumc3d, solver/mhd).  The reference's Fortran main loop
 *
 *     CALL initial_update                      (solver/mhd/initial.f90:86-116)
 *     DO while (global_time < total_time)      (solver/mhd/main.f90:98-139)
 *        CALL finddt                           (solver/mhd/rungekutta.f90:221-332)
 *        IF (global_time + dt > total_time) dt = total_time - global_time
 *        CALL rungekutta(n_step)               (solver/mhd/rungekutta.f90:12-208)
 *     END DO
 *
 * becomes a sequence of calls on one opaque handle.  Every entry point is a
 * plain C function taking plain pointers and sizes; nothing here depends on
 * PyTorch or on CUDA headers.  All calls return 0 on success and a non-zero
 * CUMC_E* code on failure; cumc_last_error() gives the message.  A handle
 * owns its device buffers and one CUDA stream, and must not be shared between
 * host threads.  There is no CPU fallback: when no CUDA device is present
 * cumc_create fails with CUMC_ECUDA.
 *
 * Array layout exchanged with the host is the reference's Fortran layout:
 *   prim(imin:imax, -2:nx+3, -2:ny+3, -2:nz+3)   column-major, imax = 8
 *   epsilon(-2:nx+3, -2:ny+3, -2:nz+3)
 * i.e. a flat double array with the variable index fastest, then x, y, z.
 * Variable order is (rho, vx, vy, vz, p, Bx_face, By_face, Bz_face) as set up
 * by SETUP_EQNS (solver/mhd/setup.f90:39-90).
 */
#ifndef CUMC3D_GPU_H
#define CUMC3D_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------- status codes ---------------- */
#define CUMC_OK          0
#define CUMC_EINVAL      1   /* bad argument or unsupported configuration      */
#define CUMC_ECUDA       2   /* CUDA runtime error / no device                 */
#define CUMC_ENOMEM      3   /* device allocation failed                       */
#define CUMC_ESTATE      4   /* non-finite or non-positive state found (guard) */
#define CUMC_ENOTREADY   5   /* call order violated (e.g. step before state)   */

/* ---------------- option enums ---------------- */
/* reconstruction, solver/mhd/parameter.h:102-115 */
#define CUMC_RECON_TVD_MM 0
#define CUMC_RECON_TVD_VL 1
#define CUMC_RECON_TVD_MC 2
#define CUMC_RECON_PPM    3
#define CUMC_RECON_WENO   4
/* Riemann solver, solver/mhd/parameter.h:90-100 */
#define CUMC_RS_LF   0
#define CUMC_RS_HLL  1
#define CUMC_RS_HLLC 2
#define CUMC_RS_HLLD 3
/* arithmetic form */
#define CUMC_FP64 0   /* plain: FP64 end to end                                  */
#define CUMC_FP32 1   /* FP32 reconstruction + Riemann flux, FP64 elsewhere      */
/* per-stage floors (CUSTOM_CHECKRHO + FINDPRESSURE of the model) */
#define CUMC_FLOOR_NONE  0
#define CUMC_FLOOR_EPS   1   /* model/riemann/src/custom.f90:103-127          */
#define CUMC_FLOOR_TORUS 2   /* model/torus-cyn/src/custom.f90:240-275,
                                model/torus-cyn/src/findpressure.f90:7-37    */
#define CUMC_FLOOR_COLLAPSAR 3 /* model/collapsar/src/custom.f90:269-330: the
                                atmosphere prim_a = (rho_floor, v = 0, eps_floor)
                                blended in below it; ideal-gas FINDPRESSURE
                                (model/collapsar/src/findpressure.f90)         */
/* model source terms (CUSTOM_SOURCE) */
#define CUMC_SRC_NONE     0
#define CUMC_SRC_CONST_GY 1  /* model/riemann/src/custom.f90:132-159          */
#define CUMC_SRC_PM_CYL   2  /* model/torus-cyn/src/custom.f90:280-320        */
#define CUMC_SRC_PM_SPH   3  /* model/torus-sph/src/custom.f90 (radial form)  */
#define CUMC_SRC_COLLAPSAR 4 /* model/collapsar/src/custom.f90:340-395: gravity of
                                the potential of cumc_poisson_* plus the black
                                hole m_bh/(r - r_sh)^2; the hole's mass grows
                                each stage by the inner-face mass flux
                                (custom.f90:450-478, cumc_collapsar_set)       */
/* model boundary hooks (CUSTOM_BOUNDARY_X/Y/Z) */
/* boundary_flag value of a z side shared with a neighbouring slab (no
 * counterpart in the reference): its ghost planes come from the neighbour
 * (cumc_group_*) instead of a boundary rule */
#define CUMC_BOUNDARY_EXCHANGE 9
#define CUMC_BC_NONE      0
#define CUMC_BC_TORUS_CYL 1  /* model/torus-cyn/src/custom.f90:146-208        */
#define CUMC_BC_TORUS_SPH 2  /* model/torus-sph/src/custom.f90 (x clamp only) */

/* Model descriptor: replaces the per-stage device hooks each reference model
 * links in (EOS, floors, sources, custom boundaries). */
typedef struct cumc_model {
    double gamma;        /* ggas: ideal-gas adiabatic index                       */
    int    floor_kind;   /* CUMC_FLOOR_*                                          */
    double rho_floor;    /* torus floor: rho_floor, eps_floor, p_floor            */
    double eps_floor;
    double p_floor;
    int    source_kind;  /* CUMC_SRC_*                                            */
    double g_const;      /* constant gravity magnitude for CUMC_SRC_CONST_GY (0.1) */
    double r_sh;         /* pseudo-Newtonian radius for point-mass gravity        */
    int    bc_kind;      /* CUMC_BC_*                                             */
} cumc_model;

/* Solver configuration: the compile-time PARAMETERs of solver/mhd/parameter.h
 * moved to run time, plus the face coordinates CUSTOM_GRID/GETGRID produce. */
typedef struct cumc_config {
    int nx, ny, nz;              /* interior zones (ny = nz = 1 for 1D)           */
    int n_dim;                   /* 1, 2 or 3                                     */
    int coordinate_flag;         /* 0 Cartesian, 1 cylindrical, 2 spherical       */
    int boundary_flag[6];        /* xin xout yin yout zin zout: 0 periodic,
                                    1 outflow, 2 reflect, 3 axis, 4 equator;
                                    zin/zout may be CUMC_BOUNDARY_EXCHANGE (a
                                    slab of a z-decomposed grid, cumc_group_*)  */
    const double *xF;            /* face coordinates, indices -3..nx+3 (nx+7)     */
    const double *yF;            /* indices -3..ny+3 (ny+7)                       */
    const double *zF;            /* indices -3..nz+3 (nz+7)                       */
    double cfl;                  /* Courant number                                */
    int recon;                   /* CUMC_RECON_*                                  */
    int riemann;                 /* CUMC_RS_*                                     */
    int precision;               /* CUMC_FP64 / CUMC_FP32                         */
    int learned;                 /* 1: learned smooth-face flag in WENO (FP32 form)*/
    int fixpole;                 /* -DFIXPOLE: axis EMF average (spherical only)  */
    int fix_periodic_normal_faces; /* 0 = reference behaviour: a periodic
                                    direction's face 0 keeps its initial normal
                                    field (boundary.f90 never fills it);
                                    1 = face 0 follows face n                     */
    int positivity_fallback;     /* 0 = reference behaviour; 1 = a cell whose
                                    reconstructed edge density or pressure is not
                                    positive falls back to first order (no
                                    counterpart in the reference)                 */
    cumc_model model;
} cumc_config;

typedef struct cumc_handle cumc_handle;

/* ---------------- lifecycle ----------------
 * cumc_create replaces BUILD_HYDRO/BUILD_MHD/BUILD_RIEMANN/GETGRID/{TVD,PPM,WENO}_WEIGHT
 * and POPULATE_DEVICE (solver/mhd/initial.f90:7-78, setup.f90:340-395,
 * getgrid.f90:13-168, openacc.f90:5-24).  Boundary-flag combinations the
 * reference rejects with STOP (setup.f90:111-325) return CUMC_EINVAL. */
int cumc_create(const cumc_config *cfg, cumc_handle **out);
/* replaces CLEAR_DEVICE (solver/mhd/openacc.f90:30-47) */
int cumc_destroy(cumc_handle *h);

/* Upload/download the primitive state in the Fortran layout described above.
 * set_state is what GET_MODEL leaves behind (solver/mhd/initial.f90:68-74);
 * get_state is the !$ACC UPDATE HOST(prim, epsilon) of dataio.f90:25-27. */
int cumc_set_state(cumc_handle *h, const double *prim, const double *eps);
int cumc_get_state(cumc_handle *h, double *prim, double *eps);

/* Download one internal array in Fortran layout (diagnostics and tests).
 * which: 0 cons(8,...), 1 bcell(3,...), 2 cs(...), 3 u_old(8,...) */
#define CUMC_ARR_CONS  0
#define CUMC_ARR_BCELL 1
#define CUMC_ARR_CS    2
int cumc_get_array(cumc_handle *h, int which, double *out, size_t n_doubles);

/* INITIAL_UPDATE: CUSTOM_CHECKRHO -> FROMRVETOU -> BOUNDARY -> UPDATE(0)
 * (solver/mhd/initial.f90:86-116). */
int cumc_initial_update(cumc_handle *h);

/* FINDDT (solver/mhd/rungekutta.f90:221-332): CFL step, min-reduced on the
 * device.  Copies dt back to the host. */
int cumc_finddt(cumc_handle *h, double *dt);

/* RUNGEKUTTA (solver/mhd/rungekutta.f90:12-208) with the given dt. */
int cumc_rk3_step(cumc_handle *h, double dt);

/* The main loop of solver/mhd/main.f90:98-139 on the device: repeat
 * FINDDT, clamp to t_end, RUNGEKUTTA, t += dt, until t >= t_end or
 * max_steps steps were taken.  dt never leaves the device; steps are
 * replayed from a captured CUDA graph.  *t_inout is the simulation time
 * before and after; *steps_out the number of steps taken. */
int cumc_evolve(cumc_handle *h, double t_end, int max_steps,
                double *t_inout, int *steps_out);

/* FIND_DIVB (solver/mhd/mhd_module.f90:110-201): max |div B| over the
 * interior from the face fields. */
int cumc_max_divb(cumc_handle *h, double *max_divb);

/* Synchronise the handle's stream (for timing). */
int cumc_sync(cumc_handle *h);

/* Number of kernel launches the handle issued since creation. */
int64_t cumc_launch_count(cumc_handle *h);

/* The handle's CUDA stream (a cudaStream_t), so callers can order their own
 * work and timing events after the engine's. */
void *cumc_stream(cumc_handle *h);

/* Diagnostics (no counterpart in the reference, which only has -DDEBUG
 * system_clock prints, e.g. solver/mhd/rungekutta.f90:22-29): run nsteps
 * eager steps with CUDA events around each kernel class and return the summed
 * milliseconds in ms_out[0..7] = flux_x, flux_y, flux_z, emf (cell/face/edge
 * EMFs and their ghosts), rk (du/dt + stage combination), recover (prim/cons
 * recovery + floors + EOS), boundary (ghost fill), dt (CFL reduction). */
int cumc_profile_step(cumc_handle *h, int nsteps, double *ms_out, int n_out);

/* Autotuner (no counterpart in the reference): times the candidate launch
 * shapes of the face-flux kernels (fused or split recon/Riemann, threads per
 * block, register budget of the Riemann kernel) on the handle's live state and
 * keeps the fastest for all later steps.  choice_out[0..4] = (split?, recon
 * threads/block, Riemann threads/block, Riemann min blocks/SM (1, 4, 5, 6; 14,
 * 15, 16 = the kernel that prefetches its next face's states into shared
 * memory with asynchronous copies, at 4, 5, 6 blocks/SM), staged
 * reconstruction: 0 = per-cell loads, 1 or 2 = stencils staged in shared
 * memory with that many cells per thread, 3 = tiles staged by TMA
 * (persistent, double-buffered; FP64 plain form with an even padded x
 * extent), 4 = as 1 at 64 registers per thread); best_ms_out = the flux time
 * of one stage with that choice.  Either pointer may be NULL. */
int cumc_autotune(cumc_handle *h, int *choice_out, double *best_ms_out);

/* Set the launch shape by hand, same five integers as choice_out above. */
int cumc_set_tuning(cumc_handle *h, const int *choice);

/* on = 1: each stage's three face-flux sweeps (reconstruction + Riemann
 * per direction) run as concurrent branches -- sweeps y and z on streams of
 * their own with their own face-state buffers (14 more arrays of the padded
 * grid each), joined before the EMFs; results are bit-identical either way.
 * Not used with the learned flag or while cumc_profile_step records. */
int cumc_set_concurrent_sweeps(cumc_handle *h, int on);

/* Positivity-fallback counter (no counterpart in the reference, which has no
 * fallback): enable = 1 starts counting from zero the cells whose
 * reconstruction took the optional first-order fallback (one count per cell
 * per sweep and stage); enable = 0 stops counting; enable = -1 leaves the
 * state as it is.  count_out (may be NULL) receives the count so far (the
 * call synchronises the handle's stream).  Counting costs one atomic per
 * fallback cell and nothing otherwise. */
int cumc_fallback_count(cumc_handle *h, int enable, unsigned long long *count_out);

/* Numerics self-check (no counterpart in the reference): compares the FP64
 * engine's FMA-corrected division by 3 with the IEEE quotient on n generated
 * normal inputs; *mismatches counts differing bit patterns. */
int cumc_check_div3(unsigned long long seed, long long n, unsigned long long *mismatches, double *example);

/* Numerics self-check (no counterpart in the reference): compares the FP64
 * engine's division (the IEEE quotient with a shortcut for a zero numerator)
 * with x / y on n generated pairs, zeros, infinities, NaNs and subnormals
 * among them; *mismatches counts differing results (any NaN equals any NaN),
 * example[0..1] = one differing pair. */
int cumc_check_dv(unsigned long long seed, long long n, unsigned long long *mismatches, double *example);

/* Measured FP64 fused-multiply-add throughput of the current device in
 * TFLOP/s (the denominator of the FP64-pipe roofline). */
int cumc_fp64_peak(double *tflops);

/* ---------------- batched 1D problems ----------------
 * Many independent 1D MHD problems of uneven size (the reference's n_dim = 1
 * build, one problem per run, solver/mhd/main.f90) advanced in ONE persistent
 * launch: each CTA runs INITIAL_UPDATE and the whole time loop of one problem
 * (own dt, own t_end, own step count) before taking the next, largest first.
 * Scope: Cartesian 1D, outflow boundaries on every side (the reference's 1D
 * Riemann tests, model/riemann/src/riemann1d.f90), ideal gas, no sources;
 * results are bit-identical to running each problem through cumc_create with
 * ny = nz = 1. */
typedef struct cumc_batch_config {
    int n_problems;
    const int *nx;               /* zones per problem                            */
    const double *const *xF;     /* per problem: face coordinates -3..nx+3       */
    const double *t_end;         /* per problem total_time                        */
    double cfl, gamma;
    int recon, riemann, precision;
    int floor_kind;              /* CUMC_FLOOR_NONE or CUMC_FLOOR_EPS            */
    int positivity_fallback;
} cumc_batch_config;
typedef struct cumc_batch cumc_batch;
int cumc_batch_create(const cumc_batch_config *cfg, cumc_batch **out);
int cumc_batch_destroy(cumc_batch *b);
/* prim(8, -2:nx+3, -2:4, -2:4) and epsilon(-2:nx+3, -2:4, -2:4) of problem p
 * in the reference's 1D layout (GET_MODEL output) */
int cumc_batch_set_state(cumc_batch *b, int p, const double *prim, const double *eps);
/* prim(8, -2:nx+3) and epsilon(-2:nx+3) of the (k,l) = (1,1) row of problem p */
int cumc_batch_get_state(cumc_batch *b, int p, double *prim_row, double *eps_row);
/* INITIAL_UPDATE + the time loop of every problem, one launch.  Per problem:
 * t_out = time reached, steps_out = steps taken, status_out = 0 or CUMC_ESTATE. */
int cumc_batch_run(cumc_batch *b, int max_steps, double *t_out, int *steps_out, int *status_out);
/* Launch shape of the next runs (no reference counterpart): problems of more
 * than coop_min_n cells are shared by a thread-block cluster of cluster_size
 * CTAs (1, 2, 4, 8 or 16; 16 is a non-portable size and falls back to one
 * CTA per problem where the device cannot place it), smaller ones run one
 * per CTA.  Defaults: 8, and 1024 for batches larger than the clusters the
 * device holds at once, 256 for smaller ones (whose problems then get a
 * cluster each).  Results do not depend on it. */
int cumc_batch_set_cluster(cumc_batch *b, int cluster_size, int coop_min_n);
int cumc_batch_sync(cumc_batch *b);
void *cumc_batch_stream(cumc_batch *b);
/* Number of kernel launches the batch issued since creation (one per
 * cumc_batch_run). */
int64_t cumc_batch_launch_count(cumc_batch *b);
const char *cumc_batch_last_error(cumc_batch *b);

/* ---------------- learned smooth-face flag (WENO, FP32 or FP64 form) ----------------
 * No reference counterpart: the reference always applies the WENO-Z
 * nonlinear weights (solver/mhd/weno_module.f90:363-404).  A 35-32-32-1 MLP
 * over scale-free stencil features flags cells whose WENO-Z face values are
 * within a tolerance of the linear optimal-weight fifth-order values; warps
 * of 32 flagged cells reconstruct with the linear weights.  Inference is
 * fused into the reconstruction kernel (BF16 tcgen05 MMA, FP32 accumulators
 * in tensor memory); every audit_interval steps a full WENO-Z audit marks
 * 128-cell tiles whose flagged cells are off by more than audit_tol to fall
 * back to WENO-Z until the next audit.
 * Parameters: float[CUMC_LEARN_NP] = W1[32][48] (out, in; inputs 35..47
 * unused), b1[32], W2[32][32], b2[32], w3[32], b3.
 * Samples: rows of CUMC_LEARN_ROW floats = 35 features, the relative
 * face-value change the linear weights make (FP64 WENO-Z of the plain
 * method), the largest nonlinear-weight deviation |omega_k - g_k|. */
#define CUMC_LEARN_NP   2657
#define CUMC_LEARN_NF   35
#define CUMC_LEARN_ROW  37
typedef struct cumc_train_config {
    int steps, batch;            /* Adam steps, samples per step               */
    float lr, delta;             /* learning rate; label: change < delta       */
    float beta1, beta2, eps;     /* Adam (0: 0.9, 0.999, 1e-8)                 */
    unsigned long long seed;     /* minibatch sampling                         */
} cumc_train_config;
/* enable (params != NULL) or disable the flag on a handle created with
 * learned = 1 (WENO; FP32 form: the network is fused into the FP32
 * reconstruction of its stage; FP64 form: the network only sets the flags
 * and the FP64 reconstruction reads them; with no cell flagged the FP64 form
 * is bit-identical to the plain form); resets the fallback tiles and the
 * counters.  Audits are taken on refresh steps: set audit_interval to a
 * multiple of flag_interval.
 * The network runs at stage 1 of every flag_interval-th step (>= 1); the
 * other stages reuse its flags, dilated by two cells along the sweep. */
int cumc_learn_set(cumc_handle *h, const float *params, float threshold, int flag_interval, int audit_interval,
                   float audit_tol);
/* audit counters: cells audited, cells flagged, tiles set to fall back, audits */
int cumc_learn_stats(cumc_handle *h, unsigned long long *out4);
/* ---------------- self-gravity potential of the collapsar model ----------------
 * Red-black successive over-relaxation of the Poisson equation on the
 * handle's spherical grid (coordinate_flag 2), as CUSTOM_UPDATE of the
 * collapsar model does it (model/collapsar/src/custom.f90:489-620; the
 * coefficients are POISSON_COEF, model/collapsar/src/poisson.f90:34-64).
 * phi lives on cells 0..n+1 of each axis.
 *
 * cumc_poisson_setup: computes the coefficients once (GET_POISSON,
 * poisson.f90:6-27), sets phi = 0 everywhere (the initial model's guess,
 * custom.f90:498-507).  rho_atm = the atmosphere density prim_a(irho): cells
 * at or below it carry no mass in the source; omega = omega_weight (1.9 in
 * the reference's def.f90).  CUMC_EINVAL for a non-spherical grid. */
int cumc_poisson_setup(cumc_handle *h, double rho_atm, double omega);
/* The relaxation loop (custom.f90:511-620) from the current phi, with the
 * density of the handle's current state: per iteration the red cells
 * ((-1)**(j+k+l) > 0), the black cells, the ghost layers (phi(0) = phi(1),
 * phi(nx+1) = -1, copies along theta, periodic along phi) and the test
 * max |dphi / phi_old| <= tol over the interior.  iters_out = iterations
 * taken, err_out = that maximum at the last one, converged_out = 1 if it
 * reached tol, 0 if max_iter ran out (where the reference STOPs).  An error
 * that is NaN (0/0 where phi stays exactly zero) counts as not converged. */
int cumc_poisson_solve(cumc_handle *h, int max_iter, double tol, int *iters_out, double *err_out,
                       int *converged_out);
/* phi (nx+2)*(ny+2)*(nz+2) doubles, j fastest, j,k,l = 0..n+1: read it back,
 * or set it (a warm start, or a restart from a checkpoint). */
int cumc_poisson_get(cumc_handle *h, double *phi);
int cumc_poisson_set(cumc_handle *h, const double *phi);

/* z-slab groups (the multi-GPU layout of the 3D path; no counterpart in the
 * reference, which runs one grid on one device).  A grid cut along z into
 * n >= 2 slabs, one handle per slab in z order, created with the slab's z
 * faces (its cells plus three ghost faces per side) and
 * boundary_flag[4]/[5] = CUMC_BOUNDARY_EXCHANGE on every side shared with a
 * neighbour (both ends too for a periodic z axis: the slabs form a ring).
 * The handles may live on different GPUs of this process (each created with
 * its GPU current); the ghost planes travel between them as contiguous
 * peer copies into the receiver's memory, twice per RK stage.  The group's
 * state equals the undivided grid's bit for bit.  Steps run host-driven
 * (no cumc_evolve); not with the learned flag, the collapsar source or
 * FIXPOLE, which need the whole grid at once.
 * cumc_group_initial_update: INITIAL_UPDATE on every slab, ghosts exchanged;
 * cumc_group_finddt: FINDDT, the minimum over the slabs;
 * cumc_group_step: one SSP-RK3 step of every slab. */
int cumc_group_initial_update(cumc_handle **slabs, int n);
int cumc_group_finddt(cumc_handle **slabs, int n, double *dt);
int cumc_group_step(cumc_handle **slabs, int n, double dt);

/* One slab per process (one rank per GPU; no counterpart in the reference).
 * The same slabs, stage split and ghost planes as cumc_group_*, with the
 * planes carried by the caller: at each exchange point pack the three
 * planes next to every exchanged z side into a contiguous device buffer,
 * send it to that side's neighbour (NCCL send/recv, or a host-staged copy),
 * and unpack what the neighbour sent into the side's ghost planes.  A
 * buffer packed at side s is unpacked by the neighbour at side 1 - s; both
 * ends of one cut agree on its size.  Everything is ordered on the handle's
 * stream (cumc_stream): a transport that runs on another stream orders
 * itself after the pack and before the unpack.  One step of a slab:
 *
 *   cumc_finddt ; the minimum over the ranks ; cumc_slab_step_begin(dt)
 *   for stage 1..3:
 *     cumc_slab_stage(stage, 0) ; exchange CUMC_FILL_EMF
 *     cumc_slab_stage(stage, 1) ; exchange CUMC_FILL_STATE
 *   cumc_slab_step_end
 *
 * and INITIAL_UPDATE: cumc_slab_initial_begin ; exchange CUMC_FILL_STATE ;
 * cumc_slab_initial_end.  For a periodic z axis the two end sides of the
 * ring are the whole grid's periodic boundary: mark them with
 * cumc_slab_seam (the first slab's side 0, the last slab's side 1) before
 * cumc_slab_initial_begin.  The ranks' states equal the undivided grid's bit
 * for bit.  Not with the learned flag, the collapsar source or FIXPOLE. */
#define CUMC_FILL_STATE 0  /* the state fill that ends a stage (BOUNDARY)         */
#define CUMC_FILL_EMF   1  /* the EMF fill inside a stage (BOUNDARY_EFIELD)       */
int cumc_slab_seam(cumc_handle *h, int side);
int cumc_slab_halo_bytes(cumc_handle *h, int fill, int side, size_t *bytes);
int cumc_slab_halo_pack(cumc_handle *h, int fill, int side, void *device_buffer);
int cumc_slab_halo_unpack(cumc_handle *h, int fill, int side, const void *device_buffer);
int cumc_slab_initial_begin(cumc_handle *h);
int cumc_slab_initial_end(cumc_handle *h);
int cumc_slab_step_begin(cumc_handle *h, double dt);
int cumc_slab_stage(cumc_handle *h, int stage, int part);
int cumc_slab_step_end(cumc_handle *h);

/* Output snapshot without stalling the step loop (print_hydroprofile,
 * solver/mhd/dataio.f90:31-240, which updates the host copy and writes HDF5).
 * cumc_snapshot_start packs the state as the reference writes it --
 * primitive = prim(1:5, 0:nx+1, 0:ny+1, 0:nz+1) (5*(nx+2)*(ny+2)*(nz+2)
 * doubles), epsilon = epsilon(0:nx+1, 0:ny+1, 0:nz+1), bfield =
 * prim(ibx:ibz, -1:nx+1, -1:ny+1, -1:nz+1) (3*(nx+3)*(ny+3)*(nz+3)), all in
 * Fortran order -- into a device buffer, after the steps already issued, and
 * copies it to the three host buffers on a separate stream; steps issued
 * afterwards run meanwhile and do not change the snapshot.  The buffers may
 * not be read or freed until cumc_snapshot_wait returns.  Page-locked
 * buffers (cudaHostAlloc) make the copy asynchronous; with pageable ones
 * start returns after the copy.  One snapshot in flight per handle (start
 * waits for the previous one). */
int cumc_snapshot_start(cumc_handle *h, double *primitive, double *epsilon, double *bfield);
int cumc_snapshot_wait(cumc_handle *h);

/* The collapsar model's black hole (model/collapsar/src/custom.f90:450-485),
 * for a spherical handle with source_kind CUMC_SRC_COLLAPSAR: its mass m_bh
 * and the speed of light in code units c_code (clight * vel2code), so that
 * r_sh = 2 m_bh / c_code^2.  After every RK stage the mass grows by
 * dt * max(mdot, 0), mdot = the inner-face mass flux summed over the sphere
 * (-flux(irho,0,k,l) xF(0)^2 dcose(k) dz(l)), combined with the stage's
 * Shu-Osher weights.  A horizon reaching the inner face (r_sh >= xF(0)) ends
 * the step with CUMC_ESTATE (the reference STOPs).  The sum's order is
 * fixed (1024 strided partial sums in sequence, then a pairwise tree); the
 * reference's OpenMP reduction leaves it unspecified. */
int cumc_collapsar_set(cumc_handle *h, double m_bh, double c_code);
int cumc_collapsar_get(cumc_handle *h, double *m_bh, double *r_sh);

/* For inspection (no counterpart in the reference): the learned-flag state of
 * sweep dir as the last refresh left it.  flags = one byte per cell of the
 * sweep's enumeration (x fastest; cells 0..n+1 along the sweep, interior
 * across it), warps = the linear decision of each warp of the staged
 * reconstruction (32 consecutive x-cells of one row), tiles = the per
 * 128-cell fallback marks.  sizes_out[0..2] receives the three byte counts;
 * any of the buffers may be NULL to ask for the sizes only. */
int cumc_learn_flags(cumc_handle *h, int dir, unsigned char *flags, unsigned char *warps, unsigned char *tiles,
                     long long *sizes_out);
/* samples of every stride-th interior cell of the current state, sweep dir */
int cumc_learn_harvest(cumc_handle *h, int dir, long long stride, float *out, long long cap, long long *rows_out);
/* mean loss and gradient over n samples (FP32, deterministic order) */
int cumc_mlp_grad(const float *params, const float *samples, long long n, float delta, float *grad_out,
                  float *loss_out);
/* Adam training on the GPU; params in/out, loss per step (may be NULL) */
int cumc_mlp_train(const float *samples, long long n, const cumc_train_config *tc, float *params_inout,
                   float *loss_curve);
/* logits of n feature rows (leading dimension ld >= 35) on the tensor cores */
int cumc_mlp_infer(const float *params, const float *features, int ld, long long n, float *logits);
const char *cumc_mlp_last_error(void);

/* cumc_batch_run1_noalloc -- NO REFERENCE COUNTERPART (an addition of this
 * library; the reference allocates its arrays itself at start-up).
 * One problem of the batched 1D engine, run without any device allocation:
 * every device buffer comes from one static array per device (about 3.5 MB)
 * instead of cudaMalloc, and nothing is freed.  For host programs that own
 * all device memory and let no library allocate: a Fortran/OpenACC code that
 * maps its arrays once and sizes its pool to what remains, or a time loop that
 * must not call cudaMalloc/cudaFree because they can synchronise the device
 * and stall the host's other streams.
 *   cfg        n_problems must be 1; nx[0] <= 4096, else CUMC_EINVAL ("at most
 *              4096 zones without allocation") before any device work;
 *   prim, eps  host, the reference's 1D layout as for cumc_batch_set_state;
 *   stream     cudaStream_t to run on (NULL: the default stream); the call
 *              returns after synchronising it;
 *   prim_row, eps_row  host outputs as for cumc_batch_get_state;
 *   t_out, steps_out, status_out  as for cumc_batch_run (may be NULL);
 *   err, err_len  optional buffer for the failure message.
 * Every call looks up the static array's address in the current context
 * (cudaGetSymbolAddress), so an address never goes stale after a
 * cudaDeviceReset; the first call on each device, with that device current,
 * (and the first after a reset) loads the module: make it before any stream
 * capture.  A CUDA error already pending on the calling thread is returned
 * as CUMC_ECUDA before any device work.  Each call clears the whole static
 * array before use.  Calls that overlap in time on one device share the
 * static array and race: serialise them.  Results equal
 * cumc_batch_create/_set_state/_run/_get_state on the same single problem. */
int cumc_batch_run1_noalloc(const cumc_batch_config *cfg, const double *prim, const double *eps, int max_steps,
                            void *stream, double *prim_row, double *eps_row, double *t_out, int *steps_out,
                            int *status_out, char *err, size_t err_len);

/* Message of the last failed call on this handle (or of the last failed
 * cumc_create when h is NULL). */
const char *cumc_last_error(cumc_handle *h);

#ifdef __cplusplus
}
#endif
#endif /* CUMC3D_GPU_H */
