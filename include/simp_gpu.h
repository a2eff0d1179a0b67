/*
 * simp_gpu.h — C ABI of the B200 (sm_100a) implementation of SIMP's per-step
 * Smoothed Particle Hydrodynamics hot path.
 *
 * SIMP's Fortran host talks to its physics through argument-less subroutines
 * that read and write module globals (fortran/src/modules/data_variables.f90:
 * 26-124).  This library keeps those globals resident on the GPU between calls
 * and exposes one entry point per reference subroutine on the path, with plain
 * pointers and sizes only, so an ISO_C_BINDING interface block can bind them
 * directly (see fortran/shim/simp_gpu_mod.f90 in this repository).
 *
 * Conventions shared by every entry point:
 *   - Return value: SIMP_OK (0) or one of the SIMP_ERR_* codes below.  The
 *     reference STOPs with a banner on the same conditions; here the caller
 *     gets the code plus the banner text from simp_gpu_last_error().
 *   - Host arrays use the reference's Fortran layout: a 2-vector field such as
 *     x(dim, maxn) is interleaved [x1, y1, x2, y2, ...] (column-major), scalar
 *     fields are double[n].  Pair indices are 1-based like p_i/p_j.
 *   - All arithmetic is IEEE FP64 unless the context was created with
 *     precision = SIMP_PREC_MIXED (FP32 pair sums with Kahan compensation,
 *     FP64 positions, integrator state and reductions).
 *   - A context is bound to one CUDA stream and is not thread-safe; the
 *     reference calls single_step from one thread (time_integration.f90:204).
 *   - The library owns all device memory; host arrays stay the caller's.
 */
#ifndef SIMP_GPU_H
#define SIMP_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define SIMP_API __attribute__((visibility("default")))
#else
#define SIMP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------- */
enum {
    SIMP_OK = 0,
    SIMP_ERR_BADARG = 1,    /* unsupported switch, null pointer, bad size      */
    SIMP_ERR_MAXN = 2,      /* ntotal > maxn: initialize.f90:156-163           */
    SIMP_ERR_PAIR_CAP = 3,  /* too many pairs: nnps.f90:132-139, 415-423       */
    SIMP_ERR_IND_INT = 4,   /* > max_ind_int interactions: nnps.f90:660-668    */
    SIMP_ERR_CUDA = 5,      /* CUDA runtime error (message in last_error)      */
    SIMP_ERR_NONFINITE = 6, /* NaN/Inf in the state after a step               */
    SIMP_ERR_TIMEOUT = 7,   /* a bounded device-side wait gave up              */
    SIMP_ERR_NOMEM = 8,     /* device allocation failed                        */
    SIMP_ERR_STATE = 9,     /* entry point called before simp_gpu_set_state    */
    SIMP_ERR_BOUNDS = 10,   /* a device index check failed (only the checked
                               debug build, libsimp_gpu_checked.so, checks)  */
    SIMP_ERR_CANCELLED = 11 /* a served request was cancelled (simp_serve.h)  */
};

/* Smoothing kernel selector: the reference's skf codes (globals.f90:136-147,
 * kernel.f90:20-45, boundary_kernel.f90:20-45); scale_h as in
 * initialize.f90:208-217. */
enum {
    SIMP_SKF_QUADRATIC = 1,   /* kernel.f90:241-290, scale_h 2                       */
    SIMP_SKF_GAUSSIAN = 2,    /* kernel.f90:108-157, scale_h 3                       */
    SIMP_SKF_QUINTIC = 3,     /* kernel.f90:165-233, scale_h 3                       */
    SIMP_SKF_WENDLAND_C2 = 4, /* kernel.f90:359-408, scale_h 1                       */
    SIMP_SKF_WENDLAND_C4 = 5, /* kernel.f90:415-464, scale_h 1                       */
    SIMP_SKF_WENDLAND_C6 = 6, /* kernel.f90:471-520, boundary_kernel.f90:438-504    */
    SIMP_SKF_MARQUIS = 7,     /* kernel.f90:527-576, scale_h 3; walls: Gaussian      */
    SIMP_SKF_MARQUIS2 = 8,    /* kernel.f90:583-633, scale_h 3; walls: Gaussian      */
    SIMP_SKF_CUBIC = 9        /* kernel.f90:297-352 (commented out in the
                                 reference, restored here with scale_h = 2)          */
};

enum { SIMP_PREC_FP64 = 0, SIMP_PREC_MIXED = 1 };
enum { SIMP_WIND_UNIFORM = 0, SIMP_WIND_VORTEX = 1 };

/*
 * Every switch and constant the hot path reads.  The reference holds these as
 * compile-time PARAMETERs (globals.f90:58-187, data_variables.f90:153-180);
 * simp_params_reference_default() fills in the shipped values.
 */
typedef struct simp_params {
    /* algorithm switches, reference codes */
    int32_t int_algorithm;     /* 1 Euler, 2 predictor-corrector, 3 leap-frog
                                  (time_integration.f90:86-148, 155-282, 289-391)     */
    int32_t nnps_algorithm;    /* 2 bucket search, 1 direct find (nnps.f90:21-30)       */
    int32_t sle;               /* 0 keep hsml, 1 Benz hsml, 2 Marquis hsml
                                  (smoothing_length.f90:24-30)                          */
    int32_t tse;               /* 0 keep dt, 1 Monaghan (time_step.f90:40-124, its CFL
                                  criterion with the artificial-viscosity form when
                                  artificial_visc), 2 VP criterion (:132-157)         */
    int32_t rheology;          /* 1 elliptical yield curve, 2 Mohr-Coulomb
                                  (bulk_viscosity.f90, shear_viscosity.f90)           */
    int32_t eos_alg;           /* 1 Hibler, 2 Gutfraind, 3 Kreyscher (eos.f90)         */
    int32_t pa_sph;            /* 1 (s_i/rho_i^2 + s_j/rho_j^2) stress_1,
                                  2 (s_i + s_j)/rho_j stress_2 (internal_stress.f90)  */
    int32_t skf;               /* SIMP_SKF_*                                            */
    int32_t den_alg;           /* density.f90:20-30 in the step: 3 diagnostic,
                                  2 continuity (con_density), 1 summation (sum_density
                                  with the reference's kept kernel_zero array;
                                  simp_gpu_sum_density is the sum alone, with W(0)
                                  at each particle's own hsml)                         */
    int32_t bfa;               /* boundary force (boundary_force.f90:20-27): 1 Monaghan,
                                  2 Wang (needs simp_gpu_set_wall_normals), 3 Marquis  */
    int32_t viscosity;         /* globals.f90:180-187 logical switches (0/1)            */
    int32_t pressure_force;
    int32_t wind_force;
    int32_t water_force;
    int32_t boundary_pressure;
    int32_t boundary_friction; /* friction branch of the boundary force                */
    int32_t mass_from_area;    /* 1: mass_update_from_area when sle is 0 or 1 (as the
                                  reference); 0: particle mass held constant         */
    int32_t max_ind_int;       /* 200 (globals.f90:24)                                 */
    int32_t hsml_multiplicity; /* 3 (data_variables.f90:105)                           */
    int32_t wind_kind;         /* SIMP_WIND_*                                          */
    int32_t precision;         /* SIMP_PREC_*                                          */
    int32_t reserved0;
    /* material constants */
    double P_star, c_eos, e, delta_min, k_t;
    double rho_ice, rho_air, rho_water, c_wind, c_water;
    double b_length, kappa_n, kappa_t;
    double alpha;              /* area factor of mass_update_from_area                 */
    /* forcing */
    double wind_u, wind_v;     /* uniform wind (m/s)                                   */
    double current_u, current_v;
    double vortex_x, vortex_y, vortex_umax, vortex_radius;
    /* numerics */
    double dt;                 /* fixed (tse = 0) or initial time step (s)             */
    double max_hsml;           /* Marquis_hsml cap; <= 0: 10 * max(hsml) at set_state
                                  (initialize.f90:191)                                */
    double skin;               /* GPU cell-list skin (m); < 0: automatic               */
    /* Mohr-Coulomb rheology (data_variables.f90:153-180): viscosity caps per unit
       pressure (declared without a value in the reference, so 0 there) and the
       friction angle phi (degrees; mu = tan(phi)) */
    double zeta_max, eta_max, phi;
    /* boundary friction (data_variables.f90:157-158, 175): friction coefficient
       xi of bf_Wang, Young modulus Y and Poisson ratio nu of the sound speed
       c_yang used by bf_Monaghan's friction term */
    double xi, Y, nu;
    /* regularisation (sph/regularization.f90), called by single_step when
       xsph_regularization or artificial_visc is on (single_step.f90:99-101);
       it then applies the artificial viscosity of art_visc_alg whichever of
       the two switches is on (regularization.f90:29-35), as the reference
       does.  The pair terms are evaluated per pair: a pair outside the
       viscosity criterion contributes nothing, and the XSPH term is
       antisymmetric (x_i gets m_j (v_i - v_j), x_j gets m_i (v_j - v_i)). */
    int32_t artificial_visc;     /* globals.f90:180-187 (0/1)                    */
    int32_t xsph_regularization; /* globals.f90:180-187 (0/1)                    */
    int32_t art_visc_alg;        /* 1 Hernquist-Katz (regularization.f90:102-213),
                                    2 Monaghan (:220-308); globals.f90:103      */
    int32_t reserved1;
    double alpha_pi, beta_pi;    /* artificial viscosity coefficients
                                    (data_variables.f90:171-172)               */
    double chi;                  /* XSPH coefficient (data_variables.f90:173)   */
} simp_params;

/* Shipped values of globals.f90 and data_variables.f90, including the
 * reference's default-real literals (rho_air = 1.3 is stored as the
 * single-precision value 1.2999999523162842). */
SIMP_API void simp_params_reference_default(simp_params *p);

typedef struct simp_ctx simp_ctx;

/* Allocate device storage for up to maxn particles and maxnb boundary
 * particles (the reference's maxn / maxnb capacities, globals.f90:21-25). */
SIMP_API int32_t simp_gpu_create(const simp_params *params, int32_t maxn, int32_t maxnb,
                        simp_ctx **out);
SIMP_API int32_t simp_gpu_destroy(simp_ctx *ctx);

/* Upload the particle and boundary state (the globals initialize.f90:
 * particle_placing / boundary_placing_1 produce).  x and vx are interleaved
 * 2*ntotal arrays, xb is 2*ntotalb.  dt and current_time are the
 * integrator's.  Returns SIMP_ERR_MAXN when ntotal > maxn. */
SIMP_API int32_t simp_gpu_set_state(simp_ctx *ctx, int32_t ntotal, const double *x,
                           const double *vx, const double *mass,
                           const double *rho, const double *hsml,
                           const double *A, const double *h, int32_t ntotalb,
                           const double *xb, const double *massb, double dt,
                           double current_time);

/* Download the state in the caller's original particle order.  Any pointer
 * may be NULL to skip that field.  After simp_gpu_step without outputs it
 * also returns those steps' status (the state is written either way). */
SIMP_API int32_t simp_gpu_get_state(simp_ctx *ctx, double *x, double *vx, double *mass,
                           double *rho, double *hsml, double *A, double *h,
                           double *dt, double *current_time);

/* Diagnostics of the last kinematic pass (the globals epsilon_11..sigma_22,
 * zeta, eta, p after single_step).  Only valid when diagnostics were kept:
 * single_step always keeps them; simp_gpu_step keeps them when
 * simp_gpu_keep_diag(ctx, 1) was called. */
SIMP_API int32_t simp_gpu_keep_diag(simp_ctx *ctx, int32_t keep);
SIMP_API int32_t simp_gpu_get_diag(simp_ctx *ctx, double *eps11, double *eps12,
                          double *eps22, double *zeta, double *eta, double *p,
                          double *sig11, double *sig12, double *sig22);

/* NNPS (nnps.f90:5-30 -> bucket_search :155-517).  Emits the unordered pair
 * set with the reference's bucket-search semantics, sorted by (p_i, p_j) with
 * p_i < p_j, 1-based original indices.  r_ij and hsml_ij are bit-exact FP64.
 * Boundary pairs are (bp_i = boundary index, bp_j = particle index) sorted by
 * (bp_i, bp_j).  nip / bnip always receive the true counts; when they exceed
 * cap / bcap the arrays hold the first cap / bcap entries and
 * SIMP_ERR_PAIR_CAP is returned.  Any array pointer may be NULL. */
SIMP_API int32_t simp_gpu_nnps(simp_ctx *ctx, int32_t *nip, int32_t *p_i, int32_t *p_j,
                      double *r_ij, double *hsml_ij, int32_t cap,
                      int32_t *bnip, int32_t *bp_i, int32_t *bp_j,
                      double *br_ij, int32_t bcap);

/* One right-hand-side evaluation, single_step.f90:5-109, on the resident
 * state at the given current_time (drag is off while current_time <= 0,
 * wind_forcing.f90:35).  Outputs are interleaved 2*ntotal (dxdt, dvxdt) or
 * ntotal (dhdt, dAdt) in the original particle order; any may be NULL. */
SIMP_API int32_t simp_gpu_single_step(simp_ctx *ctx, double current_time, double *dxdt,
                             double *dvxdt, double *dhdt, double *dAdt);

/* Density pair sum, density.f90:41-100 (sum_density), on the resident state:
 * rho_out[i] = (k0_i m_i + sum_j m_j W_ij) / (k0_i m_i / rho_i +
 * sum_j m_j W_ij / rho_j), k0_i = W(0) with hsml_i. */
SIMP_API int32_t simp_gpu_sum_density(simp_ctx *ctx, double *rho_out);

/* Advance nsteps predictor-corrector steps (time_integration.f90:146-181 with
 * predictor_corrector :263-390), state resident on the device.  On return
 * *current_time and *dt hold the integrator's values; current_time advances
 * by the dt computed at the end of each step, as the reference does
 * (time_integration.f90:179).  With current_time and dt both NULL (single-
 * basin contexts) the call returns once the steps are enqueued, without
 * waiting for them: the next simp_gpu_get_state returns their status, and
 * the next simp_gpu_step, simp_gpu_single_step or simp_gpu_nnps waits for
 * them and returns it before doing anything else; simp_gpu_set_state drops
 * it (the new state replaces theirs). */
SIMP_API int32_t simp_gpu_step(simp_ctx *ctx, int32_t nsteps, double *current_time,
                      double *dt);

/* Interaction statistics of the last NNPS (nnps.f90:613-670): maximal,
 * minimal and summed per-particle interaction counts (boundary pairs
 * included) and the number of particles without interactions. */
SIMP_API int32_t simp_gpu_interaction_stats(simp_ctx *ctx, int32_t *maxip,
                                   int32_t *minip, int64_t *sumip,
                                   int32_t *noip);

/* ---- batches of basins ---------------------------------------------------
 * A batch context holds up to max_instances independent basins (instances)
 * of different sizes and forcings, resident together and advanced together
 * by simp_gpu_step: every kernel of a step covers all instances in one
 * launch.  Each instance has its own cell grid and its own current_time; all
 * share the context's simp_params (physics, fixed dt: tse = 0, fixed hsml:
 * sle = 0).  An instance's results do not depend on which other instances
 * share the batch.  No reference counterpart (the reference runs one basin
 * per process). */
typedef struct simp_forcing {
    int32_t wind_kind;         /* SIMP_WIND_*                                   */
    int32_t reserved0;
    double wind_u, wind_v;     /* uniform wind (m/s)                            */
    double vortex_x, vortex_y, vortex_umax, vortex_radius;
} simp_forcing;

/* Unit normals of the walls of a single-basin context, b_normal(2, ntotalb)
 * in the order of set_state's xb (data_variables.f90:46, set with the walls
 * by boundaries.f90:232-287, pointing into the ice).  Read by the Wang
 * boundary force (bfa = 2, boundary_force.f90:146-172), which refuses to run
 * without them.  A new set_state clears them. */
SIMP_API int32_t simp_gpu_set_wall_normals(simp_ctx *ctx, int32_t ntotalb, const double *b_normal);

/* Forcing of a single-basin context (the wind fields of its simp_params),
 * used from the next simp_gpu_set_state on and by the basin already set.
 * The reference hard-codes its wind (wind_forcing.f90:36-37). */
SIMP_API int32_t simp_gpu_set_forcing(simp_ctx *ctx, const simp_forcing *forcing);

/* maxn / maxnb: particle and wall capacities over all instances; at most
 * 2,097,151 particles per instance; max_instances <= 1024. */
SIMP_API int32_t simp_gpu_create_batch(const simp_params *params, int32_t maxn, int32_t maxnb,
                                       int32_t max_instances, simp_ctx **out);
/* Admits one basin (arrays as in simp_gpu_set_state; its current_time starts
 * at 0) into a free slot, returned in *slot.  SIMP_ERR_MAXN when the
 * capacities or the slots are exhausted. */
SIMP_API int32_t simp_gpu_batch_add(simp_ctx *ctx, const simp_forcing *forcing, int32_t ntotal,
                                    const double *x, const double *vx, const double *mass,
                                    const double *rho, const double *hsml, const double *A,
                                    const double *h, int32_t ntotalb, const double *xb,
                                    const double *massb, int32_t *slot);
/* Retires a basin and frees its slot and storage. */
SIMP_API int32_t simp_gpu_batch_remove(simp_ctx *ctx, int32_t slot);
/* State of one basin in its own particle order (pointers may be NULL). */
SIMP_API int32_t simp_gpu_batch_get_state(simp_ctx *ctx, int32_t slot, double *x, double *vx,
                                          double *mass, double *rho, double *hsml, double *A,
                                          double *h, double *current_time);
/* Particles, steps advanced and status flags (bit 0: non-finite) of a slot;
 * *ntotal = 0 for a free slot.  In a batch, a basin whose state turns
 * non-finite only sets its flag: simp_gpu_step keeps advancing the batch
 * and the caller retires that basin. */
SIMP_API int32_t simp_gpu_batch_info(simp_ctx *ctx, int32_t slot, int32_t *ntotal,
                                     int64_t *steps, int32_t *flags);

/* Summation density (the same result as simp_gpu_sum_density) for callers
 * that cannot allocate device memory.  No counterpart in the reference: it
 * exists for hosts whose device memory belongs to another runtime (CUDA
 * Fortran or OpenACC device arrays, a framework's caching allocator) and for
 * loops that may not stall on cudaMalloc, which can synchronise the device.
 *   x       device, 2*n interleaved positions   hsml, mass, rho: device, n
 *   rho_out device, n (original order)          skf: SIMP_SKF_*
 *   stream  cudaStream_t to run on (NULL: the legacy default stream)
 * The buffers must be device memory of the current device or managed
 * memory; host arrays are refused with SIMP_ERR_BADARG.
 * It calls no cudaMalloc, cudaFree or allocating library routine: its cell
 * list lives in one fixed array inside the library (about 7 MB, held on
 * every GPU that loads the library until the process exits).  n must be at
 * most SIMP_NOALLOC_MAX_PARTICLES, else SIMP_ERR_BADARG.  The first call on
 * each device (and the first after another CUDA context became current on
 * it) looks up that array's device address, so make it before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race
 * and must be serialised by the caller.  An error left by earlier work on
 * the calling thread is reported as SIMP_ERR_CUDA before anything is
 * launched.  Asynchronous: returns after enqueueing on stream. */
#define SIMP_NOALLOC_MAX_PARTICLES 65536
SIMP_API int32_t simp_gpu_sum_density_noalloc(const double *x, const double *hsml,
                                              const double *mass, const double *rho,
                                              int32_t n, int32_t skf, double *rho_out,
                                              void *stream);

/* The CUDA stream (cudaStream_t) every kernel of this context runs on, for
 * event timing and interop.  No reference counterpart (the reference has no
 * device). */
SIMP_API void *simp_gpu_stream(simp_ctx *ctx);

/* Implementation of the two pair passes (no reference counterpart):
 * SIMP_PASSES_TILED stages chunks of `threads` consecutive particles of a
 * cell row with their cell halo (at most `cap` particles) in shared memory;
 * the gather forms gather every particle's neighbours from HBM over Verlet
 * lists, with the kinematic pass as one kernel (SIMP_PASSES_GATHER_ONE) or
 * as two, pair finding then pair sums over the stored pair list
 * (SIMP_PASSES_GATHER_TWO); SIMP_PASSES_GATHER (the default) takes two
 * kernels for contexts of up to 400,000 particles, else one.
 * All give the same bits.  threads: 64..256, a multiple of 32; cap: a
 * multiple of 4, within the shared memory of one block (both checked for
 * every form). */
#define SIMP_PASSES_GATHER 0
#define SIMP_PASSES_TILED 1
#define SIMP_PASSES_GATHER_ONE 2
#define SIMP_PASSES_GATHER_TWO 3
SIMP_API int32_t simp_gpu_set_passes(simp_ctx *ctx, int32_t impl, int32_t threads, int32_t cap);
SIMP_API int32_t simp_gpu_get_passes(const simp_ctx *ctx, int32_t *impl, int32_t *threads, int32_t *cap);
/* Times one right-hand side (both passes, no state change) of the current
 * state under a set of implementations and tile shapes, `reps` times each,
 * and keeps the fastest.  *ms_best: its time per right-hand side. */
SIMP_API int32_t simp_gpu_autotune(simp_ctx *ctx, int32_t reps, double *ms_best);

/* Number of kernels this context has launched so far (graph replays count
 * each captured kernel).  No reference counterpart. */
SIMP_API int64_t simp_gpu_kernel_launches(const simp_ctx *ctx);

/* Per-kernel timing of simp_gpu_step: when on, CUDA events recorded inside
 * the step graph time each kernel of every step; simp_gpu_kernel_times then
 * returns, for the n_kernels kernels of a step (kinematic, stress-predict,
 * kinematic, stress-correct, step-finish) and, as a sixth entry, the
 * re-sorts between steps, the summed milliseconds and the number of steps
 * timed.  No reference counterpart. */
SIMP_API int32_t simp_gpu_profile(simp_ctx *ctx, int32_t on);
SIMP_API int32_t simp_gpu_kernel_times(simp_ctx *ctx, double *ms, int32_t n_kernels,
                                       int64_t *steps_timed);

/* ---- snapshot files -------------------------------------------------------
 * The reference's output files, in its formats (in_out/output.f90:61-78):
 *   particle_momentum.csv  " i , x/1000 , y/1000 , 100 vx , 100 vy"  (1x,I7,4(1x,A1,1x,e15.8E3))
 *   particle_state.csv     " i , mass , p , hsml , A , h , eps11 , eps12 , eps22 ,
 *                           sig11 , sig12 , sig22"                   (1x,I7,11(1x,A1,1x,e15.8E3))
 *   particle_other.csv     " ntotal , ntotalb , current_time/3600"   (1x,2(I7,1x,A1,1x),e15.8E3)
 *   boundary_particles.csv " j , xb/1000 , yb/1000 , massb"          (1x,I5,3(1x,A1,1x,e14.8))
 * `folder` is a directory path (with or without the trailing '/'). */

/* Creates the three particle files empty (initialize.f90:83-95). */
SIMP_API int32_t simp_csv_create_output(const char *folder);
/* Appends one snapshot of a single-basin context, as `output` does: its
 * state and the diagnostics of the last right-hand side that kept them
 * (simp_gpu_single_step, or simp_gpu_step after simp_gpu_keep_diag). */
SIMP_API int32_t simp_gpu_write_output(simp_ctx *ctx, const char *folder);
/* The same from host arrays (x, vx interleaved as x(2, ntotal)). */
SIMP_API int32_t simp_csv_append_snapshot(const char *folder, int32_t ntotal, int32_t ntotalb,
                                          double current_time, const double *x, const double *vx,
                                          const double *mass, const double *p, const double *hsml,
                                          const double *A, const double *h, const double *eps11,
                                          const double *eps12, const double *eps22, const double *sig11,
                                          const double *sig12, const double *sig22);
/* Writes boundary_particles.csv (boundaries.f90:52-63). */
SIMP_API int32_t simp_csv_write_walls(const char *folder, int32_t ntotalb, const double *xb,
                                      const double *massb);
/* Spin-up reader (replaces particle_reading, initialize.f90:234-330, which
 * reads 14 columns per state record where output writes 11, and only the
 * first snapshot).  Reads snapshot `snapshot` (0-based; negative counts
 * from the last, -1 = the last) in SI units (x in m, vx in m/s,
 * current_time in s).  With every array null it only returns the sizes;
 * more than `cap` particles is SIMP_ERR_MAXN, like the reference's STOP.
 * rho is not in the files: with the diagnostic density it is h rho_ice. */
SIMP_API int32_t simp_csv_read_snapshot(const char *folder, int32_t snapshot, int32_t cap,
                                        int32_t *ntotal, int32_t *ntotalb, double *current_time,
                                        double *x, double *vx, double *mass, double *p, double *hsml,
                                        double *A, double *h);
/* Reads boundary_particles.csv (boundary_reading, boundaries.f90:119-160;
 * all walls converted to m, where the reference converts the first ntotal). */
SIMP_API int32_t simp_csv_read_walls(const char *folder, int32_t cap, int32_t *ntotalb, double *xb,
                                     double *massb);
/* Text of the last error of the simp_csv_* calls on this thread. */
SIMP_API const char *simp_csv_last_error(void);

/* Human-readable text of the last error on this context ("" if none). */
SIMP_API const char *simp_gpu_last_error(const simp_ctx *ctx);

/* Library version string. */
SIMP_API const char *simp_gpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* SIMP_GPU_H */
