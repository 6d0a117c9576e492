/*
 * pandora_gpu.h -- C-ABI of the B200 (sm_100a) RK3 time step of the PANDORA 2.0
 * pseudo-spectral DNS code.
 *
 * Plain C, no C++ or CUDA types.  Every entry point returns an int status
 * (PANDORA_OK == 0, negative on error; pandora_strerror() names it).  The
 * state that the reference keeps module-global (the f_arrays PETSc Vecs, the
 * p_arrays particle arrays, bmat/binv in g_domain) lives in one handle, on one
 * GPU, in HBM.  One handle per host thread; calls on one handle are not
 * re-entrant; different handles are independent.
 *
 * Layout at the boundary is the reference's truncated spectral layout
 * arr_u*_3w(0:1, k=0..2KK, j=0..2KJ, i=0..KI) (src/pf_arrays.f90:267-280):
 * in C order [i][j][k][re,im], k fastest, KI = NODES_X/3, KJ = NODES_Y/3,
 * KK = NODES_Z/3 (integer division, src/pg_domain.f90:220-231).  Negative
 * wavenumbers sit at indices KJ+1..2KJ (resp. KK+1..2KK) and map to
 * index-(2K+1) (src/pf_arrays.f90:1770-1804).  FP64 always at the boundary.
 */
#ifndef PANDORA_GPU_H
#define PANDORA_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (MPI_Abort sites of the reference become return codes) ---- */
#define PANDORA_OK                 0
#define PANDORA_ERR_INVALID_ARG   -1   /* bad pointer, size or parameter value      */
#define PANDORA_ERR_OOM           -2   /* device allocation failed / budget exceeded */
#define PANDORA_ERR_CUDA          -3   /* a CUDA runtime call failed                 */
#define PANDORA_ERR_NAN           -4   /* non-finite value detected in the state     */
#define PANDORA_ERR_TIMEOUT       -5   /* a bounded device wait gave up              */
#define PANDORA_ERR_BAD_LAYOUT    -6   /* size not supported by the transform plan   */
#define PANDORA_ERR_CFL           -7   /* RK3_CFL >= 1 (src/pg_rk3.f90:240-267)      */
#define PANDORA_ERR_PARTICLE_LOST -8   /* wrap left a particle outside the domain
                                          (src/pp_control.f90:1514-1518)             */
#define PANDORA_ERR_NO_DEVICE     -9   /* no CUDA device / extension not usable      */
#define PANDORA_ERR_UNSUPPORTED  -10   /* option not built in this library           */

/* ---- enum values, identical to src/pg_parameters.f90 ---- */
#define PANDORA_F_ISOTROPIC          1   /* pg_parameters.f90:131 */
#define PANDORA_F_SHEAR_DNS          2   /* pg_parameters.f90:132 */
#define PANDORA_F_ISOTROPIC_DEFORMED 5   /* pg_parameters.f90:135 */
#define PANDORA_RK3_TIMESTEP_DECIDE  1   /* pg_parameters.f90:211 */
#define PANDORA_RK3_TIMESTEP_FIXED   2   /* pg_parameters.f90:212 */
#define PANDORA_RK3_TIMESTEP_CFL     3   /* pg_parameters.f90:213 */
#define PANDORA_NS_BF_ROT            1   /* pg_parameters.f90:219 */
#define PANDORA_NS_R_CONV            2   /* pg_parameters.f90:220, convective Rogallo form */
#define PANDORA_NS_R_ROT             3   /* pg_parameters.f90:221, rotational Rogallo form */
#define PANDORA_DEALIASING_23        1   /* 2/3 rule (cube truncation), pg_parameters.f90:224 */
#define PANDORA_DEALIASING_SPHERICAL 2   /* 2/3 sphere |k_lab| <= KMAX, pg_parameters.f90:225 */
#define PANDORA_DEALIASING_LES       3   /* |k_lab| <= LES_CUTOFF * KMAX, pg_parameters.f90:226 */
#define PANDORA_F_INIT_NULL          0   /* pg_parameters.f90:150 */
#define PANDORA_F_INIT_GAUSS         3
#define PANDORA_F_INIT_KERR          4
#define PANDORA_F_INIT_PULSE         5
#define PANDORA_F_INIT_SQUARE        6
#define PANDORA_F_INIT_MINUSFIVETHIRD 8
#define PANDORA_F_INIT_MATSUMOTO     9
#define PANDORA_F_INIT_AHMED_ELGHOBASHI 10
#define PANDORA_P_INIT_RANDOM        2   /* pg_parameters.f90:236 */
#define PANDORA_PREC_FP64            0
/* FP32-mixed form (no counterpart in the reference, which is FP64 throughout): fields,
 * transforms and the nonlinear term in FP32; twiddles generated in long double, the
 * clock, the Rogallo frame B(t), the remesh, the forcing coefficients, the per-mode
 * RHS/RK3 arithmetic, the particles and the E(k)/epsilon shell sums in FP64.  Every
 * boundary call still takes and returns FP64 arrays. */
#define PANDORA_PREC_FP32_MIXED      1
/* Viscous term of the RK3 step (pandora_params.rk3_viscous).  EXPLICIT is the
 * reference's: -F_NU k^2 u inside the right-hand side of every stage
 * (src/pf_rk3.f90:2388-2390, combined at 2471).  INTEGRATING_FACTOR has no
 * counterpart in the reference: the low-storage RK3 runs on v = exp(F_NU k^2 t) u,
 * which with u and the register kept in physical units reads, per stage s,
 *   r_s = E_s (beta_s r_{s-1} + N(u_{s-1})),  u_s = E_s u_{s-1} + gamma_s dt r_s,
 *   E_s = exp(-F_NU k^2 (c_{s+1} - c_s) dt),  c = 0, 1/3, 3/4, 1,
 * N the right-hand side without the viscous term; the exponent is formed in FP64 in
 * both precisions.  Isotropic flow only (the wavenumbers of the sheared frame move
 * with time); other flow types return PANDORA_ERR_UNSUPPORTED. */
#define PANDORA_VISCOUS_EXPLICIT     0
#define PANDORA_VISCOUS_INTEGRATING_FACTOR 1

/*
 * Namelist fields of ip_file.in that the RK3 step reads (src/pg_control.f90:385-436),
 * mirrored one-to-one.  Seeds replace RANDOM_SEED_FLUID / RANDOM_SEED_PARTICLES:
 * the reference draws from gfortran's random_number, which cannot be replayed here,
 * so this library defines one counter-based generator (SplitMix64 finaliser over a
 * stream index) that the oracle shares; draw ORDER follows the reference.
 */
typedef struct pandora_params {
    /* nl_domain */
    int32_t nodes_x, nodes_y, nodes_z;
    int32_t b110, b220, b330;
    /* nl_fluid */
    double  f_rho, f_nu;
    /* nl_flow */
    int32_t f_type;
    double  f_deform_s;
    int32_t f_remesh_t;
    /* nl_numerics */
    int32_t rk3_timestep;
    double  rk3_cfl, rk3_dt;
    int32_t ns_deformed;
    int32_t dealiasing;
    /* nl_control */
    int32_t tsteps;
    /* nl_f_init */
    int32_t f_init_type;
    double  f_init_u0, f_init_kp, f_init_kv;
    double  f_init_kstart, f_init_kend, f_init_epsilon;
    /* nl_force */
    double  force_tf, force_sigma, force_kf;
    int32_t force_stop;
    /* nl_particle / nl_part_properties */
    int32_t p_track_part;
    int32_t p_init_type;
    int64_t p_np_global;    /* at most 2^31 - 1 (the per-step spatial sort counts in 32 bits) */
    int32_t p_interp_order;
    int32_t p_ts_release;
    double  p_rho;
    double  p_dia_vals;     /* single diameter level (P_DIA_LVLS = 1); 0 => tracers */
    /* random seeds (see above) */
    uint64_t seed_fluid, seed_force, seed_particles;
    /* arithmetic of the step: PANDORA_PREC_FP64 or PANDORA_PREC_FP32_MIXED */
    int32_t precision;
    /* viscous term: PANDORA_VISCOUS_EXPLICIT (0, the reference's) or
     * PANDORA_VISCOUS_INTEGRATING_FACTOR (1) */
    int32_t rk3_viscous;
    /* nl_numerics LES_CUTOFF: cutoff of DEALIASING = 3 as a multiple of KMAX */
    double  les_cutoff;
    /* schedule of the x pass (no counterpart in the reference; results do not depend on
     * it): x lines per warp, 1, 2 or 4 for x lengths of at most 64 points (0: the
     * library's choice for the length); other lengths take 0 or 1 */
    int32_t x_lines_per_warp;
    int32_t reserved[3];
} pandora_params;

typedef struct pandora_handle pandora_handle;

/* Fills *p with the defaults of conf/ip_file.in for the fields above. */
int pandora_params_default(pandora_params* p);

/* Library / device queries.  pandora_params_sizeof() lets a binding check its
 * mirror of the struct layout (ctypes, iso_c_binding). */
const char* pandora_strerror(int status);
int pandora_params_sizeof(void);
int pandora_device_count(int* count);

/* Sizes of the truncated spectral layout: NKI = KI+1, NKJ = 2KJ+1, NKK = 2KK+1;
 * S = NKI*NKJ*NKK complex modes per component; kkmax = number of E(k) shells
 * (src/pf_fluidstats.f90:348-374). */
int pandora_sizes(const pandora_params* p, int32_t* nki, int32_t* nkj, int32_t* nkk,
                  int64_t* modes, int32_t* kkmax);

/*
 * Allocates the device state for one simulation on the current CUDA device
 * (replaces ProgramInit's f_ArraysInit/f_FftwInit/f_ForceInit,
 * src/pg_control.f90:52-146).  The state starts at zero.
 */
int pandora_create(const pandora_params* p, pandora_handle** out);
int pandora_destroy(pandora_handle* h);

/* Runs all of this handle's work on a caller-owned cudaStream_t (NULL: the
 * handle's own stream). */
int pandora_set_stream(pandora_handle* h, void* cuda_stream);

/* ---- state in / out (host buffers, reference layout, synchronous) ---- */
int pandora_set_state(pandora_handle* h, const double* u1, const double* u2, const double* u3);
int pandora_get_state(pandora_handle* h, double* u1, double* u2, double* u3);
/* RK3 low-storage registers rk3_3w_1..3 (src/pf_arrays.f90:67-72). */
int pandora_set_rk(pandora_handle* h, const double* r1, const double* r2, const double* r3);
int pandora_get_rk(pandora_handle* h, double* r1, double* r2, double* r3);
/* OU forcing coefficients fluid_f1..3(0:1,-NK:NK,-NK:NK,0:NK) as [i][j][k][2]
 * (src/pf_force.f90:289-300); n = 3 * (NK+1)*(2NK+1)^2 * 2 doubles in total. */
int pandora_forcing_size(pandora_handle* h, int64_t* ndoubles_per_component);
int pandora_set_forcing(pandora_handle* h, const double* f1, const double* f2, const double* f3);
int pandora_get_forcing(pandora_handle* h, double* f1, double* f2, double* f3);
/* Device pointers of u1..u3 (for zero-copy users; valid until destroy), in the
 * stored precision: double2 [i][j][k] (FP64 form) or float2 (FP32-mixed form). */
int pandora_state_device_ptrs(pandora_handle* h, void** u1, void** u2, void** u3);

/* Seeded solenoidal initial field, f_InitialiseFluid (src/pf_initialise.f90:97-512),
 * computed on the device. */
int pandora_init_fluid(pandora_handle* h);

/* ---- particles (p_arrays, src/pp_arrays.f90:92-429), SoA-free host view:
 *      xp[3*np] = (x1,x2,x3) per particle, likewise up, up_rk3, rk3; dp[np]. */
int pandora_set_particles(pandora_handle* h, int64_t np, const double* xp, const double* up,
                          const double* up_rk3, const double* rk3, const double* dp);
int pandora_get_particles(pandora_handle* h, int64_t np, double* xp, double* up,
                          double* up_rk3, double* rk3, double* dp);
/* P_INIT_RANDOM positions (src/pp_control.f90:663-707), on the device. */
int pandora_init_particles(pandora_handle* h);

/*
 * One RK3 time step, g_RK3Calc (src/pg_rk3.f90:82-129): three stages, each
 * f_RK3Stage{1,2,3} (src/pf_rk3.f90:40-200) including the E(k)/epsilon
 * statistics at stage 1, forcing at every stage and the particle advance.
 * On return *simtime = t0 + dt and *dt holds the step's dt (synchronous).
 */
int pandora_rk3_step(pandora_handle* h, int32_t tstep, double* simtime, double* dt);
/* nsteps steps tstep0 .. tstep0+nsteps-1, enqueued on the stream without host
 * synchronisation (simtime/dt live on the device); *simtime is updated when
 * sync != 0. */
int pandora_rk3_advance(pandora_handle* h, int32_t tstep0, int32_t nsteps, int32_t sync,
                        double* simtime);
/* One stage (1..3) of step tstep at time `time`; *dt in/out as in f_RK3Stage*. */
int pandora_rk3_stage(pandora_handle* h, int32_t stage, int32_t tstep, double time, double* dt);

/*
 * Statistics of the current state, f_FluidstatsFsPrimaryQuants
 * (src/pf_fluidstats.f90:1423-1576): ek[kkmax] = shell energy / mode density,
 * *tke = 0.5 (u1u1+u2u2+u3u3), *eps = f_dis = sum 2 nu k^2 e(k).
 * *ucfl = max |u1|+|u2|+|u3| of the last stage-1 physical field
 * (src/pf_fluidstats.f90:913-917).  Any output pointer may be NULL.
 */
int pandora_stats(pandora_handle* h, double* ek, int32_t kkmax, double* tke, double* eps,
                  double* ucfl);
/* Statistics recorded at stage 1 of the most recent step (state at step start). */
int pandora_last_step_stats(pandora_handle* h, double* ek, int32_t kkmax, double* tke,
                            double* eps, double* ucfl);

/* Nonlinear term omega x u of the current state in spectral layout (normalised),
 * the product of f_RK3PrepareRealSpace + f_RK3RealSpace + the forward
 * transforms (test hook of src/ptf_rk3.f90:1115-1191). */
int pandora_nonlinear(pandora_handle* h, double* n1, double* n2, double* n3);

/* ---- statistics beyond E(k) ----
 * Real-space statistics of the current state (f_FluidstatsRs2D, src/pf_fluidstats.f90:
 * 827-958; the transforms of one stage, no state change): out[0..20] raw sums over the
 * NX NY NZ points of u1u1 u2u2 u3u3 u1u2 u1u3 u2u3, u1^3 u2^3 u3^3, u1^4 u2^4 u3^4
 * (laboratory-frame velocity), w1^2 w2^2 w3^2, w1^3.., w1^4..; out[21] max |u1|+|u2|+|u3|,
 * out[22..24] max |w_i|.  n >= 25.  Normalisation as f_FluidstatsRsCollect
 * (src/pf_fluidstats.f90:960-1100) is the caller's.  In the R-conv form w is
 * d(u1,u2,u3)/dx1, the fields the reference holds in u4..u6 there. */
int pandora_realspace_stats(pandora_handle* h, double* out, int32_t n);

/* TS_CORR's longitudinal autocorrelation of the current state (f_FluidstatsRs2D,
 * src/pf_fluidstats.f90:933-945): r[l] = sum over the NX NY NZ points of u1(x) u1(x + l dx),
 * l = 0..NX/2, periodic in x, u1(x) in the laboratory frame for shear and u1(x + l dx) the
 * stored component (the reference's temp_r1i).  n >= NX/2 + 1.  r1i = r / (rs_u1u1 N^3)
 * and rs_lint11 = dx_laboratoryframe sum_l r[l] / (rs_u1u1 N^3) are the caller's
 * (src/pf_fluidstats.f90:1092-1105). */
int pandora_x_correlation(pandora_handle* h, double* r, int32_t n);
/* Particle statistics (p_StatsPrimary, src/pp_stats.f90:119-200): out[0..5] sums of
 * up_i up_j, out[6] sum of (1/2)(pi/6 dp^3 P_RHO)|up|^2.  n >= 7. */
int pandora_particle_stats(pandora_handle* h, double* out, int32_t n);

/* Physical-space velocity of the last stage (x fastest, [z][y][x]), as
 * materialised for particle interpolation (arr_u*_3r, src/pf_rk3.f90:1108-1115). */
int pandora_get_physical_velocity(pandora_handle* h, double* u1, double* u2, double* u3);

/* Moving frame of a shear flow: bmat(1,3) and binv(1,3) of g_domain
 * (src/pg_domain.f90:202-214), as g_RK3UpdateB (src/pg_rk3.f90:280-385) and the
 * remesh (src/pf_rk3.f90:4056-4178) leave them; both 0 for isotropic flow. */
int pandora_frame(pandora_handle* h, double* bmat13, double* binv13);

/* Device status word: non-zero bits record NaN detection / bounded-wait timeouts /
 * lost particles since the last call; clears it. */
int pandora_check_status(pandora_handle* h);

/* Number of kernel launches one pandora_rk3_step/advance enqueues per step. */
int pandora_launches_per_step(pandora_handle* h, int32_t* n);

/* Profiling hook: enqueues `reps` launches of one pass of a stage-2 step on the
 * handle's stream, without synchronising (callers bracket it with their own
 * events).  pass: 1 z-inverse, 2 y-inverse, 3 x-pass (NL), 4 y-forward,
 * 5 z-forward then the per-mode RK update (two launches), 6 particles,
 * 7 spectral statistics.  Passes 5 and 6
 * advance the state; use only on a scratch simulation. */
int pandora_profile_pass(pandora_handle* h, int32_t pass, int32_t reps);
/* Algorithmic HBM bytes of one launch of `pass` (each input read once, each
 * output written once, at the stored, unpadded extents; for the particles the field
 * values their stencils need, at most the whole field, and their state). */
int pandora_pass_bytes(pandora_handle* h, int32_t pass, double* bytes);

/* Instrumentation (no counterpart in the reference): every step records a CUDA
 * event pair around each pass p whose bit p-1 is set in `passes` (passes 1..6 as
 * in pandora_profile_pass), in each stage, inside
 * the step graph; passes = 0 turns it off.  pandora_pass_times waits for the
 * handle's stream and writes the durations of the most recent step,
 * ms[(stage-1)*6 + pass-1] in milliseconds (-1 where a pass was not timed). */
int pandora_set_pass_timing(pandora_handle* h, int32_t passes);
int pandora_pass_times(pandora_handle* h, float* ms);

/*
 * Batches (no counterpart in the reference: the device side of the ensemble
 * server).  A batch holds `capacity` slots of one class -- grid size, precision,
 * flow type with its B110..B330, particles per member and their interpolation
 * order, forcing radius -- each slot a full simulation with its own state.
 * Members may differ in seeds, viscosity, dt, forcing amplitude and time scale and
 * shear rate.  One step of the batch advances every occupied slot: each kernel
 * launch serves up to 32 members, and members admitted at different times advance
 * side by side, each with its own step counter and time.  Results are those of
 * the same simulation run alone (the kernels do the same arithmetic per member).
 * All calls on one batch run in its stream order and, except the readers
 * (member_time, get_state, get_particles, last_step_stats, sync), none waits on
 * the host; the batch is not re-entrant.
 */
typedef struct pandora_batch pandora_batch;
/* Device bytes a batch of this class and capacity allocates (for admission control). */
int pandora_batch_bytes(const pandora_params* cls, int32_t capacity, int64_t* bytes);
/* Capacity > 1 needs grid lengths of 32, 48, 64, 96, 128, 192 or 256 on every axis (the
 * ensemble's sizes; other lengths: PANDORA_ERR_UNSUPPORTED, or capacity 1). */
int pandora_batch_create(const pandora_params* cls, int32_t capacity, pandora_batch** out);
int pandora_batch_destroy(pandora_batch* b);
int pandora_batch_capacity(pandora_batch* b, int32_t* capacity, int32_t* free_slots);
/* Start a member in a free slot: seeded initial field (and particles), step 1 at
 * time 0.  *slot < 0 on entry: any free slot; else that slot (it must be free).
 * PANDORA_ERR_BAD_LAYOUT if `member` is not of the batch's class, PANDORA_ERR_OOM
 * if no slot is free. */
int pandora_batch_admit(pandora_batch* b, const pandora_params* member, int32_t* slot);
/* Free a slot (in stream order; its member stops after the work already enqueued). */
int pandora_batch_release(pandora_batch* b, int32_t slot);
/* Free a slot and keep its member's last-step statistics: enqueues the copy of its
 * shell sums to pinned host memory, then marks the slot free; *ticket completes
 * when both are done (pandora_batch_ticket_done), after which
 * pandora_batch_result_stats reads them without waiting.  Never waits itself. */
int pandora_batch_finish(pandora_batch* b, int32_t slot, int64_t* ticket);
int pandora_batch_result_stats(pandora_batch* b, int32_t slot, double* ek, int32_t kkmax, double* tke,
                               double* eps);
/* Enqueue nsteps RK3 steps of every occupied slot (asynchronous); *ticket (may be
 * null) completes when they are done. */
int pandora_batch_step(pandora_batch* b, int32_t nsteps, int64_t* ticket);
int pandora_batch_ticket_done(pandora_batch* b, int64_t ticket, int32_t* done);
int pandora_batch_sync(pandora_batch* b);
int pandora_batch_launches_per_step(pandora_batch* b, int32_t* n);
/* Next step number, time and dt of a slot's member (waits for the batch). */
int pandora_batch_member_time(pandora_batch* b, int32_t slot, int32_t* tstep, double* simtime, double* dt);
int pandora_batch_get_state(pandora_batch* b, int32_t slot, double* u1, double* u2, double* u3);
int pandora_batch_get_particles(pandora_batch* b, int32_t slot, int64_t np, double* xp, double* up,
                                double* up_rk3, double* rk3, double* dp);
/* Statistics of the member's state at stage 1 of its last step. */
int pandora_batch_last_step_stats(pandora_batch* b, int32_t slot, double* ek, int32_t kkmax, double* tke,
                                  double* eps);

/*
 * No counterpart in the reference.  The nonlinear term omega x u of a spectral
 * velocity field (the output of pandora_nonlinear), for callers that may not
 * allocate device memory: they pass device buffers u1..u3 (input) and n1..n3
 * (output), S complex values each in the layout above, and the call allocates
 * nothing.  Its scratch is a set of fixed __device__ arrays (about 16 MB on every
 * GPU that loads the library, held until exit), so grids are limited to 64
 * points per direction (larger sizes return PANDORA_ERR_BAD_LAYOUT) and to
 * isotropic flow.  All calls share that scratch: calls that overlap on the GPU
 * race, so serialise them.  The first call on a device sets up the scratch
 * addresses and should come before any stream capture on that device.  The call
 * returns after the result is written (it synchronises `cuda_stream`, NULL = the
 * legacy default stream).
 */
int pandora_nonlinear_static(const pandora_params* p, const double* u1, const double* u2,
                             const double* u3, double* n1, double* n2, double* n3,
                             void* cuda_stream);

#ifdef __cplusplus
}
#endif
#endif /* PANDORA_GPU_H */
