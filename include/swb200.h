/*
 * swb200.h -- C ABI of the B200 time-integration library (libswb200.so).
 *
 * The library replaces the body of ShallowWaters.jl's time loop,
 *   time_integration(Prog, Diag, S) -> PrognosticVars      (src/time_integration.jl:2-250)
 * called from run_model(T, P)                              (src/run_model.jl:25-39).
 * Everything inside that function -- rhs!, continuity!, the RK/SSPRK stage
 * combination, ghost_points!, bottom drag, biharmonic diffusion, the
 * semi-Lagrangian tracer and the NaN check -- runs as CUDA kernels for sm_100a.
 * The host keeps Parameter, Grid, Constants, Forcing and the initial
 * conditions and hands their (already rounded) values to this library.
 *
 * Array convention (all entry points): a 2-D field of size (m, n) in the
 * reference's notation is a contiguous host buffer with x fastest, element
 * (i, j) (1-based, as in Julia) at offset (i-1) + (j-1)*m.  That is Julia's
 * column-major Array{T,2}, i.e. C's row-major a[j][i].  The element type of
 * prognostic fields (u, v, eta, sst) is the config's Tprog, the element type
 * of the static fields (f_q, f_u, f_v, Fx, Fy, H, eta_ref, Feta) is its T.
 *
 * Shapes, with N = nx, M = ny, nux = N (periodic) or N-1 (nonperiodic)
 * (src/grid.jl:26-31, src/initial_conditions.jl:6-21, src/forcing.jl:11-53):
 *   u    (nux+4) x (M+4)      v    (N+4) x (M+3)
 *   eta  (N+2)   x (M+2)      sst  (N+2) x M          -- with halo
 *   f_q  (N+1)   x (M+1)      f_u  nux x M      f_v  N x (M-1)
 *   Fx   nux     x M          Fy   N x (M-1)
 *   H    (N+2)   x (M+2)      eta_ref  N x M    Feta  N x M
 *
 * Errors: every entry point returns an sw_error code; the library never
 * aborts or exits.  sw_last_error(ctx) gives a message for the last failure.
 * A context owns one CUDA stream and is not thread-safe; distinct contexts may
 * be used from distinct threads.  Host pointers are never retained after a
 * call returns.
 */
#ifndef SWB200_H
#define SWB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SWB200_ABI_VERSION 1

/* Number formats of Parameter.T / Tprog / Tcomm (src/default_parameters.jl:3-6). */
enum sw_number_format {
    SW_FLOAT16 = 1,
    SW_FLOAT32 = 2,
    SW_FLOAT64 = 3
};

/* Parameter.time_scheme (src/default_parameters.jl:50). */
enum sw_time_scheme { SW_RK = 0, SW_SSPRK2 = 1, SW_SSPRK3 = 2, SW_4SSPRK3 = 3 };
/* Parameter.dynamics (src/default_parameters.jl:68). */
enum sw_dynamics { SW_NONLINEAR = 0, SW_LINEAR = 1 };
/* Parameter.adv_scheme (src/default_parameters.jl:67). */
enum sw_adv_scheme { SW_ARAKAWA_HSU = 0, SW_SADOURNY = 1 };
/* Parameter.bottom_drag (src/default_parameters.jl:71). */
enum sw_bottom_drag { SW_DRAG_QUADRATIC = 0, SW_DRAG_LINEAR = 1, SW_DRAG_NONE = 2 };
/* Parameter.diffusion (src/default_parameters.jl:76). */
enum sw_diffusion { SW_DIFF_CONSTANT = 0, SW_DIFF_SMAGORINSKY = 1 };
/* Device storage of the prognostic fields.  NATIVE keeps Tprog.  BF16/F16
 * store u, v, eta and sst in 16 bits (u, v scaled by storage_scale_uv) with
 * FP32 tendencies and FP32-compensated (Kahan) accumulation; Tprog must be
 * Float32.  This form has no counterpart in the reference. */
enum sw_storage { SW_STORE_NATIVE = 0, SW_STORE_BF16 = 1, SW_STORE_F16 = 2 };

enum sw_error {
    SW_OK = 0,
    SW_ERR_ARG = 1,          /* bad shape, option or pointer                     */
    SW_ERR_CUDA = 2,         /* a CUDA call failed                               */
    SW_NAN_DETECTED = 3,     /* feedback.nans_detected (src/feedback.jl:61-72)   */
    SW_ERR_TIMEOUT = 4,      /* a bounded device wait ran out                    */
    SW_ERR_UNSUPPORTED = 5,  /* option combination not built                     */
    SW_ERR_NOMEM = 6,        /* device allocation failed                         */
    SW_ERR_DEPARTURE = 7,    /* tracer departure point left the wrapped domain   */
    SW_ERR_NODEVICE = 8      /* no CUDA device                                   */
};

/* Everything time_integration reads from S.parameters, S.grid and
 * S.constants.  Scalar constants are the reference's values AFTER rounding to
 * T or Tprog (src/constants.jl:58-115, src/grid.jl:68-83), carried in double
 * (exact for Float16/Float32 values). */
typedef struct sw_config {
    int32_t abi_version;         /* = SWB200_ABI_VERSION                        */

    /* Grid sizes (src/grid.jl:21-56). */
    int32_t nx, ny;
    int32_t periodic;            /* 1: bc == "periodic" (ep = 1), 0: nonperiodic */
    int32_t halo, haloeta;       /* must be 2 and 1 (src/grid.jl:50-51)          */
    int32_t halosstx, halossty;  /* must be 1 and 0 (src/grid.jl:52-53)          */

    /* Number formats (src/default_parameters.jl:3-6). */
    int32_t T, Tprog, Tcomm;     /* enum sw_number_format                        */

    /* Time stepping (src/default_parameters.jl:50-58, src/grid.jl:68-87). */
    int32_t time_scheme;         /* enum sw_time_scheme                          */
    int32_t RKo, RKs, RKn;
    int32_t nstep_diff, nstep_advcor;
    int32_t nadvstep, nadvstep_half;
    int32_t nout;
    int32_t dtint;
    int64_t nt;                  /* steps run by sw_time_integration             */

    /* Physics options. */
    int32_t dynamics, adv_scheme, bottom_drag, diffusion;
    int32_t tracer_advection, tracer_consumption;
    int32_t surface_relax, surface_forcing;
    int32_t seasonal_wind_x, seasonal_wind_y;

    /* Constants in Tprog (src/constants.jl:58-72, 93; src/grid.jl:74). */
    double RKaDt[4], RKbDt[3];
    double Dt_Ds, Dt_D, Dt_D_half;
    double one_minus_alpha;
    double Dt_diff;
    /* SSPRK3 coefficients (src/constants.jl:4-27). */
    int32_t ssp_n, ssp_s, ssp_kn, ssp_mn;
    double ssp_Dt_Dn, ssp_kna, ssp_knb, ssp_Dt_Dnc;

    /* Constants in T (src/constants.jl:94-108, src/grid.jl:80-83). */
    double g, cD, rD, gamma, cSmag, nuB, rSST, jSST, SSTmin;
    double dtadvu, dtadvv, half_dtadvu, half_dtadvv;
    /* Float64 frequencies (src/constants.jl:110-113). */
    double omegaFeta, omegaFx, omegaFy;

    /* Device storage form (no reference counterpart). */
    int32_t storage;             /* enum sw_storage                              */
    double storage_scale_uv;     /* power of two, e.g. 1024                      */
    int32_t reserved[8];
} sw_config;

/* S.grid's Coriolis fields and S.forcing (src/grid.jl:93-95,
 * src/forcing.jl:1-53).  Element type T.  f_u/f_v are only read for linear
 * dynamics, eta_ref only with surface_relax, Feta only with surface_forcing;
 * the others must be given. */
typedef struct sw_static {
    const void* f_q;
    const void* f_u;
    const void* f_v;
    const void* Fx;
    const void* Fy;
    const void* H;
    const void* eta_ref;
    const void* Feta;
} sw_static;

/* Outcome of a run. */
typedef struct sw_status {
    int64_t steps_done;   /* time steps completed by this call                  */
    int64_t step;         /* model step counter after the call (i of the loop)  */
    int64_t nan_step;     /* step at which NaNs were found, or -1               */
    int32_t code;         /* enum sw_error of the run                           */
    int32_t reserved;
} sw_status;

/* Global diagnostics of the current state, reduced on the device in FP64. */
typedef struct sw_diag {
    double mass;          /* sum of eta over the interior                       */
    double energy;        /* 1/2 sum h*(Ix(u^2)+Iy(v^2)) + 1/2 g sum eta^2      */
    double max_speed;     /* max |u|, |v| over the interior (for a CFL check)   */
    int64_t nan_count;    /* NaNs in u, v, eta, sst                             */
} sw_diag;

/* Per-kernel device times of a profiled run (CUDA events on the context's
 * stream).  Kinds: 0 rk stage, 1 tail (drag+diffusion), 2 tracer,
 * 3 advection/Coriolis refresh, 4 NaN check, 5 other. */
#define SW_PROFILE_KINDS 6
typedef struct sw_profile {
    double step_ms_total;              /* sum of per-step device times          */
    double kernel_ms[SW_PROFILE_KINDS];
    int64_t launches[SW_PROFILE_KINDS];
    int64_t steps;
} sw_profile;

typedef struct sw_ctx sw_ctx;

/* Drop-in for time_integration (src/time_integration.jl:2-250): uploads the
 * state (with halo, as built by initial_conditions/add_halo,
 * src/initial_conditions.jl:26-164, src/ghost_points.jl:2-27), runs cfg->nt
 * steps and writes the final state back into the same buffers.  On NaN
 * detection it stops like the reference (src/time_integration.jl:235-237):
 * u, v, eta are those before the failing step, sst after it, and the return
 * value is SW_NAN_DETECTED. */
int sw_time_integration(const sw_config* cfg, const sw_static* st,
                        void* u, void* v, void* eta, void* sst,
                        sw_status* status);

/* Context API (the same loop, split so state can stay on the device).
 * sw_create mirrors preallocate + the constant uploads of run_model
 * (src/run_model.jl:29-36, src/preallocate.jl:454-471). */
int sw_create(const sw_config* cfg, const sw_static* st, sw_ctx** out);
/* Upload a state with halo (Tprog, shapes above).  Resets the step counter. */
int sw_set_state(sw_ctx* ctx, const void* u, const void* v,
                 const void* eta, const void* sst);
/* Advance nsteps time steps (the loop body src/time_integration.jl:45-243),
 * continuing the step counter.  Blocks until done. */
int sw_run(sw_ctx* ctx, int64_t nsteps, sw_status* status);
/* Download the current state with halo (Tprog). */
int sw_get_state(sw_ctx* ctx, void* u, void* v, void* eta, void* sst);
/* The u, v, eta (with halo, Tprog) that the last right-hand-side evaluation
 * of the last step read: the input of its last RK stage or SSP sub-stage, or
 * the current state before any step.  The reference's output writes q and the
 * relative vorticity from its work arrays (src/output.jl:105-115), which hold
 * the values of that evaluation (src/PV_advection.jl:2-18, src/rhs.jl:89-128);
 * they follow from this state, H and f_q.  Native storage only. */
int sw_get_rhs_input(sw_ctx* ctx, void* u, void* v, void* eta);
/* FP64 reductions over the current state. */
int sw_diagnostics(sw_ctx* ctx, sw_diag* out);
/* sw_diagnostics for callers that cannot allocate device memory (for example
 * a host whose pool allocator owns the GPU's memory, or a time loop that must
 * not be stalled by the device-wide synchronisation of cudaMalloc/cudaFree).
 * No counterpart in the reference.  The fields are the caller's DEVICE
 * buffers in the host-array layout and shapes above (u, v, eta, sst in Tprog,
 * H in T); only cfg->nx, ny, periodic, T, Tprog and g are read.  Reduction
 * scratch is a fixed array inside the library, so it allocates nothing and
 * accepts at most 16,777,216 cells (nx*ny), returning SW_ERR_ARG beyond that.
 * The first call on a device, and the first after the device's CUDA context
 * was created again (cudaDeviceReset), looks up that array (make it before any
 * stream capture); a CUDA error already pending at entry is returned as
 * SW_ERR_CUDA and left pending; calls whose kernels overlap on one device share the array and
 * race.  Runs on `stream` (a cudaStream_t, NULL for the default stream) and
 * returns after the result has reached *out. */
int sw_diagnostics_noalloc(const sw_config* cfg, const void* u, const void* v,
                           const void* eta, const void* sst, const void* H,
                           void* stream, sw_diag* out);
/* sw_run with per-kernel CUDA-event timing; when l2_flush_bytes > 0 a buffer
 * of that size is written between steps (outside the timed intervals). */
int sw_run_profiled(sw_ctx* ctx, int64_t nsteps, int64_t l2_flush_bytes,
                    sw_profile* prof, sw_status* status);
/* sw_run with one CUDA-event interval per time step; when l2_flush_bytes > 0
 * a buffer of that size is written between steps (outside the intervals).
 * *step_ms_total is the sum of the intervals.  Steps run as on sw_run (from
 * CUDA graphs where possible).  No reference counterpart (measurement). */
int sw_run_timed(sw_ctx* ctx, int64_t nsteps, int64_t l2_flush_bytes,
                 double* step_ms_total, sw_status* status);
/* Number of CUDA kernel launches the library has issued on this context. */
int64_t sw_kernel_launches(const sw_ctx* ctx);
/* Ends a context.  Its device blocks are kept by the library for reuse by
 * later contexts of the same sizes (up to 16 GiB in all), so repeated drop-in
 * calls do not pay for cudaMalloc/cudaFree; sw_trim_memory frees them.  No
 * reference counterpart (the reference's preallocate! arrays are freed by
 * Julia's garbage collector). */
void sw_destroy(sw_ctx* ctx);
/* Returns every device and pinned block kept for reuse to CUDA.  Call it with
 * no context in use. */
int sw_trim_memory(void);

/* Ensembles advanced together: n members, each with its own config and static
 * fields (any grid size and parameters), advanced with one kernel launch per
 * sub-step for all members that share the boundary type, options and state
 * storage.  Members must be Float32, RK, nonlinear, nstep_diff = 1, without
 * nstep_advcor, seasonal wind or surface forcing (else SW_ERR_UNSUPPORTED);
 * their storage may be native or one of the 16-bit forms (with that form's
 * own restrictions).  Every member computes exactly what a lone context with
 * its config computes.  No reference counterpart (an ensemble there is a loop
 * of run_model calls). */
typedef struct sw_batch sw_batch;
int sw_batch_create(int32_t n, const sw_config* cfgs, const sw_static* statics, sw_batch** out);
/* Upload member m's state (as sw_set_state); resets the batch to step 0. */
int sw_batch_set_state(sw_batch* b, int32_t member, const void* u, const void* v,
                       const void* eta, const void* sst);
/* Advance up to nsteps global steps; a member stops after its own nt steps (or
 * a NaN stop).  statuses: n entries, the member's steps done and code. */
int sw_batch_run(sw_batch* b, int64_t nsteps, sw_status* statuses);
int sw_batch_get_state(sw_batch* b, int32_t member, void* u, void* v, void* eta, void* sst);
int64_t sw_batch_launches(const sw_batch* b);
/* Rows per warp strip of the batched stage and tail kernels: 4, 8, 16 or 32,
 * or 0 before the first run that could choose.  sw_batch_run chooses it on
 * its first call of more than 44 global steps: each candidate advances 2
 * untimed steps, then 3 interleaved rounds time 3 steps of each (real steps
 * of the run: every candidate computes identical values) and the best round
 * of each decides.  The choice is remembered for later batches of the same
 * member shapes in the process.  SWB200_BATCH_TY=4|8|16|32 in the environment
 * forces one; SWB200_TUNE_LOG=1 prints the timings. */
int32_t sw_batch_tile_rows(const sw_batch* b);
/* Member m's context (owned by the batch: do not destroy it), e.g. for
 * sw_diagnostics after a run. */
sw_ctx* sw_batch_member(sw_batch* b, int32_t member);
void sw_batch_destroy(sw_batch* b);

/* Reverse-mode gradient (adjoint) of an eta misfit through the time loop:
 *   J = sum over the interior i <= nx, j <= ny of (eta(i+1, j+1) after
 *       nsteps steps - eta_obs(i, j))^2
 * differentiated with respect to the initial state (u, v, eta with their
 * halos, shapes above) and the wind forcing Fx (nux x M).  Replaces the
 * ForwardDiff/ChainRules route of the Julia ecosystem, which the reference
 * cannot take (its number types are restricted to AbstractFloat), so it has no
 * counterpart in the reference; the forward model it differentiates is
 * src/time_integration.jl:45-233.  Supported: T = Tprog = Tcomm in
 * Float32 or Float64; RK2/3/4, SSPRK2 (2-4 sub-stages), SSPRK3 (n = 2 or 3)
 * or 4SSPRK3 (the SSP schemes with their semi-implicit continuity); linear dynamics, or nonlinear with Arakawa-Hsu
 * or Sadourny and nstep_advcor = 0; any nstep_diff, drag and diffusion;
 * either boundary; surface relaxation or forcing; seasonal wind.  Other
 * options give SW_ERR_UNSUPPORTED.  The tracer is passive and plays no part.
 * Inputs and outputs are HOST buffers in T: u, v, eta the initial state,
 * eta_obs nx x ny; g_u, g_v, g_eta (state shapes), g_Fx and eta_final (the eta
 * after nsteps, with halo) may be NULL.  ncheckpoints >= nsteps keeps every
 * step state on the device and, memory permitting (off with
 * SWB200_ADJ_STORE=0), every step's RK stage inputs and tail input as well, so
 * the reverse sweep recomputes only each pass's intermediates.  With fewer
 * checkpoints than steps the schedule is two-level: a state slot at the start
 * of each segment of ceil(nsteps / ncheckpoints) steps, and the reverse sweep
 * recomputes one segment at a time while keeping its steps' stage inputs, so
 * every step is recomputed once; when a segment's stage inputs do not fit in
 * device memory (or with SWB200_ADJ_SCHEDULE=binomial) the binomial
 * checkpoint schedule recomputes states from the slots alone.  ncheckpoints
 * is an upper bound: when that many state slots do not fit in device memory,
 * half as many are tried (down to one, binomial schedule);
 * stats->checkpoints reports the number used.  The derivative of sqrt at 0 (drag and Smagorinsky at
 * rest) is taken as 0.  Gradients are summed with atomics, so repeated calls
 * agree to rounding, not bit for bit.  stats may be NULL. */
typedef struct sw_adjoint_stats {
    double forward_ms;                 /* device time of the first forward sweep      */
    double reverse_ms;                 /* device time of the reverse sweep            */
    int64_t forward_steps;             /* steps advanced, recomputation included      */
    int64_t adjoint_steps;             /* adjoint steps (= nsteps)                    */
    int32_t checkpoints;               /* state slots used                            */
    int32_t launches_per_forward_step;
    int32_t launches_per_adjoint_step;
    int32_t stored_stage_states;       /* 1: every step's stage inputs were kept (no forward recomputation);
                                          2: kept per segment (two-level schedule); 3: the same, with
                                          each segment recomputed on a second stream while the next
                                          one is reversed; 0: not kept */
} sw_adjoint_stats;
int sw_adjoint_run(const sw_config* cfg, const sw_static* st,
                   const void* u, const void* v, const void* eta, const void* eta_obs,
                   int64_t nsteps, int32_t ncheckpoints, double* J,
                   void* g_u, void* g_v, void* g_eta, void* g_Fx, void* eta_final,
                   sw_adjoint_stats* stats);

/* Which build of the library this is.  SW_BUILD_PARITY (libswb200.so) is
 * compiled without FMA contraction and reproduces the reference's Float32 and
 * Float64 arithmetic bit for bit; SW_BUILD_FAST (libswb200_fast.so) contracts
 * a*b+c into fused multiply-adds and agrees with the reference to rounding.
 * No reference counterpart (the reference has one build). */
enum sw_build { SW_BUILD_PARITY = 0, SW_BUILD_FAST = 1 };
int sw_build_kind(void);

const char* sw_strerror(int code);
const char* sw_last_error(const sw_ctx* ctx);
int sw_abi_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SWB200_H */
