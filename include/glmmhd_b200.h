/* glmmhd_b200.h -- C ABI of libglmmhd_b200.so, the B200 (sm_100a) GLM-MHD / CT-MHD time step.
 *
 * Two layers:
 *
 *  1. The legacy bridge symbols, with the exact signatures the reference's Julia bridge binds
 *     (march_bridge/MarchBridge.jl:34-81 via dlsym + ccall, march_bridge/cu/spike_mhd.cu:321-340,
 *     march_bridge/cu/spike_ctm.cu:299-328).  `march_*` run the transverse-free 1-D Hancock + HLL
 *     + Dedner march scheme; `ct_run` runs the constrained-transport march.  As in the reference,
 *     they return elapsed ms and report no errors; the extended API below does.
 *
 *  2. The extended API (`gmt_*`): a context per configuration, explicit streams, FP32 and FP64,
 *     runtime grid size, every scheme of the reference's Julia step API (glmmhd_turb.jl step_plm!
 *     :878, step_tiled! :746, step_multi! :1981, compute_dt :1973; ct_mhd.jl CTMHD.step! :174),
 *     status codes, and the deterministic mode-sum forcing.
 *
 * State layout everywhere: SoA planes of nx*ny*nz reals, x fastest,
 * index = i + nx*(j + ny*k) -- the memory image of the reference's (N,N,N,9) Float32 array
 * (glmmhd_turb.jl:57,63-64).  GLM: 9 planes [rho, rho vx, rho vy, rho vz, E, Bx, By, Bz, psi].
 * CT: 8 planes [rho, rho vx, rho vy, rho vz, E, bxf, byf, bzf], bxf[i,j,k] = Bx on the lower-x
 * face (ct_mhd.jl:10-11).  All data pointers are device pointers owned by the caller; `stream`
 * is a cudaStream_t (NULL = legacy default stream).
 */
#ifndef GLMMHD_B200_H
#define GLMMHD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GMT_ABI_VERSION 1
#define GMT_MAX_SPECIES 8

/* status codes (0 = success) */
enum {
    GMT_OK = 0,
    GMT_ERR_ARG = 1,         /* invalid argument / unsupported size */
    GMT_ERR_CUDA = 2,        /* a CUDA call failed; see gmt_last_error() */
    GMT_ERR_UNSUPPORTED = 3, /* configuration not built */
    GMT_ERR_STATE = 4,       /* non-finite or non-positive state detected */
    GMT_ERR_NOMEM = 5,
    GMT_ERR_TIMEOUT = 6      /* a bounded in-kernel wait gave up; results of that step are invalid */
};
enum { GMT_F32 = 0, GMT_F64 = 1 };
enum { GMT_SCHEME_UNSPLIT = 0, GMT_SCHEME_MARCH1D = 1, GMT_SCHEME_CT = 2 };
enum { GMT_RECON_MC = 0, GMT_RECON_MINMOD = 1, GMT_RECON_PPM = 2 };
enum { GMT_RIEMANN_HLLD = 0, GMT_RIEMANN_HLL = 1, GMT_RIEMANN_LLF = 2, GMT_RIEMANN_LLF_BOUND = 3 };
enum { GMT_EMF_AVERAGE = 0, GMT_EMF_CONTACT = 1 };

/* Configuration.  Physical defaults follow `Params` (glmmhd_turb.jl:28-52); call
 * gmt_params_init() and override fields. */
typedef struct gmt_params {
    int32_t abi_version;      /* GMT_ABI_VERSION */
    int32_t nx, ny, nz;
    int32_t dtype;            /* GMT_F32 | GMT_F64 */
    int32_t scheme;           /* GMT_SCHEME_* */
    int32_t recon;            /* GMT_RECON_* */
    int32_t riemann;          /* GMT_RIEMANN_* */
    int32_t iflo;             /* 1: revert unphysical interface states (glmmhd_turb.jl:618) */
    int32_t emf;              /* CT edge EMF: GMT_EMF_* */
    int32_t ct_halfslope;     /* CT: 1 = ct_mhd.jl's extra factor 1/2 on the slope (:49-50) */
    int32_t tile_x, tile_y, tile_z; /* 0 = automatic */
    int32_t nsp;              /* march scheme: passive species (0..GMT_MAX_SPECIES); planes 9.. of the
                               * state hold rho*X, carried by the face mass flux (spike_mhd.cu:218-221) */
    double boxlen, gamma, courant, smallr, smallc;
    double smallp;            /* march / CT pressure floor (spike_mhd.cu:52) */
    double glm_ch_scale, glm_cp_coef;
    double llf_dmin, llf_pmin;
    double turb_min_rho;
    double turb_amp;          /* stationary rms acceleration of the forcing field */
    double turb_T;            /* OU autocorrelation time */
    int32_t turb_ndt;         /* OU updates per turb_T */
    uint32_t turb_seed;
} gmt_params;

/* One step. */
typedef struct gmt_step_args {
    double dt;
    double t;                 /* simulation time (forcing ramp min(t/turb_T, 1)) */
    double ch;                /* GLM cleaning speed */
    double glm_fac;           /* psi *= glm_fac after the update */
    int32_t do_turb;          /* apply the forcing kick */
    int32_t want_cfl;         /* fuse the next step's CFL reduction into this step */
} gmt_step_args;

typedef struct gmt_diag {
    double mass, ke2, vrms, divbmax, rhomin, etot, divb_l2, psi_l2;
    int32_t finite, nonfinite_cells;
} gmt_diag;

typedef struct gmt_ctx gmt_ctx;

/* --- library / context ------------------------------------------------------------------ */
const char* gmt_version(void);
/* last error message of the calling thread ("" if none) */
const char* gmt_last_error(void);
/* fill reference defaults for an n^3 box (glmmhd_turb.jl:28-52) */
int gmt_params_init(gmt_params* p, int n);
/* allocate a context on the current device: scratch for reductions, forcing tables, tiles */
int gmt_create(const gmt_params* p, gmt_ctx** out);
int gmt_destroy(gmt_ctx* ctx);
/* kernel resource report: registers, dynamic shared bytes and tile of the step kernel */
int gmt_kernel_info(gmt_ctx* ctx, int32_t* regs, int64_t* smem_bytes, int32_t tile[3]);

/* --- GLM step (unsplit: step_plm!/step_tiled!/step_multi!; march1d: march_run_dev) ------- */
/* uold/unew: base pointers of 9 contiguous planes (plane stride nx*ny*nz), 9 + nsp with species */
int gmt_step(gmt_ctx* ctx, const void* uold, void* unew, const gmt_step_args* a, void* stream);
/* same with one pointer per plane (the bridge's float*[9 + nsp] layout) */
int gmt_step_planes(gmt_ctx* ctx, const void* const* uold, void* const* unew, const gmt_step_args* a,
                    void* stream);

/* --- CFL (compute_dt, glmmhd_turb.jl:1963-1978) ------------------------------------------ */
/* reduce max_cells sum_d(|v_d|+c_f) and max_cells max_d(|v_d|+c_f) into the context (async) */
int gmt_cfl_async(gmt_ctx* ctx, const void* u, void* stream);
/* synchronise `stream` and read the last CFL maxima (from gmt_cfl_async or a want_cfl step);
 * also reports GMT_ERR_TIMEOUT if a step since the last check abandoned a bounded wait */
int gmt_cfl_result(gmt_ctx* ctx, double out[2], void* stream);
/* dt = courant*dx/max ctot (synchronous, as compute_dt) */
int gmt_compute_dt(gmt_ctx* ctx, const void* u, double* dt, void* stream);

/* --- diagnostics (glmmhd_turb.jl:1996-2018), FP64, deterministic ------------------------- */
int gmt_diagnostics(gmt_ctx* ctx, const void* u, gmt_diag* out, void* stream);

/* --- device-resident time loop (no counterpart in the reference: its loop is host Julia,
 *     glmmhd_turb.jl:2216-2230) ---------------------------------------------------------------- */
enum { GMT_RUN_CH_MAXSIGNAL = 1, GMT_RUN_FORCING = 2, GMT_RUN_GRAPH = 4 };
/* Run up to nsteps unsplit steps with every decision on the device: dt = courant*dx/max ctot from
 * the CFL fused into the previous step, ch (the global max signal speed with GMT_RUN_CH_MAXSIGNAL,
 * else courant*dx/dt/3*glm_ch_scale), glm_fac, the forcing ramp and the OU cadence
 * (GMT_RUN_FORCING: advance when t >= next forcing time), dt clipped to the next forcing time and
 * to t_end.  With GMT_RUN_GRAPH the two-step unit u->w->u is captured once into a CUDA graph and
 * replayed.  Starts at t0 with the context's forcing state.  Returns the time reached (*t_out) and
 * the buffer holding the result (*which: 0 = u, 1 = w); synchronous on return. */
int gmt_run(gmt_ctx* ctx, void* u, void* w, int32_t nsteps, double t0, double t_end, int32_t flags, void* stream,
            double* t_out, int32_t* which);

/* --- batched ensemble: many periodic boxes of different sizes in one persistent launch per step -
 * (no counterpart in the reference).  Every box: its own n^3 grid (n a multiple of 16), forcing
 * amplitude and seed; the physics of `base`.  Each step: one tick per box, the conditional forcing
 * updates, and one persistent kernel over a queue of tile work items of all boxes (32x16 columns
 * in FP32, 16x16 in FP64, z-chunks of at most 64 planes). */
typedef struct gmt_ensemble gmt_ensemble;
int gmt_ensemble_create(const gmt_params* base, int32_t nbox, const int32_t* n, const double* turb_amp,
                        const uint32_t* seeds, gmt_ensemble** out);
int gmt_ensemble_destroy(gmt_ensemble* e);
/* u[b], w[b]: device base pointers of box b's two 9-plane registers; the result is in u after an
 * even number of steps, in w after an odd one; t_out[b] = time reached by box b */
int gmt_ensemble_run(gmt_ensemble* e, void* const* u, void* const* w, int32_t nsteps, double t_end, int32_t flags,
                     void* stream, double* t_out);

/* --- turbulence statistics (no counterpart in the reference's step path; used by its turbulence
 *     checks, GPU_SOLVER_OPTIMIZATION_PLAYBOOK.md:283-284) ------------------------------------ */
/* shell-binned kinetic-energy spectrum of w = sqrt(rho) v: out[k] = 1/2 sum over the shell
 * k-1/2 <= |k'| < k+1/2 of |w^(k')|^2 for k = 0..kmax (sum_k out[k] = mean kinetic energy density).
 * FP64, deterministic; the context keeps the scratch of the largest kmax used.  Synchronous. */
int gmt_ke_spectrum(gmt_ctx* ctx, const void* u, int32_t kmax, double* out, void* stream);
/* log-density statistics of a GLM state: s = ln(rho/<rho>); pdf[b] = fraction of cells with s in bin b
 * of [smin, smax) divided by the bin width (nbins <= 4096); stats = {<rho>, <s>, sigma_s}.  FP64,
 * deterministic; synchronous. */
#define GMT_PDF_MAX_BINS 4096
int gmt_density_pdf(gmt_ctx* ctx, const void* u, int32_t nbins, double smin, double smax, double* pdf, double stats[3],
                    void* stream);
/* band-limited kinetic-energy loss L = sum_{kmin <= k <= kmax} out[k] of gmt_ke_spectrum and its
 * gradient dL/du, written to ubar as 9 planes of u's dtype (the E, B and psi planes are zero).
 * Synchronous. */
int gmt_ke_band_loss(gmt_ctx* ctx, const void* u, int32_t kmin, int32_t kmax, double* loss, void* ubar, void* stream);

/* --- discrete adjoint of the unsplit step (no counterpart in the reference) ----------------------
 * ubar = (du'/du)^T ubar_next for u' = gmt_step(ctx, u, u', a): PLM reconstruction (MC or minmod),
 * any Riemann solver, GLM, interface-state reverts, the void floor, psi damping and the forcing kick,
 * with a->dt, a->ch, a->glm_fac and the context's current forcing table frozen at the values the
 * forward step used (restore them with gmt_forcing_set_modes when recomputing from a checkpoint).
 * At a limiter kink, an HLLD branch switch, a floor or a revert the derivative of the branch that
 * the forward step took is used.  The step's part of dL/d(turb_amp) is added to an accumulator in
 * the context (gmt_adjoint_amp_grad).  Scratch of 207 state planes is allocated on the first call.
 * ubar must not alias u or ubar_next.  PPM and non-unsplit contexts return GMT_ERR_ARG. */
int gmt_adjoint_step(gmt_ctx* ctx, const void* u, const void* ubar_next, void* ubar, const gmt_step_args* a,
                     void* stream);
/* *out = the accumulated dL/d(turb_amp); reset != 0 zeroes the accumulator afterwards.  Synchronous.
 * Returns GMT_ERR_TIMEOUT (and clears the condition) if an adjoint step since the last call abandoned
 * a bounded wait: the gradients accumulated since then are invalid. */
int gmt_adjoint_amp_grad(gmt_ctx* ctx, double* out, int32_t reset, void* stream);
/* The FP32 adjoint runs its first three passes (interface states, fluxes, update-epilogue adjoint)
 * as the forward step's tile march in record mode; percell != 0 makes it run them as per-cell passes
 * instead (the FP64 path always does).  Both give the same gradient to round-off; the per-cell form
 * is the check of the tile form.  No counterpart in the reference. */
int gmt_adjoint_set_passes(gmt_ctx* ctx, int32_t percell);

/* --- diagnostics without allocation --------------------------------------------------------
 * No counterpart in the reference.  Same quantities as gmt_diagnostics for a 9-plane GLM state,
 * for callers that must not allocate device memory: a driver loop that cannot afford the device
 * synchronisation of cudaMalloc/cudaFree, a host framework whose own pool owns the memory budget,
 * or a hook holding only a state pointer and no context.  Allocates nothing: its scratch is a
 * static device array in the library image (one row per z-plane), so nz is limited to
 * GMT_NOALLOC_MAX_PLANES (GMT_ERR_ARG beyond it).  The first call on a device looks up that
 * array's device address; make it before any stream capture.  All calls share the array: calls
 * that overlap on the GPU race and must be serialised by the caller.  Synchronous on `stream`. */
#define GMT_NOALLOC_MAX_PLANES 2048
int gmt_diagnostics_noalloc(const void* u, int32_t nx, int32_t ny, int32_t nz, int32_t dtype, double boxlen,
                            double smallr, gmt_diag* out, void* stream);

/* --- failure-path testing (no counterpart in the reference) ------------------------------------
 * The tile kernels (GLM, march, CT, the adjoint's record tile) wait for each staged plane on an
 * mbarrier with a bounded wait: after budget_cycles SM clock cycles (default 2^30, about 0.5 s) a
 * wait gives up, sets the context's error flag and the kernel finishes; the host then reports
 * GMT_ERR_TIMEOUT (gmt_cfl_result, gmt_run, gmt_adjoint_amp_grad) and the step's output is invalid.
 * This sets the budget (budget_cycles = 0: the default) and, with withhold != 0, makes the tiles
 * skip staging the next plane and withhold their arrivals, so that every wait runs out with no
 * copy in flight.  (0, 0) restores production behaviour.  For tests of the failure path only. */
int gmt_test_wait_limit(gmt_ctx* ctx, int64_t budget_cycles, int32_t withhold);

/* --- forcing: 61 +/- integer modes, 1 <= |k|^2 <= 9, solenoidal OU, Philox4x32-10 -------- */
int gmt_forcing_reset(gmt_ctx* ctx, void* stream);
/* one OU update (interval turb_T/turb_ndt) + refresh of the per-row mode table */
int gmt_forcing_advance(gmt_ctx* ctx, void* stream);
/* host copies of the complex mode amplitudes, layout [61][3][2] doubles */
int gmt_forcing_set_modes(gmt_ctx* ctx, const double* modes, void* stream);
int gmt_forcing_get_modes(gmt_ctx* ctx, double* modes, void* stream);
int gmt_forcing_counter(gmt_ctx* ctx, uint32_t* counter);
/* the whole forcing state: the modes, the Philox counter of the next OU update and the time of the
 * next update (gmt_run's cadence), to checkpoint a run or carry it to another context or grid (the
 * mode-sum forcing does not depend on the grid).  set_state also refreshes the mode table. */
int gmt_forcing_get_state(gmt_ctx* ctx, double* modes, uint32_t* counter, double* next_time, void* stream);
int gmt_forcing_set_state(gmt_ctx* ctx, const double* modes, uint32_t counter, double next_time, void* stream);

/* --- initial conditions on the device ---------------------------------------------------- */
int gmt_ic_orszag_tang(gmt_ctx* ctx, void* u, void* stream);            /* glmmhd_turb.jl:2021 */
int gmt_ic_uniform(gmt_ctx* ctx, void* u, double rho0, double p0, double bx0, double by0, double bz0,
                   void* stream);                                          /* glmmhd_turb.jl:2164 */
/* seeded synthetic turbulent state (stand-in for a pre-evolved checkpoint): the uniform state plus
 * v = mach*c_s*a(x), dB = db*a(x), rho = rho0*exp(0.2 a_y(x)), a = one unit-rms draw of the 61-mode
 * solenoidal field with Philox seed `seed`.  In a CT context the face fields are
 * B0 + curl(db/(4 pi) a) taken on the cell edges, so the face divergence is zero to round-off. */
int gmt_ic_turbulent(gmt_ctx* ctx, void* u, double rho0, double p0, double bx0, double by0, double bz0,
                     double mach, double db, uint32_t seed, void* stream);

/* --- constrained transport (CTMHD.step!, ct_mhd.jl:174; ct_run, spike_ctm.cu:305) --------- */
/* q: base pointer of 8 planes [rho, mx, my, mz, E, bxf, byf, bzf] */
int gmt_ct_step(gmt_ctx* ctx, const void* qold, void* qnew, const gmt_step_args* a, void* stream);
int gmt_ct_cfl_async(gmt_ctx* ctx, const void* q, void* stream);
/* max |div B| from the face field (ct_mhd.jl:190-194) */
int gmt_ct_divb_max(gmt_ctx* ctx, const void* q, double* out, void* stream);
int gmt_ct_ic_orszag_tang(gmt_ctx* ctx, void* q, void* stream);

/* --- legacy bridge ABI (march_bridge/MarchBridge.jl, spike_mhd.cu:321-340) --------------- */
/* The grid size of the legacy entry points is fixed when the library is built (GMT_LEGACY_NX,
 * as build_mhd.sh's -DNX) and may be changed at run time with march_set_nx. */
int march_nv(void);                              /* 9 (+ passive species: 0) */
int march_nx(void);
int march_nsp(void);
void march_set_dtdx(float v);
void march_set_glm(float ch, float glmfac);
void march_set_gamma(float g);
double march_run_dev(float* const* qv, float* const* ov, int nsteps);
void march_set_nx(int n);                        /* extension: runtime grid size */
/* CT march (spike_ctm.cu:299-328): qv/ov = 5 conserved + 3 face-B planes, cc = 3 scratch planes */
double ct_run(float* const* qv, float* const* ov, float* const* cc, int nsteps);
int ct_regs(void);
int ct_shmem(void);

#ifdef __cplusplus
}
#endif
#endif /* GLMMHD_B200_H */
