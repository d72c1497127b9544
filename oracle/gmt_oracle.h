/* gmt_oracle.h -- C ABI of the CPU oracle for the GLM-MHD / CT-MHD time step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is a plain C++ restatement of the
 * reference physics (glmmhd_turb.jl, ct_mhd.jl, march_bridge/cu/spike_mhd.cu,
 * march_bridge/cu/spike_ctm.cu).  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference legs may load it, and only as the
 * checker or the timed CPU baseline.  The product library never links it.
 *
 * State layout (all entry points): 9 (GLM) or 5+3 (CT) contiguous planes of
 * nx*ny*nz reals, x fastest -- the memory image of the reference's
 * (N,N,N,9) column-major array (glmmhd_turb.jl:57,63-64) and of the bridge's
 * float*[9] SoA planes (march_bridge/MarchBridge.jl:10,64).
 */
#ifndef GMT_ORACLE_H
#define GMT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_RECON_MC = 0, ORC_RECON_MINMOD = 1, ORC_RECON_PPM = 2 };
enum { ORC_RIEMANN_HLLD = 0, ORC_RIEMANN_HLL = 1, ORC_RIEMANN_LLF = 2, ORC_RIEMANN_LLF_BOUND = 3 };
enum { ORC_EMF_AVERAGE = 0, ORC_EMF_CONTACT = 1 };
#define ORC_NMODES 61

/* branch counters (orc_count_reset / orc_count_get): each guarded branch of the reference */
enum {
    ORC_CNT_HANCOCK_REVERT = 0, /* unsplit predictor rho <= smallr or p <= pfl -> m0 (glmmhd_turb.jl:393-395) */
    ORC_CNT_IFLO_REVERT,        /* interface state rho < smallr or p < pfl -> m0 (glmmhd_turb.jl:618) */
    ORC_CNT_VOID_FLOOR,         /* updated rho < smallr -> void state (glmmhd_turb.jl:450-453) */
    ORC_CNT_LLF_SWITCH,         /* HLLD face switched to LLF by llf_dmin / llf_pmin (glmmhd_turb.jl:287-289) */
    ORC_CNT_HLLD_DEGEN,         /* |denK| < 1e-12 star state used by the sampled region (glmmhd_turb.jl:225-238) */
    ORC_CNT_HLLD_L,             /* HLLD sampled region: F_L* (SL* >= 0) */
    ORC_CNT_HLLD_LS,            /* F_L** (SL* < 0 <= SM) */
    ORC_CNT_HLLD_RS,            /* F_R** (SM < 0 <= SR*) */
    ORC_CNT_HLLD_R,             /* F_R* (SR* < 0) */
    ORC_CNT_PPM_FALLBACK,       /* PPM cell falls back to PLM faces on a pressure jump (spj, glmmhd_turb.jl:952-975) */
    ORC_CNT_FACE_FLOOR,         /* march / CT face state floored at smallr / smallp (spike_mhd.cu:199-223) */
    ORC_CNT_PRED1D_FLOOR,       /* march / CT 1-D predictor floored (spike_mhd.cu:149-161) */
    ORC_CNT_N
};

typedef struct orc_params {
    int32_t nx, ny, nz;
    int32_t recon;      /* ORC_RECON_* */
    int32_t riemann;    /* ORC_RIEMANN_* */
    int32_t iflo;       /* 1: revert unphysical interface states to m0 (glmmhd_turb.jl:618) */
    int32_t emf;        /* CT only: ORC_EMF_* */
    int32_t ct_halfslope; /* CT only: 1 = ct_mhd.jl's extra factor 1/2 on the half slope */
    double boxlen, gamma, smallr, smallc;
    double smallp;      /* march/CT pressure floor (spike_mhd.cu:52); GLM uses smallr*smallc^2/gamma */
    double llf_dmin, llf_pmin;
    double turb_min_rho;
    int32_t nsp;        /* march only: passive species, planes 9..9+nsp-1 hold rho*X */
    int32_t pad;
} orc_params;

typedef struct orc_step_args {
    double dt;
    double ch;          /* GLM cleaning speed */
    double glm_fac;     /* psi *= glm_fac after the update */
    double ramp;        /* forcing ramp min(t/T,1) */
    int32_t do_turb;
    int32_t pad;
    const double* modes; /* [ORC_NMODES][3][2] complex forcing coefficients, or NULL */
} orc_step_args;

typedef struct orc_diag {
    double mass, ke2, vrms, divbmax, rhomin, etot, divb_l2, psi_l2;
    int32_t finite, pad;
} orc_diag;

int  orc_set_threads(int n);
/* zero the branch counters and switch counting on (on != 0) or off */
void orc_count_reset(int on);
/* copy min(n, ORC_CNT_N) counters to out */
void orc_count_get(int64_t* out, int n);
int  orc_num_modes(void);
void orc_mode_k(int32_t* k3);                   /* 3*ORC_NMODES ints */
void orc_trig_table(int n, double* out);        /* [4 m][2 (cos,sin)][n] */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double orc_forcing_sigma0(double amp, double alpha, double beta);
void orc_ou_update(double* modes, uint32_t seed, uint32_t counter, double alpha, double beta,
                   double sigma0);
void orc_accel_f64(const orc_params* p, const double* modes, double ramp, double* a3);

/* unsplit PLM/PPM + MUSCL-Hancock + Riemann + GLM step (glmmhd_turb.jl:374-480, 599-767) */
int orc_step_unsplit_f64(const orc_params* p, const orc_step_args* a, const double* uold, double* unew);
int orc_step_unsplit_f32(const orc_params* p, const orc_step_args* a, const float* uold, float* unew);
/* the same step evaluated on forward-mode tangents (the ForwardDiff counterpart) along ndir <=
 * ORC_JVP_MAXDIR directions at once: dunew[k] = J duold[k] + (d unew / d amplitude) amp_rel[k],
 * the directional derivative of the step along the state direction duold[k] (duold may be null)
 * and the relative forcing-amplitude change amp_rel[k] (may be null; the modes scale with the
 * amplitude).  duold and dunew hold ndir states one after another; unew (may be null) receives the
 * ordinary FP64 step output.  Returns nonzero for an invalid ndir. */
#define ORC_JVP_MAXDIR 8
int orc_jvp_unsplit_f64(const orc_params* p, const orc_step_args* a, const double* uold, int32_t ndir,
                        const double* duold, const double* amp_rel, double* unew, double* dunew);
/* transverse-free 1-D Hancock march (spike_mhd.cu:227-302), f32 update base */
int orc_step_march1d_f64(const orc_params* p, const orc_step_args* a, const double* uold, double* unew);
int orc_step_march1d_f32(const orc_params* p, const orc_step_args* a, const float* uold, float* unew);
/* CT step (ct_mhd.jl:85-184, spike_ctm.cu): q = 5 conserved + 3 lower-face B planes */
int orc_ct_step_f64(const orc_params* p, const orc_step_args* a, const double* qold, double* qnew);
int orc_ct_step_f32(const orc_params* p, const orc_step_args* a, const float* qold, float* qnew);

/* CFL (glmmhd_turb.jl:1963-1978): out[0] = max_cells sum_d(|v_d|+cf_d),
 * out[1] = max_cells max_d(|v_d|+cf_d) */
void orc_cfl_f64(const orc_params* p, const double* u, double* out);
void orc_cfl_f32(const orc_params* p, const float* u, double* out);
void orc_ct_cfl_f64(const orc_params* p, const double* q, double* out);
void orc_diag_f64(const orc_params* p, const double* u, orc_diag* d);
void orc_diag_f32(const orc_params* p, const float* u, orc_diag* d);
double orc_ct_divb_max_f64(const orc_params* p, const double* q);

void orc_ic_ot_f64(const orc_params* p, double* u);
void orc_ic_uniform_f64(const orc_params* p, double rho0, double p0, double bx0, double by0,
                        double bz0, double* u);
void orc_ct_ic_ot_f64(const orc_params* p, double* q);

#ifdef __cplusplus
}
#endif
#endif
