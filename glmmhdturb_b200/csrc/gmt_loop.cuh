// gmt_loop.cuh -- device-resident time loop: the host loop of run_turb (glmmhd_turb.jl:2216-2230)
// moved onto the GPU so that many steps run without a host round trip and can be captured in a
// CUDA graph.
//
// Per step and per box: the tick kernel turns the CFL maxima that the previous step fused into
// its write-out into dt, ch, glm_fac and the forcing ramp, decides whether the OU forcing advances
// this step (t >= next_time, glmmhd_turb.jl:2217) and clips dt to the forcing cadence and t_end
// (:2221); the conditional OU / mode-table kernels then run only on boxes that advance, and the
// step kernel reads its dt, ch, glm_fac and ramp from the same record.
#pragma once
#include "gmt_internal.h"

namespace gmt {

// per-box loop record in device memory; dt, ch, glm_fac, ramp first (the step kernel's dparams)
struct LoopState {
    double dt, ch, glm_fac, ramp;
    double t, t_end, next_time;
    uint32_t counter;   // OU updates done
    int advance;        // 1: the forcing advances before this step
    int status;         // 1: no positive finite CFL maximum (state invalid); steps then have dt = 0
    int pad;
};

// per-box constants of the loop
struct LoopConst {
    double courant, dx, boxlen, cp_coef, glm_ch_scale, turb_T, dtf, alpha, beta, sigma0;
    int ch_max_signal;  // 1: ch = global max signal speed; 0: ch = courant*dx/dt/3*glm_ch_scale
    int do_turb;
    uint32_t seed;
    int pad;
};

__global__ void tick_kernel(LoopState* st, const LoopConst* cs, const unsigned long long* cfl, int nbox) {
    int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= nbox) return;
    LoopState S = st[b];
    const LoopConst C = cs[b];
    double cmax = __longlong_as_double((long long)cfl[2 * b]);
    double smax = __longlong_as_double((long long)cfl[2 * b + 1]);
    S.advance = 0;
    if (C.do_turb && S.t >= S.next_time) {
        S.advance = 1;
        S.next_time += C.dtf;
    }
    double dt = 0.0;
    if (cmax > 0.0 && isfinite(cmax)) {
        dt = C.courant * C.dx / cmax;
    } else {
        S.status = 1;
    }
    if (C.do_turb) dt = fmin(dt, S.next_time - S.t);
    dt = fmin(dt, S.t_end - S.t);
    if (!(dt > 0.0)) dt = 0.0;
    double ch = S.ch;
    if (dt > 0.0) ch = C.ch_max_signal ? smax : C.courant * C.dx / dt / 3.0 * C.glm_ch_scale;
    if (!(ch > 0.0)) ch = 1.0;
    S.dt = dt;
    S.ch = ch;
    S.glm_fac = C.cp_coef > 0.0 ? exp(-(ch * ch / (C.cp_coef * C.boxlen * ch)) * dt) : 1.0;
    S.ramp = C.turb_T > 0.0 ? fmin(S.t / C.turb_T, 1.0) : 1.0;
    S.t += dt;
    st[b] = S;
}

// one block per box: OU update of the 61 modes of boxes whose record says advance
__global__ void ou_cond_kernel(double* modes, LoopState* st, const LoopConst* cs, const int* mode_k) {
    const int b = blockIdx.x, q = threadIdx.x;
    const LoopState& S = st[b];
    if (!S.advance) return;
    const LoopConst& C = cs[b];
    uint32_t counter = S.counter;
    if (q < 61)
        ou_mode_update(modes + (size_t)b * 61 * 6, q, mode_k[3 * q], mode_k[3 * q + 1], mode_k[3 * q + 2], C.seed,
                       counter, C.alpha, C.beta, C.sigma0);
    __syncthreads();
    if (q == 0) st[b].counter = counter + 1;
}

// mode-table rows of advancing boxes; grid (rows, boxes)
template <class R> struct BoxTables {
    const double* modes;   // [61][3][2] of this box
    const R* trigy;
    const R* trigz;
    R* btab;
    int ny, nz;
};
template <class R>
__global__ void __launch_bounds__(256) btab_cond_kernel(const BoxTables<R>* bt, const LoopState* st, const int* mode_k) {
    const int b = blockIdx.y;
    if (!st[b].advance) return;
    const BoxTables<R> T = bt[b];
    int row = blockIdx.x * blockDim.x + threadIdx.x;
    if (row >= T.ny * T.nz) return;
    btab_row(T.modes, mode_k, T.trigy, T.trigz, T.ny, T.nz, row % T.ny, row / T.ny, T.btab + (size_t)row * 24);
}

}  // namespace gmt
