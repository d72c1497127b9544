// gmt_api.cu -- C ABI of libglmmhd_b200.so (declared in include/glmmhd_b200.h).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/glmmhd_b200.h"
#include "gmt_internal.h"
#include "gmt_unsplit.cuh"
#include "gmt_loop.cuh"

using namespace gmt;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}
int cuda_fail(cudaError_t e, const char* where) {
    g_err = std::string(where) + ": " + cudaGetErrorString(e);
    return GMT_ERR_CUDA;
}
#define GMT_CUDA(call)                                           \
    do {                                                         \
        cudaError_t e_ = (call);                                 \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);      \
    } while (0)

const double kTwoPi = 6.283185307179586476925286766559;

std::vector<double> trig_table(int n) {
    std::vector<double> t(8 * (size_t)n);
    for (int m = 0; m < 4; ++m)
        for (int i = 0; i < n; ++i) {
            double th = kTwoPi * (double)m * ((double)i + 0.5) / (double)n;
            t[(size_t)(2 * m) * n + i] = std::cos(th);
            t[(size_t)(2 * m + 1) * n + i] = std::sin(th);
        }
    return t;
}

// the FP32 x table of force_accel_f32: per column the pairs (2 cos, -2 sin) of the 4 x modes
std::vector<float> trig8_table(const std::vector<double>& t, int n) {
    std::vector<float> t8((size_t)8 * n);
    for (int i = 0; i < n; ++i)
        for (int m = 0; m < 4; ++m) {
            t8[(size_t)8 * i + 2 * m] = (float)(2.0 * t[(size_t)(2 * m) * n + i]);
            t8[(size_t)8 * i + 2 * m + 1] = (float)(-2.0 * t[(size_t)(2 * m + 1) * n + i]);
        }
    return t8;
}

// sigma0 such that the stationary rms |a| equals amp, sqrt(P(k)) = 1/|k|
double forcing_sigma0(double amp, double alpha, double beta) {
    double s = 0.0;
    for (int kx = 0; kx <= 3; ++kx)
        for (int ky = -3; ky <= 3; ++ky)
            for (int kz = -3; kz <= 3; ++kz) {
                int k2 = kx * kx + ky * ky + kz * kz;
                bool half = kx > 0 || (kx == 0 && ky > 0) || (kx == 0 && ky == 0 && kz > 0);
                if (k2 >= 1 && k2 <= 9 && half) s += 1.0 / k2;
            }
    return amp * std::sqrt((1.0 - alpha * alpha) / (8.0 * beta * beta * s));
}

bool divides(int n, int t) { return t > 0 && n % t == 0; }

}  // namespace

struct gmt_ctx {
    gmt_params p;
    int device = 0;
    int esize = 4;            // bytes per real
    size_t n = 0;             // cells
    int ox = 0, oy = 0, lz = 0;
    unsigned long long* cfl = nullptr;   // [2]
    double* diag_part = nullptr;
    double* diag_out = nullptr;
    int diag_blocks = 592;
    double* modes = nullptr;  // [61][3][2]
    void* btab = nullptr;     // [nz][ny][24] reals
    void* trig[3] = {nullptr, nullptr, nullptr};
    void* trig8 = nullptr;    // FP32: x table [nx][4][2] of 2 cos, -2 sin for the vectorised forcing kick
    void* ct_scratch = nullptr;
    void* fmass = nullptr;         // march with species: lower-face mass fluxes (3 planes)
    unsigned long long* divb = nullptr;
    int* err = nullptr;       // device flag set by kernels whose bounded waits gave up
    LoopState* loop = nullptr;     // device-resident time loop record (gmt_run)
    LoopConst* loopc = nullptr;
    void* bt = nullptr;            // BoxTables<R> of this box
    const int* mode_k_dev = nullptr;
    cudaStream_t cap = nullptr;    // private stream for graph capture
    struct Graph { const void* u; const void* w; int flags; cudaGraphExec_t exec; };
    std::vector<Graph> graphs;
    double next_time = 0.0;        // next forcing update time
    void* spec = nullptr;          // spectrum scratch (grown on demand)
    size_t spec_bytes = 0;
    uint32_t counter = 0;
    double sigma0 = 0, alpha = 0, beta = 0;
    void* adj = nullptr;           // adjoint scratch (207 planes, allocated on first use)
    double* adj_damp = nullptr;    // dL/d(turb_amp) accumulator
    int* adj_err = nullptr;        // set when the adjoint's record tile abandons a bounded wait
    int adj_percell = 0;           // 1: the adjoint runs its first three passes per cell
    long long wait_cycles = GMT_WAIT_CYCLES;   // budget of the tile kernels' bounded waits
    int wait_test = 0;             // failure-path tests: staging withheld, so every bounded wait runs out
    struct TmaMap { const void* base; CUtensorMap map; };
    TmaMap tma[2] = {};            // tensor maps of the last two input states (tile staging)
    int tma_next = 0;
    struct CtTmaMap { const void* base; CUtensorMap map8, map1; };
    CtTmaMap ct_tma[2] = {};       // the same for the CT state (8 variables, and bzf alone)
    int ct_tma_next = 0;
};

namespace {

template <class R> Consts<R> consts_of(const gmt_params& p) {
    Consts<R> K;
    K.gamma = (R)p.gamma;
    K.smallr = (R)p.smallr;
    K.smallc = (R)p.smallc;
    K.pfl = K.smallr * (K.smallc * K.smallc) / K.gamma;
    K.smallp = (R)p.smallp;
    K.llf_dmin = (R)p.llf_dmin;
    K.llf_pmin = (R)p.llf_pmin;
    K.turb_min_rho = (R)p.turb_min_rho;
    return K;
}

int choose_tile(gmt_ctx* c, bool ct = false) {
    const gmt_params& p = c->p;
    const int maxt = ct ? ct_max_threads(c->esize) : unsplit_max_threads(c->esize);
    auto smem = [&](int ox, int oy) { return ct ? ct_smem_of(c->esize, ox, oy) : unsplit_smem(c->esize, ox, oy); };
    // largest first: 32x16 (512 threads, one block per SM) measured fastest at 512^3 FP32 for
    // both the unsplit and the march scheme; FP64 stops at 256 threads
    static const int cand[][2] = {{32, 16}, {32, 8}, {32, 4}, {16, 8}, {16, 4}, {8, 8}, {8, 4}, {4, 4},
                                  {8, 2}, {4, 2}, {2, 2}, {8, 1}, {4, 1}, {2, 1}, {1, 1}};
    int ox = p.tile_x, oy = p.tile_y;
    auto fits = [&](int tx, int ty) {
        return divides(p.nx, tx) && divides(p.ny, ty) && tx * ty <= maxt && smem(tx, ty) <= 227 * 1024;
    };
    if (ox <= 0 || oy <= 0) {
        ox = oy = 0;
        if (!ct && c->esize == 8 && fits(16, 16)) {
            // the FP64 step: 16x16 (a compile-time tile) has less halo than 32x8 and measured
            // 3.8 % faster at 512^3 than the runtime 32x8 tile
            ox = oy = 16;
        } else {
            for (auto& t : cand)
                if (fits(t[0], t[1])) {
                    ox = t[0];
                    oy = t[1];
                    break;
                }
        }
    }
    if (!divides(p.nx, ox) || !divides(p.ny, oy))
        return fail(GMT_ERR_ARG, "tile " + std::to_string(ox) + "x" + std::to_string(oy) + " does not divide the grid");
    if (ox * oy > maxt) return fail(GMT_ERR_ARG, "tile_x*tile_y must be <= " + std::to_string(maxt));
    if (smem(ox, oy) > 227 * 1024) return fail(GMT_ERR_ARG, "tile needs more than 227 KB shared memory");
    int lz = p.tile_z;
    if (lz <= 0) {
        long cols = (long)(p.nx / ox) * (p.ny / oy);
        lz = p.nz;
        while (lz > 8 && cols * ((p.nz + lz - 1) / lz) < 148L * 8) lz = (lz + 1) / 2;
    }
    c->ox = ox; c->oy = oy; c->lz = std::min(lz, p.nz);
    return GMT_OK;
}

// cuTensorMapEncodeTiled, looked up once through the runtime (the library does not link libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// The tile marches stage their planes by TMA when the input state is one array of its planes
// (plane stride nx*ny*nz), 16-byte aligned, with nx and the tile width multiples of 4 (16-byte
// rows and box origins in either precision): a 4-D map (x, y, z, variable) whose box is the tile's
// staged region, (ox+8) x (oy+4 or 5) x 1 plane x the variables.  Otherwise use_tma stays 0 and
// every tile uses cp.async.
// a 4-D map (x, y, z, variable) of nvar planes of nx*ny*nz reals from base, box bx x by x 1 x bv;
// false if it cannot be made (then the caller stages by cp.async)
template <class R>
bool encode_state_map(CUtensorMap* m, const R* base, int nx, int ny, int nz, int nvar, int bx, int by, int bv) {
    EncodeTiledFn enc = encode_tiled_fn();
    if (!enc) return false;
    const size_t n = (size_t)nx * ny * nz, es = sizeof(R);
    const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nvar};
    const cuuint64_t strides[3] = {(cuuint64_t)nx * es, (cuuint64_t)nx * ny * es, (cuuint64_t)n * es};
    const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, 1, (cuuint32_t)bv};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    const CUtensorMapDataType dt = es == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    return enc(m, dt, 4, const_cast<R*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// the TMA preconditions shared by both tile marches: one array of nvar planes, 16-byte aligned,
// nx and the tile width multiples of 4, box extents within 256 and the grid at least one box
template <class R, class P>
const R* tma_base(const P& planes, int nvar, int nx, int ny, int nz, int ox, int oy, int rows) {
    if (nx % 4 != 0 || ox % 4 != 0 || ox + 8 > 256 || oy + rows > 256 || nx < ox + 8 || ny < oy + rows) return nullptr;
    const size_t n = (size_t)nx * ny * nz;
    const R* base = planes.p[0];
    for (int v = 1; v < nvar; ++v)
        if (planes.p[v] != base + (size_t)v * n) return nullptr;
    if (reinterpret_cast<uintptr_t>(base) % 16 != 0) return nullptr;
    return base;
}

template <class R> void set_tma(gmt_ctx* c, UnsplitArgs<R>& A) {
    A.use_tma = 0;
    std::memset(&A.tmap, 0, sizeof(A.tmap));
    const R* base = tma_base<R>(A.u, 9, A.nx, A.ny, A.nz, A.ox, A.oy, 4);
    if (!base) return;
    for (const gmt_ctx::TmaMap& t : c->tma)
        if (t.base == base) {
            A.tmap = t.map;
            A.use_tma = 1;
            return;
        }
    CUtensorMap m;
    if (!encode_state_map(&m, base, A.nx, A.ny, A.nz, 9, A.ox + 8, A.oy + 4, 9)) return;
    c->tma[c->tma_next].base = base;
    c->tma[c->tma_next].map = m;
    c->tma_next ^= 1;
    A.tmap = m;
    A.use_tma = 1;
}

// CT: the staged region is (ox+8) x (oy+5) cells; one map moves the 8 state variables, one bzf
template <class R> void set_ct_tma(gmt_ctx* c, CTArgs<R>& A) {
    A.use_tma = 0;
    std::memset(&A.tmap8, 0, sizeof(A.tmap8));
    std::memset(&A.tmap1, 0, sizeof(A.tmap1));
    const R* base = tma_base<R>(A.q, 8, A.nx, A.ny, A.nz, A.ox, A.oy, 5);
    if (!base) return;
    for (const gmt_ctx::CtTmaMap& t : c->ct_tma)
        if (t.base == base) {
            A.tmap8 = t.map8;
            A.tmap1 = t.map1;
            A.use_tma = 1;
            return;
        }
    CUtensorMap m8, m1;
    if (!encode_state_map(&m8, base, A.nx, A.ny, A.nz, 8, A.ox + 8, A.oy + 5, 8)) return;
    if (!encode_state_map(&m1, base, A.nx, A.ny, A.nz, 8, A.ox + 8, A.oy + 5, 1)) return;
    c->ct_tma[c->ct_tma_next].base = base;
    c->ct_tma[c->ct_tma_next].map8 = m8;
    c->ct_tma[c->ct_tma_next].map1 = m1;
    c->ct_tma_next ^= 1;
    A.tmap8 = m8;
    A.tmap1 = m1;
    A.use_tma = 1;
}

template <class R> CPlanes<R> cplanes(const void* base, size_t n) {
    CPlanes<R> P;
    for (int v = 0; v < 9; ++v) P.p[v] = static_cast<const R*>(base) + (size_t)v * n;
    return P;
}
template <class R> Planes<R> planes(void* base, size_t n) {
    Planes<R> P;
    for (int v = 0; v < 9; ++v) P.p[v] = static_cast<R*>(base) + (size_t)v * n;
    return P;
}

template <class R>
int step_impl(gmt_ctx* c, const CPlanes<R>& u, const Planes<R>& o, const gmt_step_args* a, cudaStream_t s,
              const void* const* sp_in = nullptr, void* const* sp_out = nullptr) {
    const gmt_params& p = c->p;
    const double dx = p.boxlen / p.nx;
    if (!(a->dt > 0.0) || !std::isfinite(a->dt)) return fail(GMT_ERR_ARG, "dt must be positive and finite");
    if (p.scheme == GMT_SCHEME_UNSPLIT) {
        if (!(a->ch > 0.0)) return fail(GMT_ERR_ARG, "ch must be positive");
        UnsplitArgs<R> A;
        A.u = u; A.o = o;
        A.nx = p.nx; A.ny = p.ny; A.nz = p.nz;
        A.ox = c->ox; A.oy = c->oy; A.lz = c->lz;
        A.dt = (R)a->dt; A.dtdx = A.dt / (R)dx;
        A.ch = (R)a->ch; A.glm_fac = (R)a->glm_fac;
        A.ramp = (R)(p.turb_T > 0 ? std::min(a->t / p.turb_T, 1.0) : 1.0);
        A.K = consts_of<R>(p);
        A.iflo = p.iflo; A.use_llf = p.riemann == GMT_RIEMANN_LLF; A.do_turb = a->do_turb;
        A.btab = a->do_turb ? static_cast<const R*>(c->btab) : nullptr;
        A.trigx = static_cast<const R*>(c->trig[0]);
        A.trig8 = static_cast<const R*>(c->trig8);
        A.cfl_out = nullptr;
        A.err = c->err;
        A.wait_cycles = c->wait_cycles;
        A.wait_test = c->wait_test;
        A.dx = (R)dx;
        A.dparams = nullptr;
        A.fmass = nullptr;
        set_tma(c, A);
        if (a->want_cfl) {
            GMT_CUDA(cudaMemsetAsync(c->cfl, 0, 2 * sizeof(unsigned long long), s));
            A.cfl_out = c->cfl;
        }
        int riem = p.riemann == GMT_RIEMANN_LLF ? GMT_RIEMANN_HLLD : p.riemann;
        cudaError_t e = launch_unsplit(A, p.recon, riem, s);
        if (e != cudaSuccess) return cuda_fail(e, "unsplit step");
        return GMT_OK;
    }
    if (p.scheme == GMT_SCHEME_MARCH1D) {
        // the tiled march: the unsplit tile with the march scheme (one solve per face); with
        // passive species it also stores the face mass fluxes for the species pass
        if (p.nsp > 0 && (!sp_in || !sp_out)) return fail(GMT_ERR_ARG, "gmt_step: species planes missing");
        UnsplitArgs<R> A;
        A.u = u; A.o = o;
        A.nx = p.nx; A.ny = p.ny; A.nz = p.nz;
        A.ox = c->ox; A.oy = c->oy; A.lz = c->lz;
        A.dt = (R)a->dt; A.dtdx = (R)(a->dt / dx);
        A.ch = (R)a->ch; A.glm_fac = (R)a->glm_fac;
        A.ramp = R(1);
        A.K = consts_of<R>(p);
        A.iflo = 0; A.use_llf = 0; A.do_turb = 0;
        A.btab = nullptr;
        A.trigx = static_cast<const R*>(c->trig[0]);
        A.trig8 = static_cast<const R*>(c->trig8);
        A.cfl_out = nullptr;
        A.err = c->err;
        A.wait_cycles = c->wait_cycles;
        A.wait_test = c->wait_test;
        A.dx = (R)dx;
        A.dparams = nullptr;
        A.fmass = p.nsp > 0 ? static_cast<R*>(c->fmass) : nullptr;
        set_tma(c, A);
        if (a->want_cfl) {
            GMT_CUDA(cudaMemsetAsync(c->cfl, 0, 2 * sizeof(unsigned long long), s));
            A.cfl_out = c->cfl;
        }
        cudaError_t e = launch_march_tiled(A, p.recon, s);
        if (e != cudaSuccess) return cuda_fail(e, "march step");
        if (p.nsp > 0) {
            MarchArgs<R> M;
            M.u = u; M.o = o;
            M.nx = p.nx; M.ny = p.ny; M.nz = p.nz;
            M.ox = c->ox; M.oy = c->oy; M.lz = c->lz;
            M.dtdx = A.dtdx;
            M.ch = A.ch; M.glm_fac = A.glm_fac;
            M.K = A.K;
            M.ppm = p.recon == GMT_RECON_PPM;
            M.nsp = p.nsp;
            for (int k = 0; k < MAX_SPECIES; ++k) { M.su[k] = nullptr; M.so[k] = nullptr; }
            for (int k = 0; k < p.nsp; ++k) {
                M.su[k] = static_cast<const R*>(sp_in[k]);
                M.so[k] = static_cast<R*>(sp_out[k]);
                if (!M.su[k] || !M.so[k]) return fail(GMT_ERR_ARG, "gmt_step: null species plane");
            }
            e = launch_species(M, static_cast<const R*>(c->fmass), s);
            if (e != cudaSuccess) return cuda_fail(e, "species step");
        }
        return GMT_OK;
    }
    return fail(GMT_ERR_ARG, "gmt_step: this context is a CT context; use gmt_ct_step");
}

template <class R> int refresh_btab(gmt_ctx* c, cudaStream_t s) {
    cudaError_t e = launch_btab<R>(c->modes, static_cast<const R*>(c->trig[1]), static_cast<const R*>(c->trig[2]),
                                   c->p.ny, c->p.nz, static_cast<R*>(c->btab), s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "forcing table");
}
int refresh_btab_any(gmt_ctx* c, cudaStream_t s) {
    return c->esize == 8 ? refresh_btab<double>(c, s) : refresh_btab<float>(c, s);
}

template <class R> CPlanes8<R> cplanes8(const void* base, size_t n) {
    CPlanes8<R> P;
    for (int v = 0; v < 8; ++v) P.p[v] = static_cast<const R*>(base) + (size_t)v * n;
    return P;
}
template <class R> Planes8<R> planes8(void* base, size_t n) {
    Planes8<R> P;
    for (int v = 0; v < 8; ++v) P.p[v] = static_cast<R*>(base) + (size_t)v * n;
    return P;
}

template <class R>
int ct_step_impl(gmt_ctx* c, const CPlanes8<R>& q, const Planes8<R>& o, const gmt_step_args* a, cudaStream_t s) {
    const gmt_params& p = c->p;
    if (!(a->dt > 0.0) || !std::isfinite(a->dt)) return fail(GMT_ERR_ARG, "dt must be positive and finite");
    CTArgs<R> A;
    A.q = q; A.o = o;
    A.nx = p.nx; A.ny = p.ny; A.nz = p.nz;
    A.ox = c->ox; A.oy = c->oy; A.lz = c->lz;
    A.dt = (R)a->dt;
    A.dtdx = A.dt / (R)(p.boxlen / p.nx);
    A.ramp = (R)(p.turb_T > 0 ? std::min(a->t / p.turb_T, 1.0) : 1.0);
    A.K = consts_of<R>(p);
    A.recon = p.recon; A.riem = p.riemann; A.emf = p.emf; A.halfslope = p.ct_halfslope;
    A.do_turb = a->do_turb;
    A.btab = a->do_turb ? static_cast<const R*>(c->btab) : nullptr;
    A.trigx = static_cast<const R*>(c->trig[0]);
    A.trig8 = static_cast<const R*>(c->trig8);
    A.scratch = static_cast<R*>(c->ct_scratch);
    A.err = c->err;
    A.wait_cycles = c->wait_cycles;
    A.wait_test = c->wait_test;
    set_ct_tma(c, A);
    cudaError_t e = launch_ct(A, s);
    if (e != cudaSuccess) return cuda_fail(e, "ct step");
    if (a->want_cfl) {
        CPlanes8<R> oc;
        for (int v = 0; v < 8; ++v) oc.p[v] = o.p[v];
        e = launch_ct_cfl<R>(oc, p.nx, p.ny, p.nz, A.K, c->cfl, s);
        if (e != cudaSuccess) return cuda_fail(e, "ct cfl");
    }
    return GMT_OK;
}

std::once_flag g_mode_once;
cudaError_t g_mode_err = cudaSuccess;

}  // namespace

extern "C" {

const char* gmt_version(void) { return "glmmhd_b200 1.0 (sm_100a)"; }
const char* gmt_last_error(void) { return g_err.c_str(); }

int gmt_params_init(gmt_params* p, int n) {
    if (!p || n <= 0) return fail(GMT_ERR_ARG, "gmt_params_init: null params or n <= 0");
    std::memset(p, 0, sizeof(*p));
    p->abi_version = GMT_ABI_VERSION;
    p->nx = p->ny = p->nz = n;
    p->dtype = GMT_F32;
    p->scheme = GMT_SCHEME_UNSPLIT;
    p->recon = GMT_RECON_MC;
    p->riemann = GMT_RIEMANN_HLLD;
    p->iflo = 1;
    p->emf = GMT_EMF_AVERAGE;
    p->boxlen = 1.0;
    p->gamma = 1.01;
    p->courant = 0.7;
    p->smallr = 1e-6;
    p->smallc = 1e-4;
    p->smallp = 1e-6;
    p->glm_ch_scale = 0.25;
    p->glm_cp_coef = 0.18;
    p->turb_min_rho = 1e-5;
    p->turb_amp = 0.0;
    p->turb_T = 0.3;
    p->turb_ndt = 100;
    p->turb_seed = 1;
    return GMT_OK;
}

int gmt_create(const gmt_params* p, gmt_ctx** out) {
    if (!p || !out) return fail(GMT_ERR_ARG, "gmt_create: null argument");
    *out = nullptr;
    if (p->abi_version != GMT_ABI_VERSION) return fail(GMT_ERR_ARG, "gmt_create: abi_version mismatch");
    if (p->nx < 1 || p->ny < 1 || p->nz < 1) return fail(GMT_ERR_ARG, "gmt_create: grid dimensions must be >= 1");
    if ((double)p->nx * p->ny * p->nz > 4.0e9) return fail(GMT_ERR_ARG, "gmt_create: grid too large (> 4e9 cells)");
    if (p->dtype != GMT_F32 && p->dtype != GMT_F64) return fail(GMT_ERR_ARG, "gmt_create: dtype must be GMT_F32 or GMT_F64");
    if (p->scheme < 0 || p->scheme > 2) return fail(GMT_ERR_ARG, "gmt_create: unknown scheme");
    if (p->recon < 0 || p->recon > 2) return fail(GMT_ERR_ARG, "gmt_create: unknown recon");
    if (p->riemann < 0 || p->riemann > 3) return fail(GMT_ERR_ARG, "gmt_create: unknown riemann");
    if (p->nsp < 0 || p->nsp > GMT_MAX_SPECIES) return fail(GMT_ERR_ARG, "gmt_create: nsp must be 0..GMT_MAX_SPECIES");
    if (p->nsp > 0 && p->scheme != GMT_SCHEME_MARCH1D)
        return fail(GMT_ERR_UNSUPPORTED, "gmt_create: passive species ride the march scheme (spike_mhd.cu NSP)");
    if (p->scheme == GMT_SCHEME_MARCH1D && p->riemann != GMT_RIEMANN_HLL)
        return fail(GMT_ERR_UNSUPPORTED, "gmt_create: the march scheme uses HLL (spike_mhd.cu:199-223)");
    if (p->scheme == GMT_SCHEME_CT && p->riemann != GMT_RIEMANN_HLL && p->riemann != GMT_RIEMANN_HLLD)
        return fail(GMT_ERR_UNSUPPORTED, "gmt_create: CT supports HLL and HLLD");
    if (!(p->gamma > 1.0) || !(p->boxlen > 0.0) || !(p->smallr > 0.0))
        return fail(GMT_ERR_ARG, "gmt_create: gamma > 1, boxlen > 0 and smallr > 0 are required");
    if (p->scheme == GMT_SCHEME_CT && p->recon == GMT_RECON_MINMOD)
        return fail(GMT_ERR_UNSUPPORTED, "gmt_create: CT supports MC and PPM reconstruction");
    std::call_once(g_mode_once, [] { g_mode_err = upload_mode_table(); });
    if (g_mode_err != cudaSuccess) return cuda_fail(g_mode_err, "mode table");
    {
        cudaError_t e = p->dtype == GMT_F64 ? unsplit_prepare_f64() : unsplit_prepare_f32();
        if (e == cudaSuccess && p->scheme == GMT_SCHEME_CT) e = p->dtype == GMT_F64 ? ct_prepare_f64() : ct_prepare_f32();
        if (e != cudaSuccess) return cuda_fail(e, "kernel attributes");
    }

    gmt_ctx* c = new gmt_ctx();
    c->p = *p;
    c->esize = p->dtype == GMT_F64 ? 8 : 4;
    c->n = (size_t)p->nx * p->ny * p->nz;
    cudaGetDevice(&c->device);
    (void)encode_tiled_fn();   // the driver entry point, looked up outside any capture
    int rc = GMT_OK;
    if (p->scheme == GMT_SCHEME_UNSPLIT || p->scheme == GMT_SCHEME_MARCH1D) rc = choose_tile(c);
    if (p->scheme == GMT_SCHEME_CT) rc = choose_tile(c, true);
    if (rc != GMT_OK) { delete c; return rc; }
    auto alloc = [&](void** ptr, size_t bytes) -> bool {
        cudaError_t e = cudaMalloc(ptr, bytes);
        if (e != cudaSuccess) { cuda_fail(e, "cudaMalloc"); return false; }
        return true;
    };
    bool ok = alloc((void**)&c->cfl, 4 * sizeof(unsigned long long)) &&
              alloc((void**)&c->diag_part, (size_t)c->diag_blocks * 8 * sizeof(double)) &&
              alloc((void**)&c->diag_out, 16 * sizeof(double)) &&
              alloc((void**)&c->modes, NMODES * 6 * sizeof(double)) &&
              alloc(&c->btab, (size_t)p->ny * p->nz * 24 * c->esize);
    const int dims[3] = {p->nx, p->ny, p->nz};
    for (int a = 0; ok && a < 3; ++a) ok = alloc(&c->trig[a], (size_t)8 * dims[a] * c->esize);
    if (ok && p->scheme == GMT_SCHEME_CT) ok = alloc(&c->ct_scratch, (size_t)15 * c->n * c->esize);
    if (ok && p->scheme == GMT_SCHEME_MARCH1D && p->nsp > 0) ok = alloc(&c->fmass, (size_t)3 * c->n * c->esize);
    if (ok) ok = alloc((void**)&c->divb, sizeof(unsigned long long));
    if (ok) ok = alloc((void**)&c->err, sizeof(int));
    if (ok) ok = alloc((void**)&c->loop, sizeof(LoopState)) && alloc((void**)&c->loopc, sizeof(LoopConst)) &&
                 alloc(&c->bt, sizeof(BoxTables<double>));
    if (ok && cudaMemset(c->err, 0, sizeof(int)) != cudaSuccess) ok = false;
    if (!ok) { gmt_destroy(c); return GMT_ERR_NOMEM; }
    for (int a = 0; a < 3; ++a) {
        std::vector<double> t = trig_table(dims[a]);
        cudaError_t e;
        if (c->esize == 8) {
            e = cudaMemcpy(c->trig[a], t.data(), t.size() * 8, cudaMemcpyHostToDevice);
        } else {
            std::vector<float> f(t.begin(), t.end());
            e = cudaMemcpy(c->trig[a], f.data(), f.size() * 4, cudaMemcpyHostToDevice);
        }
        if (e != cudaSuccess) { gmt_destroy(c); return cuda_fail(e, "trig upload"); }
    }
    if (c->esize == 4) {
        std::vector<float> t8 = trig8_table(trig_table(p->nx), p->nx);
        cudaError_t e = cudaMalloc(&c->trig8, t8.size() * 4);
        if (e == cudaSuccess) e = cudaMemcpy(c->trig8, t8.data(), t8.size() * 4, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { gmt_destroy(c); return cuda_fail(e, "trig upload"); }
    }
    int nd = p->turb_ndt > 0 ? p->turb_ndt : 100;
    double dtf = p->turb_T / nd;
    c->alpha = 1.0 - dtf / p->turb_T;
    c->beta = std::sqrt(2.0 * dtf / p->turb_T);
    c->sigma0 = forcing_sigma0(p->turb_amp, c->alpha, c->beta);
    rc = gmt_forcing_reset(c, nullptr);
    if (rc == GMT_OK) {
        cudaError_t e = mode_table_device(&c->mode_k_dev);
        if (e == cudaSuccess) {
            if (c->esize == 8) {
                BoxTables<double> T{c->modes, (const double*)c->trig[1], (const double*)c->trig[2], (double*)c->btab, p->ny, p->nz};
                e = cudaMemcpy(c->bt, &T, sizeof(T), cudaMemcpyHostToDevice);
            } else {
                BoxTables<float> T{c->modes, (const float*)c->trig[1], (const float*)c->trig[2], (float*)c->btab, p->ny, p->nz};
                e = cudaMemcpy(c->bt, &T, sizeof(T), cudaMemcpyHostToDevice);
            }
        }
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking);
        if (e != cudaSuccess) rc = cuda_fail(e, "gmt_create");
    }
    if (rc == GMT_OK) {
        cudaError_t e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = cuda_fail(e, "gmt_create");
    }
    if (rc != GMT_OK) { gmt_destroy(c); return rc; }
    *out = c;
    return GMT_OK;
}

int gmt_destroy(gmt_ctx* c) {
    if (!c) return GMT_OK;
    cudaFree(c->cfl);
    cudaFree(c->diag_part);
    cudaFree(c->diag_out);
    cudaFree(c->modes);
    cudaFree(c->btab);
    cudaFree(c->trig8);
    for (auto& t : c->trig) cudaFree(t);
    cudaFree(c->ct_scratch);
    cudaFree(c->fmass);
    cudaFree(c->divb);
    cudaFree(c->err);
    for (auto& g : c->graphs) cudaGraphExecDestroy(g.exec);
    cudaFree(c->spec);
    cudaFree(c->adj);
    cudaFree(c->adj_damp);
    cudaFree(c->adj_err);
    if (c->cap) cudaStreamDestroy(c->cap);
    cudaFree(c->loop);
    cudaFree(c->loopc);
    cudaFree(c->bt);
    delete c;
    return GMT_OK;
}

int gmt_kernel_info(gmt_ctx* c, int32_t* regs, int64_t* smem, int32_t tile[3]) {
    if (!c) return fail(GMT_ERR_ARG, "null context");
    int r = -1;
    int64_t sm = 0;
    if (c->p.scheme == GMT_SCHEME_UNSPLIT) {
        r = unsplit_regs(c->esize, c->p.recon, c->p.riemann == GMT_RIEMANN_LLF ? GMT_RIEMANN_HLLD : c->p.riemann,
                         c->ox * c->oy);
        sm = (int64_t)unsplit_smem(c->esize, c->ox, c->oy);
    } else if (c->p.scheme == GMT_SCHEME_MARCH1D) {
        r = c->esize == 8 ? march_tiled_regs((const UnsplitArgs<double>*)nullptr, c->p.recon, c->ox * c->oy)
                          : march_tiled_regs((const UnsplitArgs<float>*)nullptr, c->p.recon, c->ox * c->oy);
        sm = (int64_t)unsplit_smem(c->esize, c->ox, c->oy);
    } else {
        r = ct_regs_of(c->esize, c->p.recon, c->p.riemann, c->ox * c->oy);
        sm = (int64_t)ct_smem_of(c->esize, c->ox, c->oy);
    }
    if (regs) *regs = r;
    if (smem) *smem = sm;
    if (tile) { tile[0] = c->ox; tile[1] = c->oy; tile[2] = c->lz; }
    return GMT_OK;
}

int gmt_step(gmt_ctx* c, const void* uold, void* unew, const gmt_step_args* a, void* stream) {
    if (!c || !uold || !unew || !a) return fail(GMT_ERR_ARG, "gmt_step: null argument");
    if (uold == unew) return fail(GMT_ERR_ARG, "gmt_step: uold and unew must be different buffers");
    cudaStream_t s = (cudaStream_t)stream;
    const void* si[MAX_SPECIES];
    void* so[MAX_SPECIES];
    for (int k = 0; k < c->p.nsp; ++k) {
        si[k] = static_cast<const char*>(uold) + (size_t)(9 + k) * c->n * c->esize;
        so[k] = static_cast<char*>(unew) + (size_t)(9 + k) * c->n * c->esize;
    }
    if (c->esize == 8)
        return step_impl<double>(c, cplanes<double>(uold, c->n), planes<double>(unew, c->n), a, s, si, so);
    return step_impl<float>(c, cplanes<float>(uold, c->n), planes<float>(unew, c->n), a, s, si, so);
}

int gmt_step_planes(gmt_ctx* c, const void* const* uold, void* const* unew, const gmt_step_args* a, void* stream) {
    if (!c || !uold || !unew || !a) return fail(GMT_ERR_ARG, "gmt_step_planes: null argument");
    for (int v = 0; v < 9; ++v)
        if (!uold[v] || !unew[v]) return fail(GMT_ERR_ARG, "gmt_step_planes: null plane pointer");
    cudaStream_t s = (cudaStream_t)stream;
    if (c->esize == 8) {
        CPlanes<double> u; Planes<double> o;
        for (int v = 0; v < 9; ++v) { u.p[v] = (const double*)uold[v]; o.p[v] = (double*)unew[v]; }
        return step_impl<double>(c, u, o, a, s, uold + 9, unew + 9);
    }
    CPlanes<float> u; Planes<float> o;
    for (int v = 0; v < 9; ++v) { u.p[v] = (const float*)uold[v]; o.p[v] = (float*)unew[v]; }
    return step_impl<float>(c, u, o, a, s, uold + 9, unew + 9);
}

int gmt_cfl_async(gmt_ctx* c, const void* u, void* stream) {
    if (!c || !u) return fail(GMT_ERR_ARG, "gmt_cfl_async: null argument");
    if (c->p.scheme == GMT_SCHEME_CT) return gmt_ct_cfl_async(c, u, stream);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = c->esize == 8 ? launch_cfl<double>(cplanes<double>(u, c->n), c->n, consts_of<double>(c->p), c->cfl, s)
                                  : launch_cfl<float>(cplanes<float>(u, c->n), c->n, consts_of<float>(c->p), c->cfl, s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "cfl");
}

int gmt_cfl_result(gmt_ctx* c, double out[2], void* stream) {
    if (!c || !out) return fail(GMT_ERR_ARG, "gmt_cfl_result: null argument");
    unsigned long long h[2];
    int herr = 0;
    GMT_CUDA(cudaMemcpyAsync(h, c->cfl, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    GMT_CUDA(cudaMemcpyAsync(&herr, c->err, sizeof(int), cudaMemcpyDeviceToHost, (cudaStream_t)stream));
    GMT_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
    if (herr) {
        cudaMemsetAsync(c->err, 0, sizeof(int), (cudaStream_t)stream);
        return fail(GMT_ERR_TIMEOUT, "a step kernel abandoned a bounded wait; its output is invalid");
    }
    std::memcpy(&out[0], &h[0], 8);
    std::memcpy(&out[1], &h[1], 8);
    if (!std::isfinite(out[0]) || !(out[0] > 0.0)) return fail(GMT_ERR_STATE, "CFL maximum is not positive and finite");
    return GMT_OK;
}

int gmt_compute_dt(gmt_ctx* c, const void* u, double* dt, void* stream) {
    if (!dt) return fail(GMT_ERR_ARG, "gmt_compute_dt: null dt");
    int rc = gmt_cfl_async(c, u, stream);
    if (rc) return rc;
    double m[2];
    rc = gmt_cfl_result(c, m, stream);
    if (rc) return rc;
    *dt = c->p.courant * (c->p.boxlen / c->p.nx) / m[0];
    return GMT_OK;
}

int gmt_diagnostics(gmt_ctx* c, const void* u, gmt_diag* out, void* stream) {
    if (!c || !u || !out) return fail(GMT_ERR_ARG, "gmt_diagnostics: null argument");
    if (c->p.scheme == GMT_SCHEME_CT) return fail(GMT_ERR_ARG, "gmt_diagnostics: GLM state only; use gmt_ct_divb_max");
    cudaStream_t s = (cudaStream_t)stream;
    const double dx = c->p.boxlen / c->p.nx;
    cudaError_t e = c->esize == 8
                        ? launch_diag<double>(cplanes<double>(u, c->n), c->p.nx, c->p.ny, c->p.nz, dx, c->p.smallr,
                                              c->diag_part, c->diag_blocks, c->diag_out, s)
                        : launch_diag<float>(cplanes<float>(u, c->n), c->p.nx, c->p.ny, c->p.nz, dx, c->p.smallr,
                                             c->diag_part, c->diag_blocks, c->diag_out, s);
    if (e != cudaSuccess) return cuda_fail(e, "diagnostics");
    double h[8];
    GMT_CUDA(cudaMemcpyAsync(h, c->diag_out, sizeof(h), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaStreamSynchronize(s));
    out->mass = h[0]; out->ke2 = h[1]; out->etot = h[2];
    out->psi_l2 = std::sqrt(h[3] / (double)c->n);
    out->divb_l2 = std::sqrt(h[4] / (double)c->n);
    out->divbmax = h[5]; out->rhomin = h[6];
    out->vrms = std::sqrt(h[1] / h[0]);
    out->nonfinite_cells = (int32_t)h[7];
    out->finite = h[7] == 0.0;
    return GMT_OK;
}

int gmt_ke_spectrum(gmt_ctx* c, const void* u, int32_t kmax, double* out, void* stream) {
    if (!c || !u || !out) return fail(GMT_ERR_ARG, "gmt_ke_spectrum: null argument");
    if (c->p.scheme == GMT_SCHEME_CT) return fail(GMT_ERR_ARG, "gmt_ke_spectrum: GLM state only");
    if (kmax < 1 || 2 * kmax + 1 > std::min(c->p.ny, c->p.nz) || kmax + 1 > c->p.nx)
        return fail(GMT_ERR_ARG, "gmt_ke_spectrum: need 1 <= kmax and 2*kmax+1 <= grid size");
    size_t need = spectrum_scratch_bytes(c->p.nx, c->p.ny, c->p.nz, kmax);
    if (need > c->spec_bytes) {
        cudaFree(c->spec);
        c->spec = nullptr;
        c->spec_bytes = 0;
        GMT_CUDA(cudaMalloc(&c->spec, need));
        c->spec_bytes = need;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = c->esize == 8
                        ? launch_spectrum<double>(cplanes<double>(u, c->n), c->p.nx, c->p.ny, c->p.nz, kmax, c->spec, out, s)
                        : launch_spectrum<float>(cplanes<float>(u, c->n), c->p.nx, c->p.ny, c->p.nz, kmax, c->spec, out, s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "gmt_ke_spectrum");
}

int gmt_density_pdf(gmt_ctx* c, const void* u, int32_t nbins, double smin, double smax, double* pdf, double stats[3],
                    void* stream) {
    if (!c || !u || !pdf || !stats) return fail(GMT_ERR_ARG, "gmt_density_pdf: null argument");
    if (nbins < 1 || nbins > GMT_PDF_MAX_BINS) return fail(GMT_ERR_ARG, "gmt_density_pdf: nbins must be 1..4096");
    if (!(smax > smin) || !std::isfinite(smin) || !std::isfinite(smax))
        return fail(GMT_ERR_ARG, "gmt_density_pdf: need finite smin < smax");
    size_t need = pdf_scratch_bytes(nbins);
    if (need > c->spec_bytes) {
        cudaFree(c->spec);
        c->spec = nullptr;
        c->spec_bytes = 0;
        GMT_CUDA(cudaMalloc(&c->spec, need));
        c->spec_bytes = need;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = c->esize == 8
        ? launch_density_pdf<double>(static_cast<const double*>(u), c->n, nbins, smin, smax, c->spec, pdf, stats, s)
        : launch_density_pdf<float>(static_cast<const float*>(u), c->n, nbins, smin, smax, c->spec, pdf, stats, s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "gmt_density_pdf");
}

int gmt_ke_band_loss(gmt_ctx* c, const void* u, int32_t kmin, int32_t kmax, double* loss, void* ubar, void* stream) {
    if (!c || !u || !loss) return fail(GMT_ERR_ARG, "gmt_ke_band_loss: null argument");
    if (c->p.scheme == GMT_SCHEME_CT) return fail(GMT_ERR_ARG, "gmt_ke_band_loss: GLM state only");
    if (kmin < 0 || kmax < kmin || kmax < 1 || 2 * kmax + 1 > std::min(c->p.ny, c->p.nz) || kmax + 1 > c->p.nx)
        return fail(GMT_ERR_ARG, "gmt_ke_band_loss: need 0 <= kmin <= kmax, 1 <= kmax, 2*kmax+1 <= grid size");
    size_t need = band_scratch_bytes(c->p.nx, c->p.ny, c->p.nz, kmax);
    if (need > c->spec_bytes) {
        cudaFree(c->spec);
        c->spec = nullptr;
        c->spec_bytes = 0;
        GMT_CUDA(cudaMalloc(&c->spec, need));
        c->spec_bytes = need;
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (!ubar) return fail(GMT_ERR_ARG, "gmt_ke_band_loss: ubar is required (9 planes of the state's dtype)");
    void* ub = ubar;
    cudaError_t e = c->esize == 8
        ? launch_band_loss<double>(cplanes<double>(u, c->n), c->p.nx, c->p.ny, c->p.nz, kmin, kmax, c->spec, loss,
                                   planes<double>(ub, c->n), s)
        : launch_band_loss<float>(cplanes<float>(u, c->n), c->p.nx, c->p.ny, c->p.nz, kmin, kmax, c->spec, loss,
                                  planes<float>(ub, c->n), s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "gmt_ke_band_loss");
}

int gmt_adjoint_step(gmt_ctx* c, const void* u, const void* ubar_next, void* ubar, const gmt_step_args* a,
                     void* stream) {
    if (!c || !u || !ubar_next || !ubar || !a) return fail(GMT_ERR_ARG, "gmt_adjoint_step: null argument");
    const gmt_params& p = c->p;
    if (p.scheme != GMT_SCHEME_UNSPLIT) return fail(GMT_ERR_ARG, "gmt_adjoint_step: unsplit GLM contexts only");
    if (p.recon == GMT_RECON_PPM) return fail(GMT_ERR_ARG, "gmt_adjoint_step: PLM (MC or minmod) only");
    if (ubar == u || ubar == ubar_next) return fail(GMT_ERR_ARG, "gmt_adjoint_step: ubar aliases an input");
    if (!(a->dt > 0.0) || !std::isfinite(a->dt)) return fail(GMT_ERR_ARG, "dt must be positive and finite");
    if (!(a->ch > 0.0)) return fail(GMT_ERR_ARG, "ch must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    if (!c->adj) {
        GMT_CUDA(cudaMalloc(&c->adj, adjoint_scratch_reals(c->n) * c->esize));
        GMT_CUDA(cudaMalloc(&c->adj_damp, sizeof(double)));
        GMT_CUDA(cudaMalloc(&c->adj_err, sizeof(int)));
        GMT_CUDA(cudaMemsetAsync(c->adj_damp, 0, sizeof(double), s));
        GMT_CUDA(cudaMemsetAsync(c->adj_err, 0, sizeof(int), s));
    }
    const double dx = p.boxlen / p.nx;
    auto go = [&](auto zero) -> int {
        using R = decltype(zero);
        AdjArgs<R> A;
        A.u = cplanes<R>(u, c->n);
        A.ubn = cplanes<R>(ubar_next, c->n);
        A.ub = planes<R>(ubar, c->n);
        A.nx = p.nx; A.ny = p.ny; A.nz = p.nz;
        A.dt = (R)a->dt; A.dtdx = A.dt / (R)dx;
        A.ch = (R)a->ch; A.glm_fac = (R)a->glm_fac;
        A.ramp = (R)(p.turb_T > 0 ? std::min(a->t / p.turb_T, 1.0) : 1.0);
        A.amp = (R)p.turb_amp;
        A.K = consts_of<R>(p);
        A.iflo = p.iflo; A.use_llf = p.riemann == GMT_RIEMANN_LLF; A.do_turb = a->do_turb;
        A.recon = p.recon;
        A.riem = p.riemann == GMT_RIEMANN_LLF ? GMT_RIEMANN_HLLD : p.riemann;
        A.btab = a->do_turb ? static_cast<const R*>(c->btab) : nullptr;
        A.trigx = static_cast<const R*>(c->trig[0]);
        R* base = static_cast<R*>(c->adj);
        A.FS = base;
        A.FL = A.FS + 54 * c->n;
        A.R1b = A.FL + 27 * c->n;
        A.FSb = A.R1b + 9 * c->n;
        A.QB = A.FSb + 54 * c->n;
        A.damp = c->adj_damp;
        // passes 1-3 by the forward step's tile march in record mode (the context's tile)
        UnsplitArgs<R> T;
        T.u = A.u;
        T.o = planes<R>(ubar, c->n);   // not written in record mode
        T.nx = p.nx; T.ny = p.ny; T.nz = p.nz;
        T.ox = c->ox; T.oy = c->oy; T.lz = c->lz;
        T.dt = A.dt; T.dtdx = A.dtdx; T.ch = A.ch; T.glm_fac = A.glm_fac; T.ramp = A.ramp;
        T.K = A.K;
        T.iflo = A.iflo; T.use_llf = A.use_llf; T.do_turb = A.do_turb;
        T.btab = A.btab; T.trigx = A.trigx; T.trig8 = static_cast<const R*>(c->trig8);
        T.cfl_out = nullptr;
        T.err = c->adj_err;
        T.wait_cycles = c->wait_cycles;
        T.wait_test = c->wait_test;
        T.dx = (R)dx;
        T.dparams = nullptr;
        T.fmass = nullptr;
        set_tma(c, T);
        T.rec_fs = A.FS;
        T.rec_ubn = A.ubn.p[0];
        T.rec_r1b = A.R1b;
        T.rec_ub = A.ub.p[0];
        T.rec_damp = A.damp;
        T.rec_amp = A.amp;
        const bool record = c->ox > 0 && c->oy > 0 && c->lz > 0 && !c->adj_percell;
        cudaError_t e = launch_adjoint<R>(A, record ? &T : nullptr, s);
        return e == cudaSuccess ? GMT_OK : cuda_fail(e, "gmt_adjoint_step");
    };
    return c->esize == 8 ? go(0.0) : go(0.0f);
}

int gmt_adjoint_amp_grad(gmt_ctx* c, double* out, int32_t reset, void* stream) {
    if (!c || !out) return fail(GMT_ERR_ARG, "gmt_adjoint_amp_grad: null argument");
    cudaStream_t s = (cudaStream_t)stream;
    if (!c->adj_damp) { *out = 0.0; return GMT_OK; }
    int herr = 0;
    GMT_CUDA(cudaMemcpyAsync(out, c->adj_damp, sizeof(double), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaMemcpyAsync(&herr, c->adj_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (reset) GMT_CUDA(cudaMemsetAsync(c->adj_damp, 0, sizeof(double), s));
    GMT_CUDA(cudaStreamSynchronize(s));
    if (herr) {
        GMT_CUDA(cudaMemsetAsync(c->adj_err, 0, sizeof(int), s));
        GMT_CUDA(cudaStreamSynchronize(s));
        return fail(GMT_ERR_TIMEOUT, "an adjoint step abandoned a bounded wait in its record tile; the gradients "
                                     "accumulated since the last check are invalid");
    }
    return GMT_OK;
}

int gmt_adjoint_set_passes(gmt_ctx* c, int32_t percell) {
    if (!c) return fail(GMT_ERR_ARG, "gmt_adjoint_set_passes: null context");
    c->adj_percell = percell != 0;
    return GMT_OK;
}

int gmt_test_wait_limit(gmt_ctx* c, int64_t budget_cycles, int32_t withhold) {
    if (!c) return fail(GMT_ERR_ARG, "gmt_test_wait_limit: null context");
    if (budget_cycles < 0) return fail(GMT_ERR_ARG, "gmt_test_wait_limit: budget_cycles must be >= 0");
    c->wait_cycles = budget_cycles > 0 ? (long long)budget_cycles : GMT_WAIT_CYCLES;
    c->wait_test = withhold != 0;
    for (auto& g : c->graphs) cudaGraphExecDestroy(g.exec);   // they hold the old kernel arguments
    c->graphs.clear();
    return GMT_OK;
}

int gmt_forcing_reset(gmt_ctx* c, void* stream) {
    if (!c) return fail(GMT_ERR_ARG, "null context");
    cudaStream_t s = (cudaStream_t)stream;
    GMT_CUDA(cudaMemsetAsync(c->modes, 0, NMODES * 6 * sizeof(double), s));
    c->counter = 0;
    c->next_time = 0.0;
    return refresh_btab_any(c, s);
}

int gmt_forcing_advance(gmt_ctx* c, void* stream) {
    if (!c) return fail(GMT_ERR_ARG, "null context");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = launch_ou_update(c->modes, c->p.turb_seed, c->counter, c->alpha, c->beta, c->sigma0, s);
    if (e != cudaSuccess) return cuda_fail(e, "OU update");
    c->counter++;
    c->next_time += c->p.turb_T / (c->p.turb_ndt > 0 ? c->p.turb_ndt : 100);
    return refresh_btab_any(c, s);
}

int gmt_forcing_set_modes(gmt_ctx* c, const double* modes, void* stream) {
    if (!c || !modes) return fail(GMT_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    GMT_CUDA(cudaMemcpyAsync(c->modes, modes, NMODES * 6 * sizeof(double), cudaMemcpyHostToDevice, s));
    GMT_CUDA(cudaStreamSynchronize(s));
    return refresh_btab_any(c, s);
}

int gmt_forcing_get_modes(gmt_ctx* c, double* modes, void* stream) {
    if (!c || !modes) return fail(GMT_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    GMT_CUDA(cudaMemcpyAsync(modes, c->modes, NMODES * 6 * sizeof(double), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaStreamSynchronize(s));
    return GMT_OK;
}

int gmt_forcing_get_state(gmt_ctx* c, double* modes, uint32_t* counter, double* next_time, void* stream) {
    if (!c || !modes || !counter || !next_time) return fail(GMT_ERR_ARG, "gmt_forcing_get_state: null argument");
    int rc = gmt_forcing_get_modes(c, modes, stream);
    if (rc) return rc;
    *counter = c->counter;
    *next_time = c->next_time;
    return GMT_OK;
}

int gmt_forcing_set_state(gmt_ctx* c, const double* modes, uint32_t counter, double next_time, void* stream) {
    if (!c || !modes) return fail(GMT_ERR_ARG, "gmt_forcing_set_state: null argument");
    if (!std::isfinite(next_time)) return fail(GMT_ERR_ARG, "gmt_forcing_set_state: next_time must be finite");
    int rc = gmt_forcing_set_modes(c, modes, stream);
    if (rc) return rc;
    c->counter = counter;
    c->next_time = next_time;
    return GMT_OK;
}

int gmt_forcing_counter(gmt_ctx* c, uint32_t* counter) {
    if (!c || !counter) return fail(GMT_ERR_ARG, "null argument");
    *counter = c->counter;
    return GMT_OK;
}

int gmt_ic_orszag_tang(gmt_ctx* c, void* u, void* stream) {
    if (!c || !u) return fail(GMT_ERR_ARG, "null argument");
    if (c->p.scheme == GMT_SCHEME_CT) return gmt_ct_ic_orszag_tang(c, u, stream);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = c->esize == 8 ? launch_ic_ot<double>(planes<double>(u, c->n), c->p.nx, c->p.ny, c->p.nz, c->p.gamma, s)
                                  : launch_ic_ot<float>(planes<float>(u, c->n), c->p.nx, c->p.ny, c->p.nz, c->p.gamma, s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "ic");
}

int gmt_ic_uniform(gmt_ctx* c, void* u, double rho0, double p0, double bx0, double by0, double bz0, void* stream) {
    if (!c || !u) return fail(GMT_ERR_ARG, "null argument");
    if (c->p.scheme == GMT_SCHEME_CT) return fail(GMT_ERR_ARG, "gmt_ic_uniform: GLM state only");
    double v9[9] = {rho0, 0, 0, 0, p0 / (c->p.gamma - 1.0) + 0.5 * (bx0 * bx0 + by0 * by0 + bz0 * bz0), bx0, by0, bz0, 0};
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = c->esize == 8 ? launch_ic_uniform<double>(planes<double>(u, c->n), c->n, v9, s)
                                  : launch_ic_uniform<float>(planes<float>(u, c->n), c->n, v9, s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "ic");
}

int gmt_ic_turbulent(gmt_ctx* c, void* u, double rho0, double p0, double bx0, double by0, double bz0, double mach,
                     double db, uint32_t seed, void* stream) {
    if (!c || !u) return fail(GMT_ERR_ARG, "null argument");
    if (!(rho0 > 0) || !(p0 > 0)) return fail(GMT_ERR_ARG, "gmt_ic_turbulent: rho0 and p0 must be positive");
    cudaStream_t s = (cudaStream_t)stream;
    double* m = nullptr;
    void* bt = nullptr;
    GMT_CUDA(cudaMalloc(&m, NMODES * 6 * sizeof(double)));
    cudaError_t e = cudaMalloc(&bt, (size_t)c->p.ny * c->p.nz * 24 * c->esize);
    if (e == cudaSuccess) e = cudaMemsetAsync(m, 0, NMODES * 6 * sizeof(double), s);
    if (e == cudaSuccess) e = launch_ou_update(m, seed, 0u, 0.0, 1.0, forcing_sigma0(1.0, 0.0, 1.0), s);
    const double b0[3] = {bx0, by0, bz0};
    const double vscale = mach * std::sqrt(c->p.gamma * p0 / rho0);
    if (e == cudaSuccess && c->p.scheme == GMT_SCHEME_CT) {
        // face fields from an edge vector potential (divergence-free to round-off); the CT scratch
        // holds the three potential planes
        e = c->esize == 8 ? launch_ct_ic_turb<double>(planes8<double>(u, c->n), c->p.nx, c->p.ny, c->p.nz, m,
                                                      static_cast<double*>(c->ct_scratch), rho0, p0, b0, vscale, db,
                                                      c->p.gamma, s)
                          : launch_ct_ic_turb<float>(planes8<float>(u, c->n), c->p.nx, c->p.ny, c->p.nz, m,
                                                     static_cast<float*>(c->ct_scratch), rho0, p0, b0, vscale, db,
                                                     c->p.gamma, s);
    } else if (e == cudaSuccess) {
        if (c->esize == 8) {
            e = launch_btab<double>(m, (const double*)c->trig[1], (const double*)c->trig[2], c->p.ny, c->p.nz,
                                    (double*)bt, s);
            if (e == cudaSuccess)
                e = launch_ic_turb<double>(planes<double>(u, c->n), c->p.nx, c->p.ny, c->p.nz, (const double*)bt,
                                           (const double*)c->trig[0], rho0, p0, b0, vscale, db, c->p.gamma, s);
        } else {
            e = launch_btab<float>(m, (const float*)c->trig[1], (const float*)c->trig[2], c->p.ny, c->p.nz,
                                   (float*)bt, s);
            if (e == cudaSuccess)
                e = launch_ic_turb<float>(planes<float>(u, c->n), c->p.nx, c->p.ny, c->p.nz, (const float*)bt,
                                          (const float*)c->trig[0], rho0, p0, b0, vscale, db, c->p.gamma, s);
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    cudaFree(m);
    cudaFree(bt);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "gmt_ic_turbulent");
}

// ------------------------------------------------------------------------------------------
// device-resident time loop (gmt_run)
// ------------------------------------------------------------------------------------------
}  // extern "C"

namespace {

LoopConst loop_const_of(const gmt_params& p, double alpha, double beta, double sigma0, int flags) {
    LoopConst C{};
    C.courant = p.courant;
    C.dx = p.boxlen / p.nx;
    C.boxlen = p.boxlen;
    C.cp_coef = p.glm_cp_coef;
    C.glm_ch_scale = p.glm_ch_scale;
    C.turb_T = p.turb_T;
    C.dtf = p.turb_T / (p.turb_ndt > 0 ? p.turb_ndt : 100);
    C.alpha = alpha;
    C.beta = beta;
    C.sigma0 = sigma0;
    C.ch_max_signal = (flags & GMT_RUN_CH_MAXSIGNAL) ? 1 : 0;
    C.do_turb = (flags & GMT_RUN_FORCING) ? 1 : 0;
    C.seed = p.turb_seed;
    return C;
}

template <class R>
cudaError_t run_enqueue(gmt_ctx* c, const void* src, void* dst, int flags, cudaStream_t s) {
    const gmt_params& p = c->p;
    tick_kernel<<<1, 32, 0, s>>>(c->loop, c->loopc, c->cfl, 1);
    if (flags & GMT_RUN_FORCING) {
        ou_cond_kernel<<<1, 64, 0, s>>>(c->modes, c->loop, c->loopc, c->mode_k_dev);
        btab_cond_kernel<R><<<dim3((p.ny * p.nz + 255) / 256, 1), 256, 0, s>>>((const BoxTables<R>*)c->bt, c->loop,
                                                                              c->mode_k_dev);
    }
    cudaError_t e = cudaMemsetAsync(c->cfl, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) return e;
    UnsplitArgs<R> A;
    A.u = cplanes<R>(src, c->n);
    A.o = planes<R>(dst, c->n);
    A.nx = p.nx; A.ny = p.ny; A.nz = p.nz;
    A.ox = c->ox; A.oy = c->oy; A.lz = c->lz;
    A.dt = A.dtdx = A.ch = A.glm_fac = A.ramp = R(0);
    A.K = consts_of<R>(p);
    A.iflo = p.iflo; A.use_llf = p.riemann == GMT_RIEMANN_LLF; A.do_turb = (flags & GMT_RUN_FORCING) ? 1 : 0;
    A.btab = A.do_turb ? static_cast<const R*>(c->btab) : nullptr;
    A.trigx = static_cast<const R*>(c->trig[0]);
    A.trig8 = static_cast<const R*>(c->trig8);
    A.cfl_out = c->cfl;
    A.err = c->err;
    A.wait_cycles = c->wait_cycles;
    A.wait_test = c->wait_test;
    A.dx = (R)(p.boxlen / p.nx);
    A.dparams = reinterpret_cast<const double*>(c->loop);
    A.fmass = nullptr;
    set_tma(c, A);
    int riem = p.riemann == GMT_RIEMANN_LLF ? GMT_RIEMANN_HLLD : p.riemann;
    return launch_unsplit(A, p.recon, riem, s);
}

cudaError_t run_enqueue_any(gmt_ctx* c, const void* src, void* dst, int flags, cudaStream_t s) {
    return c->esize == 8 ? run_enqueue<double>(c, src, dst, flags, s) : run_enqueue<float>(c, src, dst, flags, s);
}

}  // namespace

extern "C" {

int gmt_run(gmt_ctx* c, void* u, void* w, int32_t nsteps, double t0, double t_end, int32_t flags, void* stream,
            double* t_out, int32_t* which) {
    if (!c || !u || !w || u == w || nsteps < 0) return fail(GMT_ERR_ARG, "gmt_run: invalid arguments");
    if (c->p.scheme != GMT_SCHEME_UNSPLIT) return fail(GMT_ERR_UNSUPPORTED, "gmt_run: unsplit scheme only");
    if (!(t_end >= t0)) return fail(GMT_ERR_ARG, "gmt_run: t_end < t0");
    cudaStream_t s = (cudaStream_t)stream;
    LoopState S{};
    S.dt = 0.0; S.ch = 1.0; S.glm_fac = 1.0; S.ramp = 0.0;
    S.t = t0; S.t_end = t_end; S.next_time = c->next_time; S.counter = c->counter;
    LoopConst C = loop_const_of(c->p, c->alpha, c->beta, c->sigma0, flags);
    GMT_CUDA(cudaMemcpyAsync(c->loop, &S, sizeof(S), cudaMemcpyHostToDevice, s));
    GMT_CUDA(cudaMemcpyAsync(c->loopc, &C, sizeof(C), cudaMemcpyHostToDevice, s));
    int rc = gmt_cfl_async(c, u, stream);   // CFL of the initial state; later steps fuse it
    if (rc) return rc;
    const int pairs = nsteps / 2;
    if ((flags & GMT_RUN_GRAPH) && pairs > 0) {
        cudaGraphExec_t exec = nullptr;
        for (auto& g : c->graphs)
            if (g.u == u && g.w == w && g.flags == flags) exec = g.exec;
        if (!exec) {
            cudaGraph_t graph;
            GMT_CUDA(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeRelaxed));
            cudaError_t e1 = run_enqueue_any(c, u, w, flags, c->cap);
            cudaError_t e2 = run_enqueue_any(c, w, u, flags, c->cap);
            cudaError_t e3 = cudaStreamEndCapture(c->cap, &graph);
            if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
                cudaGetLastError();
                return cuda_fail(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3), "gmt_run capture");
            }
            cudaError_t e4 = cudaGraphInstantiate(&exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e4 != cudaSuccess) return cuda_fail(e4, "gmt_run instantiate");
            if (c->graphs.size() >= 8) {
                cudaGraphExecDestroy(c->graphs.front().exec);
                c->graphs.erase(c->graphs.begin());
            }
            c->graphs.push_back({u, w, flags, exec});
        }
        for (int i = 0; i < pairs; ++i) GMT_CUDA(cudaGraphLaunch(exec, s));
    } else {
        for (int i = 0; i < pairs; ++i) {
            GMT_CUDA(run_enqueue_any(c, u, w, flags, s));
            GMT_CUDA(run_enqueue_any(c, w, u, flags, s));
        }
    }
    if (nsteps & 1) GMT_CUDA(run_enqueue_any(c, u, w, flags, s));
    int herr = 0;
    GMT_CUDA(cudaMemcpyAsync(&S, c->loop, sizeof(S), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaMemcpyAsync(&herr, c->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaStreamSynchronize(s));
    c->next_time = S.next_time;
    c->counter = S.counter;
    if (t_out) *t_out = S.t;
    if (which) *which = nsteps & 1;
    if (herr) {
        cudaMemset(c->err, 0, sizeof(int));
        return fail(GMT_ERR_TIMEOUT, "gmt_run: a step kernel abandoned a bounded wait");
    }
    if (S.status) return fail(GMT_ERR_STATE, "gmt_run: CFL maximum not positive and finite (invalid state)");
    return GMT_OK;
}

// ------------------------------------------------------------------------------------------
// ensemble
// ------------------------------------------------------------------------------------------
}  // extern "C"

// z-chunk of a box's ensemble work items: the box's nz split into ceil(n/64) equal chunks, so the
// per-chunk prologue (two extra planes) stays near 3-6% while a 64-box ensemble still yields
// thousands of items for the persistent grid
inline int ens_lz(int n) {
    const int nch = (n + 63) / 64;
    return (n + nch - 1) / nch;
}

struct gmt_ensemble {
    gmt_params p;
    int nbox = 0;
    int esize = 4;
    int nsm = 148;
    std::vector<int> n;
    std::vector<double> amp;
    std::vector<uint32_t> seed;
    LoopState* loop = nullptr;       // [nbox]
    LoopConst* loopc = nullptr;      // [nbox]
    unsigned long long* cfl = nullptr;  // [2 nbox]
    double* modes = nullptr;         // [nbox][61][3][2]
    std::vector<void*> btab, trig;   // per box: row table; trig x, y, z
    void* bt = nullptr;              // BoxTables<R>[nbox]
    void* args = nullptr;            // UnsplitArgs<R>[2][nbox]
    EnsItem* items = nullptr;
    int nitems = 0;
    unsigned* queue = nullptr;       // [2] one counter per parity
    int* err = nullptr;
    const int* mode_k_dev = nullptr;
    cudaStream_t cap = nullptr;
    std::vector<const void*> bound_u, bound_w;
    cudaGraphExec_t exec = nullptr;
    int exec_flags = -1;
    int rows_max = 0;
    std::vector<double> alpha, beta, sigma0;
};

namespace {

template <class R> int ens_bind(gmt_ensemble* E, void* const* u, void* const* w, int flags) {
    std::vector<UnsplitArgs<R>> A(2 * E->nbox);
    for (int par = 0; par < 2; ++par)
        for (int b = 0; b < E->nbox; ++b) {
            UnsplitArgs<R>& a = A[par * E->nbox + b];
            const int n = E->n[b];
            const size_t cells = (size_t)n * n * n;
            a.u = cplanes<R>(par == 0 ? u[b] : w[b], cells);
            a.o = planes<R>(par == 0 ? w[b] : u[b], cells);
            a.nx = a.ny = a.nz = n;
            a.ox = ens_tile_x<R>(); a.oy = 16; a.lz = ens_lz(n);
            a.dt = a.dtdx = a.ch = a.glm_fac = a.ramp = R(0);
            a.K = consts_of<R>(E->p);
            a.iflo = E->p.iflo; a.use_llf = E->p.riemann == GMT_RIEMANN_LLF;
            a.do_turb = (flags & GMT_RUN_FORCING) ? 1 : 0;
            a.btab = a.do_turb ? static_cast<const R*>(E->btab[b]) : nullptr;
            a.trigx = static_cast<const R*>(E->trig[3 * b]);
            a.trig8 = nullptr;   // the ensemble kernel reads the generic tables (force_accel)
            a.cfl_out = E->cfl + 2 * b;
            a.err = E->err;
            a.wait_cycles = GMT_WAIT_CYCLES;
            a.wait_test = 0;
            a.dx = (R)(E->p.boxlen / n);
            a.dparams = reinterpret_cast<const double*>(E->loop + b);
            a.fmass = nullptr;
            a.use_tma = 0;   // the ensemble kernel stages by cp.async
            std::memset(&a.tmap, 0, sizeof(a.tmap));
        }
    cudaError_t e = cudaMemcpy(E->args, A.data(), A.size() * sizeof(UnsplitArgs<R>), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "ensemble bind");
}

template <class R> cudaError_t ens_enqueue(gmt_ensemble* E, int par, int flags, cudaStream_t s) {
    tick_kernel<<<(E->nbox + 63) / 64, 64, 0, s>>>(E->loop, E->loopc, E->cfl, E->nbox);
    if (flags & GMT_RUN_FORCING) {
        ou_cond_kernel<<<E->nbox, 64, 0, s>>>(E->modes, E->loop, E->loopc, E->mode_k_dev);
        btab_cond_kernel<R><<<dim3((E->rows_max + 255) / 256, E->nbox), 256, 0, s>>>((const BoxTables<R>*)E->bt, E->loop,
                                                                                     E->mode_k_dev);
    }
    cudaError_t e = cudaMemsetAsync(E->cfl, 0, 2 * E->nbox * sizeof(unsigned long long), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(E->queue + par, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    const UnsplitArgs<R>* args = static_cast<const UnsplitArgs<R>*>(E->args) + par * E->nbox;
    int riem = E->p.riemann == GMT_RIEMANN_LLF ? GMT_RIEMANN_HLLD : E->p.riemann;
    return launch_ensemble(args, E->items, E->nitems, E->queue + par, E->p.recon, riem, E->nsm, s);
}

cudaError_t ens_enqueue_any(gmt_ensemble* E, int par, int flags, cudaStream_t s) {
    return E->esize == 8 ? ens_enqueue<double>(E, par, flags, s) : ens_enqueue<float>(E, par, flags, s);
}

}  // namespace

extern "C" {

int gmt_ensemble_destroy(gmt_ensemble* E) {
    if (!E) return GMT_OK;
    if (E->exec) cudaGraphExecDestroy(E->exec);
    if (E->cap) cudaStreamDestroy(E->cap);
    cudaFree(E->loop);
    cudaFree(E->loopc);
    cudaFree(E->cfl);
    cudaFree(E->modes);
    for (void* x : E->btab) cudaFree(x);
    for (void* x : E->trig) cudaFree(x);
    cudaFree(E->bt);
    cudaFree(E->args);
    cudaFree(E->items);
    cudaFree(E->queue);
    cudaFree(E->err);
    delete E;
    return GMT_OK;
}

int gmt_ensemble_create(const gmt_params* base, int32_t nbox, const int32_t* n, const double* amp,
                        const uint32_t* seeds, gmt_ensemble** out) {
    if (!base || !n || !out || nbox < 1) return fail(GMT_ERR_ARG, "gmt_ensemble_create: invalid arguments");
    *out = nullptr;
    if (base->abi_version != GMT_ABI_VERSION) return fail(GMT_ERR_ARG, "gmt_ensemble_create: abi_version mismatch");
    if (base->scheme != GMT_SCHEME_UNSPLIT) return fail(GMT_ERR_UNSUPPORTED, "gmt_ensemble_create: unsplit scheme only");
    if (!((base->recon == GMT_RECON_MC && (base->riemann == GMT_RIEMANN_HLLD || base->riemann == GMT_RIEMANN_HLL ||
                                          base->riemann == GMT_RIEMANN_LLF)) ||
          (base->recon == GMT_RECON_PPM && base->riemann == GMT_RIEMANN_HLL)))
        return fail(GMT_ERR_UNSUPPORTED, "gmt_ensemble_create: built for PLM-MC with HLLD/HLL/LLF and PPM with HLL");
    if (base->dtype != GMT_F32 && base->dtype != GMT_F64) return fail(GMT_ERR_ARG, "gmt_ensemble_create: bad dtype");
    for (int b = 0; b < nbox; ++b)
        if (n[b] < 16 || n[b] % 16 != 0)
            return fail(GMT_ERR_ARG, "gmt_ensemble_create: every box size must be a positive multiple of 16");
    std::call_once(g_mode_once, [] { g_mode_err = upload_mode_table(); });
    if (g_mode_err != cudaSuccess) return cuda_fail(g_mode_err, "mode table");
    {
        cudaError_t e = base->dtype == GMT_F64 ? unsplit_prepare_f64() : unsplit_prepare_f32();
        if (e != cudaSuccess) return cuda_fail(e, "kernel attributes");
    }
    gmt_ensemble* E = new gmt_ensemble();
    E->p = *base;
    E->nbox = nbox;
    E->esize = base->dtype == GMT_F64 ? 8 : 4;
    E->n.assign(n, n + nbox);
    E->amp.resize(nbox);
    E->seed.resize(nbox);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&E->nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = cudaSuccess;
    auto A = [&](void** ptr, size_t bytes) {
        if (e == cudaSuccess) e = cudaMalloc(ptr, bytes);
    };
    A((void**)&E->loop, nbox * sizeof(LoopState));
    A((void**)&E->loopc, nbox * sizeof(LoopConst));
    A((void**)&E->cfl, 2 * nbox * sizeof(unsigned long long));
    A((void**)&E->modes, (size_t)nbox * NMODES * 6 * sizeof(double));
    A(&E->bt, nbox * sizeof(BoxTables<double>));
    A(&E->args, 2 * nbox * sizeof(UnsplitArgs<double>));
    A((void**)&E->queue, 2 * sizeof(unsigned));
    A((void**)&E->err, sizeof(int));
    E->btab.assign(nbox, nullptr);
    E->trig.assign(3 * nbox, nullptr);
    for (int b = 0; b < nbox; ++b) {
        A(&E->btab[b], (size_t)n[b] * n[b] * 24 * E->esize);
        for (int a = 0; a < 3; ++a) A(&E->trig[3 * b + a], (size_t)8 * n[b] * E->esize);
        E->rows_max = std::max(E->rows_max, n[b] * n[b]);
    }

    // work items: biggest boxes first, tiles of ens_tile_x x 16 columns (a box whose width is not a
    // multiple of the tile gets an overhanging last tile) x ens_lz-plane chunks (the last chunk of
    // a box may be shorter)
    const int etx = E->esize == 8 ? ens_tile_x<double>() : ens_tile_x<float>();
    std::vector<int> order(nbox);
    for (int b = 0; b < nbox; ++b) order[b] = b;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] > n[b]; });
    std::vector<EnsItem> items;
    for (int b : order) {
        const int lz = ens_lz(n[b]);
        for (int bz = 0; bz < (n[b] + lz - 1) / lz; ++bz)
            for (int by = 0; by < n[b] / 16; ++by)
                for (int bx = 0; bx < (n[b] + etx - 1) / etx; ++bx) items.push_back({b, bx, by, bz});
    }
    E->nitems = (int)items.size();
    A((void**)&E->items, items.size() * sizeof(EnsItem));
    if (e == cudaSuccess) e = cudaMemcpy(E->items, items.data(), items.size() * sizeof(EnsItem), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(E->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(E->modes, 0, (size_t)nbox * NMODES * 6 * sizeof(double));
    if (e == cudaSuccess) e = mode_table_device(&E->mode_k_dev);
    // trig tables, forcing constants, loop records, box tables
    int nd = base->turb_ndt > 0 ? base->turb_ndt : 100;
    double dtf = base->turb_T / nd;
    double alpha = 1.0 - dtf / base->turb_T, beta = std::sqrt(2.0 * dtf / base->turb_T);
    std::vector<LoopState> S(nbox);
    std::vector<LoopConst> Cs(nbox);
    std::vector<BoxTables<double>> Td(nbox);
    std::vector<BoxTables<float>> Tf(nbox);
    for (int b = 0; b < nbox && e == cudaSuccess; ++b) {
        std::vector<double> t = trig_table(n[b]);
        for (int a = 0; a < 3 && e == cudaSuccess; ++a) {
            if (E->esize == 8) {
                e = cudaMemcpy(E->trig[3 * b + a], t.data(), t.size() * 8, cudaMemcpyHostToDevice);
            } else {
                std::vector<float> f(t.begin(), t.end());
                e = cudaMemcpy(E->trig[3 * b + a], f.data(), f.size() * 4, cudaMemcpyHostToDevice);
            }
        }

        E->amp[b] = amp ? amp[b] : base->turb_amp;
        E->seed[b] = seeds ? seeds[b] : base->turb_seed + (uint32_t)b;
        gmt_params pb = *base;
        pb.nx = pb.ny = pb.nz = n[b];
        pb.turb_seed = E->seed[b];
        Cs[b] = loop_const_of(pb, alpha, beta, forcing_sigma0(E->amp[b], alpha, beta),
                              GMT_RUN_CH_MAXSIGNAL | GMT_RUN_FORCING);
        S[b] = LoopState{};
        S[b].ch = 1.0; S[b].glm_fac = 1.0;
        S[b].t = 0.0; S[b].t_end = 0.0; S[b].next_time = 0.0; S[b].counter = 0;
        const double* mb = E->modes + (size_t)b * NMODES * 6;
        Td[b] = BoxTables<double>{mb, (const double*)E->trig[3 * b + 1], (const double*)E->trig[3 * b + 2],
                                  (double*)E->btab[b], n[b], n[b]};
        Tf[b] = BoxTables<float>{mb, (const float*)E->trig[3 * b + 1], (const float*)E->trig[3 * b + 2],
                                 (float*)E->btab[b], n[b], n[b]};
    }
    if (e == cudaSuccess) e = cudaMemcpy(E->loop, S.data(), nbox * sizeof(LoopState), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(E->loopc, Cs.data(), nbox * sizeof(LoopConst), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = E->esize == 8 ? cudaMemcpy(E->bt, Td.data(), nbox * sizeof(Td[0]), cudaMemcpyHostToDevice)
                          : cudaMemcpy(E->bt, Tf.data(), nbox * sizeof(Tf[0]), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&E->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        gmt_ensemble_destroy(E);
        return cuda_fail(e, "gmt_ensemble_create");
    }
    *out = E;
    return GMT_OK;
}

int gmt_ensemble_run(gmt_ensemble* E, void* const* u, void* const* w, int32_t nsteps, double t_end, int32_t flags,
                     void* stream, double* t_out) {
    if (!E || !u || !w || nsteps < 0) return fail(GMT_ERR_ARG, "gmt_ensemble_run: invalid arguments");
    for (int b = 0; b < E->nbox; ++b)
        if (!u[b] || !w[b] || u[b] == w[b]) return fail(GMT_ERR_ARG, "gmt_ensemble_run: bad state pointers");
    cudaStream_t s = (cudaStream_t)stream;
    const int nb = E->nbox;
    bool rebind = (int)E->bound_u.size() != nb || E->exec_flags != flags;
    for (int b = 0; !rebind && b < nb; ++b) rebind = E->bound_u[b] != u[b] || E->bound_w[b] != w[b];
    if (rebind) {
        GMT_CUDA(cudaStreamSynchronize(s));
        int rc = E->esize == 8 ? ens_bind<double>(E, u, w, flags) : ens_bind<float>(E, u, w, flags);
        if (rc) return rc;
        E->bound_u.assign(u, u + nb);
        E->bound_w.assign(w, w + nb);
        if (E->exec) { cudaGraphExecDestroy(E->exec); E->exec = nullptr; }
        E->exec_flags = flags;
        // per-run flags live in the loop constants
        std::vector<LoopConst> Cs(nb);
        GMT_CUDA(cudaMemcpy(Cs.data(), E->loopc, nb * sizeof(LoopConst), cudaMemcpyDeviceToHost));
        for (auto& C : Cs) {
            C.ch_max_signal = (flags & GMT_RUN_CH_MAXSIGNAL) ? 1 : 0;
            C.do_turb = (flags & GMT_RUN_FORCING) ? 1 : 0;
        }
        GMT_CUDA(cudaMemcpy(E->loopc, Cs.data(), nb * sizeof(LoopConst), cudaMemcpyHostToDevice));
    }
    // t_end of every box, then the CFL maxima of the initial states
    std::vector<LoopState> S(nb);
    GMT_CUDA(cudaMemcpyAsync(S.data(), E->loop, nb * sizeof(LoopState), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaStreamSynchronize(s));
    for (auto& x : S) x.t_end = t_end;
    GMT_CUDA(cudaMemcpyAsync(E->loop, S.data(), nb * sizeof(LoopState), cudaMemcpyHostToDevice, s));
    for (int b = 0; b < nb; ++b) {
        const size_t cells = (size_t)E->n[b] * E->n[b] * E->n[b];
        cudaError_t e = E->esize == 8
                            ? launch_cfl<double>(cplanes<double>(u[b], cells), cells, consts_of<double>(E->p), E->cfl + 2 * b, s)
                            : launch_cfl<float>(cplanes<float>(u[b], cells), cells, consts_of<float>(E->p), E->cfl + 2 * b, s);
        if (e != cudaSuccess) return cuda_fail(e, "ensemble cfl");
    }
    const int pairs = nsteps / 2;
    if ((flags & GMT_RUN_GRAPH) && pairs > 0) {
        if (!E->exec) {
            cudaGraph_t graph;
            GMT_CUDA(cudaStreamBeginCapture(E->cap, cudaStreamCaptureModeRelaxed));
            cudaError_t e1 = ens_enqueue_any(E, 0, flags, E->cap);
            cudaError_t e2 = ens_enqueue_any(E, 1, flags, E->cap);
            cudaError_t e3 = cudaStreamEndCapture(E->cap, &graph);
            if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess) {
                cudaGetLastError();
                return cuda_fail(e1 != cudaSuccess ? e1 : (e2 != cudaSuccess ? e2 : e3), "ensemble capture");
            }
            cudaError_t e4 = cudaGraphInstantiate(&E->exec, graph, 0);
            cudaGraphDestroy(graph);
            if (e4 != cudaSuccess) return cuda_fail(e4, "ensemble instantiate");
        }
        for (int i = 0; i < pairs; ++i) GMT_CUDA(cudaGraphLaunch(E->exec, s));
    } else {
        for (int i = 0; i < pairs; ++i) {
            GMT_CUDA(ens_enqueue_any(E, 0, flags, s));
            GMT_CUDA(ens_enqueue_any(E, 1, flags, s));
        }
    }
    if (nsteps & 1) GMT_CUDA(ens_enqueue_any(E, 0, flags, s));
    int herr = 0;
    GMT_CUDA(cudaMemcpyAsync(S.data(), E->loop, nb * sizeof(LoopState), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaMemcpyAsync(&herr, E->err, sizeof(int), cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaStreamSynchronize(s));
    int bad = 0;
    for (int b = 0; b < nb; ++b) {
        if (t_out) t_out[b] = S[b].t;
        bad |= S[b].status;
    }
    if (herr) {
        cudaMemset(E->err, 0, sizeof(int));
        return fail(GMT_ERR_TIMEOUT, "gmt_ensemble_run: a step kernel abandoned a bounded wait");
    }
    if (bad) return fail(GMT_ERR_STATE, "gmt_ensemble_run: a box has no positive finite CFL maximum");
    return GMT_OK;
}

// ------------------------------------------------------------------------------------------
// CT
// ------------------------------------------------------------------------------------------
int gmt_ct_step(gmt_ctx* c, const void* qold, void* qnew, const gmt_step_args* a, void* stream) {
    if (!c || !qold || !qnew || !a) return fail(GMT_ERR_ARG, "gmt_ct_step: null argument");
    if (c->p.scheme != GMT_SCHEME_CT) return fail(GMT_ERR_ARG, "gmt_ct_step: context scheme is not GMT_SCHEME_CT");
    if (qold == qnew) return fail(GMT_ERR_ARG, "gmt_ct_step: qold and qnew must be different buffers");
    cudaStream_t s = (cudaStream_t)stream;
    if (c->esize == 8) return ct_step_impl<double>(c, cplanes8<double>(qold, c->n), planes8<double>(qnew, c->n), a, s);
    return ct_step_impl<float>(c, cplanes8<float>(qold, c->n), planes8<float>(qnew, c->n), a, s);
}

int gmt_ct_cfl_async(gmt_ctx* c, const void* q, void* stream) {
    if (!c || !q) return fail(GMT_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = c->esize == 8
                        ? launch_ct_cfl<double>(cplanes8<double>(q, c->n), c->p.nx, c->p.ny, c->p.nz,
                                                consts_of<double>(c->p), c->cfl, s)
                        : launch_ct_cfl<float>(cplanes8<float>(q, c->n), c->p.nx, c->p.ny, c->p.nz,
                                               consts_of<float>(c->p), c->cfl, s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "ct cfl");
}

int gmt_ct_divb_max(gmt_ctx* c, const void* q, double* out, void* stream) {
    if (!c || !q || !out) return fail(GMT_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    const double dx = c->p.boxlen / c->p.nx;
    cudaError_t e = c->esize == 8
                        ? launch_ct_divb<double>(cplanes8<double>(q, c->n), c->p.nx, c->p.ny, c->p.nz, dx, c->divb, s)
                        : launch_ct_divb<float>(cplanes8<float>(q, c->n), c->p.nx, c->p.ny, c->p.nz, dx, c->divb, s);
    if (e != cudaSuccess) return cuda_fail(e, "divb");
    unsigned long long h;
    GMT_CUDA(cudaMemcpyAsync(&h, c->divb, 8, cudaMemcpyDeviceToHost, s));
    GMT_CUDA(cudaStreamSynchronize(s));
    std::memcpy(out, &h, 8);
    return GMT_OK;
}

int gmt_ct_ic_orszag_tang(gmt_ctx* c, void* q, void* stream) {
    if (!c || !q) return fail(GMT_ERR_ARG, "null argument");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = c->esize == 8 ? launch_ct_ic_ot<double>(planes8<double>(q, c->n), c->p.nx, c->p.ny, c->p.nz, c->p.gamma, s)
                                  : launch_ct_ic_ot<float>(planes8<float>(q, c->n), c->p.nx, c->p.ny, c->p.nz, c->p.gamma, s);
    return e == cudaSuccess ? GMT_OK : cuda_fail(e, "ct ic");
}

// ------------------------------------------------------------------------------------------
// legacy bridge ABI: __constant__-style setters become process-wide state (spike_mhd.cu:52,
// 321-340); each grid size gets its own lazily created FP32 context.
// ------------------------------------------------------------------------------------------
#ifndef GMT_LEGACY_NSP
#define GMT_LEGACY_NSP 0     // passive species of the legacy march build (spike_mhd.cu -DNSP)
#endif
#ifndef GMT_LEGACY_NX
#define GMT_LEGACY_NX 480
#endif
static std::mutex g_legacy_mu;
static int g_legacy_nx = GMT_LEGACY_NX;
static float g_dtdx = 0.02f, g_ch = 1.0f, g_glmfac = 1.0f, g_gamma = 1.4f;
static gmt_ctx* g_legacy_ctx[2] = {nullptr, nullptr};   // [0] march, [1] CT
static float g_legacy_gamma_of[2] = {0.f, 0.f};

static gmt_ctx* legacy_ctx(int which) {
    gmt_ctx*& c = g_legacy_ctx[which];
    if (c && (c->p.nx != g_legacy_nx || g_legacy_gamma_of[which] != g_gamma)) { gmt_destroy(c); c = nullptr; }
    if (!c) {
        gmt_params p;
        gmt_params_init(&p, g_legacy_nx);
        p.scheme = which == 0 ? GMT_SCHEME_MARCH1D : GMT_SCHEME_CT;
        p.riemann = GMT_RIEMANN_HLL;
        p.gamma = g_gamma;
        p.smallr = 1e-6;
        p.smallp = 1e-6;
        p.boxlen = 1.0;
        if (which == 0) p.nsp = GMT_LEGACY_NSP;
        if (gmt_create(&p, &c) != GMT_OK) c = nullptr;
        g_legacy_gamma_of[which] = g_gamma;
    }
    return c;
}

int march_nv(void) { return 9 + GMT_LEGACY_NSP; }
int march_nx(void) { return g_legacy_nx; }
int march_nsp(void) { return GMT_LEGACY_NSP; }
void march_set_nx(int n) {
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    if (n > 0) g_legacy_nx = n;
}
void march_set_dtdx(float v) { g_dtdx = v; }
void march_set_glm(float ch, float fac) { g_ch = ch; g_glmfac = fac; }
void march_set_gamma(float g) { g_gamma = g; }

double march_run_dev(float* const* qv, float* const* ov, int nsteps) {
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    gmt_ctx* c = legacy_ctx(0);
    if (!c || !qv || !ov || nsteps < 0) return -1.0;
    const double dx = c->p.boxlen / c->p.nx;
    gmt_step_args a{};
    a.dt = (double)g_dtdx * dx;
    a.ch = g_ch;
    a.glm_fac = g_glmfac;
    constexpr int NV = 9 + GMT_LEGACY_NSP;
    const void* q[NV];
    void* o[NV];
    for (int v = 0; v < NV; ++v) { q[v] = qv[v]; o[v] = ov[v]; }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0);
    bool in_q = true;
    for (int it = 0; it < nsteps; ++it) {
        if (gmt_step_planes(c, in_q ? q : (const void* const*)o, in_q ? o : (void* const*)q, &a, nullptr) != GMT_OK) break;
        in_q = !in_q;
    }
    cudaEventRecord(t1);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (!in_q)
        for (int v = 0; v < NV; ++v) cudaMemcpy(qv[v], ov[v], c->n * sizeof(float), cudaMemcpyDeviceToDevice);
    return (double)ms;
}

double ct_run(float* const* qv, float* const* ov, float* const* cc, int nsteps) {
    (void)cc;  // the face-averaged field is formed inside the kernels; the scratch planes are unused
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    gmt_ctx* c = legacy_ctx(1);
    if (!c || !qv || !ov || nsteps < 0) return -1.0;
    const double dx = c->p.boxlen / c->p.nx;
    gmt_step_args a{};
    a.dt = (double)g_dtdx * dx;
    CPlanes8<float> q, o;
    Planes8<float> qw, ow;
    for (int v = 0; v < 8; ++v) { q.p[v] = qv[v]; o.p[v] = ov[v]; qw.p[v] = qv[v]; ow.p[v] = ov[v]; }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0);
    bool in_q = true;
    for (int it = 0; it < nsteps; ++it) {
        int rc = in_q ? ct_step_impl<float>(c, q, ow, &a, nullptr) : ct_step_impl<float>(c, o, qw, &a, nullptr);
        if (rc != GMT_OK) break;
        in_q = !in_q;
    }
    cudaEventRecord(t1);
    cudaEventSynchronize(t1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (!in_q)
        for (int v = 0; v < 8; ++v) cudaMemcpy(qv[v], ov[v], c->n * sizeof(float), cudaMemcpyDeviceToDevice);
    return (double)ms;
}

int ct_regs(void) {
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    gmt_ctx* c = legacy_ctx(1);
    return c ? ct_regs_of(4, c->p.recon, c->p.riemann, c->ox * c->oy) : -1;
}
int ct_shmem(void) {
    std::lock_guard<std::mutex> lk(g_legacy_mu);
    gmt_ctx* c = legacy_ctx(1);
    return c ? (int)ct_smem_of(4, c->ox, c->oy) : -1;
}

}  // extern "C"

namespace gmt {
void set_last_error(const std::string& msg) { g_err = msg; }
int unsplit_regs_f32(int recon, int riem, int nthreads);
int unsplit_regs_f64(int recon, int riem, int nthreads);
int unsplit_regs(int esize, int recon, int riem, int nthreads) {
    return esize == 8 ? unsplit_regs_f64(recon, riem, nthreads) : unsplit_regs_f32(recon, riem, nthreads);
}
int unsplit_max_threads(int esize) { return esize == 8 ? 256 : 512; }
size_t unsplit_smem(int esize, int ox, int oy) {
    return esize == 8 ? unsplit_smem_bytes<double>(ox, oy) : unsplit_smem_bytes<float>(ox, oy);
}
}  // namespace gmt
