// gmt_internal.h -- launchers shared between the kernel translation units and the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "gmt_common.cuh"

namespace gmt {

constexpr int NMODES = 61;

// unsplit GLM step (gmt_unsplit_f32.cu / gmt_unsplit_f64.cu)
cudaError_t launch_unsplit(const UnsplitArgs<float>& A, int recon, int riem, cudaStream_t s);
cudaError_t launch_unsplit(const UnsplitArgs<double>& A, int recon, int riem, cudaStream_t s);
int unsplit_max_threads(int dtype_bytes);
cudaError_t unsplit_prepare_f32();   // shared-memory attributes of every step kernel
cudaError_t unsplit_prepare_f64();
struct EnsItem;
// tile of the ensemble kernel: ens_tile_x<R>() columns by 16 rows (32 in FP32, 16 in FP64)
template <class R> constexpr int ens_tile_x() { return sizeof(R) == 4 ? 32 : 16; }
cudaError_t launch_ensemble(const UnsplitArgs<float>* boxes, const EnsItem* items, int nitems, unsigned* queue,
                            int recon, int riem, int nsm, cudaStream_t s);
cudaError_t launch_ensemble(const UnsplitArgs<double>* boxes, const EnsItem* items, int nitems, unsigned* queue,
                            int recon, int riem, int nsm, cudaStream_t s);
size_t unsplit_smem(int dtype_bytes, int ox, int oy);
// tiled march (the unsplit tile with the march scheme; no passive species)
cudaError_t launch_march_tiled(const UnsplitArgs<float>& A, int recon, cudaStream_t s);
cudaError_t launch_march_tiled(const UnsplitArgs<double>& A, int recon, cudaStream_t s);
int march_tiled_regs(const UnsplitArgs<float>*, int recon, int nthreads);
int march_tiled_regs(const UnsplitArgs<double>*, int recon, int nthreads);
int unsplit_regs(int dtype_bytes, int recon, int riem, int nthreads);

// transverse-free 1-D Hancock march (gmt_march1d.cu)
constexpr int MAX_SPECIES = 8;
template <class R> struct MarchArgs {   // the species pass of the march scheme
    CPlanes<R> u;
    Planes<R> o;
    int nx, ny, nz, ox, oy, lz;
    R dtdx, ch, glm_fac;
    Consts<R> K;
    int ppm;
    int nsp;                       // passive species: su[s] = rho*X in, so[s] out
    const R* su[MAX_SPECIES];
    R* so[MAX_SPECIES];
};
// passive species of the march scheme, after the tiled step stored the face mass fluxes
cudaError_t launch_species(const MarchArgs<float>& A, const float* fmass, cudaStream_t s);
cudaError_t launch_species(const MarchArgs<double>& A, const double* fmass, cudaStream_t s);

// constrained transport (gmt_ct.cu): q = [rho, mx, my, mz, E, bxf, byf, bzf]
template <class R> struct CTArgs {
    CPlanes8<R> q;
    Planes8<R> o;
    int nx, ny, nz, ox, oy, lz;
    R dt, dtdx, ramp;
    Consts<R> K;
    int recon, riem, emf, halfslope, do_turb;
    const R* btab;
    const R* trigx;
    const R* trig8;        // FP32 or null: x table of 2 cos, -2 sin (force_accel_f32)
    R* scratch;            // 15 planes: lower-face EMF data and cell EMFs (12), edge EMFs (3)
    int* err;              // device flag set when a bounded wait gives up
    int use_tma;           // tmap8/tmap1 describe q: tiles clear of the box edges stage by TMA
    CUtensorMap tmap8;     // 4-D map (x, y, z, variable) of q, box (ox+8) x (oy+5) x 1 x 8
    CUtensorMap tmap1;     // the same tensor, box (ox+8) x (oy+5) x 1 x 1 (bzf of the next plane)
    long long wait_cycles; // budget of each bounded wait (GMT_WAIT_CYCLES)
    int wait_test;         // failure-path tests only (see UnsplitArgs::wait_test)
};
cudaError_t launch_ct(const CTArgs<float>& A, cudaStream_t s);
cudaError_t launch_ct(const CTArgs<double>& A, cudaStream_t s);
cudaError_t ct_prepare_f32();   // shared-memory attributes of the CT tile kernels
cudaError_t ct_prepare_f64();
int ct_regs_of(int dtype_bytes, int recon, int riem, int nthreads);
size_t ct_smem_of(int dtype_bytes, int ox, int oy);
int ct_max_threads(int dtype_bytes);

// auxiliary kernels (gmt_aux.cu)
template <class R> cudaError_t launch_cfl(const CPlanes<R>& u, size_t n, const Consts<R>& K,
                                          unsigned long long* out, cudaStream_t s);
template <class R> cudaError_t launch_ct_cfl(const CPlanes8<R>& q, int nx, int ny, int nz, const Consts<R>& K,
                                             unsigned long long* out, cudaStream_t s);
// diagnostics partials -> double out[10] = {mass, ke2, etot, psi2, divb2, divbmax, rhomin, nonfinite, -, -}
template <class R> cudaError_t launch_diag(const CPlanes<R>& u, int nx, int ny, int nz, double dx, double smallr,
                                           double* partials, int nblocks, double* out, cudaStream_t s);
template <class R> cudaError_t launch_ct_divb(const CPlanes8<R>& q, int nx, int ny, int nz, double dx,
                                              unsigned long long* out, cudaStream_t s);
cudaError_t launch_ou_update(double* modes, uint32_t seed, uint32_t counter, double alpha, double beta,
                             double sigma0, cudaStream_t s);
template <class R> cudaError_t launch_btab(const double* modes, const R* trigy, const R* trigz, int ny, int nz,
                                           R* btab, cudaStream_t s);
template <class R> cudaError_t launch_ic_ot(const Planes<R>& u, int nx, int ny, int nz, double gamma, cudaStream_t s);
template <class R> cudaError_t launch_ic_uniform(const Planes<R>& u, size_t n, const double v9[9], cudaStream_t s);
template <class R> cudaError_t launch_ct_ic_ot(const Planes8<R>& q, int nx, int ny, int nz, double gamma, cudaStream_t s);
template <class R> cudaError_t launch_ct_ic_turb(const Planes8<R>& q, int nx, int ny, int nz, const double* modes,
                                                 R* scratch, double rho0, double p0, const double b0[3], double vscale,
                                                 double db, double gamma, cudaStream_t s);
template <class R> cudaError_t launch_ic_turb(const Planes<R>& u, int nx, int ny, int nz, const R* btab,
                                             const R* trigx, double rho0, double p0, const double b0[3],
                                             double vscale, double bscale, double gamma, cudaStream_t s);
size_t spectrum_scratch_bytes(int nx, int ny, int nz, int kmax);
template <class R> cudaError_t launch_spectrum(const CPlanes<R>& u, int nx, int ny, int nz, int kmax, void* scratch,
                                               double* E_host, cudaStream_t s);
size_t band_scratch_bytes(int nx, int ny, int nz, int kmax);
size_t pdf_scratch_bytes(int nbins);
template <class R> cudaError_t launch_density_pdf(const R* rho, size_t n, int nbins, double smin, double smax,
                                                  void* scratch, double* pdf_host, double* stats_host, cudaStream_t s);
template <class R> cudaError_t launch_band_loss(const CPlanes<R>& u, int nx, int ny, int nz, int kmin, int kmax,
                                                void* scratch, double* L_host, const Planes<R>& ub, cudaStream_t s);
// discrete adjoint of one unsplit PLM step, dt frozen (gmt_adjoint.cu)
template <class R> struct AdjArgs {
    CPlanes<R> u;          // input state of the forward step
    CPlanes<R> ubn;        // adjoint of the step's output
    Planes<R> ub;          // adjoint of the step's input (written)
    int nx, ny, nz;
    R dt, dtdx, ch, glm_fac, ramp, amp;
    Consts<R> K;
    int iflo, use_llf, do_turb, recon, riem;
    const R* btab;
    const R* trigx;
    R* FS;                 // 54 planes: the 6 interface states of every cell
    R* FL;                 // 27 planes: the +x, +y, +z face fluxes
    R* R1b;                // 9 planes: adjoint of the pre-epilogue update
    R* FSb;                // 54 planes: adjoint of the interface states
    R* QB;                 // 63 planes: own primitive adjoint (9), slope-stencil terms A_d (27), B_d (27)
    double* damp;          // dL/d(forcing amplitude) accumulator
};
size_t adjoint_scratch_reals(size_t n);
// rec: the forward step's tile arguments for the record tile (passes 1-3 in one march), or null
template <class R> cudaError_t launch_adjoint(const AdjArgs<R>& A, const UnsplitArgs<R>* rec, cudaStream_t s);
cudaError_t upload_mode_table();   // the 61 wavevectors into constant memory
cudaError_t mode_table_device(const int** ptr);   // device address of that table
void set_last_error(const std::string& msg);   // message returned by gmt_last_error() on this thread

}  // namespace gmt
