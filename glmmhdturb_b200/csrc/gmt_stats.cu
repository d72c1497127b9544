// gmt_stats.cu -- turbulence statistics on the device: the shell-binned kinetic-energy spectrum.
//
// E(k) = 1/2 sum_{k-1/2 <= |k'| < k+1/2} |w^(k')|^2 with w = sqrt(rho) v = m / sqrt(rho) and
// w^(k) = N^-3 sum_x w(x) e^{-2 pi i k.x/N}, so that sum_k E(k) is the mean kinetic energy density
// (Parseval).  Only |k_i| <= kmax is needed, so the transform is three separable low-k DFT stages
// (x: kx = 0..kmax, y and z: -kmax..kmax), O(N^3 kmax) work, FP64 accumulation, and a fixed-order
// final reduction (no atomics: the spectrum is bit-reproducible).
#include <cmath>
#include <vector>

#include "gmt_internal.h"

namespace gmt {

// stage x: A[c][kx][row] = sum_x w_c(x,row) e^{-i 2pi kx x/nx}, row = y + ny z
template <class R>
__global__ void __launch_bounds__(128) spec_x_kernel(const CPlanes<R> u, int nx, int ny, int nz, int kmax,
                                                     const double2* tw, double2* A) {
    const size_t rows = (size_t)ny * nz;
    const size_t total = 3 * (size_t)(kmax + 1) * rows;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t row = t % rows;
        const int kx = (int)((t / rows) % (kmax + 1));
        const int c = (int)(t / (rows * (kmax + 1)));
        const R* rho = u.p[0] + row * nx;
        const R* m = u.p[1 + c] + row * nx;
        const double2* e = tw + (size_t)kx * nx;
        double re = 0.0, im = 0.0;
        for (int x = 0; x < nx; ++x) {
            double w = (double)m[x] / sqrt(fmax((double)rho[x], 1e-300));
            re += w * e[x].x;
            im += w * e[x].y;
        }
        A[t] = make_double2(re, im);
    }
}

// stage y: B[c][kx][jy][z] = sum_y A[c][kx][y + ny z] e^{-i 2pi ky y/ny}, ky = jy - kmax
__global__ void __launch_bounds__(128) spec_y_kernel(const double2* A, int ny, int nz, int kmax, const double2* tw,
                                                     double2* B) {
    const int K1 = kmax + 1, K2 = 2 * kmax + 1;
    const size_t total = 3 * (size_t)K1 * K2 * nz;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(t % nz);
        const int jy = (int)((t / nz) % K2);
        const size_t ckx = t / ((size_t)nz * K2);   // c*K1 + kx
        const double2* a = A + ckx * (size_t)ny * nz + (size_t)z * ny;
        const double2* e = tw + (size_t)jy * ny;
        double re = 0.0, im = 0.0;
        for (int y = 0; y < ny; ++y) {
            re += a[y].x * e[y].x - a[y].y * e[y].y;
            im += a[y].x * e[y].y + a[y].y * e[y].x;
        }
        B[t] = make_double2(re, im);
    }
}

// stage z + power: P[kx][jy][jz] = sum_c |sum_z B e^{-i 2pi kz z/nz}|^2 / N^6
__global__ void __launch_bounds__(128) spec_z_kernel(const double2* B, int nz, int kmax, const double2* tw, double norm,
                                                     double* P) {
    const int K1 = kmax + 1, K2 = 2 * kmax + 1;
    const size_t total = (size_t)K1 * K2 * K2;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int jz = (int)(t % K2);
        const size_t kxjy = t / K2;               // kx*K2 + jy
        const double2* e = tw + (size_t)jz * nz;
        double p = 0.0;
        for (int c = 0; c < 3; ++c) {
            const double2* b = B + ((size_t)c * K1 * K2 + kxjy) * nz;
            double re = 0.0, im = 0.0;
            for (int z = 0; z < nz; ++z) {
                re += b[z].x * e[z].x - b[z].y * e[z].y;
                im += b[z].x * e[z].y + b[z].y * e[z].x;
            }
            p += (re * re + im * im) * norm;
        }
        P[t] = p;
    }
}

// shells, in a fixed order by one thread
__global__ void spec_shell_kernel(const double* P, int kmax, double* E) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int K1 = kmax + 1, K2 = 2 * kmax + 1;
    for (int s = 0; s <= kmax; ++s) E[s] = 0.0;
    for (int kx = 0; kx < K1; ++kx)
        for (int jy = 0; jy < K2; ++jy)
            for (int jz = 0; jz < K2; ++jz) {
                const int ky = jy - kmax, kz = jz - kmax;
                const double k = sqrt((double)(kx * kx + ky * ky + kz * kz));
                const int s = (int)floor(k + 0.5);
                if (s > kmax) continue;
                const double wgt = kx > 0 ? 2.0 : 1.0;   // the -kx half by Hermitian symmetry
                E[s] += 0.5 * wgt * P[((size_t)kx * K2 + jy) * K2 + jz];
            }
}

std::vector<double> spectrum_twiddles(int n, int kmin, int kmax) {
    std::vector<double> t(2 * (size_t)(kmax - kmin + 1) * n);
    const double twopi = 6.283185307179586476925286766559;
    for (int k = kmin; k <= kmax; ++k)
        for (int x = 0; x < n; ++x) {
            double th = twopi * (double)k * (double)x / (double)n;
            size_t i = ((size_t)(k - kmin) * n + x) * 2;
            t[i] = std::cos(th);
            t[i + 1] = -std::sin(th);
        }
    return t;
}

size_t spectrum_scratch_bytes(int nx, int ny, int nz, int kmax) {
    const size_t K1 = kmax + 1, K2 = 2 * kmax + 1;
    size_t tw = 2 * sizeof(double) * (K1 * nx + K2 * ny + K2 * nz);
    size_t A = 3 * K1 * (size_t)ny * nz * sizeof(double2);
    size_t B = 3 * K1 * K2 * (size_t)nz * sizeof(double2);
    size_t P = K1 * K2 * K2 * sizeof(double) + K1 * sizeof(double);
    return tw + A + B + P + 256;
}

template <class R>
cudaError_t launch_spectrum(const CPlanes<R>& u, int nx, int ny, int nz, int kmax, void* scratch, double* E_host,
                            cudaStream_t s) {
    const size_t K1 = kmax + 1, K2 = 2 * kmax + 1;
    char* p = static_cast<char*>(scratch);
    double2* twx = reinterpret_cast<double2*>(p);
    double2* twy = twx + K1 * nx;
    double2* twz = twy + K2 * ny;
    double2* A = twz + K2 * nz;
    double2* B = A + 3 * K1 * (size_t)ny * nz;
    double* P = reinterpret_cast<double*>(B + 3 * K1 * K2 * (size_t)nz);
    double* E = P + K1 * K2 * K2;
    std::vector<double> tx = spectrum_twiddles(nx, 0, kmax), ty = spectrum_twiddles(ny, -kmax, kmax),
                        tz = spectrum_twiddles(nz, -kmax, kmax);
    cudaError_t e = cudaMemcpyAsync(twx, tx.data(), tx.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(twy, ty.data(), ty.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(twz, tz.data(), tz.size() * 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    const double n3 = (double)nx * ny * nz;
    auto grid = [](size_t total) { return (int)std::min<size_t>((total + 127) / 128, 148 * 32); };
    spec_x_kernel<R><<<grid(3 * K1 * ny * nz), 128, 0, s>>>(u, nx, ny, nz, kmax, twx, A);
    spec_y_kernel<<<grid(3 * K1 * K2 * nz), 128, 0, s>>>(A, ny, nz, kmax, twy, B);
    spec_z_kernel<<<grid(K1 * K2 * K2), 128, 0, s>>>(B, nz, kmax, twz, 1.0 / (n3 * n3), P);
    spec_shell_kernel<<<1, 1, 0, s>>>(P, kmax, E);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(E_host, E, K1 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

// ---------------------------------------------------------------------------------------------
// Band-limited kinetic-energy loss L = sum_{kmin <= shell <= kmax} E(shell) and its gradient.
// dL/dw(x) = w_S(x)/N^3 with w_S the band-passed field, pulled back through w = m/sqrt(rho).
// ---------------------------------------------------------------------------------------------
// stage z of the forward transform, complex: C[c][kx][jy][jz] = N^-3 sum_z B e^{-i kz z}
__global__ void __launch_bounds__(128) band_z_kernel(const double2* B, int nz, int kmax, const double2* tw, double norm,
                                                     double2* Cc) {
    const int K1 = kmax + 1, K2 = 2 * kmax + 1;
    const size_t total = 3 * (size_t)K1 * K2 * K2;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int jz = (int)(t % K2);
        const size_t ckxjy = t / K2;
        const double2* b = B + ckxjy * nz;
        const double2* e = tw + (size_t)jz * nz;
        double re = 0.0, im = 0.0;
        for (int z = 0; z < nz; ++z) {
            re += b[z].x * e[z].x - b[z].y * e[z].y;
            im += b[z].x * e[z].y + b[z].y * e[z].x;
        }
        Cc[t] = make_double2(re * norm, im * norm);
    }
}

__device__ __forceinline__ int shell_of(int kx, int ky, int kz) {
    return (int)floor(sqrt((double)(kx * kx + ky * ky + kz * kz)) + 0.5);
}

// loss, one thread, fixed order
__global__ void band_loss_kernel(const double2* Cc, int kmax, int kmin, int kmaxb, double* L) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int K1 = kmax + 1, K2 = 2 * kmax + 1;
    double acc = 0.0;
    for (int c = 0; c < 3; ++c)
        for (int kx = 0; kx < K1; ++kx)
            for (int jy = 0; jy < K2; ++jy)
                for (int jz = 0; jz < K2; ++jz) {
                    int sh = shell_of(kx, jy - kmax, jz - kmax);
                    if (sh < kmin || sh > kmaxb) continue;
                    double2 v = Cc[(((size_t)c * K1 + kx) * K2 + jy) * K2 + jz];
                    acc += 0.5 * (kx > 0 ? 2.0 : 1.0) * (v.x * v.x + v.y * v.y);
                }
    *L = acc;
}

// inverse z: G[c][kx][jy][z] = sum_jz mask * C e^{+i kz z}   (tw holds e^{-i k z}: use its conjugate)
__global__ void __launch_bounds__(128) band_iz_kernel(const double2* Cc, int nz, int kmax, int kmin, int kmaxb,
                                                      const double2* tw, double2* G) {
    const int K1 = kmax + 1, K2 = 2 * kmax + 1;
    const size_t total = 3 * (size_t)K1 * K2 * nz;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int z = (int)(t % nz);
        const size_t ckxjy = t / nz;
        const int jy = (int)(ckxjy % K2), kx = (int)((ckxjy / K2) % K1);
        double re = 0.0, im = 0.0;
        for (int jz = 0; jz < K2; ++jz) {
            int sh = shell_of(kx, jy - kmax, jz - kmax);
            if (sh < kmin || sh > kmaxb) continue;
            double2 cv = Cc[ckxjy * K2 + jz];
            double2 e = tw[(size_t)jz * nz + z];   // e^{-i kz z}; conj = e^{+i kz z}
            re += cv.x * e.x + cv.y * e.y;
            im += cv.y * e.x - cv.x * e.y;
        }
        G[t] = make_double2(re, im);
    }
}

// inverse y: H[c][kx][y + ny z] = sum_jy G[c][kx][jy][z] e^{+i ky y}
__global__ void __launch_bounds__(128) band_iy_kernel(const double2* G, int ny, int nz, int kmax, const double2* tw,
                                                      double2* H) {
    const int K1 = kmax + 1, K2 = 2 * kmax + 1;
    const size_t rows = (size_t)ny * nz;
    const size_t total = 3 * (size_t)K1 * rows;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t row = t % rows;
        const size_t ckx = t / rows;
        const int y = (int)(row % ny), z = (int)(row / ny);
        double re = 0.0, im = 0.0;
        for (int jy = 0; jy < K2; ++jy) {
            double2 g = G[(ckx * K2 + jy) * nz + z];
            double2 e = tw[(size_t)jy * ny + y];
            re += g.x * e.x + g.y * e.y;
            im += g.y * e.x - g.x * e.y;
        }
        H[t] = make_double2(re, im);
    }
}

// inverse x + chain rule: wS_c = sum_kx wgt Re(H e^{+i kx x}); ubar = dL/du
template <class R>
__global__ void __launch_bounds__(128) band_ix_kernel(const CPlanes<R> u, int nx, int ny, int nz, int kmax,
                                                      const double2* H, const double2* tw, double norm, Planes<R> ub) {
    const size_t rows = (size_t)ny * nz;
    const size_t n = rows * nx;
    const int K1 = kmax + 1;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(c % nx);
        const size_t row = c / nx;
        double rho = fmax((double)u.p[0][c], 1e-300), isr = 1.0 / sqrt(rho);
        double rhob = 0.0;
        for (int comp = 0; comp < 3; ++comp) {
            double ws = 0.0;
            for (int kx = 0; kx < K1; ++kx) {
                double2 h = H[((size_t)comp * K1 + kx) * rows + row];
                double2 e = tw[(size_t)kx * nx + x];
                ws += (kx > 0 ? 2.0 : 1.0) * (h.x * e.x + h.y * e.y);   // Re(h * conj(e))
            }
            double wb = ws * norm;
            double m = (double)u.p[1 + comp][c];
            ub.p[1 + comp][c] = (R)(wb * isr);
            rhob += -0.5 * wb * m * isr / rho;
        }
        ub.p[0][c] = (R)rhob;
        for (int v = 4; v < 9; ++v) ub.p[v][c] = (R)0;
    }
}

template <class R>
cudaError_t launch_band_loss(const CPlanes<R>& u, int nx, int ny, int nz, int kmin, int kmax, void* scratch, double* L_host,
                             const Planes<R>& ub, cudaStream_t s) {
    const size_t K1 = kmax + 1, K2 = 2 * kmax + 1;
    char* p = static_cast<char*>(scratch);
    double2* twx = reinterpret_cast<double2*>(p);
    double2* twy = twx + K1 * nx;
    double2* twz = twy + K2 * ny;
    double2* A = twz + K2 * nz;
    double2* B = A + 3 * K1 * (size_t)ny * nz;
    double2* Cc = B + 3 * K1 * K2 * (size_t)nz;
    double2* G = Cc + 3 * K1 * K2 * K2;
    double* L = reinterpret_cast<double*>(G + 3 * K1 * K2 * (size_t)nz);
    std::vector<double> tx = spectrum_twiddles(nx, 0, kmax), ty = spectrum_twiddles(ny, -kmax, kmax),
                        tz = spectrum_twiddles(nz, -kmax, kmax);
    cudaError_t e = cudaMemcpyAsync(twx, tx.data(), tx.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(twy, ty.data(), ty.size() * 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(twz, tz.data(), tz.size() * 8, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    const double n3 = (double)nx * ny * nz;
    auto grid = [](size_t total) { return (int)std::min<size_t>((total + 127) / 128, 148 * 32); };
    spec_x_kernel<R><<<grid(3 * K1 * ny * nz), 128, 0, s>>>(u, nx, ny, nz, kmax, twx, A);
    spec_y_kernel<<<grid(3 * K1 * K2 * nz), 128, 0, s>>>(A, ny, nz, kmax, twy, B);
    band_z_kernel<<<grid(3 * K1 * K2 * K2), 128, 0, s>>>(B, nz, kmax, twz, 1.0 / n3, Cc);
    band_loss_kernel<<<1, 1, 0, s>>>(Cc, kmax, kmin, kmax, L);
    band_iz_kernel<<<grid(3 * K1 * K2 * nz), 128, 0, s>>>(Cc, nz, kmax, kmin, kmax, twz, G);
    band_iy_kernel<<<grid(3 * K1 * ny * nz), 128, 0, s>>>(G, ny, nz, kmax, twy, A);
    band_ix_kernel<R><<<grid((size_t)nx * ny * nz), 128, 0, s>>>(u, nx, ny, nz, kmax, A, twx, 1.0 / n3, ub);
    e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(L_host, L, sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    return e;
}

size_t band_scratch_bytes(int nx, int ny, int nz, int kmax) {
    const size_t K1 = kmax + 1, K2 = 2 * kmax + 1;
    return 2 * sizeof(double) * (K1 * nx + K2 * ny + K2 * nz) + 3 * K1 * (size_t)ny * nz * sizeof(double2) +
           3 * K1 * K2 * (size_t)nz * sizeof(double2) * 2 + 3 * K1 * K2 * K2 * sizeof(double2) + 256;
}

template cudaError_t launch_band_loss<float>(const CPlanes<float>&, int, int, int, int, int, void*, double*,
                                             const Planes<float>&, cudaStream_t);
template cudaError_t launch_band_loss<double>(const CPlanes<double>&, int, int, int, int, int, void*, double*,
                                              const Planes<double>&, cudaStream_t);

// ---------------------------------------------------------------------------------------------
// Log-density PDF: s = ln(rho / <rho>), its histogram on [smin, smax) and its mean and standard
// deviation sigma_s.  Per-block FP64 partials in a fixed tree order and a one-thread final sum
// (deterministic); the histogram is integer counts.
// ---------------------------------------------------------------------------------------------
constexpr int PDF_BLOCKS = 592, PDF_THREADS = 256;

template <class R>
__device__ __forceinline__ double block_sum256(double v, double* red) {
    red[threadIdx.x] = v;
    __syncthreads();
    for (int st = PDF_THREADS / 2; st > 0; st >>= 1) {
        if ((int)threadIdx.x < st) red[threadIdx.x] += red[threadIdx.x + st];
        __syncthreads();
    }
    double r = red[0];
    __syncthreads();
    return r;
}

template <class R>
__global__ void __launch_bounds__(PDF_THREADS) pdf_mass_kernel(const R* rho, size_t n, double* part) {
    __shared__ double red[PDF_THREADS];
    double m = 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
        m += (double)rho[c];
    double t = block_sum256<R>(m, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void pdf_mean_kernel(const double* part, int nb, size_t n, double* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double m = 0.0;
    for (int b = 0; b < nb; ++b) m += part[b];
    out[0] = m / (double)n;
}

template <class R>
__global__ void __launch_bounds__(PDF_THREADS) pdf_hist_kernel(const R* rho, size_t n, const double* mean, int nbins,
                                                               double smin, double smax, double* part,
                                                               unsigned long long* hist) {
    __shared__ double red[PDF_THREADS];
    extern __shared__ unsigned int hs[];
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) hs[b] = 0u;
    __syncthreads();
    const double irm = 1.0 / mean[0];
    const double idel = (double)nbins / (smax - smin);
    double s1 = 0.0, s2 = 0.0;
    for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x) {
        double sv = log((double)rho[c] * irm);
        s1 += sv;
        s2 += sv * sv;
        double f = (sv - smin) * idel;
        if (f >= 0.0 && f < (double)nbins) atomicAdd(&hs[(int)f], 1u);
    }
    double t1 = block_sum256<R>(s1, red);
    double t2 = block_sum256<R>(s2, red);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = t1; part[2 * blockIdx.x + 1] = t2; }
    for (int b = threadIdx.x; b < nbins; b += blockDim.x)
        if (hs[b]) atomicAdd(&hist[b], (unsigned long long)hs[b]);
}

__global__ void pdf_final_kernel(const double* part, int nb, size_t n, double* out) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double s1 = 0.0, s2 = 0.0;
    for (int b = 0; b < nb; ++b) { s1 += part[2 * b]; s2 += part[2 * b + 1]; }
    const double m = s1 / (double)n;
    out[1] = m;
    out[2] = sqrt(fmax(s2 / (double)n - m * m, 0.0));
}

size_t pdf_scratch_bytes(int nbins) { return (size_t)(3 * PDF_BLOCKS + 8) * sizeof(double) + (size_t)nbins * 8; }

template <class R>
cudaError_t launch_density_pdf(const R* rho, size_t n, int nbins, double smin, double smax, void* scratch,
                               double* pdf_host, double* stats_host, cudaStream_t s) {
    double* part = static_cast<double*>(scratch);          // [3 * PDF_BLOCKS]
    double* out = part + 3 * PDF_BLOCKS;                    // [mean rho, mean s, sigma_s]
    unsigned long long* hist = reinterpret_cast<unsigned long long*>(out + 8);
    cudaError_t e = cudaMemsetAsync(hist, 0, (size_t)nbins * 8, s);
    if (e != cudaSuccess) return e;
    pdf_mass_kernel<R><<<PDF_BLOCKS, PDF_THREADS, 0, s>>>(rho, n, part);
    pdf_mean_kernel<<<1, 1, 0, s>>>(part, PDF_BLOCKS, n, out);
    pdf_hist_kernel<R><<<PDF_BLOCKS, PDF_THREADS, (size_t)nbins * sizeof(unsigned), s>>>(rho, n, out, nbins, smin, smax,
                                                                                        part, hist);
    pdf_final_kernel<<<1, 1, 0, s>>>(part, PDF_BLOCKS, n, out);
    e = cudaGetLastError();
    std::vector<unsigned long long> h((size_t)nbins);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h.data(), hist, (size_t)nbins * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(stats_host, out, 3 * sizeof(double), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    const double ds = (smax - smin) / nbins;
    for (int b = 0; b < nbins; ++b) pdf_host[b] = (double)h[b] / ((double)n * ds);
    return cudaSuccess;
}

template cudaError_t launch_density_pdf<float>(const float*, size_t, int, double, double, void*, double*, double*,
                                               cudaStream_t);
template cudaError_t launch_density_pdf<double>(const double*, size_t, int, double, double, void*, double*, double*,
                                                cudaStream_t);

template cudaError_t launch_spectrum<float>(const CPlanes<float>&, int, int, int, int, void*, double*, cudaStream_t);
template cudaError_t launch_spectrum<double>(const CPlanes<double>&, int, int, int, int, void*, double*, cudaStream_t);

}  // namespace gmt
