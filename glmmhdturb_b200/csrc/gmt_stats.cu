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

template cudaError_t launch_spectrum<float>(const CPlanes<float>&, int, int, int, int, void*, double*, cudaStream_t);
template cudaError_t launch_spectrum<double>(const CPlanes<double>&, int, int, int, int, void*, double*, cudaStream_t);

}  // namespace gmt
