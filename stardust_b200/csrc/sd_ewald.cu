// sd_ewald.cu -- FP64 reference forces by Ewald summation (the accuracy reference).
//
// The model is the one the periodic PM step approximates (Green's function of
// kPoissonPeriodic, Sim.cu:528-557): Newtonian gravity in the unit periodic box,
// G = 1, each source of mass 1/n_src, the mean density removed (k = 0 mode
// dropped), masses smoothed by a Gaussian of width s (the PM softening
// softening_cells/G in box units). Without any grid, its potential is
//   Phi_hat(k) = -4 pi rho_hat(k) exp(-k^2 s^2 / 2) / k^2,   k = 2 pi n, n != 0.
// Ewald split with b^2 = 2 s^2 + 1/alpha^2:
//   exp(-k^2 s^2/2)/k^2 = exp(-k^2 b^2/4)/k^2  +  [exp(-k^2 s^2/2) - exp(-k^2 b^2/4)]/k^2
// The first term is summed over modes |n| <= n_max (structure factors of all
// sources); the second is, in real space, the pair potential
//   phi_s(r) = -m [erf(r/a) - erf(r/b)] / r,   a = sqrt(2) s,
// which decays like a Gaussian of width b and is summed over all sources at
// their nearest periodic image (r_cut = 0.5 must exceed a few b).
// Everything is FP64. These kernels measure force errors; they are not on the
// simulation path.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "sd_internal.h"

namespace sd {
namespace {

constexpr int kEwThreads = 256;
constexpr double kPi = 3.14159265358979323846;

// rho_hat(n) = sum_j m exp(-2 pi i n . x_j) for one mode per thread, sources
// staged through shared memory.
__global__ void __launch_bounds__(kEwThreads) k_structure(const float4* __restrict__ src, int n_src,
                                                         const int3* __restrict__ modes, int n_modes,
                                                         double2* __restrict__ rho_hat) {
    __shared__ double3 tile[kEwThreads];
    const int mi = blockIdx.x * blockDim.x + threadIdx.x;
    int3 n = make_int3(0, 0, 0);
    if (mi < n_modes) n = modes[mi];
    double re = 0.0, im = 0.0;
    for (int base = 0; base < n_src; base += kEwThreads) {
        const int j = base + threadIdx.x;
        if (j < n_src) {
            const float4 p = src[j];
            tile[threadIdx.x] = make_double3(p.x, p.y, p.z);
        }
        __syncthreads();
        const int cnt = min(kEwThreads, n_src - base);
        for (int t = 0; t < cnt; ++t) {
            const double3 x = tile[t];
            const double ph = -2.0 * kPi * ((double)n.x * x.x + (double)n.y * x.y + (double)n.z * x.z);
            double sn, cs;
            sincos(ph, &sn, &cs);
            re += cs;
            im += sn;
        }
        __syncthreads();
    }
    if (mi < n_modes) rho_hat[mi] = make_double2(re / (double)n_src, im / (double)n_src);
}

__device__ __forceinline__ double min_image(double d) { return d - rint(d); }

// a(x_t) = long-range mode sum + short-range pair sum, one target per thread.
__global__ void __launch_bounds__(kEwThreads) k_ewald_force(const float4* __restrict__ src, int n_src,
                                                           const float4* __restrict__ tgt, int n_tgt,
                                                           const int3* __restrict__ modes,
                                                           const double* __restrict__ coef,
                                                           const double2* __restrict__ rho_hat, int n_modes,
                                                           double a_len, double b_len, double3* __restrict__ out) {
    __shared__ double3 tile[kEwThreads];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double3 x = make_double3(0.0, 0.0, 0.0);
    if (i < n_tgt) {
        const float4 p = tgt[i];
        x = make_double3(p.x, p.y, p.z);
    }
    double ax = 0.0, ay = 0.0, az = 0.0;
    // long range: a = -sum_k c_k k Im[rho_hat(k) exp(i k.x)], both halves folded into c_k
    if (i < n_tgt) {
        for (int mi = 0; mi < n_modes; ++mi) {
            const int3 n = modes[mi];
            const double ph = 2.0 * kPi * ((double)n.x * x.x + (double)n.y * x.y + (double)n.z * x.z);
            double sn, cs;
            sincos(ph, &sn, &cs);
            const double2 r = rho_hat[mi];
            const double imv = r.x * sn + r.y * cs;
            const double f = -coef[mi] * imv * 2.0 * kPi;
            ax += f * n.x;
            ay += f * n.y;
            az += f * n.z;
        }
    }
    // short range over all sources at their nearest image
    const double inv_a = 1.0 / a_len, inv_b = 1.0 / b_len;
    const double ca = 2.0 / (sqrt(kPi) * a_len), cb = 2.0 / (sqrt(kPi) * b_len);
    const double m = 1.0 / (double)n_src;
    for (int base = 0; base < n_src; base += kEwThreads) {
        const int j = base + threadIdx.x;
        if (j < n_src) {
            const float4 p = src[j];
            tile[threadIdx.x] = make_double3(p.x, p.y, p.z);
        }
        __syncthreads();
        const int cnt = min(kEwThreads, n_src - base);
        if (i < n_tgt) {
            for (int t = 0; t < cnt; ++t) {
                const double3 s = tile[t];
                const double dx = min_image(x.x - s.x), dy = min_image(x.y - s.y), dz = min_image(x.z - s.z);
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 < 1e-24 || r2 > 0.25) continue;
                const double r = sqrt(r2);
                // f(r) = [erf(r/a) - erf(r/b)] / r ; a = m f'(r) r_hat
                const double e = erf(r * inv_a) - erf(r * inv_b);
                const double dfdr = (ca * exp(-r2 * inv_a * inv_a) - cb * exp(-r2 * inv_b * inv_b)) / r - e / r2;
                const double g = m * dfdr / r;
                ax += g * dx;
                ay += g * dy;
                az += g * dz;
            }
        }
        __syncthreads();
    }
    if (i < n_tgt) out[i] = make_double3(ax, ay, az);
}

}  // namespace
}  // namespace sd

using namespace sd;

extern "C" {

// Number of half-space modes with 0 < |n|^2 <= nmax^2 (the workspace layout).
int sd_ewald_modes(int nmax) {
    int c = 0;
    for (int nz = 0; nz <= nmax; ++nz)
        for (int ny = -nmax; ny <= nmax; ++ny)
            for (int nx = -nmax; nx <= nmax; ++nx) {
                if (nz == 0 && (ny < 0 || (ny == 0 && nx <= 0))) continue;
                if (nx * nx + ny * ny + nz * nz > nmax * nmax) continue;
                ++c;
            }
    return c;
}

size_t sd_ewald_workspace_bytes(int nmax) {
    const size_t m = (size_t)sd_ewald_modes(nmax);
    return align_up(m * sizeof(int3), 256) + align_up(m * sizeof(double), 256) + align_up(m * sizeof(double2), 256);
}

int sd_ewald_forces(const float* src, int n_src, const float* tgt, int n_tgt, double softening, double split_b,
                    int nmax, double* acc_out, void* workspace, size_t workspace_bytes, void* stream) {
    if (!src || !tgt || !acc_out || !workspace || n_src <= 0 || n_tgt < 0 || nmax < 1 || softening <= 0.0 ||
        split_b * split_b <= 2.0 * softening * softening || split_b > 0.1)
        return fail(SD_E_ARG, "ewald: bad arguments (need 0 < 2 s^2 < b^2, b <= 0.1, nmax >= 1)");
    if (workspace_bytes < sd_ewald_workspace_bytes(nmax)) return fail(SD_E_ARG, "ewald: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const int nm = sd_ewald_modes(nmax);
    std::vector<int3> modes;
    std::vector<double> coef;
    modes.reserve(nm);
    coef.reserve(nm);
    for (int nz = 0; nz <= nmax; ++nz)
        for (int ny = -nmax; ny <= nmax; ++ny)
            for (int nx = -nmax; nx <= nmax; ++nx) {
                if (nz == 0 && (ny < 0 || (ny == 0 && nx <= 0))) continue;
                const int n2 = nx * nx + ny * ny + nz * nz;
                if (n2 > nmax * nmax) continue;
                const double k2 = 4.0 * kPi * kPi * (double)n2;
                modes.push_back(make_int3(nx, ny, nz));
                // 4 pi exp(-k^2 b^2/4)/k^2, times 2 for the conjugate mode -n
                coef.push_back(2.0 * 4.0 * kPi * exp(-0.25 * k2 * split_b * split_b) / k2);
            }
    char* w = (char*)workspace;
    int3* d_modes = (int3*)w;
    double* d_coef = (double*)(w + align_up((size_t)nm * sizeof(int3), 256));
    double2* d_rho = (double2*)(w + align_up((size_t)nm * sizeof(int3), 256) + align_up((size_t)nm * sizeof(double), 256));
    if (SD_CUDA(cudaMemcpyAsync(d_modes, modes.data(), sizeof(int3) * nm, cudaMemcpyHostToDevice, st)) ||
        SD_CUDA(cudaMemcpyAsync(d_coef, coef.data(), sizeof(double) * nm, cudaMemcpyHostToDevice, st)))
        return SD_E_CUDA;
    k_structure<<<(nm + kEwThreads - 1) / kEwThreads, kEwThreads, 0, st>>>(reinterpret_cast<const float4*>(src), n_src,
                                                                        d_modes, nm, d_rho);
    SD_LAUNCHED(st);
    if (n_tgt > 0) {
        k_ewald_force<<<(n_tgt + kEwThreads - 1) / kEwThreads, kEwThreads, 0, st>>>(
            reinterpret_cast<const float4*>(src), n_src, reinterpret_cast<const float4*>(tgt), n_tgt, d_modes, d_coef,
            d_rho, nm, sqrt(2.0) * softening, split_b, reinterpret_cast<double3*>(acc_out));
        SD_LAUNCHED(st);
    }
    // the host vectors must outlive the asynchronous copies
    return SD_CUDA(cudaStreamSynchronize(st));
}

}  // extern "C"
