// sd_poisson.cu -- periodic Poisson solve: five passes over the grid, all
// hand-written (the reference calls cuFFT R2C, kPoissonPeriodic, cuFFT C2R:
// Sim.cu:3586-3603, 528-557).
//
// Layouts (complex = float2, H = G/2, P = H+1 kx bins):
//   rho, phi : real [z][y][x]
//   specA    : [z][kx][y]  (y contiguous)    -- written by A and D
//   specB    : [kx][ky][z] (z contiguous)    -- written by B and C
// Passes:
//   A  x-lines real->complex (+ int64 fixed-point -> float conversion), write specA
//   B  y-lines forward, write specB transposed so z becomes contiguous
//   C  z-lines: forward, Green's function multiply, inverse (in place)
//   D  y-lines inverse, write specA layout
//   E  x-lines complex->real, write phi
// Every pass reads and writes each element once; transposes happen through the
// shared-memory tile, so global accesses are whole lines or 64-128 B segments.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "sd_common.cuh"
#include "sd_fft.cuh"
#include "sd_internal.h"

namespace sd {

namespace {

constexpr int kFftThreads = 256;

template <int G>
struct Tiles {
    static constexpr int H = G / 2;
    static constexpr int P = H + 1;
    static constexpr int TY = (G < 16) ? G : 16;  // rows per CTA in passes A and E
    static constexpr int TZ = (G < 8) ? G : 8;    // lines per CTA in passes B and D
    static constexpr int LC = (G < 8) ? G : 8;    // lines per CTA in pass C
    static constexpr int LSH = fft::line_stride(H);
    static constexpr int LSG = fft::line_stride(G);
};

template <int G>
__global__ void __launch_bounds__(kFftThreads) k_pass_a(const long long* __restrict__ acc, const float* __restrict__ rho,
                                                        int clear_acc, float* __restrict__ rho_keep,
                                                        float2* __restrict__ specA, const float2* __restrict__ tw_g) {
    using T = Tiles<G>;
    constexpr int H = T::H, P = T::P, TY = T::TY, LS = T::LSH;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* s = sm + G;
    const int y0 = blockIdx.x * TY, z = blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    for (int t = threadIdx.x; t < TY * H; t += kFftThreads) {
        const int yy = t / H, m = t % H;
        const size_t row = ((size_t)z * G + y0 + yy) * G;
        float2 v;
        if (acc) {
            longlong2* p = reinterpret_cast<longlong2*>(const_cast<long long*>(acc) + row) + m;
            const longlong2 q = *p;
            v = make_float2(fixed_to_float(q.x), fixed_to_float(q.y));
            if (clear_acc) *p = make_longlong2(0, 0);
            if (rho_keep) reinterpret_cast<float2*>(rho_keep + row)[m] = v;
        } else {
            v = reinterpret_cast<const float2*>(rho + row)[m];
        }
        s[yy * LS + fft::pad(m)] = v;
    }
    __syncthreads();
    fft::lines<H, TY, LS, kFftThreads, 2, false>(s, tw);
    // Z -> X:  X[k] = E[k] + W_G^k O[k],  E = (Z[k] + conj Z[H-k])/2,  O = (Z[k] - conj Z[H-k])/(2i)
    for (int t = threadIdx.x; t < P * TY; t += kFftThreads) {
        const int kx = t / TY, yy = t % TY;
        const float2* line = s + yy * LS;
        const float2 zk = line[fft::pad(kx == H ? 0 : kx)];
        const float2 zc = line[fft::pad(kx == 0 ? 0 : H - kx)];
        const float er = 0.5f * (zk.x + zc.x), ei = 0.5f * (zk.y - zc.y);
        const float orr = 0.5f * (zk.y + zc.y), oi = -0.5f * (zk.x - zc.x);
        const float2 w = tw[kx];
        specA[((size_t)z * P + kx) * G + y0 + yy] =
            make_float2(er + (w.x * orr - w.y * oi), ei + (w.x * oi + w.y * orr));
    }
}

template <int G>
__global__ void __launch_bounds__(kFftThreads) k_pass_b(const float2* __restrict__ specA, float2* __restrict__ specB,
                                                        const float2* __restrict__ tw_g) {
    using T = Tiles<G>;
    constexpr int P = T::P, TZ = T::TZ, LS = T::LSG;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* s = sm + G;
    const int z0 = blockIdx.x * TZ, kx = blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    for (int t = threadIdx.x; t < TZ * G; t += kFftThreads) {
        const int l = t / G, y = t % G;
        s[l * LS + fft::pad(y)] = specA[((size_t)(z0 + l) * P + kx) * G + y];
    }
    __syncthreads();
    fft::lines<G, TZ, LS, kFftThreads, 1, false>(s, tw);
    for (int t = threadIdx.x; t < TZ * G; t += kFftThreads) {
        const int l = t % TZ, ky = t / TZ;
        specB[((size_t)kx * G + ky) * G + z0 + l] = s[l * LS + fft::pad(ky)];
    }
}

template <int G>
__global__ void __launch_bounds__(kFftThreads) k_pass_c(float2* __restrict__ specB, const float2* __restrict__ tw_g,
                                                        const float* __restrict__ gexp_g, float scale) {
    using T = Tiles<G>;
    constexpr int LC = T::LC, LS = T::LSG, H = T::H;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float* gexp = reinterpret_cast<float*>(sm + G);
    float2* s = sm + G + (H + 2) / 2 + 1;
    const int ky0 = blockIdx.x * LC, kx = blockIdx.y;
    float2* base = specB + ((size_t)kx * G + ky0) * G;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    for (int i = threadIdx.x; i <= H; i += kFftThreads) gexp[i] = gexp_g[i];
    for (int t = threadIdx.x; t < LC * G; t += kFftThreads) {
        const int l = t / G, z = t % G;
        s[l * LS + fft::pad(z)] = base[t];
    }
    __syncthreads();
    fft::lines<G, LC, LS, kFftThreads, 1, false>(s, tw);
    // Green's function: -scale/k^2 * exp(-k^2 s^2/2), k = 0 -> 0 (Sim.cu:536-556).
    for (int t = threadIdx.x; t < LC * G; t += kFftThreads) {
        const int l = t / G, kz = t % G;
        const int ky = ky0 + l;
        const int kyf = (ky <= G / 2) ? ky : ky - G;
        const int kzf = (kz <= G / 2) ? kz : kz - G;
        const int k2 = kx * kx + kyf * kyf + kzf * kzf;
        float m = 0.f;
        if (k2 != 0) m = (-scale / (float)k2) * (gexp[kx] * gexp[abs(kyf)] * gexp[abs(kzf)]);
        float2& e = s[l * LS + fft::pad(kz)];
        e.x *= m;
        e.y *= m;
    }
    __syncthreads();
    fft::lines<G, LC, LS, kFftThreads, 1, true>(s, tw);
    for (int t = threadIdx.x; t < LC * G; t += kFftThreads) {
        const int l = t / G, z = t % G;
        base[t] = s[l * LS + fft::pad(z)];
    }
}

template <int G>
__global__ void __launch_bounds__(kFftThreads) k_pass_d(const float2* __restrict__ specB, float2* __restrict__ specA,
                                                        const float2* __restrict__ tw_g) {
    using T = Tiles<G>;
    constexpr int P = T::P, TZ = T::TZ, LS = T::LSG;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* s = sm + G;
    const int z0 = blockIdx.x * TZ, kx = blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    for (int t = threadIdx.x; t < TZ * G; t += kFftThreads) {
        const int l = t % TZ, ky = t / TZ;
        s[l * LS + fft::pad(ky)] = specB[((size_t)kx * G + ky) * G + z0 + l];
    }
    __syncthreads();
    fft::lines<G, TZ, LS, kFftThreads, 1, true>(s, tw);
    for (int t = threadIdx.x; t < TZ * G; t += kFftThreads) {
        const int l = t / G, y = t % G;
        specA[((size_t)(z0 + l) * P + kx) * G + y] = s[l * LS + fft::pad(y)];
    }
}

template <int G>
__global__ void __launch_bounds__(kFftThreads) k_pass_e(const float2* __restrict__ specA, float* __restrict__ phi,
                                                        const float2* __restrict__ tw_g) {
    using T = Tiles<G>;
    constexpr int H = T::H, P = T::P, TY = T::TY, LS = T::LSH;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* s = sm + G;
    const int y0 = blockIdx.x * TY, z = blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    for (int t = threadIdx.x; t < P * TY; t += kFftThreads) {
        const int kx = t / TY, yy = t % TY;
        s[yy * LS + fft::pad(kx)] = specA[((size_t)z * P + kx) * G + y0 + yy];
    }
    __syncthreads();
    // X -> Z, pairs (k, H-k) in place:
    //   Z[k] = E + i O,  E = X[k] + conj X[H-k],  O = (X[k] - conj X[H-k]) * exp(+2 pi i k / G)
    // (imaginary parts of the k = 0 and k = H bins are dropped, as a C2R transform does)
    constexpr int HP = H / 2 + 1;
    for (int t = threadIdx.x; t < TY * HP; t += kFftThreads) {
        const int yy = t / HP, k = t % HP;
        float2* line = s + yy * LS;
        float2 a = line[fft::pad(k)], b = line[fft::pad(H - k)];
        if (k == 0) { a.y = 0.f; b.y = 0.f; }
        {
            const float2 w = tw[k];
            const float er = a.x + b.x, ei = a.y - b.y, dr = a.x - b.x, di = a.y + b.y;
            const float orr = dr * w.x + di * w.y, oi = di * w.x - dr * w.y;
            line[fft::pad(k)] = make_float2(er - oi, ei + orr);
        }
        if (k != 0 && 2 * k != H) {
            const float2 w = tw[H - k];
            const float er = b.x + a.x, ei = b.y - a.y, dr = b.x - a.x, di = b.y + a.y;
            const float orr = dr * w.x + di * w.y, oi = di * w.x - dr * w.y;
            line[fft::pad(H - k)] = make_float2(er - oi, ei + orr);
        }
    }
    __syncthreads();
    fft::lines<H, TY, LS, kFftThreads, 2, true>(s, tw);
    for (int t = threadIdx.x; t < TY * H; t += kFftThreads) {
        const int yy = t / H, m = t % H;
        reinterpret_cast<float2*>(phi + ((size_t)z * G + y0 + yy) * G)[m] = s[yy * LS + fft::pad(m)];
    }
}

template <int G>
struct Launcher {
    using T = Tiles<G>;
    static size_t smem_a() { return sizeof(float2) * ((size_t)G + (size_t)T::TY * T::LSH); }
    static size_t smem_b() { return sizeof(float2) * ((size_t)G + (size_t)T::TZ * T::LSG); }
    static size_t smem_c() { return sizeof(float2) * ((size_t)G + (T::H + 2) / 2 + 1 + (size_t)T::LC * T::LSG); }

    static int configure() {
        static bool done = false;
        if (done) return SD_OK;
        int rc = SD_OK;
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_a<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_b<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_c<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_d<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_e<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a()));
        if (rc == SD_OK) done = true;
        return rc == SD_OK ? SD_OK : SD_E_CUDA;
    }

    static int run(const PoissonPlan& p, const long long* acc, const float* rho, int clear, float* keep, float2* A,
                   float2* B, float* phi, cudaStream_t s) {
        int rc = configure();
        if (rc != SD_OK) return rc;
        k_pass_a<G><<<dim3(G / T::TY, G), kFftThreads, smem_a(), s>>>(acc, rho, clear, keep, A, p.tw);
        SD_LAUNCHED(s);
        k_pass_b<G><<<dim3(G / T::TZ, T::P), kFftThreads, smem_b(), s>>>(A, B, p.tw);
        SD_LAUNCHED(s);
        k_pass_c<G><<<dim3(G / T::LC, T::P), kFftThreads, smem_c(), s>>>(B, p.tw, p.gexp, p.scale);
        SD_LAUNCHED(s);
        k_pass_d<G><<<dim3(G / T::TZ, T::P), kFftThreads, smem_b(), s>>>(B, A, p.tw);
        SD_LAUNCHED(s);
        k_pass_e<G><<<dim3(G / T::TY, G), kFftThreads, smem_a(), s>>>(A, phi, p.tw);
        SD_LAUNCHED(s);
        return SD_OK;
    }
};

}  // namespace

size_t poisson_spectrum_elems(int G) { return (size_t)G * G * (size_t)(G / 2 + 1); }

static int poisson_configure(int G) {
    switch (G) {
        case 16: return Launcher<16>::configure();
        case 32: return Launcher<32>::configure();
        case 64: return Launcher<64>::configure();
        case 128: return Launcher<128>::configure();
        case 256: return Launcher<256>::configure();
        case 512: return Launcher<512>::configure();
        default: return fail(SD_E_UNSUPPORTED, "poisson: grid size %d not supported", G);
    }
}

int poisson_plan_build(PoissonPlan& p, int G, float soft) {
    if (p.G == G && p.soft == soft && p.tw) return SD_OK;
    poisson_plan_free(p);
    // kernel attributes are set here, outside any stream capture
    if (int rc = poisson_configure(G)) return rc;
    std::vector<float2> tw((size_t)G);
    const double two_pi = 6.283185307179586476925286766559;
    for (int m = 0; m < G; ++m) {
        const double a = -two_pi * (double)m / (double)G;
        tw[m] = make_float2((float)cos(a), (float)sin(a));
    }
    std::vector<float> ge((size_t)G / 2 + 1);
    const double s = two_pi * (double)(soft > 0.f ? soft : 0.f) / (double)G;
    for (int k = 0; k <= G / 2; ++k) ge[k] = (float)exp(-0.5 * s * s * (double)k * (double)k);
    if (SD_CUDA(cudaMalloc(&p.tw, sizeof(float2) * tw.size())) != SD_OK) return SD_E_NOMEM;
    if (SD_CUDA(cudaMalloc(&p.gexp, sizeof(float) * ge.size())) != SD_OK) return SD_E_NOMEM;
    if (SD_CUDA(cudaMemcpy(p.tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice)) != SD_OK ||
        SD_CUDA(cudaMemcpy(p.gexp, ge.data(), sizeof(float) * ge.size(), cudaMemcpyHostToDevice)) != SD_OK)
        return SD_E_CUDA;
    p.scale = (float)(1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846 * (double)G * G * G));
    p.G = G;
    p.soft = soft;
    return SD_OK;
}

void poisson_plan_free(PoissonPlan& p) {
    if (p.tw) cudaFree(p.tw);
    if (p.gexp) cudaFree(p.gexp);
    p.tw = nullptr;
    p.gexp = nullptr;
    p.G = 0;
}

int launch_poisson(const PoissonPlan& p, const long long* acc, const float* rho, int clear, float* keep, float2* A,
                   float2* B, float* phi, cudaStream_t s) {
    switch (p.G) {
        case 16: return Launcher<16>::run(p, acc, rho, clear, keep, A, B, phi, s);
        case 32: return Launcher<32>::run(p, acc, rho, clear, keep, A, B, phi, s);
        case 64: return Launcher<64>::run(p, acc, rho, clear, keep, A, B, phi, s);
        case 128: return Launcher<128>::run(p, acc, rho, clear, keep, A, B, phi, s);
        case 256: return Launcher<256>::run(p, acc, rho, clear, keep, A, B, phi, s);
        case 512: return Launcher<512>::run(p, acc, rho, clear, keep, A, B, phi, s);
        default: return fail(SD_E_UNSUPPORTED, "poisson: grid size %d not supported", p.G);
    }
}

}  // namespace sd
