// sd_fft.cuh -- shared-memory Stockham FFT for many lines per CTA (sm_100a).
//
// A CTA holds L lines of N complex values in shared memory and transforms all
// of them at once. Stages are mixed radix (8, then 4 or 2 for the remainder),
// in the self-sorting Stockham form: stage with radix R and sub-transform
// length Ns reads in[j + r*N/R], multiplies by W_{Ns*R}^{(j mod Ns)*r}, does an
// R-point DFT in registers and writes out[(j/Ns)*Ns*R + (j mod Ns) + r*Ns].
// Output is in natural order. Each stage loads all its butterflies into
// registers, synchronises and stores back in place, so one buffer suffices.
//
// Shared-memory layout: element i of a line sits at i + (i >> 4) (one pad slot
// per 16 float2), which keeps every stage's accesses at or near the two
// wavefronts per warp that 8-byte accesses need.
//
// Twiddles come from a table tw[m] = exp(-2 pi i m / M) of the transform's
// "table length" M = N * TWS (TWS = table stride); the inverse uses conjugates.
// Transforms are unnormalised.
#pragma once

#include <cuda_runtime.h>

namespace sd {
namespace fft {

__host__ __device__ constexpr int pad(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int line_stride(int n) { return n + (n >> 4) + 1; }

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 conjf2(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (forward) or +i (inverse)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 2) {
        const float2 a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if constexpr (R == 4) {
        const float2 t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
        const float2 t2 = cadd(v[1], v[3]), t3 = mul_mi<INV>(csub(v[1], v[3]));
        v[0] = cadd(t0, t2);
        v[2] = csub(t0, t2);
        v[1] = cadd(t1, t3);
        v[3] = csub(t1, t3);
    } else {  // R == 8: two 4-point DFTs of the even and odd inputs
        float2 e[4] = {v[0], v[2], v[4], v[6]};
        float2 o[4] = {v[1], v[3], v[5], v[7]};
        dft<4, INV>(e);
        dft<4, INV>(o);
        constexpr float c = 0.70710678118654752440f;
        // W8^1 = c(1 -/+ i), W8^2 = -/+ i, W8^3 = c(-1 -/+ i)
        const float2 o1 = INV ? make_float2(c * (o[1].x - o[1].y), c * (o[1].x + o[1].y))
                              : make_float2(c * (o[1].x + o[1].y), c * (o[1].y - o[1].x));
        const float2 o2 = mul_mi<INV>(o[2]);
        const float2 o3 = INV ? make_float2(-c * (o[3].x + o[3].y), c * (o[3].x - o[3].y))
                              : make_float2(c * (o[3].y - o[3].x), -c * (o[3].x + o[3].y));
        v[0] = cadd(e[0], o[0]);
        v[4] = csub(e[0], o[0]);
        v[1] = cadd(e[1], o1);
        v[5] = csub(e[1], o1);
        v[2] = cadd(e[2], o2);
        v[6] = csub(e[2], o2);
        v[3] = cadd(e[3], o3);
        v[7] = csub(e[3], o3);
    }
}

template <int REM>
struct radix_of {
    static constexpr int value = (REM % 8 == 0) ? 8 : ((REM % 4 == 0) ? 4 : 2);
};

// One Stockham stage on L lines of length N (line stride LS), then recurse.
template <int N, int Ns, int L, int LS, int NT, int TWS, bool INV>
__device__ __forceinline__ void stages(float2* s, const float2* tw) {
    if constexpr (Ns < N) {
        constexpr int R = radix_of<N / Ns>::value;
        constexpr int NB = N / R;
        constexpr int TOT = L * NB;
        constexpr int PER = (TOT + NT - 1) / NT;
        float2 v[PER][R];
#pragma unroll
        for (int p = 0; p < PER; ++p) {
            const int t = threadIdx.x + p * NT;
            if (TOT % NT == 0 || t < TOT) {
                const int l = t / NB, j = t % NB, k = j % Ns;
                const float2* line = s + l * LS;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    float2 x = line[pad(j + r * NB)];
                    if (Ns > 1 && r > 0) {
                        float2 w = tw[(k * r * (N / (Ns * R))) * TWS];
                        if (INV) w.y = -w.y;
                        x = cmul(x, w);
                    }
                    v[p][r] = x;
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int p = 0; p < PER; ++p) {
            const int t = threadIdx.x + p * NT;
            if (TOT % NT == 0 || t < TOT) {
                const int l = t / NB, j = t % NB, k = j % Ns;
                dft<R, INV>(v[p]);
                float2* line = s + l * LS;
                const int base = (j / Ns) * Ns * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) line[pad(base + r * Ns)] = v[p][r];
            }
        }
        __syncthreads();
        stages<N, Ns * R, L, LS, NT, TWS, INV>(s, tw);
    }
}

// Transform L lines of length N held in s (line stride LS). Caller synchronises
// before the call (data in place); the routine ends with a barrier.
template <int N, int L, int LS, int NT, int TWS, bool INV>
__device__ __forceinline__ void lines(float2* s, const float2* tw) {
    stages<N, 1, L, LS, NT, TWS, INV>(s, tw);
}

}  // namespace fft
}  // namespace sd
