// sd_fft.cuh -- shared-memory Stockham FFT over 16 interleaved lines (sm_100a).
//
// A CTA holds 16 lines of N complex values in shared memory, interleaved:
// element i of line l sits at s[i*16 + l]. All 16 lines are transformed at once.
// Threads are mapped line-fastest (item u -> line u & 15, butterfly u >> 4), so
// every load and store of every stage touches two runs of 16 consecutive
// float2 per warp: the two-wavefront minimum for 8-byte accesses, with no
// padding and no bank conflicts.
//
// Stages are mixed radix (32 or 16 where every thread still gets a butterfly,
// else 8, then 4 or 2 for the remainder) in the self-sorting
// Stockham form: the stage with radix R and sub-transform length Ns reads
// in[j + r*N/R], multiplies by W_{Ns*R}^{(j mod Ns)*r}, does an R-point DFT in
// registers and writes out[(j/Ns)*Ns*R + (j mod Ns) + r*Ns]. Output is in
// natural order. Each stage loads all its butterflies into registers,
// synchronises and stores back in place.
//
// Twiddles come from a table tw[m] = exp(-2 pi i m / M) of length M = N * TWS
// (TWS = table stride); the inverse uses conjugates. Transforms are unnormalised.
#pragma once

#include <cuda_runtime.h>

namespace sd {
namespace fft {

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

// W_32^k = exp(-2 pi i k / 32), k < 16 (mathematical constants; the inverse uses
// conjugates). W_16^k = W_32^(2k).
namespace w32 {
constexpr float c1 = 0.98078528040323044913f, s1 = 0.19509032201612826785f;
constexpr float c2 = 0.92387953251128675613f, s2 = 0.38268343236508977173f;
constexpr float c3 = 0.83146961230254523708f, s3 = 0.55557023301960222474f;
constexpr float r = 0.70710678118654752440f;
__device__ __forceinline__ float2 get(int k) {  // k is a compile-time constant after unrolling
    switch (k) {
        case 0: return make_float2(1.f, 0.f);
        case 1: return make_float2(c1, -s1);
        case 2: return make_float2(c2, -s2);
        case 3: return make_float2(c3, -s3);
        case 4: return make_float2(r, -r);
        case 5: return make_float2(s3, -c3);
        case 6: return make_float2(s2, -c2);
        case 7: return make_float2(s1, -c1);
        case 8: return make_float2(0.f, -1.f);
        case 9: return make_float2(-s1, -c1);
        case 10: return make_float2(-s2, -c2);
        case 11: return make_float2(-s3, -c3);
        case 12: return make_float2(-r, -r);
        case 13: return make_float2(-c3, -s3);
        case 14: return make_float2(-c2, -s2);
        default: return make_float2(-c1, -s1);
    }
}
}  // namespace w32

template <int R, bool INV>
__device__ __forceinline__ void dft(float2* v) {
    if constexpr (R == 16 || R == 32) {
        // radix-2 split: DFTs of the even and odd inputs, combined with W_R^k
        constexpr int H = R / 2;
        float2 e[H], o[H];
#pragma unroll
        for (int i = 0; i < H; ++i) {
            e[i] = v[2 * i];
            o[i] = v[2 * i + 1];
        }
        dft<H, INV>(e);
        dft<H, INV>(o);
#pragma unroll
        for (int k = 0; k < H; ++k) {
            float2 w = w32::get(k * (32 / R));
            if (INV) w.y = -w.y;
            const float2 t = (k == 0) ? o[k] : cmul(o[k], w);
            v[k] = cadd(e[k], t);
            v[k + H] = csub(e[k], t);
        }
    } else if constexpr (R == 2) {
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

// Radix of the next stage for a remaining length REM of an N-point transform on
// NT threads: the largest of 32, 16 that divides REM and still gives every thread
// a butterfly (16 N / R >= NT), else 8, 4 or 2. Fewer, wider stages mean fewer
// shared-memory round trips.
template <int REM, int N, int NT>
struct radix_of {
    static constexpr int value = (REM % 32 == 0 && 16 * N / 32 >= NT)   ? 32
                                 : (REM % 16 == 0 && 16 * N / 16 >= NT) ? 16
                                 : (REM % 8 == 0)                       ? 8
                                 : (REM % 4 == 0)                       ? 4
                                                                        : 2;
};

// One Stockham stage on the 16 interleaved lines, then recurse.
// radix_of as a constexpr function, and the sub-transform length Ns of the last
// stage of an N-point transform on NT threads.
constexpr int radix_for(int rem, int N, int NT) {
    return (rem % 32 == 0 && 16 * N / 32 >= NT)   ? 32
           : (rem % 16 == 0 && 16 * N / 16 >= NT) ? 16
           : (rem % 8 == 0)                       ? 8
           : (rem % 4 == 0)                       ? 4
                                                  : 2;
}
constexpr int last_stage_ns(int N, int NT) {
    int ns = 1;
    while (ns * radix_for(N / ns, N, NT) < N) ns *= radix_for(N / ns, N, NT);
    return ns;
}

// Element `pos` of line l as the first stage reads it: plainly, or through a
// caller's functor that forms it from what s holds (a pre-processing step fused
// into the first stage's loads, saving a shared-memory round trip and a barrier).
struct PlainLoad {
    __device__ __forceinline__ float2 operator()(const float2* s, int l, int pos) const { return s[pos * 16 + l]; }
};

// Stages from sub-transform length Ns on, stopping before the stage at STOP; the
// stage at Ns = 1 reads through `load`.
template <int N, int Ns, int NT, int TWS, bool INV, int STOP = N, class Load = PlainLoad>
__device__ __forceinline__ void stages16(float2* s, const float2* tw, Load load = Load()) {
    if constexpr (Ns < N && Ns < STOP) {
        constexpr int R = radix_of<N / Ns, N, NT>::value;
        constexpr int NB = N / R;
        constexpr int TOT = 16 * NB;
        constexpr int PER = (TOT + NT - 1) / NT;
        float2 v[PER][R];
#pragma unroll
        for (int p = 0; p < PER; ++p) {
            const int u = threadIdx.x + p * NT;
            if (TOT % NT == 0 || u < TOT) {
                const int l = u & 15, j = u >> 4, k = j % Ns;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    float2 x = (Ns == 1) ? load(s, l, j + r * NB) : s[(j + r * NB) * 16 + l];
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
            const int u = threadIdx.x + p * NT;
            if (TOT % NT == 0 || u < TOT) {
                const int l = u & 15, j = u >> 4, k = j % Ns;
                dft<R, INV>(v[p]);
                const int base = (j / Ns) * Ns * R + k;
#pragma unroll
                for (int r = 0; r < R; ++r) s[(base + r * Ns) * 16 + l] = v[p][r];
            }
        }
        __syncthreads();
        stages16<N, Ns * R, NT, TWS, INV, STOP>(s, tw);
    }
}

// Transform the 16 interleaved lines of length N in s. The caller synchronises
// before the call; the routine ends with a barrier.
template <int N, int NT, int TWS, bool INV>
__device__ __forceinline__ void lines16(float2* s, const float2* tw) {
    stages16<N, 1, NT, TWS, INV>(s, tw);
}

// Forward transform, a pointwise multiply, inverse transform of the 16 lines.
// The forward's last stage (radix R, sub-length Ns = N / R) leaves, in each
// thread's registers, the outputs at positions j + r Ns -- exactly the inputs of
// an inverse first stage of the same radix. So that stage, the multiply
// mul(line, position, value) and the inverse's first stage run in registers with
// no shared-memory round trip or barrier between them; the inverse then goes on
// from sub-length R. The caller synchronises before the call; it ends with a
// barrier.
template <int N, int NT, int TWS, class Mul>
__device__ __forceinline__ void convolve16(float2* s, const float2* tw, Mul mul) {
    constexpr int NsL = last_stage_ns(N, NT);
    constexpr int R = N / NsL;
    constexpr int NB = N / R;  // == NsL
    constexpr int TOT = 16 * NB;
    constexpr int PER = (TOT + NT - 1) / NT;
    stages16<N, 1, NT, TWS, false, NsL>(s, tw);
    float2 v[PER][R];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int u = threadIdx.x + p * NT;
        if (TOT % NT == 0 || u < TOT) {
            const int l = u & 15, j = u >> 4;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                float2 x = s[(j + r * NB) * 16 + l];
                if (NsL > 1 && r > 0) x = cmul(x, tw[(j * r) * TWS]);
                v[p][r] = x;
            }
        }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int u = threadIdx.x + p * NT;
        if (TOT % NT == 0 || u < TOT) {
            const int l = u & 15, j = u >> 4;
            dft<R, false>(v[p]);
#pragma unroll
            for (int r = 0; r < R; ++r) v[p][r] = mul(l, j + r * NsL, v[p][r]);
            dft<R, true>(v[p]);
#pragma unroll
            for (int r = 0; r < R; ++r) s[(j * R + r) * 16 + l] = v[p][r];
        }
    }
    __syncthreads();
    stages16<N, R, NT, TWS, true>(s, tw);
}

// lines16, with the last stage writing its outputs row-major (line l at
// s[l * RS + position]) instead of interleaved, for callers that store rows; the
// first stage reads through `load`.
template <int N, int NT, int TWS, bool INV, int RS, class Load = PlainLoad>
__device__ __forceinline__ void lines16_rows(float2* s, const float2* tw, Load load = Load()) {
    constexpr int NsL = last_stage_ns(N, NT);
    constexpr int R = N / NsL;
    constexpr int NB = N / R;
    constexpr int TOT = 16 * NB;
    constexpr int PER = (TOT + NT - 1) / NT;
    stages16<N, 1, NT, TWS, INV, NsL>(s, tw, load);
    float2 v[PER][R];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int u = threadIdx.x + p * NT;
        if (TOT % NT == 0 || u < TOT) {
            const int l = u & 15, j = u >> 4;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                float2 x = (NsL == 1) ? load(s, l, j + r * NB) : s[(j + r * NB) * 16 + l];
                if (NsL > 1 && r > 0) {
                    float2 w = tw[(j * r) * TWS];
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
        const int u = threadIdx.x + p * NT;
        if (TOT % NT == 0 || u < TOT) {
            const int l = u & 15, j = u >> 4;
            dft<R, INV>(v[p]);
#pragma unroll
            for (int r = 0; r < R; ++r) s[l * RS + j + r * NsL] = v[p][r];
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

}  // namespace fft
}  // namespace sd
