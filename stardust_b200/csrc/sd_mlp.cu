// sd_mlp.cu -- learned sub-grid force correction: features, BF16 tensor-core
// MLP (30 -> 64 -> 64 -> 3, SiLU), its training kernels and the fused inference
// that feeds the kick. No counterpart in the reference; the correction is added
// on top of the plain PM acceleration (kIntegrate's accG sample, Sim.cu:822).
//
// Numerics: weights and activations are BF16, every matrix product accumulates
// in FP32 on the tensor cores (mma.sync m16n8k16 bf16), biases and the SiLU are
// FP32, master weights and Adam moments are FP32.
//
// Parameter vector (FP32, kMlpParams floats): W1[32][64] (inputs padded 30->32),
// b1[64], W2[64][64], b2[64], W3[64][8] (outputs padded 3->8), b3[8]; W[k][n]
// maps input k to output n.
//
// Features of a particle at p (grid G, mean count per cell rho_bar):
//   f[(dz+1)*9 + (dy+1)*3 + (dx+1)] = log(1 + rho(c + d) / rho_bar) - log 2,  d in {-1,0,1}^3
//   f[27..29] = p*G - c - 1/2 (sub-cell offset), f[30] = f[31] = 0,
// with c = floor(p*G) the containing cell and rho the CIC density (count units).
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "sd_common.cuh"
#include "sd_internal.h"

namespace sd {
namespace {

constexpr int kIn = 32, kH = 64, kOut = 8;
constexpr int oW1 = 0, oB1 = oW1 + kIn * kH, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH,
              oB3 = oW3 + kH * kOut, kParams = oB3 + kOut;
static_assert(kParams == 6792, "parameter layout");

__device__ __forceinline__ unsigned pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);  // .x = lo (low 16 bits)
    return *reinterpret_cast<const unsigned*>(&v);
}

__device__ __forceinline__ void mma16816(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// SiLU through the hardware tanh (one MUFU op): sigmoid(z) = (1 + tanh(z/2)) / 2.
// Its relative error (about 2^-11) is below the BF16 rounding of the activations;
// training and inference use the same function.
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigmoid(float z) { return fmaf(0.5f, tanh_approx(0.5f * z), 0.5f); }

// SiLU of two pre-activations, computed and returned as packed BF16 (the inference's
// next-layer input): z is rounded to BF16 first, then z * (1/2 + tanh(z/2) / 2) with
// the packed BF16 tanh, so one special-function instruction serves two units.
__device__ __forceinline__ unsigned silu_bf16x2(float z0, float z1) {
    const __nv_bfloat162 z = __floats2bfloat162_rn(z0, z1);
    const __nv_bfloat162 half = __floats2bfloat162_rn(0.5f, 0.5f);
    const __nv_bfloat162 hz = __hmul2(z, half);  // exact: a power of two
    unsigned t;
    asm("tanh.approx.bf16x2 %0, %1;" : "=r"(t) : "r"(*reinterpret_cast<const unsigned*>(&hz)));
    const __nv_bfloat162 s = __hfma2(*reinterpret_cast<const __nv_bfloat162*>(&t), half, half);
    const __nv_bfloat162 r = __hmul2(z, s);
    return *reinterpret_cast<const unsigned*>(&r);
}
__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = sigmoid(z);
    return s * fmaf(z, 1.f - s, 1.f);
}

// ---- features -------------------------------------------------------------------
__device__ __forceinline__ void particle_features(const float* __restrict__ rho, int G, float inv_mean, float4 p,
                                                  float* f) {
    const int m = G - 1;
    const int cx = min(max((int)(p.x * (float)G), 0), m);
    const int cy = min(max((int)(p.y * (float)G), 0), m);
    const int cz = min(max((int)(p.z * (float)G), 0), m);
    const float ln2 = 0.69314718055994531f;
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const float r =
                    __ldg(rho + ((size_t)((cz + dz) & m) * G + ((cy + dy) & m)) * G + ((cx + dx) & m));
                f[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] = __logf(1.f + r * inv_mean) - ln2;
            }
    f[27] = p.x * (float)G - (float)cx - 0.5f;
    f[28] = p.y * (float)G - (float)cy - 0.5f;
    f[29] = p.z * (float)G - (float)cz - 0.5f;
    f[30] = 0.f;
    f[31] = 0.f;
}

__global__ void k_features(const float4* __restrict__ pos, const int* __restrict__ perm, int n,
                           const float* __restrict__ rho, int G, float inv_mean, __nv_bfloat16* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[perm ? perm[i] : i];
    float f[32];
    if (p.x < 0.f) {
#pragma unroll
        for (int j = 0; j < 32; ++j) f[j] = 0.f;
    } else {
        particle_features(rho, G, inv_mean, p, f);
    }
    uint4* o = reinterpret_cast<uint4*>(out + (size_t)i * kIn);
#pragma unroll
    for (int q = 0; q < 4; ++q)
        o[q] = make_uint4(pack_bf16(f[8 * q], f[8 * q + 1]), pack_bf16(f[8 * q + 2], f[8 * q + 3]),
                          pack_bf16(f[8 * q + 4], f[8 * q + 5]), pack_bf16(f[8 * q + 6], f[8 * q + 7]));
}

// ---- fused inference: 16 particles per warp-iteration -----------------------------
// B fragments of the three weight matrices, laid out per lane: for matrix W[K][N],
// k-chunk kc and n-tile nt, lane (g = lane/4, t = lane%4) holds
//   b0 = {W[16kc + 2t][8nt + g], W[16kc + 2t + 1][8nt + g]},  b1 = same rows + 8.
constexpr int kFragW1 = (kIn / 16) * (kH / 8) * 32, kFragW2 = (kH / 16) * (kH / 8) * 32,
              kFragW3 = (kH / 16) * (kOut / 8) * 32;

__device__ __forceinline__ uint2 b_frag(const float* W, int N, int kc, int nt, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int k0 = 16 * kc + 2 * t, n = 8 * nt + g;
    return make_uint2(pack_bf16(W[(k0)*N + n], W[(k0 + 1) * N + n]), pack_bf16(W[(k0 + 8) * N + n], W[(k0 + 9) * N + n]));
}

constexpr int kInferWarps = 8;
constexpr int kXPad = kIn + 8;  // bf16 row stride of the feature tile: 80 B, conflict-light fragment loads

// Output rows [r0, r0 + 16) of the warp's feature tile through the three layers;
// y[] receives rows r0 + g and r0 + g + 8, columns 2t, 2t + 1 (no bias).
__device__ __forceinline__ void mlp_tile(const __nv_bfloat16 (*xs)[kXPad], int r0, const uint2* f1, const uint2* f2,
                                         const uint2* f3, const float* bias, int lane, float (&y)[4]) {
    const int g = lane >> 2, t = lane & 3;
    float acc[kH / 8][4];
#pragma unroll
    for (int nt = 0; nt < kH / 8; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
#pragma unroll
    for (int kc = 0; kc < kIn / 16; ++kc) {
        unsigned a[4];
        a[0] = *reinterpret_cast<const unsigned*>(&xs[r0 + g][16 * kc + 2 * t]);
        a[1] = *reinterpret_cast<const unsigned*>(&xs[r0 + g + 8][16 * kc + 2 * t]);
        a[2] = *reinterpret_cast<const unsigned*>(&xs[r0 + g][16 * kc + 2 * t + 8]);
        a[3] = *reinterpret_cast<const unsigned*>(&xs[r0 + g + 8][16 * kc + 2 * t + 8]);
#pragma unroll
        for (int nt = 0; nt < kH / 8; ++nt) {
            const uint2 b = f1[(kc * (kH / 8) + nt) * 32 + lane];
            mma16816(acc[nt], a, b.x, b.y);
        }
    }
    // bias + SiLU; the C fragments of n-tiles (2j, 2j+1) are the A fragment of k-chunk j
    unsigned h[kH / 16][4];
#pragma unroll
    for (int j = 0; j < kH / 16; ++j) {
        const int c0 = 16 * j + 2 * t, c1 = c0 + 8;
        h[j][0] = silu_bf16x2(acc[2 * j][0] + bias[c0], acc[2 * j][1] + bias[c0 + 1]);
        h[j][1] = silu_bf16x2(acc[2 * j][2] + bias[c0], acc[2 * j][3] + bias[c0 + 1]);
        h[j][2] = silu_bf16x2(acc[2 * j + 1][0] + bias[c1], acc[2 * j + 1][1] + bias[c1 + 1]);
        h[j][3] = silu_bf16x2(acc[2 * j + 1][2] + bias[c1], acc[2 * j + 1][3] + bias[c1 + 1]);
    }
#pragma unroll
    for (int nt = 0; nt < kH / 8; ++nt)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[nt][q] = 0.f;
#pragma unroll
    for (int kc = 0; kc < kH / 16; ++kc)
#pragma unroll
        for (int nt = 0; nt < kH / 8; ++nt) {
            const uint2 b = f2[(kc * (kH / 8) + nt) * 32 + lane];
            mma16816(acc[nt], h[kc], b.x, b.y);
        }
#pragma unroll
    for (int j = 0; j < kH / 16; ++j) {
        const int c0 = 16 * j + 2 * t, c1 = c0 + 8;
        h[j][0] = silu_bf16x2(acc[2 * j][0] + bias[kH + c0], acc[2 * j][1] + bias[kH + c0 + 1]);
        h[j][1] = silu_bf16x2(acc[2 * j][2] + bias[kH + c0], acc[2 * j][3] + bias[kH + c0 + 1]);
        h[j][2] = silu_bf16x2(acc[2 * j + 1][0] + bias[kH + c1], acc[2 * j + 1][1] + bias[kH + c1 + 1]);
        h[j][3] = silu_bf16x2(acc[2 * j + 1][2] + bias[kH + c1], acc[2 * j + 1][3] + bias[kH + c1 + 1]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) y[q] = 0.f;
#pragma unroll
    for (int kc = 0; kc < kH / 16; ++kc) {
        const uint2 b = f3[kc * 32 + lane];
        mma16816(y, h[kc], b.x, b.y);
    }
}

// 32 particles per warp pass: every lane builds one particle's features, then
// the warp runs two 16-row tiles through the network on the tensor cores.
__global__ void __launch_bounds__(kInferWarps * 32) k_mlp_infer(const float* __restrict__ params,
                                                               const float4* __restrict__ pos,
                                                               const int* __restrict__ perm, int n,
                                                               const float* __restrict__ rho, int G, float inv_mean,
                                                               float out_scale, float4* __restrict__ out) {
    __shared__ uint2 f1[kFragW1], f2[kFragW2], f3[kFragW3];
    __shared__ float bias[kH + kH + kOut];
    __shared__ __nv_bfloat16 xs[kInferWarps][32][kXPad];
    __shared__ float ys[kInferWarps][32][4];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kFragW1; i += blockDim.x) {
        const int l = i & 31, nt = (i >> 5) % (kH / 8), kc = (i >> 5) / (kH / 8);
        f1[i] = b_frag(params + oW1, kH, kc, nt, l);
    }
    for (int i = threadIdx.x; i < kFragW2; i += blockDim.x) {
        const int l = i & 31, nt = (i >> 5) % (kH / 8), kc = (i >> 5) / (kH / 8);
        f2[i] = b_frag(params + oW2, kH, kc, nt, l);
    }
    for (int i = threadIdx.x; i < kFragW3; i += blockDim.x) {
        const int l = i & 31, kc = i >> 5;
        f3[i] = b_frag(params + oW3, kOut, kc, 0, l);
    }
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        bias[i] = params[oB1 + i];
        bias[kH + i] = params[oB2 + i];
    }
    if (threadIdx.x < kOut) bias[2 * kH + threadIdx.x] = params[oB3 + threadIdx.x];
    __syncthreads();

    const int g = lane >> 2, t = lane & 3;
    const int passes = (n + 31) / 32;
    for (int ps = blockIdx.x * kInferWarps + w; ps < passes; ps += gridDim.x * kInferWarps) {
        const int i = ps * 32 + lane;
        float4 p = make_float4(-1.f, -1.f, -1.f, 0.f);
        if (i < n) p = pos[perm ? perm[i] : i];
        {
            float f[32];
            if (p.x < 0.f) {
#pragma unroll
                for (int j = 0; j < 32; ++j) f[j] = 0.f;
            } else {
                particle_features(rho, G, inv_mean, p, f);
            }
#pragma unroll
            for (int j = 0; j < 32; j += 8)
                *reinterpret_cast<uint4*>(&xs[w][lane][j]) =
                    make_uint4(pack_bf16(f[j], f[j + 1]), pack_bf16(f[j + 2], f[j + 3]),
                               pack_bf16(f[j + 4], f[j + 5]), pack_bf16(f[j + 6], f[j + 7]));
        }
        __syncwarp();
#pragma unroll 1
        for (int half = 0; half < 2; ++half) {
            float y[4];
            mlp_tile(xs[w], 16 * half, f1, f2, f3, bias, lane, y);
            // y: rows g, g+8 of this half; cols 2t, 2t+1 (outputs 0..2 are meaningful)
            if (t < 2) {
                const int r = 16 * half + g;
                ys[w][r][2 * t] = y[0] + bias[2 * kH + 2 * t];
                ys[w][r][2 * t + 1] = y[1] + bias[2 * kH + 2 * t + 1];
                ys[w][r + 8][2 * t] = y[2] + bias[2 * kH + 2 * t];
                ys[w][r + 8][2 * t + 1] = y[3] + bias[2 * kH + 2 * t + 1];
            }
        }
        __syncwarp();
        if (i < n)
            out[i] = (p.x >= 0.f) ? make_float4(ys[w][lane][0] * out_scale, ys[w][lane][1] * out_scale,
                                                ys[w][lane][2] * out_scale, 0.f)
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncwarp();
    }
}

// ---- training: generic BF16 GEMM with FP32 accumulation ------------------------------
// C_part[split][m][n] = sum_{k in split} opA[m][k] * opB[k][n]
//   opA[m][k] = TA ? A[k*lda + m] : A[m*lda + k],  opB[k][n] = TB ? B[n*ldb + k] : B[k*ldb + n]
// One warp per 16x8 output tile; M a multiple of 16, N a multiple of 8; K is
// arbitrary (products past K, or past the split's end, read as zero).
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm(const __nv_bfloat16* __restrict__ A, int lda,
                                              const __nv_bfloat16* __restrict__ B, int ldb, float* __restrict__ C,
                                              int M, int N, int K, int ksplit) {
    const int lane = threadIdx.x & 31;
    const int tile = blockIdx.x * 4 + (threadIdx.x >> 5);
    const int tn = N / 8, tiles = (M / 16) * tn;
    if (tile >= tiles) return;
    const int m0 = (tile / tn) * 16, n0 = (tile % tn) * 8;
    const int split = blockIdx.y;
    const int kbeg = split * ksplit, kend = min(K, kbeg + ksplit);
    const int g = lane >> 2, t = lane & 3;
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    auto a_at = [&](int m, int k) -> __nv_bfloat16 {
        if (k >= kend) return zero;
        return TA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k];
    };
    auto b_at = [&](int k, int nn) -> __nv_bfloat16 {
        if (k >= kend) return zero;
        return TB ? B[(size_t)nn * ldb + k] : B[(size_t)k * ldb + nn];
    };
    auto pk = [](__nv_bfloat16 lo, __nv_bfloat16 hi) {
        return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
    };
    float acc[4] = {0.f, 0.f, 0.f, 0.f};
    for (int k0 = kbeg; k0 < kend; k0 += 16) {
        unsigned a[4];
        a[0] = pk(a_at(m0 + g, k0 + 2 * t), a_at(m0 + g, k0 + 2 * t + 1));
        a[1] = pk(a_at(m0 + g + 8, k0 + 2 * t), a_at(m0 + g + 8, k0 + 2 * t + 1));
        a[2] = pk(a_at(m0 + g, k0 + 2 * t + 8), a_at(m0 + g, k0 + 2 * t + 9));
        a[3] = pk(a_at(m0 + g + 8, k0 + 2 * t + 8), a_at(m0 + g + 8, k0 + 2 * t + 9));
        const unsigned b0 = pk(b_at(k0 + 2 * t, n0 + g), b_at(k0 + 2 * t + 1, n0 + g));
        const unsigned b1 = pk(b_at(k0 + 2 * t + 8, n0 + g), b_at(k0 + 2 * t + 9, n0 + g));
        mma16816(acc, a, b0, b1);
    }
    float* c = C + (size_t)split * M * N;
    c[(size_t)(m0 + g) * N + n0 + 2 * t] = acc[0];
    c[(size_t)(m0 + g) * N + n0 + 2 * t + 1] = acc[1];
    c[(size_t)(m0 + g + 8) * N + n0 + 2 * t] = acc[2];
    c[(size_t)(m0 + g + 8) * N + n0 + 2 * t + 1] = acc[3];
}

// sum the split partials in fixed order: out[i] = sum_s part[s][i]
__global__ void k_sum_splits(const float* __restrict__ part, int splits, size_t count, float* __restrict__ out) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float s = 0.f;
    for (int p = 0; p < splits; ++p) s += part[(size_t)p * count + i];
    out[i] = s;
}

// Z = acc + bias (FP32, kept for the backward pass); H = bf16(SiLU(Z)).
__global__ void k_bias_silu(const float* __restrict__ acc, const float* __restrict__ bias, int rows, int cols,
                            float* __restrict__ z, __nv_bfloat16* __restrict__ h) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)rows * cols) return;
    const float v = acc[i] + bias[i % cols];
    z[i] = v;
    h[i] = __float2bfloat16_rn(silu(v));
}

// Output layer: Y = acc + b3; dY = 2 (Y - T) / (3 rows) on the 3 real outputs
// (bf16 for the products), squared error per row into err[row].
__global__ void k_out_grad(const float* __restrict__ acc, const float* __restrict__ b3, const float* __restrict__ tgt,
                           int rows, __nv_bfloat16* __restrict__ dy, float* __restrict__ err) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    float e = 0.f;
    for (int c = 0; c < kOut; ++c) {
        float d = 0.f;
        if (c < 3) {
            const float y = acc[(size_t)r * kOut + c] + b3[c];
            const float diff = y - tgt[(size_t)r * 3 + c];
            e += diff * diff;
            d = 2.f * diff / (3.f * (float)rows);
        }
        dy[(size_t)r * kOut + c] = __float2bfloat16_rn(d);
    }
    err[r] = e;
}

// dZ = bf16(dH * SiLU'(Z))
__global__ void k_silu_back(const float* __restrict__ dh, const float* __restrict__ z, size_t count,
                            __nv_bfloat16* __restrict__ dz) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    dz[i] = __float2bfloat16_rn(dh[i] * silu_grad(z[i]));
}

// column sums of a bf16 [rows][cols] matrix, one block per column, fixed order
__global__ void __launch_bounds__(256) k_colsum(const __nv_bfloat16* __restrict__ a, int rows, int cols,
                                                float* __restrict__ out) {
    __shared__ float red[256];
    float s = 0.f;
    for (int r = threadIdx.x; r < rows; r += 256) s += __bfloat162float(a[(size_t)r * cols + blockIdx.x]);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

__global__ void k_sum_f32(const float* __restrict__ a, int n, float* __restrict__ out) {
    __shared__ float red[256];
    float s = 0.f;
    for (int i = threadIdx.x; i < n; i += 256) s += a[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

__global__ void k_to_bf16(const float* __restrict__ a, int n, __nv_bfloat16* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2bfloat16_rn(a[i]);
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ grad, int n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.f - b1) * g;
    const float vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

}  // namespace

size_t mlp_param_count() { return kParams; }

int launch_mlp_infer(const float* params, const float4* pos, const int* perm, int n, const float* rho, int G,
                     float inv_mean, float out_scale, float4* out, cudaStream_t s) {
    if (n <= 0) return SD_OK;
    const int passes = (n + 31) / 32;
    int blocks = (passes + kInferWarps - 1) / kInferWarps;
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_mlp_infer<<<blocks, kInferWarps * 32, 0, s>>>(params, pos, perm, n, rho, G, inv_mean, out_scale, out);
    SD_LAUNCHED(s);
    return SD_OK;
}

// Workspace of one training batch of `rows` samples (rows a multiple of 16).
static size_t mlp_train_ws(int rows, int splits) {
    const size_t r = (size_t)rows;
    size_t b = 0;
    b += align_up(r * kH * 4, 256) * 4;         // z1, z2, dh (fp32) + acc scratch
    b += align_up(r * kH * 2, 256) * 4;         // h1, h2, dz2, dz1 (bf16)
    b += align_up(r * kOut * 4, 256);           // y acc
    b += align_up(r * kOut * 2, 256);           // dy (bf16)
    b += align_up(r * 4, 256);                  // per-row error
    b += align_up((size_t)kParams * 2, 256);    // bf16 weights
    b += align_up((size_t)splits * kH * kH * 4, 256);  // split partials of weight grads
    b += 256;
    return b;
}

}  // namespace sd

using namespace sd;

extern "C" {

int sd_mlp_param_count(void) { return kParams; }

int sd_mlp_features(const float* pos, const int32_t* perm, int n, const float* rho, int G, float inv_mean,
                    void* features_bf16, void* stream) {
    if (!pos || !rho || !features_bf16 || n < 0 || G < 16 || (G & (G - 1)))
        return fail(SD_E_ARG, "mlp_features: bad arguments");
    if (n == 0) return SD_OK;
    cudaStream_t st = (cudaStream_t)stream;
    k_features<<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float4*>(pos), perm, n, rho, G, inv_mean,
                                                 reinterpret_cast<__nv_bfloat16*>(features_bf16));
    SD_LAUNCHED(st);
    return SD_OK;
}

int sd_mlp_infer(const float* params, const float* pos, const int32_t* perm, int n, const float* rho, int G,
                 float inv_mean, float out_scale, float* out, void* stream) {
    if (!params || !pos || !rho || !out || n < 0 || G < 16 || (G & (G - 1)))
        return fail(SD_E_ARG, "mlp_infer: bad arguments");
    return launch_mlp_infer(params, reinterpret_cast<const float4*>(pos), perm, n, rho, G, inv_mean, out_scale,
                            reinterpret_cast<float4*>(out), (cudaStream_t)stream);
}

// split-K slices of the weight-gradient products (K = rows): one per 1024 rows
static int mlp_splits(int rows) { return (rows + 1023) / 1024; }

size_t sd_mlp_train_workspace_bytes(int rows) {
    const int splits = mlp_splits(rows);
    return mlp_train_ws(rows, splits);
}

// Loss and gradients of one batch: features X (bf16 [rows][32]), targets T
// (fp32 [rows][3]) -> grad (fp32 [kParams]) of the mean squared error over rows
// and the 3 components, and *sse = the sum of squared errors (device float).
// rows must be a multiple of 16.
int sd_mlp_loss_grad(const float* params, const void* features_bf16, const float* targets, int rows, float* grad,
                     float* sse, void* ws, size_t ws_bytes, void* stream) {
    if (!params || !features_bf16 || !targets || !grad || !sse || !ws || rows <= 0 || rows % 16)
        return fail(SD_E_ARG, "mlp_loss_grad: bad arguments (rows must be a positive multiple of 16)");
    const int splits = mlp_splits(rows);
    if (ws_bytes < mlp_train_ws(rows, splits)) return fail(SD_E_ARG, "mlp_loss_grad: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const size_t r = (size_t)rows;
    char* p = (char*)ws;
    auto take = [&](size_t bytes) {
        char* q = p;
        p += align_up(bytes, 256);
        return q;
    };
    float* z1 = (float*)take(r * kH * 4);
    float* z2 = (float*)take(r * kH * 4);
    float* dh = (float*)take(r * kH * 4);
    float* accb = (float*)take(r * kH * 4);
    __nv_bfloat16* h1 = (__nv_bfloat16*)take(r * kH * 2);
    __nv_bfloat16* h2 = (__nv_bfloat16*)take(r * kH * 2);
    __nv_bfloat16* dz2 = (__nv_bfloat16*)take(r * kH * 2);
    __nv_bfloat16* dz1 = (__nv_bfloat16*)take(r * kH * 2);
    float* yacc = (float*)take(r * kOut * 4);
    __nv_bfloat16* dy = (__nv_bfloat16*)take(r * kOut * 2);
    float* err = (float*)take(r * 4);
    __nv_bfloat16* wb = (__nv_bfloat16*)take((size_t)kParams * 2);
    float* part = (float*)take((size_t)splits * kH * kH * 4);
    const __nv_bfloat16* X = (const __nv_bfloat16*)features_bf16;

    auto blocks = [](size_t count) { return (unsigned)((count + 255) / 256); };
    k_to_bf16<<<blocks(kParams), 256, 0, st>>>(params, kParams, wb);
    SD_LAUNCHED(st);
    const __nv_bfloat16 *W1 = wb + oW1, *W2 = wb + oW2, *W3 = wb + oW3;
    // gemm helper: C[M][N] = opA * opB over K (split-K into `sp` slices, summed in fixed order)
    auto gemm = [&](bool ta, bool tb, const __nv_bfloat16* A, int lda, const __nv_bfloat16* B, int ldb, float* C,
                    int M, int N, int K) -> int {
        const int tiles = (M / 16) * (N / 8);
        const int sp = (K >= 2048) ? splits : 1;
        const int ks = ((K / sp + 15) / 16) * 16;
        dim3 grid((tiles + 3) / 4, sp);
        float* dst = (sp == 1) ? C : part;
        if (ta && tb) k_gemm<true, true><<<grid, 128, 0, st>>>(A, lda, B, ldb, dst, M, N, K, ks);
        else if (ta) k_gemm<true, false><<<grid, 128, 0, st>>>(A, lda, B, ldb, dst, M, N, K, ks);
        else if (tb) k_gemm<false, true><<<grid, 128, 0, st>>>(A, lda, B, ldb, dst, M, N, K, ks);
        else k_gemm<false, false><<<grid, 128, 0, st>>>(A, lda, B, ldb, dst, M, N, K, ks);
        SD_LAUNCHED(st);
        if (sp > 1) {
            k_sum_splits<<<blocks((size_t)M * N), 256, 0, st>>>(part, sp, (size_t)M * N, C);
            SD_LAUNCHED(st);
        }
        return SD_OK;
    };
    int rc;
    // forward
    if ((rc = gemm(false, false, X, kIn, W1, kH, accb, rows, kH, kIn))) return rc;
    k_bias_silu<<<blocks(r * kH), 256, 0, st>>>(accb, params + oB1, rows, kH, z1, h1);
    SD_LAUNCHED(st);
    if ((rc = gemm(false, false, h1, kH, W2, kH, accb, rows, kH, kH))) return rc;
    k_bias_silu<<<blocks(r * kH), 256, 0, st>>>(accb, params + oB2, rows, kH, z2, h2);
    SD_LAUNCHED(st);
    if ((rc = gemm(false, false, h2, kH, W3, kOut, yacc, rows, kOut, kH))) return rc;
    k_out_grad<<<blocks(r), 256, 0, st>>>(yacc, params + oB3, targets, rows, dy, err);
    SD_LAUNCHED(st);
    k_sum_f32<<<1, 256, 0, st>>>(err, rows, sse);
    SD_LAUNCHED(st);
    // backward: layer 3
    if ((rc = gemm(true, false, h2, kH, dy, kOut, grad + oW3, kH, kOut, rows))) return rc;
    k_colsum<<<kOut, 256, 0, st>>>(dy, rows, kOut, grad + oB3);
    SD_LAUNCHED(st);
    if ((rc = gemm(false, true, dy, kOut, W3, kOut, dh, rows, kH, kOut))) return rc;
    k_silu_back<<<blocks(r * kH), 256, 0, st>>>(dh, z2, r * kH, dz2);
    SD_LAUNCHED(st);
    // layer 2
    if ((rc = gemm(true, false, h1, kH, dz2, kH, grad + oW2, kH, kH, rows))) return rc;
    k_colsum<<<kH, 256, 0, st>>>(dz2, rows, kH, grad + oB2);
    SD_LAUNCHED(st);
    if ((rc = gemm(false, true, dz2, kH, W2, kH, dh, rows, kH, kH))) return rc;
    k_silu_back<<<blocks(r * kH), 256, 0, st>>>(dh, z1, r * kH, dz1);
    SD_LAUNCHED(st);
    // layer 1
    if ((rc = gemm(true, false, X, kIn, dz1, kH, grad + oW1, kIn, kH, rows))) return rc;
    k_colsum<<<kH, 256, 0, st>>>(dz1, rows, kH, grad + oB1);
    SD_LAUNCHED(st);
    return SD_OK;
}

int sd_mlp_adam(float* params, float* m, float* v, const float* grad, int step, float lr, float beta1, float beta2,
                float eps, void* stream) {
    if (!params || !m || !v || !grad || step < 1) return fail(SD_E_ARG, "mlp_adam: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const float c1 = 1.f / (1.f - powf(beta1, (float)step)), c2 = 1.f / (1.f - powf(beta2, (float)step));
    k_adam<<<(kParams + 255) / 256, 256, 0, st>>>(params, m, v, grad, kParams, lr, beta1, beta2, eps, c1, c2);
    SD_LAUNCHED(st);
    return SD_OK;
}

}  // extern "C"
