// sd_mlp.cu -- learned sub-grid force correction: features, BF16 tensor-core
// MLP (30 -> 64 -> 64 -> 3, SiLU), its training kernels and the fused inference
// that feeds the kick. No counterpart in the reference; the correction is added
// on top of the plain PM acceleration (kIntegrate's accG sample, Sim.cu:822).
//
// Numerics: weights and activations are BF16, every matrix product accumulates
// in FP32 on the tensor cores (the inference with tcgen05.mma into tensor memory,
// the training's GEMMs with mma.sync m16n8k16), biases and the SiLU are FP32,
// master weights and Adam moments are FP32.
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

__device__ __forceinline__ float silu(float z) { return z * sigmoid(z); }
__device__ __forceinline__ float silu_grad(float z) {
    const float s = sigmoid(z);
    return s * fmaf(z, 1.f - s, 1.f);
}

// ---- features -------------------------------------------------------------------
// the density feature of one cell: log(1 + rho / rho_bar) - log 2
__device__ __forceinline__ float cell_feature(float r, float inv_mean) {
    return __logf(1.f + r * inv_mean) - 0.69314718055994531f;
}

__device__ __forceinline__ void particle_features(const float* __restrict__ rho, int G, float inv_mean, float4 p,
                                                  float* f) {
    const int m = G - 1;
    const int cx = min(max((int)(p.x * (float)G), 0), m);
    const int cy = min(max((int)(p.y * (float)G), 0), m);
    const int cz = min(max((int)(p.z * (float)G), 0), m);
#pragma unroll
    for (int dz = -1; dz <= 1; ++dz)
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const float r =
                    __ldg(rho + ((size_t)((cz + dz) & m) * G + ((cy + dy) & m)) * G + ((cx + dx) & m));
                f[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] = cell_feature(r, inv_mean);
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

// ---- fused inference on the 5th-generation tensor cores (tcgen05) -------------------
// One CTA of 128 threads takes tiles of 128 particles, thread r <-> row r of the
// tile <-> tensor-memory lane r. Each layer is one tcgen05.mma chain (M = 128,
// N = 64 or 16, K in steps of 16, BF16 x BF16 -> FP32) issued by thread 0: the
// activations (operand A) sit in tensor memory, the weights (operand B) in
// shared memory, the FP32 accumulator in 64 tensor-memory columns. Completion
// arrives on an mbarrier (tcgen05.commit); every thread reads its row back with
// tcgen05.ld, adds the bias, applies the SiLU and writes its row of the next
// layer's A with tcgen05.st -- no shared-memory round trip for the activations.
//
// A: row r in lane r, element k in column kAcol + k / 2 (two BF16 per 32-bit
// column, k even in the low half); k-step s reads columns kAcol + 8 s.
// B: the canonical K-major layout without swizzle, 8 x 16-byte core matrices
// (8 rows x 8 BF16): element (row n, k) of a matrix with K columns at byte
// (n / 8) * SBO + (k / 8) * 128 + (n % 8) * 16 + (k % 8) * 2, SBO = K * 16; the
// descriptor of k-step s starts 256 s bytes in (leading offset 128 bytes: the two
// 8-column halves of the step).
//
// Measured against the mma.sync kernel it replaced (2,097,152 particles on 128^3,
// identical outputs): 0.165 against 0.153 ms. The tensor pipe is 8 % busy; the
// kernel waits on the feature gathers from L2 and on the SiLU's dependent chains
// at four CTAs per SM (the tensor-memory columns), not on the products.
namespace tc {
constexpr int kThreads = 128;                  // one warpgroup: TMEM lanes 0..127
constexpr int kTmemCols = 128;                 // FP32 accumulator (columns 0..63) + BF16 operand A (64..95)
constexpr int kAcol = 64;                      // A: row r in lane r, BF16 pairs along K in consecutive columns
constexpr int kN3 = 16;                        // output layer N (3 outputs padded)
constexpr int kB1 = 0;                         // W1^T [64][32]
constexpr int kB2 = kB1 + kH * kIn * 2;        // W2^T [64][64]
constexpr int kB3 = kB2 + kH * kH * 2;         // W3^T [16][64] (rows 8..15 zero)
constexpr int kBias = kB3 + kN3 * kH * 2;      // b1[64], b2[64], b3[8] (float)
constexpr int kBar = kBias + (2 * kH + kOut) * 4 + 8;  // mbarrier (8-byte aligned)
constexpr int kTaddr = kBar + 8;
constexpr int kSmem = kTaddr + 8;
constexpr int kSmemLaunch = 46 * 1024;  // at most four CTAs per SM (see launch_mlp_infer)
static_assert(kBar % 8 == 0 && kB2 % 16 == 0 && kB3 % 16 == 0, "alignment");

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// byte offset of element (r, k) in a K-major shared-memory operand with K columns
__device__ __forceinline__ int op_off(int r, int k, int K) { return (r >> 3) * (K * 16) + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2; }

__device__ __forceinline__ uint64_t desc(uint32_t addr, int K) {
    const uint64_t lbo = 128 >> 4, sbo = (uint64_t)(K * 16) >> 4;
    return (uint64_t)((addr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);  // version 1, no swizzle
}

// instruction descriptor: BF16 x BF16 -> FP32, both K-major, M = 128
__host__ __device__ constexpr uint32_t idesc(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// A from tensor memory (the activations), B from shared memory (the weights)
__device__ __forceinline__ void mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b), "r"(id), "r"(acc));
}

// 16 32-bit words into columns [col, col + 16) of this thread's TMEM lane
__device__ __forceinline__ void st16(uint32_t taddr, const unsigned (&w)[16]) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(
            taddr),
        "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(w[8]), "r"(w[9]),
        "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]), "r"(w[14]), "r"(w[15])
        : "memory");
}
__device__ __forceinline__ void wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Bounded wait for phase `parity` of the mbarrier; false if it gave up.
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity) {
    for (int it = 0; it < (1 << 22); ++it) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred q;\n\tmbarrier.try_wait.parity.shared::cta.b64 q, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, q;\n\t}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// FP32 columns [col, col + 16 X) of this thread's TMEM lane: X loads of 16 columns
// in flight together, one wait
__device__ __forceinline__ void ld16_issue(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
template <int X>
__device__ __forceinline__ void ld_cols(uint32_t taddr, float (&v)[16 * X]) {
    uint32_t r[X][16];
#pragma unroll
    for (int x = 0; x < X; ++x) ld16_issue(taddr + 16 * x, r[x]);
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int x = 0; x < X; ++x)
#pragma unroll
        for (int q = 0; q < 16; ++q) v[16 * x + q] = __uint_as_float(r[x][q]);
}
}  // namespace tc

// Waits that gave up (an mbarrier phase that never completed): the tile's outputs
// are NaN and the count is readable through sd_mlp_wait_timeouts.
__device__ unsigned g_mlp_wait_timeouts = 0;

// The two hidden layers run on weights and biases scaled by 1/2 (exact in BF16 and
// FP32), so each accumulator holds u = z / 2 and SiLU(z) = z sigmoid(z) =
// u + u tanh(u): one tanh and one FMA per unit, rounded to BF16 once.
__global__ void __launch_bounds__(tc::kThreads, 4) k_mlp_infer_tc(const float* __restrict__ params,
                                                              const float4* __restrict__ pos,
                                                              const int* __restrict__ perm, int n,
                                                              const float* __restrict__ rho, int G,
                                                              float inv_mean, float out_scale,
                                                              float4* __restrict__ out) {
    extern __shared__ __align__(1024) unsigned char sm[];
    const int r = threadIdx.x, warp = r >> 5;
    float* bias = reinterpret_cast<float*>(sm + tc::kBias);
    const uint32_t bar = tc::smem_u32(sm + tc::kBar);
    uint32_t* taddr_s = reinterpret_cast<uint32_t*>(sm + tc::kTaddr);
    // weights as K-major operands (W[k][n] -> row n, column k), the same BF16 rounding
    // as the training's copies
    for (int e = r; e < kH * kIn; e += tc::kThreads) {
        const int nn = e / kIn, k = e % kIn;
        *reinterpret_cast<__nv_bfloat16*>(sm + tc::kB1 + tc::op_off(nn, k, kIn)) =
            __float2bfloat16_rn(0.5f * params[oW1 + k * kH + nn]);
    }
    for (int e = r; e < kH * kH; e += tc::kThreads) {
        const int nn = e / kH, k = e % kH;
        *reinterpret_cast<__nv_bfloat16*>(sm + tc::kB2 + tc::op_off(nn, k, kH)) =
            __float2bfloat16_rn(0.5f * params[oW2 + k * kH + nn]);
    }
    for (int e = r; e < tc::kN3 * kH; e += tc::kThreads) {
        const int nn = e / kH, k = e % kH;
        *reinterpret_cast<__nv_bfloat16*>(sm + tc::kB3 + tc::op_off(nn, k, kH)) =
            __float2bfloat16_rn(nn < kOut ? params[oW3 + k * kOut + nn] : 0.f);
    }
    for (int e = r; e < kH; e += tc::kThreads) {
        bias[e] = 0.5f * params[oB1 + e];
        bias[kH + e] = 0.5f * params[oB2 + e];
    }
    if (r < kOut) bias[2 * kH + r] = params[oB3 + r];
    if (r == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc::smem_u32(taddr_s)),
                     "r"(tc::kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc::fence_proxy();  // the weights, written by the threads, are read by the tensor cores
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tmem = *taddr_s;
    const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);  // this warp's 32 lanes
    const uint32_t a_lane = lane_addr + tc::kAcol;  // this thread's row of the operand A
    const uint32_t b1 = tc::smem_u32(sm + tc::kB1), b2 = tc::smem_u32(sm + tc::kB2),
                   b3 = tc::smem_u32(sm + tc::kB3);
    uint32_t phase = 0;
    bool ok = true;
    const int tiles = (n + tc::kThreads - 1) / tc::kThreads;
    // this thread's particle of the CTA's next tile, loaded while the current tile
    // runs through the network
    float4 pn = make_float4(-1.f, -1.f, -1.f, 0.f);
    if (blockIdx.x * tc::kThreads + r < n) {
        const int i0 = blockIdx.x * tc::kThreads + r;
        pn = pos[perm ? perm[i0] : i0];
    }
    for (int t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
        const int i = t * tc::kThreads + r;
        const float4 p = pn;
        {
            const int inx = i + gridDim.x * tc::kThreads;
            pn = make_float4(-1.f, -1.f, -1.f, 0.f);
            if (inx < n) pn = pos[perm ? perm[inx] : inx];
        }
        {
            unsigned w[16];
            if (p.x < 0.f) {
#pragma unroll
                for (int j = 0; j < 16; ++j) w[j] = 0u;
            } else {
                float f[32];
                particle_features(rho, G, inv_mean, p, f);
#pragma unroll
                for (int j = 0; j < 16; ++j) w[j] = pack_bf16(f[2 * j], f[2 * j + 1]);
            }
            tc::st16(a_lane, w);
            tc::wait_st();
        }
        // three layers; layer l reads A (K = 32 for the first, 64 after) and B_l
#pragma unroll 1
        for (int layer = 0; layer < 3; ++layer) {
            const int K = layer == 0 ? kIn : kH;
            tc::fence_before();  // this thread's operand row (tcgen05.st, waited) before the MMA
            __syncthreads();
            if (r == 0) {
                tc::fence_after();
                const uint32_t bb = layer == 0 ? b1 : (layer == 1 ? b2 : b3);
                const uint32_t id = tc::idesc(layer == 2 ? tc::kN3 : kH);
                // k-step s: A columns kAcol + 8 s (16 BF16 per row), B rows from byte 256 s
                for (int s = 0; s < K / 16; ++s)
                    tc::mma_ts(tmem, tmem + tc::kAcol + 8 * s, tc::desc(bb + 256 * s, K), id, s > 0);
                tc::commit(bar);
            }
            // every thread waits; the verdict is made uniform so the CTA's barriers stay matched
            if (!__syncthreads_and(tc::wait_bar(bar, phase))) {
                ok = false;
                if (r == 0) atomicAdd(&g_mlp_wait_timeouts, 1u);
                break;
            }
            phase ^= 1;
            tc::fence_after();
            if (layer < 2) {
                // this row's 64 pre-activations -> SiLU -> the next layer's operand row
                // (the MMA that read A has completed)
#pragma unroll
                for (int c2 = 0; c2 < kH / 32; ++c2) {
                    float v[32];
                    tc::ld_cols<2>(lane_addr + 32 * c2, v);
                    const float* b = bias + layer * kH + 32 * c2;
                    unsigned h[16];
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const float u0 = v[2 * q] + b[2 * q], u1 = v[2 * q + 1] + b[2 * q + 1];
                        h[q] = pack_bf16(fmaf(u0, tanh_approx(u0), u0), fmaf(u1, tanh_approx(u1), u1));
                    }
                    tc::st16(a_lane + 16 * c2, h);  // units 32 c2 .. 32 c2 + 31
                }
                tc::wait_st();
            } else {
                float v[16];
                tc::ld_cols<1>(lane_addr, v);
                const float* b = bias + 2 * kH;
                if (i < n)
                    out[i] = (p.x >= 0.f) ? make_float4((v[0] + b[0]) * out_scale, (v[1] + b[1]) * out_scale,
                                                        (v[2] + b[2]) * out_scale, 0.f)
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        if (!ok && i < n) out[i] = make_float4(__int_as_float(0x7fc00000), __int_as_float(0x7fc00000),
                                               __int_as_float(0x7fc00000), 0.f);
    }
    // every tcgen05.ld has completed (wait::ld) and no MMA is in flight once the
    // last wait returned; a CTA whose wait gave up drains with a second bounded wait
    if (!ok && r == 0) tc::wait_bar(bar, phase);
    tc::fence_before();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tc::kTmemCols)
                     : "memory");
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
    // tiles of 128 particles; four CTAs fill an SM's 512 tensor-memory columns (128 each).
    // The dynamic shared memory is padded so that no fifth CTA is placed on an SM, where
    // its tcgen05.alloc would wait for one of the four to finish.
    static_assert(tc::kSmemLaunch >= tc::kSmem && 5 * (tc::kSmemLaunch + 1024) > 228 * 1024, "four CTAs per SM");
    const int tiles = (n + tc::kThreads - 1) / tc::kThreads;
    const int blocks = tiles < 148 * 4 ? tiles : 148 * 4;
    k_mlp_infer_tc<<<blocks, tc::kThreads, tc::kSmemLaunch, s>>>(params, pos, perm, n, rho, G, inv_mean, out_scale,
                                                                 out);
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

int sd_mlp_wait_timeouts(void) {
    unsigned v = 0;
    if (SD_CUDA(cudaMemcpyFromSymbol(&v, g_mlp_wait_timeouts, sizeof(v)))) return SD_E_CUDA;
    return (int)v;
}

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
