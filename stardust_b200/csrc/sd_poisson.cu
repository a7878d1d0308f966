// sd_poisson.cu -- periodic Poisson solve rho -> phi, all passes hand-written
// (the reference calls cuFFT R2C, kPoissonPeriodic, cuFFT C2R: Sim.cu:3586-3603,
// 528-557).
//
// Spectrum layout: one buffer of 4x4x4 complex "bricks" (512 B each). The kx
// axis holds the H+1 = G/2+1 bins of the real transform padded to H+4 (the last
// brick carries the Nyquist bin and three zero columns). Brick (bx,by,bz) starts
// at (((bz*NBY + by)*NBX + bx) * 64); inside a brick element (kx_l, y_l, z_l)
// sits at z_l*16 + y_l*4 + kx_l.
//
// Passes (CTA = one 4x4 bundle of 16 lines, held interleaved in shared memory):
//   A  x-rows real -> complex (input: float grid or int64 fixed-point grid)
//   B  y-lines forward            (in place)
//   C  z-lines forward, Green's function, z-lines inverse (in place)
//   D  y-lines inverse            (in place)
//   E  x-rows complex -> real, write phi
// Every global access moves whole 512-byte bricks or whole rows, B/C/D stage
// their bricks with cp.async, and each pass reads and writes every element once.
#include <cuda.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>
#include <vector>

#include "sd_common.cuh"
#include "sd_fft.cuh"
#include "sd_internal.h"

namespace sd {

namespace {

constexpr int kFftThreads = 256;
constexpr int kDepositThreads = 512;

template <int G>
struct Geo {
    static constexpr int H = G / 2;
    static constexpr int NBX = H / 4 + 1;  // kx bricks (last: Nyquist + padding)
    static constexpr int PX = 4 * NBX;     // padded kx positions = H + 4
    static constexpr int NBY = G / 4;
    static constexpr int NBZ = G / 4;
    __device__ __forceinline__ static size_t brick(int bx, int by, int bz) {
        return ((((size_t)bz * NBY + by) * NBX) + bx) * 64;
    }
};

// ---- pass A's x transform at G = 512: one warp per line ---------------------------
// A row of 512 reals is packed as 256 complex z[m] = x[2m] + i x[2m+1]; lane t
// holds z[t + 32k], k = 0..7. The 256-point transform is factored 8 x 32
// (m = t + 32k, f = f1 + 8 f2): a radix-8 DFT over k in registers and the twiddle
// W256^(t f1); then the 32-point DFTs over t, factored 8 x 4 (t = j + 4i,
// f2 = g1 + 8 g2) after a transpose through the warp's own shared scratch: lane
// (f1, j) takes a radix-8 DFT over i and the twiddle W32^(j g1); a second
// transpose hands lane L the output groups gA = L and gB = 64 - L (lane 0: 0 and
// 32), each finished by a radix-4 DFT over j into Z[g + 64 g2]. Both members of
// every pair (k, H - k) of the real-to-complex unpacking then sit in one lane.
// The bins go to a brick-ordered staging buffer, from which the CTA stores whole
// 512-byte bricks (a warp storing its own line would touch 65 bricks per line).
// Only __syncwarp orders the scratch; XOR swizzles keep every 8-byte access of the
// scratch and the staging buffer at two wavefronts.
namespace xl {
constexpr int kTw2 = 3 * 32 + 3 * 4;   // float2 entries of the two twiddle tables
constexpr int kStage = 16 * 4 * 65;     // float2: 65 bricks of 16 lines x 4 bins

// Twiddle tables, lane-contiguous so every load is conflict-free: tw[p*32 + t] =
// W256^(t 2^p) and then tw[96 + p*4 + j] = W32^(j 2^p), p = 0..2, copied from the
// table tw_g[m] = W512^m. Other powers are products of at most two of these.
__device__ __forceinline__ void fill_twiddles(float2* tw2, const float2* __restrict__ tw_g) {
    for (int e = threadIdx.x; e < kTw2; e += blockDim.x)
        tw2[e] = e < 96 ? tw_g[(2 * (e & 31)) << (e >> 5)] : tw_g[(16 * ((e - 96) & 3)) << ((e - 96) >> 2)];
}

// v[q] *= w^q for q = 1..7, given w, w^2, w^4
__device__ __forceinline__ void twiddle8(float2 (&v)[8], float2 w1, float2 w2, float2 w4) {
    const float2 w3 = fft::cmul(w1, w2);
    v[1] = fft::cmul(v[1], w1);
    v[2] = fft::cmul(v[2], w2);
    v[3] = fft::cmul(v[3], w3);
    v[4] = fft::cmul(v[4], w4);
    v[5] = fft::cmul(v[5], fft::cmul(w1, w4));
    v[6] = fft::cmul(v[6], fft::cmul(w2, w4));
    v[7] = fft::cmul(v[7], fft::cmul(w3, w4));
}

// Staging position of bin kx of line l = z_l*4 + y_l: brick kx/4, element
// z_l*16 + y_l*4 + kx%4 (the spectrum's brick layout), bits 2-3 of the element
// XORed with the brick's low bits. 16-byte pairs (kx even, kx + 1) stay adjacent.
__device__ __forceinline__ int stage_pos(int kx, int l) {
    const int b = kx >> 2;
    return b * 64 + ((((l >> 2) << 4) + ((l & 3) << 2) + (kx & 3)) ^ ((b & 3) << 2));
}

// One pair of the unpacking: from Z[k] and Z[H-k], X[k] = E + W512^k O and
// X[H-k] = conj E + W512^(H-k) conj O with E = (Z[k] + conj Z[H-k]) / 2,
// O = (Z[k] - conj Z[H-k]) / (2i); W512^(H-k) = -conj W512^k.
__device__ __forceinline__ void unpack_pair(float2 zk, float2 zc, int k, const float2* tw, float2* st, int l) {
    constexpr int H = 256;
    const float er = 0.5f * (zk.x + zc.x), ei = 0.5f * (zk.y - zc.y);
    const float orr = 0.5f * (zk.y + zc.y), oi = -0.5f * (zk.x - zc.x);
    const float2 w = tw[k];
    st[stage_pos(k, l)] = make_float2(er + (w.x * orr - w.y * oi), ei + (w.x * oi + w.y * orr));
    if (2 * k != H)
        st[stage_pos(H - k, l)] = make_float2(er + (w.y * oi - w.x * orr), -ei + (w.y * orr + w.x * oi));
}

// z: this lane's inputs z[t + 32k] (destroyed); sc: the warp's 256-float2 scratch,
// free on entry and on return; tw: W512^m in shared memory; st: the staging
// buffer, which receives bins 0..259 of line l (257..259 zero).
__device__ __forceinline__ void r2c512(float2 (&z)[8], float2* sc, const float2* tw, const float2* tw2, float2* st,
                                       int l) {
    const int lane = threadIdx.x & 31;
    fft::dft<8, false>(z);
    twiddle8(z, tw2[lane], tw2[32 + lane], tw2[64 + lane]);  // W256^(t f1)
    __syncwarp();
#pragma unroll
    for (int f1 = 0; f1 < 8; ++f1) sc[f1 * 32 + (lane ^ (4 * (f1 & 3)))] = z[f1];
    __syncwarp();
    const int f1 = lane >> 2, j = lane & 3;
#pragma unroll
    for (int i = 0; i < 8; ++i) z[i] = sc[f1 * 32 + ((j + 4 * i) ^ (4 * (f1 & 3)))];
    fft::dft<8, false>(z);
    twiddle8(z, tw2[96 + j], tw2[100 + j], tw2[104 + j]);  // W32^(j g1)
    __syncwarp();
#pragma unroll
    for (int g1 = 0; g1 < 8; ++g1) {
        const int g = f1 + 8 * g1;
        sc[4 * g + (j ^ ((g >> 2) & 3))] = z[g1];
    }
    __syncwarp();
    const int ga = lane, gb = lane ? 64 - lane : 32;
    float2 a[4], b[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        a[q] = sc[4 * ga + (q ^ ((ga >> 2) & 3))];
        b[q] = sc[4 * gb + (q ^ ((gb >> 2) & 3))];
    }
    __syncwarp();  // the scratch is free again
    fft::dft<4, false>(a);  // a[g2] = Z[ga + 64 g2]
    fft::dft<4, false>(b);  // b[g2] = Z[gb + 64 g2]
    if (lane) {
        unpack_pair(a[0], b[3], lane, tw, st, l);
        unpack_pair(a[1], b[2], 64 + lane, tw, st, l);
        unpack_pair(b[1], a[2], 128 - lane, tw, st, l);
        unpack_pair(b[0], a[3], 64 - lane, tw, st, l);
    } else {
        st[stage_pos(0, l)] = make_float2(a[0].x + a[0].y, 0.f);
        st[stage_pos(256, l)] = make_float2(a[0].x - a[0].y, 0.f);
        st[stage_pos(257, l)] = make_float2(0.f, 0.f);
        st[stage_pos(258, l)] = make_float2(0.f, 0.f);
        st[stage_pos(259, l)] = make_float2(0.f, 0.f);
        unpack_pair(a[1], a[3], 64, tw, st, l);
        unpack_pair(a[2], a[2], 128, tw, st, l);
        unpack_pair(b[0], b[3], 32, tw, st, l);
        unpack_pair(b[1], b[2], 96, tw, st, l);
    }
}

// The staged bricks (kx/4 = 0..64) of bundle (by, bz) to the spectrum, 16 bytes
// per thread: each warp instruction writes one whole brick.
template <int G>
__device__ __forceinline__ void store_bricks(const float2* st, float2* __restrict__ spec, int by, int bz) {
    for (int u = threadIdx.x; u < 65 * 32; u += blockDim.x) {
        const int b = u >> 5, c = u & 31;
        const float4 v = *reinterpret_cast<const float4*>(st + b * 64 + ((2 * c) ^ ((b & 3) << 2)));
        *reinterpret_cast<float4*>(spec + Geo<G>::brick(b, by, bz) + 2 * c) = v;
    }
}
}  // namespace xl

// ---- pass A: rows (y = 4by + y_l, z = 4bz + z_l) -> kx bins -----------------
// line l = z_l*4 + y_l; positions m < H hold z[m] = x[2m] + i x[2m+1].
// SRC 0: float grid, 1: int64 fixed-point grid (zeroed after reading). The source
// grid has side src_g <= G: a smaller one (the isolated boundary's density) sits in
// the low corner of the transform box and everything outside it reads as zero.
template <int G, int SRC>
__global__ void __launch_bounds__(kFftThreads) k_pass_a(const float* __restrict__ rho, long long* __restrict__ acc,
                                                        float* __restrict__ rho_keep, float2* __restrict__ spec,
                                                        const float2* __restrict__ tw_g, int src_g) {
    using T = Geo<G>;
    constexpr int H = T::H, NBX = T::NBX;
    constexpr int ITEMS = 16 * (H / 2);  // (line, pair of positions)
    constexpr int PER = (ITEMS + kFftThreads - 1) / kFftThreads;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* s = sm + G;
    const int by = blockIdx.x, bz = blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    if constexpr (G == 512) {
        // one warp per line, two lines per warp (the fused deposit's transform);
        // shared: tw | twiddle tables | 8 warp scratches | brick staging
        float2* tw2 = sm + G;
        xl::fill_twiddles(tw2, tw_g);
        __syncthreads();
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        float2* sc = tw2 + xl::kTw2 + warp * 256;
        float2* st = tw2 + xl::kTw2 + (kFftThreads / 32) * 256;
#pragma unroll 1
        for (int l = warp; l < 16; l += kFftThreads / 32) {
            const int y = by * 4 + (l & 3), z = bz * 4 + (l >> 2);
            const size_t row = ((size_t)z * src_g + y) * src_g;
            const bool in_rows = y < src_g && z < src_g;
            // every load of the row is issued before any store: a store that follows
            // the load of the same address in the loop body kept the next load waiting
            // behind it, one memory round trip per 512 bytes (2.46 ms at 512^3)
            float2 v[8];
            longlong2 q[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int m = lane + 32 * k;
                v[k] = make_float2(0.f, 0.f);
                q[k] = make_longlong2(0, 0);
                if (in_rows && 2 * m < src_g) {
                    if (SRC == 0)
                        v[k] = *reinterpret_cast<const float2*>(rho + row + 2 * m);
                    else
                        q[k] = *reinterpret_cast<const longlong2*>(acc + row + 2 * m);
                }
            }
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const int m = lane + 32 * k;
                if (in_rows && 2 * m < src_g) {
                    if (SRC == 1) {
                        *reinterpret_cast<longlong2*>(acc + row + 2 * m) = make_longlong2(0, 0);
                        v[k] = make_float2(fixed_to_float(q[k].x), fixed_to_float(q[k].y));
                    }
                    if (rho_keep) *reinterpret_cast<float2*>(rho_keep + row + 2 * m) = v[k];
                }
            }
            xl::r2c512(v, sc, tw, tw2, st, l);
        }
        __syncthreads();
        xl::store_bricks<G>(st, spec, by, bz);
        return;
    }

    float4 v[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int u = threadIdx.x + p * kFftThreads;
        if (ITEMS % kFftThreads == 0 || u < ITEMS) {
            const int l = u & 15, mp = u >> 4;
            const int y = by * 4 + (l & 3), z = bz * 4 + (l >> 2);
            const size_t row = ((size_t)z * src_g + y) * src_g;
            v[p] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (y < src_g && z < src_g && 4 * mp < src_g) {
                if (SRC == 0) {
                    v[p] = *reinterpret_cast<const float4*>(rho + row + 4 * mp);
                } else {
                    const longlong2 q0 = *reinterpret_cast<const longlong2*>(acc + row + 4 * mp);
                    const longlong2 q1 = *reinterpret_cast<const longlong2*>(acc + row + 4 * mp + 2);
                    v[p] = make_float4(fixed_to_float(q0.x), fixed_to_float(q0.y), fixed_to_float(q1.x),
                                       fixed_to_float(q1.y));
                }
            }
        }
    }
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int u = threadIdx.x + p * kFftThreads;
        if (ITEMS % kFftThreads == 0 || u < ITEMS) {
            const int l = u & 15, mp = u >> 4;
            const int y = by * 4 + (l & 3), z = bz * 4 + (l >> 2);
            const size_t row = ((size_t)z * src_g + y) * src_g;
            if (y < src_g && z < src_g && 4 * mp < src_g) {
                if (SRC == 1) {
                    *reinterpret_cast<longlong2*>(acc + row + 4 * mp) = make_longlong2(0, 0);
                    *reinterpret_cast<longlong2*>(acc + row + 4 * mp + 2) = make_longlong2(0, 0);
                }
                if (rho_keep) *reinterpret_cast<float4*>(rho_keep + row + 4 * mp) = v[p];
            }
            s[(2 * mp) * 16 + l] = make_float2(v[p].x, v[p].y);
            s[(2 * mp + 1) * 16 + l] = make_float2(v[p].z, v[p].w);
        }
    }
    __syncthreads();
    fft::lines16<H, kFftThreads, 2, false>(s, tw);
    // Z -> X, pairs (k, H-k):  E = (Z[k] + conj Z[H-k])/2,  O = (Z[k] - conj Z[H-k])/(2i),
    // X[k] = E + W^k O,  X[H-k] = conj E + W^(H-k) conj O;  X[0], X[H] from Z[0].
    constexpr int PAIRS = 16 * (H / 2 + 1);
    for (int u = threadIdx.x; u < PAIRS; u += kFftThreads) {
        const int l = u & 15, k = u >> 4;
        if (k == 0) {
            const float2 z0 = s[l];
            s[l] = make_float2(z0.x + z0.y, 0.f);
            s[H * 16 + l] = make_float2(z0.x - z0.y, 0.f);
            s[(H + 1) * 16 + l] = make_float2(0.f, 0.f);
            s[(H + 2) * 16 + l] = make_float2(0.f, 0.f);
            s[(H + 3) * 16 + l] = make_float2(0.f, 0.f);
            continue;
        }
        const float2 zk = s[k * 16 + l], zc = s[(H - k) * 16 + l];
        const float er = 0.5f * (zk.x + zc.x), ei = 0.5f * (zk.y - zc.y);
        const float orr = 0.5f * (zk.y + zc.y), oi = -0.5f * (zk.x - zc.x);
        const float2 w = tw[k];
        s[k * 16 + l] = make_float2(er + (w.x * orr - w.y * oi), ei + (w.x * oi + w.y * orr));
        if (2 * k != H) {
            const float2 w2 = tw[H - k];  // conj E + W^(H-k) conj O
            s[(H - k) * 16 + l] = make_float2(er + (w2.x * orr + w2.y * oi), -ei + (w2.y * orr - w2.x * oi));
        }
    }
    __syncthreads();
    // store bricks (bx, by, bz): brick element e = z_l*16 + y_l*4 + kx_l, two at a time
    for (int u = threadIdx.x; u < NBX * 32; u += kFftThreads) {
        const int bx = u >> 5, c = u & 31;
        const int l = (c >> 3) * 4 + ((c >> 1) & 3), kx = bx * 4 + (c & 1) * 2;
        const float2 a = s[kx * 16 + l], b = s[(kx + 1) * 16 + l];
        *reinterpret_cast<float4*>(spec + T::brick(bx, by, bz) + 2 * c) = make_float4(a.x, a.y, b.x, b.y);
    }
}

// ---- balanced fused deposit ---------------------------------------------------------
// Scratch (DepositWork::ints) of a grid with NB = G^2/16 row bundles, NC = ceil(NB/256):
//   items[NB]    CTAs sharing each bundle (>= 1)
//   xpre[NB]     exclusive prefix of (items - 1) inside each block of 256 bundles
//   arrive[NB]   CTAs of a shared bundle done so far (zero between uses)
//   cta_sum[NC], cta_pre[NC + 1]   per-block totals and their exclusive prefix
//   plan_done    blocks of the plan kernel done (zero between uses)
template <int G>
struct DepPlan {
    static constexpr int NB = G * G / 16;
    static constexpr int NC = (NB + 255) / 256;
    static constexpr int kItems = 0, kXpre = NB, kArrive = 2 * NB, kCtaSum = 3 * NB, kCtaPre = 3 * NB + NC,
                         kDone = 3 * NB + 2 * NC + 1, kInts = kDone + 1;
};

// The 25 base rows whose CIC stencils reach the 16 rows of bundle b = bz*(G/4)+by,
// as 7 ranges of the sorted particles: r = 0 the bundle's own rows (16 consecutive
// keys); r = 1 the rows z_l = 3 of the bundle below in z (4 consecutive keys);
// r = 2..5 the rows y_l = 3, z_l = r - 2 of the bundle below in y; r = 6 the row
// y_l = z_l = 3 of the bundle below in both. Neighbours wrap (periodic box).
template <int G>
__device__ __forceinline__ void window_range(int b, int r, const int* __restrict__ rs, int& lo, int& hi) {
    constexpr int TB = G / 4;
    const int by = b & (TB - 1), bz = b / TB;
    const int bym = (by + TB - 1) & (TB - 1), bzm = (bz + TB - 1) & (TB - 1);
    int k0, k1;
    if (r == 0) {
        k0 = 16 * b;
        k1 = k0 + 16;
    } else if (r == 1) {
        k0 = 16 * (bzm * TB + by) + 12;
        k1 = k0 + 4;
    } else if (r == 6) {
        k0 = 16 * (bzm * TB + bym) + 15;
        k1 = k0 + 1;
    } else {
        k0 = 16 * (bz * TB + bym) + 4 * (r - 2) + 3;
        k1 = k0 + 1;
    }
    lo = rs[k0];
    hi = rs[k1];
}

// Exclusive scan of one int per thread over a block of 256 threads; *total gets the sum.
__device__ __forceinline__ int block_excl_scan256(int v, int* total) {
    __shared__ int wsum[8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) wsum[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        int x = lane < 8 ? wsum[lane] : 0;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane < 8) wsum[lane] = x;
    }
    __syncthreads();
    const int excl = inc - v + (warp ? wsum[warp - 1] : 0);
    *total = wsum[7];
    __syncthreads();  // wsum may be reused by the next call
    return excl;
}

// How many CTAs share each bundle: ceil(window particles / split), at least 1,
// and where each bundle's extra CTAs start. The last block to finish turns the
// block totals into their prefix.
template <int G>
__global__ void __launch_bounds__(256) k_deposit_plan(const int* __restrict__ rs, int* __restrict__ w, int split) {
    using P = DepPlan<G>;
    const int b = blockIdx.x * 256 + threadIdx.x;
    int extra = 0;
    if (b < P::NB) {
        int total = 0;
#pragma unroll
        for (int r = 0; r < 7; ++r) {
            int lo, hi;
            window_range<G>(b, r, rs, lo, hi);
            total += hi - lo;
        }
        const int items = total > split ? (int)(((long long)total + split - 1) / split) : 1;
        w[P::kItems + b] = items;
        extra = items - 1;
    }
    int sum;
    const int excl = block_excl_scan256(extra, &sum);
    if (b < P::NB) w[P::kXpre + b] = excl;
    if (threadIdx.x == 0) w[P::kCtaSum + blockIdx.x] = sum;
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(reinterpret_cast<unsigned*>(w + P::kDone), 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    // NC <= 256 blocks (G <= 1024)
    const int v = threadIdx.x < P::NC ? __ldcg(w + P::kCtaSum + threadIdx.x) : 0;
    int all;
    const int pre = block_excl_scan256(v, &all);
    if (threadIdx.x < P::NC) w[P::kCtaPre + threadIdx.x] = pre;
    if (threadIdx.x == 0) {
        w[P::kCtaPre + P::NC] = all;
        w[P::kDone] = 0;
    }
}

// One CTA's share (slice `slice` of `items`) of bundle b: deposit its particles
// into int64 row sums in shared memory; if the bundle is shared, add the sums into
// the fixed-point grid and let the last CTA continue with the whole bundle; then
// convert, transform the 16 rows along x and store the spectrum bricks.
// (Summing equal corners across a warp's lanes first, with __match_any_sync and
// __reduce_add_sync, made dense scenes slower, not faster: 0.27 against 0.18 ms
// at 4M particles / 256^3.)
template <int G, bool SHARED>
__device__ __forceinline__ void deposit_bundle(int b, int slice, int items, const float4* __restrict__ pos,
                                               const int* __restrict__ perm, const int* __restrict__ row_start,
                                               float* __restrict__ rho_keep, float2* __restrict__ spec,
                                               const DepositWork& w, unsigned* __restrict__ arrive, bool reuse) {
    using T = Geo<G>;
    constexpr int H = T::H, NBX = T::NBX, NT = kDepositThreads, TB = G / 4;
    // The int64 fixed-point sums, as two 32-bit words per cell (lo[16][RS], hi[16][RS]),
    // share their storage with the complex line buffer used after the conversion.
    // Rows are RS = G + 4 words apart, so the row-parallel 16-byte reads of the
    // conversion fall in different banks.
    constexpr int RS = G + 4;
    extern __shared__ float2 sm[];
    const float2* tw = sm;
    unsigned* acc_lo = reinterpret_cast<unsigned*>(sm + G);
    unsigned* acc_hi = acc_lo + 16 * RS;
    float2* s = sm + G;
    __shared__ int r_lo[7], r_off[8];
    __shared__ int s_last;
    const int by = b & (TB - 1), bz = b / TB;
    const int m = G - 1;
    const int j = threadIdx.x;
    int lo = 0, len = 0;
    if (j < 7) {
        int hi;
        window_range<G>(b, j, row_start, lo, hi);
        len = hi - lo;
    }
    if (reuse) __syncthreads();  // the shared buffers of this CTA's previous bundle are free
    for (int i = threadIdx.x; i < 8 * RS; i += NT) reinterpret_cast<uint4*>(acc_lo)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (threadIdx.x < 32) {
        int inc = len;
#pragma unroll
        for (int o = 1; o < 8; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, inc, o);
            if (j >= o) inc += t;
        }
        if (j < 7) {
            r_lo[j] = lo;
            r_off[j + 1] = inc;
        }
        if (j == 0) r_off[0] = 0;
    }
    __syncthreads();
    const int total = r_off[7];
    const int f_lo = SHARED ? (int)((long long)total * slice / items) : 0;
    const int f_hi = SHARED ? (int)((long long)total * (slice + 1) / items) : total;
    // A weight q <= 2^32 is added as (q >> 16) into the high word and (q & 0xffff)
    // into the low word: with fewer than 2^16 particles in this share neither 32-bit
    // sum can overflow, so plain adds keep the 64-bit total exact. Larger shares
    // add the low 32 bits and carry into the high word instead.
    const bool split16 = f_hi - f_lo < 65536;
    const int lane = threadIdx.x & 31;
    constexpr int kBatch = 4;
    // lane f = base + q * NT + lane
    for (int base = f_lo + (threadIdx.x & ~31); base < f_hi; base += kBatch * NT) {
        int src[kBatch];
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
            const int f = base + q * NT + lane;
            src[q] = -1;
            if (f < f_hi) {
                int r = (r_off[4] <= f) ? 4 : 0;  // largest r < 7 with r_off[r] <= f
                if (r + 2 < 7 && r_off[r + 2] <= f) r += 2;
                if (r + 1 < 7 && r_off[r + 1] <= f) r += 1;
                src[q] = r_lo[r] + (f - r_off[r]);
            }
        }
        if (perm) {
#pragma unroll
            for (int q = 0; q < kBatch; ++q)
                if (src[q] >= 0) src[q] = perm[src[q]];
        }
        float4 pb[kBatch];
#pragma unroll
        for (int q = 0; q < kBatch; ++q) pb[q] = (src[q] >= 0) ? pos[src[q]] : make_float4(-1.f, -1.f, -1.f, 0.f);
#pragma unroll
        for (int q = 0; q < kBatch; ++q) {
            if (base + q * NT >= f_hi) break;
            const float4 p = pb[q];
            const bool valid = p.x >= 0.f;  // empty slots sort into row 0
            int ix, iy, iz;
            float fx, fy, fz;
            cic_axis(p.x, G, ix, fx);
            cic_axis(p.y, G, iy, fy);
            cic_axis(p.z, G, iz, fz);
            if (!valid) continue;
            const int x0 = ix & m, x1 = (ix + 1) & m;
#pragma unroll
            for (int oyz = 0; oyz < 4; ++oyz) {
                const int yl = ((iy + (oyz & 1)) & m) - 4 * by;
                const int zl = ((iz + (oyz >> 1)) & m) - 4 * bz;
                if ((unsigned)yl >= 4u || (unsigned)zl >= 4u) continue;
                const int rowc = (zl * 4 + yl) * RS;
#pragma unroll
                for (int ox = 0; ox < 2; ++ox) {
                    const unsigned long long qv =
                        (unsigned long long)fixed_weight(cic_weight(ox | (oyz << 1), fx, fy, fz));
                    const int c = rowc + (ox ? x1 : x0);
                    if (split16) {
                        atomicAdd(acc_hi + c, (unsigned)(qv >> 16));
                        atomicAdd(acc_lo + c, (unsigned)(qv & 0xffffu));
                    } else {
                        // atomicAdd returns the previous low word, so every wrap is seen by
                        // exactly one add
                        const unsigned lw = (unsigned)qv;
                        const unsigned old = atomicAdd(acc_lo + c, lw);
                        const unsigned up = (unsigned)(qv >> 32) + ((old + lw < old) ? 1u : 0u);
                        if (up) atomicAdd(acc_hi + c, up);
                    }
                }
            }
        }
    }
    __syncthreads();
    int sh = split16 ? 16 : 32;  // value of a cell: (hi << sh) + lo
    if (SHARED && items > 1) {
        // a shared bundle: every CTA adds its rows into the fixed-point grid; the last
        // to arrive reads the complete sums back (and leaves the grid zero)
        unsigned long long* g = reinterpret_cast<unsigned long long*>(w.acc);
#pragma unroll 1
        for (int u = threadIdx.x; u < 16 * G; u += NT) {
            const int l = u / G, x = u & m;
            const unsigned long long v =
                ((unsigned long long)acc_hi[l * RS + x] << sh) + (unsigned long long)acc_lo[l * RS + x];
            if (v) atomicAdd(g + ((size_t)(4 * bz + (l >> 2)) * G + 4 * by + (l & 3)) * G + x, v);
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) s_last = atomicAdd(arrive + b, 1u) == (unsigned)(items - 1);
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        // all of this thread's loads first, then the shared-memory writes and the zeroing
        // stores (a store behind each load of the same address would serialise them)
        constexpr int RB = 4;  // loads in flight per thread (more spill at the 40-register bound)
#pragma unroll 1
        for (int u0 = threadIdx.x; u0 < 16 * G; u0 += RB * NT) {
            unsigned long long rb[RB];
#pragma unroll
            for (int q = 0; q < RB; ++q) {
                const int u = u0 + q * NT, l = u / G, x = u & m;
                if (u < 16 * G) rb[q] = __ldcg(g + ((size_t)(4 * bz + (l >> 2)) * G + 4 * by + (l & 3)) * G + x);
            }
#pragma unroll
            for (int q = 0; q < RB; ++q) {
                const int u = u0 + q * NT, l = u / G, x = u & m;
                if (u < 16 * G) {
                    acc_lo[l * RS + x] = (unsigned)rb[q];
                    acc_hi[l * RS + x] = (unsigned)(rb[q] >> 32);
                    g[((size_t)(4 * bz + (l >> 2)) * G + 4 * by + (l & 3)) * G + x] = 0ull;
                }
            }
        }
        sh = 32;
        if (threadIdx.x == 0) arrive[b] = 0u;
        __syncthreads();
    }
    if constexpr (G == 512) {
        // warp l converts row l and transforms it (the generic pass A's routine, so
        // both deposit paths give the same bits); its lo row is then its scratch
        static_assert(NT == 16 * 32, "one warp per line");
        const int l = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const unsigned* lo = acc_lo + l * RS;
        const unsigned* hi = acc_hi + l * RS;
        const size_t grow = ((size_t)(bz * 4 + (l >> 2)) * G + by * 4 + (l & 3)) * G;
        float2 v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int m = lane + 32 * k;
            const uint2 lw = *reinterpret_cast<const uint2*>(lo + 2 * m);
            const uint2 hw = *reinterpret_cast<const uint2*>(hi + 2 * m);
            v[k] = make_float2(fixed_to_float((long long)(((unsigned long long)hw.x << sh) + lw.x)),
                               fixed_to_float((long long)(((unsigned long long)hw.y << sh) + lw.y)));
            if (rho_keep) *reinterpret_cast<float2*>(rho_keep + grow + 2 * m) = v[k];
        }
        // every row is in registers: the sums' storage becomes 16 warp scratches
        // (256 float2 each) and the brick staging (16 * 256 + kStage = 16 * RS float2)
        static_assert(16 * 256 + xl::kStage == 16 * RS, "scratch and staging fill the sums");
        __syncthreads();
        float2* R = reinterpret_cast<float2*>(acc_lo);
        xl::r2c512(v, R + l * 256, tw, sm + G + 16 * RS, R + 16 * 256, l);
        __syncthreads();
        xl::store_bricks<G>(R + 16 * 256, spec, by, bz);
        return;
    }
    // int64 rows -> complex positions z[m] = x[2m] + i x[2m+1] on line l = z_l*4 + y_l,
    // staged through registers because the line buffer overlays the sums.
    constexpr int CITEMS = 16 * (H / 2);
    constexpr int CPER = (CITEMS + NT - 1) / NT;
    float4 cv[CPER];
#pragma unroll
    for (int p = 0; p < CPER; ++p) {
        const int u = threadIdx.x + p * NT;
        if (CITEMS % NT == 0 || u < CITEMS) {
            const int l = u & 15, mp = u >> 4;
            const uint4 lw = *reinterpret_cast<const uint4*>(acc_lo + l * RS + 4 * mp);
            const uint4 hw = *reinterpret_cast<const uint4*>(acc_hi + l * RS + 4 * mp);
            cv[p] = make_float4(fixed_to_float((long long)(((unsigned long long)hw.x << sh) + lw.x)),
                                fixed_to_float((long long)(((unsigned long long)hw.y << sh) + lw.y)),
                                fixed_to_float((long long)(((unsigned long long)hw.z << sh) + lw.z)),
                                fixed_to_float((long long)(((unsigned long long)hw.w << sh) + lw.w)));
        }
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < CPER; ++p) {
        const int u = threadIdx.x + p * NT;
        if (CITEMS % NT == 0 || u < CITEMS) {
            const int l = u & 15, mp = u >> 4;
            if (rho_keep) {
                const size_t grow = ((size_t)(bz * 4 + (l >> 2)) * G + by * 4 + (l & 3)) * G;
                *reinterpret_cast<float4*>(rho_keep + grow + 4 * mp) = cv[p];
            }
            s[(2 * mp) * 16 + l] = make_float2(cv[p].x, cv[p].y);
            s[(2 * mp + 1) * 16 + l] = make_float2(cv[p].z, cv[p].w);
        }
    }
    __syncthreads();
    fft::lines16<H, NT, 2, false>(s, tw);
    constexpr int PAIRS = 16 * (H / 2 + 1);
    for (int u = threadIdx.x; u < PAIRS; u += NT) {
        const int l = u & 15, k = u >> 4;
        if (k == 0) {
            const float2 z0 = s[l];
            s[l] = make_float2(z0.x + z0.y, 0.f);
            s[H * 16 + l] = make_float2(z0.x - z0.y, 0.f);
            s[(H + 1) * 16 + l] = make_float2(0.f, 0.f);
            s[(H + 2) * 16 + l] = make_float2(0.f, 0.f);
            s[(H + 3) * 16 + l] = make_float2(0.f, 0.f);
            continue;
        }
        const float2 zk = s[k * 16 + l], zc = s[(H - k) * 16 + l];
        const float er = 0.5f * (zk.x + zc.x), ei = 0.5f * (zk.y - zc.y);
        const float orr = 0.5f * (zk.y + zc.y), oi = -0.5f * (zk.x - zc.x);
        const float2 wk = tw[k];
        s[k * 16 + l] = make_float2(er + (wk.x * orr - wk.y * oi), ei + (wk.x * oi + wk.y * orr));
        if (2 * k != H) {
            const float2 w2 = tw[H - k];
            s[(H - k) * 16 + l] = make_float2(er + (w2.x * orr + w2.y * oi), -ei + (w2.y * orr - w2.x * oi));
        }
    }
    __syncthreads();
    for (int u = threadIdx.x; u < NBX * 32; u += NT) {
        const int bx = u >> 5, c = u & 31;
        const int l = (c >> 3) * 4 + ((c >> 1) & 3), kx = bx * 4 + (c & 1) * 2;
        const float2 a = s[kx * 16 + l], c2 = s[(kx + 1) * 16 + l];
        *reinterpret_cast<float4*>(spec + T::brick(bx, by, bz) + 2 * c) = make_float4(a.x, a.y, c2.x, c2.y);
    }
}

// Grid: X CTAs that take the extra shares of heavy bundles (first, so they start
// early), then one CTA per bundle for its first share. 40 registers at G = 512
// keep three 70 KB CTAs per SM; smaller grids need more for their FFT stages.
template <int G>
__global__ void __launch_bounds__(kDepositThreads, G >= 128 ? 3 : 2)
    k_pass_a_deposit_bal(const float4* __restrict__ pos, const int* __restrict__ perm,
                         const int* __restrict__ row_start, float* __restrict__ rho_keep, float2* __restrict__ spec,
                         const float2* __restrict__ tw_g, DepositWork w) {
    using P = DepPlan<G>;
    extern __shared__ float2 sm[];
    const int* items = w.ints + P::kItems;
    const int* xpre = w.ints + P::kXpre;
    const int* cta_pre = w.ints + P::kCtaPre;
    unsigned* arrive = reinterpret_cast<unsigned*>(w.ints + P::kArrive);
    const int X = (int)gridDim.x - P::NB;
    const bool first = (int)blockIdx.x >= X;  // a bundle's first share, then done
    const int extras = first ? 0 : cta_pre[P::NC];
    if (!first && (int)blockIdx.x >= extras) return;  // no extra share for this CTA
    for (int i = threadIdx.x; i < G; i += kDepositThreads) sm[i] = tw_g[i];  // ordered by a later barrier
    if constexpr (G == 512) xl::fill_twiddles(sm + G + 16 * (G + 4), tw_g);  // the twiddle tables, after the sums
    for (int e = first ? 0 : (int)blockIdx.x; first || e < extras; e += X) {
        int b, slice;
        if (first) {
            b = (int)blockIdx.x - X;
            slice = 0;
        } else {
            // the bundle of extra share e: the last b whose extras start at or before e
            int lo = 0, hi = P::NB - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (cta_pre[mid >> 8] + xpre[mid] <= e) lo = mid;
                else hi = mid - 1;
            }
            b = lo;
            slice = 1 + e - (cta_pre[lo >> 8] + xpre[lo]);
        }
        // a bundle that one CTA covers whole takes the instantiation without the
        // shared-bundle code: a path that may run costs registers and time even when
        // it does not (0.513 against 0.479 ms at 16M / 512^3)
        // (at 512^3; smaller grids, whose registers the two copies would spill, keep one)
        const int nb = items[b];
        if (G >= 512 && nb == 1)
            deposit_bundle<G, false>(b, 0, 1, pos, perm, row_start, rho_keep, spec, w, arrive,
                                     !first && e != (int)blockIdx.x);
        else
            deposit_bundle<G, true>(b, slice, nb, pos, perm, row_start, rho_keep, spec, w, arrive,
                                    !first && e != (int)blockIdx.x);
        if (first) break;
    }
}

// Stage bricks into shared memory with cp.async. DIR 1: y-lines of CTA (bx,bz);
// DIR 2: z-lines of CTA (bx,by). Lines: DIR 1 -> z_l*4 + kx_l, DIR 2 -> y_l*4 + kx_l.
template <int G, int DIR>
__device__ __forceinline__ void load_lines(float2* s, const float2* __restrict__ spec, int b0, int b1) {
    using T = Geo<G>;
    constexpr int NB = (DIR == 1) ? T::NBY : T::NBZ;
    for (int u = threadIdx.x; u < NB * 32; u += kFftThreads) {
        const int b = u >> 5, c = u & 31;
        const int e = 2 * c;
        size_t src;
        int dst;
        if (DIR == 1) {  // b = by
            src = T::brick(b0, b, b1) + e;
            dst = (b * 4 + ((e >> 2) & 3)) * 16 + (e >> 4) * 4 + (e & 3);
        } else {  // b = bz: the brick lands contiguously
            src = T::brick(b0, b1, b) + e;
            dst = b * 64 + e;
        }
        fft::cp_async16(s + dst, spec + src);
    }
    fft::cp_async_wait_all();
    __syncthreads();
}

template <int G, int DIR>
__device__ __forceinline__ void store_lines(const float2* s, float2* __restrict__ spec, int bx, int b1) {
    using T = Geo<G>;
    constexpr int NB = (DIR == 1) ? T::NBY : T::NBZ;
    for (int u = threadIdx.x; u < NB * 32; u += kFftThreads) {
        const int b = u >> 5, c = u & 31;
        const int e = 2 * c;
        size_t dst;
        int src;
        if (DIR == 1) {
            dst = T::brick(bx, b, b1) + e;
            src = (b * 4 + ((e >> 2) & 3)) * 16 + (e >> 4) * 4 + (e & 3);
        } else {
            dst = T::brick(bx, b1, b) + e;
            src = b * 64 + e;
        }
        *reinterpret_cast<float4*>(spec + dst) = *reinterpret_cast<const float4*>(s + src);
    }
}

// ---- passes B and D: y-lines of CTA (bx, bz), in place -------------------------
template <int G, bool INV>
__global__ void __launch_bounds__(kFftThreads) k_pass_y(float2* __restrict__ spec, const float2* __restrict__ tw_g) {
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* s = sm + G;
    const int bx = blockIdx.x, bz = blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    load_lines<G, 1>(s, spec, bx, bz);
    fft::lines16<G, kFftThreads, 1, INV>(s, tw);
    store_lines<G, 1>(s, spec, bx, bz);
}

// ---- pass C: z-lines of CTA (bx, by): forward, Green's function, inverse ---------
// MODE 0: the periodic Green's function (analytic, Sim.cu:528-557).
// MODE 1: forward transform only (builds the isolated boundary's Green spectrum).
// MODE 2: multiply by a tabulated real Green spectrum table[|ky|][kx][|kz|]
//         ((H+1)^3 floats) times table_scale, then inverse (isolated boundary,
//         kMulSpec, Sim.cu:578-584).
template <int G, int MODE>
__global__ void __launch_bounds__(kFftThreads) k_pass_c(float2* __restrict__ spec, const float2* __restrict__ tw_g,
                                                        const float* __restrict__ gexp_g, float scale,
                                                        const float* __restrict__ table, float table_scale) {
    using T = Geo<G>;
    constexpr int H = T::H;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float* gexp = reinterpret_cast<float*>(sm + G);
    float2* s = sm + G + (H + 2) / 2 + 1;
    const int bx = blockIdx.x, by = blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    if (MODE == 0)
        for (int i = threadIdx.x; i <= H; i += kFftThreads) gexp[i] = gexp_g[i];
    __shared__ float line_g[16];
    __shared__ int line_k2[16];
    if (MODE == 0 && threadIdx.x < 16) {
        const int l = threadIdx.x;
        const int kx = bx * 4 + (l & 3), ky = by * 4 + (l >> 2);
        const int kyf = (ky <= G / 2) ? ky : ky - G;
        line_g[l] = (kx <= H) ? -scale * (gexp_g[kx] * gexp_g[abs(kyf)]) : 0.f;  // the global table: no barrier yet
        line_k2[l] = kx * kx + kyf * kyf;
    }
    load_lines<G, 2>(s, spec, bx, by);  // ends with a barrier
    if (MODE == 1) {
        fft::lines16<G, kFftThreads, 1, false>(s, tw);
        store_lines<G, 2>(s, spec, bx, by);
        return;
    }
    // forward, Green's function, inverse; the multiply happens in registers between
    // the forward's last stage and the inverse's first
    auto green = [&](int l, int kz, float2 x) {
        const int kzf = (kz <= G / 2) ? kz : kz - G;
        float m;
        if (MODE == 0) {
            // Green's function: -scale/k^2 * exp(-k^2 s^2/2), k = 0 -> 0 (Sim.cu:536-556), with
            // the per-line factors of (kx, ky) hoisted; padding columns kx > H are zeroed.
            const int k2 = line_k2[l] + kzf * kzf;
            m = (k2 != 0) ? __fdividef(line_g[l] * gexp[abs(kzf)], (float)k2) : 0.f;
        } else {
            const int kx = bx * 4 + (l & 3), ky = by * 4 + (l >> 2);
            const int kyf = (ky <= G / 2) ? ky : G - ky;
            m = (kx <= H) ? table[((size_t)kyf * (H + 1) + kx) * (H + 1) + abs(kzf)] * table_scale : 0.f;
        }
        return make_float2(x.x * m, x.y * m);
    };
    fft::convolve16<G, kFftThreads, 1>(s, tw, green);
    store_lines<G, 2>(s, spec, bx, by);
}

// Real part of a forward spectrum (bricked) into table[|ky|][kx][|kz|], ky, kz, kx <= H.
template <int G>
__global__ void k_green_table(const float2* __restrict__ spec, float* __restrict__ table) {
    using T = Geo<G>;
    constexpr int H = T::H;
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t n = (size_t)(H + 1) * (H + 1) * (H + 1);
    if (i >= n) return;
    const int kz = (int)(i % (H + 1)), kx = (int)((i / (H + 1)) % (H + 1)), ky = (int)(i / ((size_t)(H + 1) * (H + 1)));
    const size_t e = T::brick(kx >> 2, ky >> 2, kz >> 2) + (size_t)((kz & 3) * 16 + (ky & 3) * 4 + (kx & 3));
    table[i] = spec[e].x;
}

// Real-space isolated kernel on the transform box (kGreen, Sim.cu:563-576):
// g = -1 / (r + soft), r the distance in cells to the nearest corner copy.
__global__ void k_green_kernel(float* __restrict__ g, int S, float soft) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)S * S * S) return;
    const int x = (int)(i % S), y = (int)((i / S) % S), z = (int)(i / ((size_t)S * S));
    const int dx = (x <= S / 2) ? x : S - x;
    const int dy = (y <= S / 2) ? y : S - y;
    const int dz = (z <= S / 2) ? z : S - z;
    const float r = sqrtf((float)(dx * dx + dy * dy + dz * dz)) + soft;
    g[i] = -1.0f / r;
}

// ---- pass E: kx bins -> real rows (y = 4by + y_l, z = 4bz + z_l) ----------------
template <int G>
__global__ void __launch_bounds__(kFftThreads, 5) k_pass_e(const float2* __restrict__ spec, float* __restrict__ phi,
                                                        const float2* __restrict__ tw_g) {
    using T = Geo<G>;
    constexpr int H = T::H, NBX = T::NBX;
    constexpr int ITEMS = NBX * 32;
    constexpr int PER = (ITEMS + kFftThreads - 1) / kFftThreads;
    extern __shared__ float2 sm[];
    float2* tw = sm;
    float2* s = sm + G;
    // CTAs run from the last row bundle to the first: pass D ends on the high-z slabs, still in L2,
    // and the gather starts on the low-z rows of phi written last here (same results, ~8 us less)
    const int by = gridDim.x - 1 - blockIdx.x, bz = gridDim.y - 1 - blockIdx.y;
    for (int i = threadIdx.x; i < G; i += kFftThreads) tw[i] = tw_g[i];
    float4 v[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int u = threadIdx.x + p * kFftThreads;
        if (ITEMS % kFftThreads == 0 || u < ITEMS)
            v[p] = *reinterpret_cast<const float4*>(spec + T::brick(u >> 5, by, bz) + 2 * (u & 31));
    }
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int u = threadIdx.x + p * kFftThreads;
        if (ITEMS % kFftThreads == 0 || u < ITEMS) {
            const int bx = u >> 5, c = u & 31;
            const int l = (c >> 3) * 4 + ((c >> 1) & 3), kx = bx * 4 + (c & 1) * 2;
            s[kx * 16 + l] = make_float2(v[p].x, v[p].y);
            s[(kx + 1) * 16 + l] = make_float2(v[p].z, v[p].w);
        }
    }
    __syncthreads();
    // X -> Z inside the first stage's loads: Z[k] = E + i O with
    //   E = X[k] + conj X[H-k],  O = (X[k] - conj X[H-k]) * exp(+2 pi i k / G)
    // (imaginary parts of the k = 0 and k = H bins are dropped, as a C2R transform
    // does), read from the staged bins, which the stage overwrites only after its
    // barrier. This saves the separate pass over the pairs and its barrier.
    auto c2r_load = [tw](const float2* s, int l, int k) {
        float2 a = s[k * 16 + l], b = s[(H - k) * 16 + l];
        if (k == 0) { a.y = 0.f; b.y = 0.f; }
        const float2 w = tw[k];
        const float er = a.x + b.x, ei = a.y - b.y, dr = a.x - b.x, di = a.y + b.y;
        const float orr = dr * w.x + di * w.y, oi = di * w.x - dr * w.y;
        return make_float2(er - oi, ei + orr);
    };
    // The last stage leaves the lines row-major (stride H + 2 float2, 16-byte
    // aligned), so each warp then writes 512 contiguous bytes of one row instead
    // of 32 bytes of each of 16 rows.
    constexpr int RS = H + 2;
    static_assert(16 * RS <= 16 * T::PX, "row staging fits the line buffer");
    fft::lines16_rows<H, kFftThreads, 2, true, RS>(s, tw, c2r_load);
    for (int u = threadIdx.x; u < 16 * (H / 2); u += kFftThreads) {
        const int l = u / (H / 2), mp = u % (H / 2);
        const size_t row = ((size_t)(bz * 4 + (l >> 2)) * G + by * 4 + (l & 3)) * G;
        const float4 ab = *reinterpret_cast<const float4*>(s + l * RS + 2 * mp);
        *reinterpret_cast<float4*>(phi + row + 4 * mp) = ab;
    }
}

template <int G>
struct Launcher {
    using T = Geo<G>;
    static size_t smem_ae() { return sizeof(float2) * ((size_t)G + 16 * (size_t)T::PX); }
    // pass A from a grid: at G = 512 the twiddle tables, 8 warp scratches and the brick staging
    static size_t smem_a() {
        return G == 512 ? sizeof(float2) * ((size_t)G + xl::kTw2 + 8 * 256 + xl::kStage) : smem_ae();
    }
    static size_t smem_bd() { return sizeof(float2) * ((size_t)G + 16 * (size_t)G); }
    static size_t smem_c() { return sizeof(float2) * ((size_t)G + (T::H + 2) / 2 + 1 + 16 * (size_t)G); }
    // the line buffer (16 * PX float2) overlays the 32-bit sum words (2 * 16 * (G + 4));
    // at G = 512 the warp-per-line transform's twiddle tables follow the sums
    static size_t smem_bal() {
        const size_t lines = sizeof(float2) * 16 * (size_t)T::PX, sums = 2 * sizeof(unsigned) * 16 * (size_t)(G + 4);
        const size_t xtab = G == 512 ? sizeof(float2) * xl::kTw2 : 0;
        static_assert(G != 512 || 16 * (G + 4) >= 16 * T::PX, "the sums are the larger overlay");
        return sizeof(float2) * (size_t)G + (lines > sums ? lines : sums) + xtab;
    }
    // CTAs that take the extra shares of heavy bundles
    static int extra_ctas() {
        const int nb = DepPlan<G>::NB / 4;
        return nb < 8 ? 8 : (nb > 296 ? 296 : nb);
    }

    static int configure() {
        int rc = SD_OK;
        // prefer the largest shared-memory carveout so several 70 KB CTAs fit per SM
        const int carve = (int)cudaSharedmemCarveoutMaxShared;
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_a<G, 0>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_a<G, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_y<G, false>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_y<G, true>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_c<G, 0>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_c<G, 1>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_c<G, 2>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_e<G>, cudaFuncAttributePreferredSharedMemoryCarveout, carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_a_deposit_bal<G>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                           carve));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_a<G, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_a<G, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_y<G, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_bd()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_y<G, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_bd()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_c<G, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_c<G, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_c<G, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_c()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_e<G>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_ae()));
        rc |= SD_CUDA(cudaFuncSetAttribute(k_pass_a_deposit_bal<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem_bal()));
        return rc == SD_OK ? SD_OK : SD_E_CUDA;
    }

    static int run(const PoissonPlan& p, const long long* acc, const float* rho, const float4* pos, const int* perm,
                   const int* row_start, float* keep, float2* spec, float* phi, cudaStream_t s, cudaEvent_t* ev,
                   const PoissonIso* iso, const DepositWork* dw) {
        const dim3 grid_rows(T::NBY, T::NBZ), grid_y(T::NBX, T::NBZ), grid_z(T::NBX, T::NBY);
        const int src_g = (iso && iso->src_g > 0) ? iso->src_g : G;
        if (pos) {
            if (!dw || !dw->acc || !dw->ints || dw->split <= 0) return fail(SD_E_ARG, "fused deposit: no work plan");
            k_deposit_plan<G><<<DepPlan<G>::NC, 256, 0, s>>>(row_start, dw->ints, dw->split);
            SD_LAUNCHED(s);
            k_pass_a_deposit_bal<G><<<extra_ctas() + DepPlan<G>::NB, kDepositThreads, smem_bal(), s>>>(
                pos, perm, row_start, keep, spec, p.tw, *dw);
        } else if (acc)
            k_pass_a<G, 1><<<grid_rows, kFftThreads, smem_a(), s>>>(nullptr, const_cast<long long*>(acc), keep, spec,
                                                                     p.tw, src_g);
        else
            k_pass_a<G, 0><<<grid_rows, kFftThreads, smem_a(), s>>>(rho, nullptr, keep, spec, p.tw, src_g);
        SD_LAUNCHED(s);
        if (ev) cudaEventRecord(ev[0], s);
        k_pass_y<G, false><<<grid_y, kFftThreads, smem_bd(), s>>>(spec, p.tw);
        SD_LAUNCHED(s);
        if (ev) cudaEventRecord(ev[1], s);
        if (iso && iso->forward_only) {
            k_pass_c<G, 1><<<grid_z, kFftThreads, smem_c(), s>>>(spec, p.tw, p.gexp, p.scale, nullptr, 0.f);
            SD_LAUNCHED(s);
            return SD_OK;
        }
        if (iso && iso->table)
            k_pass_c<G, 2><<<grid_z, kFftThreads, smem_c(), s>>>(spec, p.tw, p.gexp, p.scale, iso->table,
                                                                 iso->table_scale);
        else
            k_pass_c<G, 0><<<grid_z, kFftThreads, smem_c(), s>>>(spec, p.tw, p.gexp, p.scale, nullptr, 0.f);
        SD_LAUNCHED(s);
        if (ev) cudaEventRecord(ev[2], s);
        k_pass_y<G, true><<<grid_y, kFftThreads, smem_bd(), s>>>(spec, p.tw);
        SD_LAUNCHED(s);
        if (ev) cudaEventRecord(ev[3], s);
        k_pass_e<G><<<grid_rows, kFftThreads, smem_ae(), s>>>(spec, phi, p.tw);
        SD_LAUNCHED(s);
        return SD_OK;
    }
};

// The Green's function's exponent table exp(-(2 pi soft / G)^2 k^2 / 2), k = 0..G/2,
// evaluated in FP64 and rounded once (both Poisson entry points build it here).
__global__ void k_fill_gexp(float* __restrict__ gexp, int G, float soft) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k > G / 2) return;
    const double s = 6.283185307179586476925286766559 * (double)(soft > 0.f ? soft : 0.f) / (double)G;
    gexp[k] = (float)exp(-0.5 * s * s * (double)k * (double)k);
}

int fill_gexp(float* gexp, int G, float soft, cudaStream_t st) {
    k_fill_gexp<<<(G / 2 + 1 + 127) / 128, 128, 0, st>>>(gexp, G, soft);
    SD_LAUNCHED(st);
    return SD_OK;
}

int poisson_configure(int G) {
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

}  // namespace

size_t deposit_work_ints(int G) {
    switch (G) {
        case 16: return DepPlan<16>::kInts;
        case 32: return DepPlan<32>::kInts;
        case 64: return DepPlan<64>::kInts;
        case 128: return DepPlan<128>::kInts;
        case 256: return DepPlan<256>::kInts;
        case 512: return DepPlan<512>::kInts;
        default: return 0;
    }
}

int deposit_split(int n, int G, int mult) {
    // by default ten times a window's mean particle count (a window spans 25 rows for a
    // bundle's 16) where the grid has at least 1024 bundles, five times below that, and at
    // least 2048: 4M particles on 256^3 (two galaxies) deposit in 0.153 ms with 10x, 0.155
    // with 5x, 0.163 with 3x; 262,144 on 64^3 (one disk, 256 bundles) in 0.048 ms with 10x,
    // 0.040 with 5x, 0.042 with 3x
    const long long nb = (long long)G * G / 16;
    if (mult <= 0) mult = nb >= 1024 ? 10 : 5;
    const long long t = (long long)mult * (long long)n / (nb > 0 ? nb : 1);
    return (int)(t < 2048 ? 2048 : (t > (1 << 30) ? (1 << 30) : t));
}

size_t poisson_spectrum_elems(int G) { return (size_t)G * G * (size_t)(G / 2 + 4); }

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
    if (SD_CUDA(cudaMalloc(&p.tw, sizeof(float2) * tw.size())) != SD_OK) return SD_E_NOMEM;
    if (SD_CUDA(cudaMalloc(&p.gexp, sizeof(float) * ((size_t)G / 2 + 1))) != SD_OK) return SD_E_NOMEM;
    if (SD_CUDA(cudaMemcpy(p.tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice)) != SD_OK)
        return SD_E_CUDA;
    // the same kernel as the allocation-free solve's, so both tables hold the same bits
    if (int rc = fill_gexp(p.gexp, G, soft, nullptr)) return rc;
    if (SD_CUDA(cudaStreamSynchronize(nullptr))) return SD_E_CUDA;
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

int launch_poisson(const PoissonPlan& p, const long long* acc, const float* rho, float* keep, float2* spec,
                   float* phi, cudaStream_t s) {
    return launch_poisson_ex(p, acc, rho, nullptr, nullptr, nullptr, keep, spec, phi, s);
}

int launch_poisson_ex(const PoissonPlan& p, const long long* acc, const float* rho, const float4* pos,
                      const int* perm, const int* row_start, float* keep, float2* spec, float* phi, cudaStream_t s,
                      cudaEvent_t* ev, const PoissonIso* iso, const DepositWork* dw) {
    switch (p.G) {
        case 16: return Launcher<16>::run(p, acc, rho, pos, perm, row_start, keep, spec, phi, s, ev, iso, dw);
        case 32: return Launcher<32>::run(p, acc, rho, pos, perm, row_start, keep, spec, phi, s, ev, iso, dw);
        case 64: return Launcher<64>::run(p, acc, rho, pos, perm, row_start, keep, spec, phi, s, ev, iso, dw);
        case 128: return Launcher<128>::run(p, acc, rho, pos, perm, row_start, keep, spec, phi, s, ev, iso, dw);
        case 256: return Launcher<256>::run(p, acc, rho, pos, perm, row_start, keep, spec, phi, s, ev, iso, dw);
        case 512: return Launcher<512>::run(p, acc, rho, pos, perm, row_start, keep, spec, phi, s, ev, iso, dw);
        default: return fail(SD_E_UNSUPPORTED, "poisson: grid size %d not supported", p.G);
    }
}

size_t green_table_elems(int S) {
    const size_t h = (size_t)S / 2 + 1;
    return h * h * h;
}

int build_green_table(const PoissonPlan& p, float softening_cells, float* kernel_grid, float2* spec, float* table,
                      cudaStream_t s) {
    const int S = p.G;
    const size_t cells = (size_t)S * S * S;
    // the reference floors the isolated softening at half a cell (buildGreen, Sim.cu:3569-3575)
    const float soft = softening_cells > 0.5f ? softening_cells : 0.5f;
    k_green_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(kernel_grid, S, soft);
    SD_LAUNCHED(s);
    PoissonIso fwd;
    fwd.forward_only = true;
    if (int rc = launch_poisson_ex(p, nullptr, kernel_grid, nullptr, nullptr, nullptr, nullptr, spec, nullptr, s,
                                   nullptr, &fwd))
        return rc;
    const size_t n = green_table_elems(S);
    switch (S) {
        case 32: k_green_table<32><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(spec, table); break;
        case 64: k_green_table<64><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(spec, table); break;
        case 128: k_green_table<128><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(spec, table); break;
        case 256: k_green_table<256><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(spec, table); break;
        case 512: k_green_table<512><<<(unsigned)((n + 255) / 256), 256, 0, s>>>(spec, table); break;
        default: return fail(SD_E_UNSUPPORTED, "isolated: transform size %d not supported", S);
    }
    SD_LAUNCHED(s);
    return SD_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free Poisson solve (sd_poisson_noalloc).
//
// For callers that must not allocate device memory: code running where
// cudaMalloc is not allowed, such as inside another library's allocator-free
// hot loop, or under a strict memory budget that forbids growth after start-up.
// Its working memory
// is file-scope device storage of fixed size, so grids are limited to
// kNoAllocMaxGrid^3. Every GPU that loads this library holds that storage
// (about 9 MB) until the process exits, and all calls on a device share it:
// calls that overlap on the GPU race on it.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxGrid = 128;
constexpr size_t kNoAllocSpecElems =
    (size_t)kNoAllocMaxGrid * kNoAllocMaxGrid * (size_t)(kNoAllocMaxGrid / 2 + 4);
constexpr int kNoAllocMaxDevices = 64;

// The bricked spectrum of the largest supported grid, the twiddle tables of
// G = 16, 32, 64, 128 (one row of kNoAllocMaxGrid entries each) and the
// Green's-function exponent table of the current call.
static __device__ __align__(256) float2 g_noalloc_spec[kNoAllocSpecElems];
static __device__ __align__(256) float2 g_noalloc_tw[4 * kNoAllocMaxGrid];
static __device__ __align__(256) float g_noalloc_gexp[kNoAllocMaxGrid / 2 + 1];

struct NoAllocDevice {
    bool ready = false;
    unsigned long long ctx_id = 0;  // the context the addresses and tables belong to
    float2* spec = nullptr;
    float2* tw = nullptr;
    float* gexp = nullptr;
};

// The unique ID of the current context (cuCtxGetId through the runtime's driver
// entry points; 0 if unavailable). A device reset ends the context: its file-scope
// arrays come back zeroed under a new ID, so the cached set-up is redone.
unsigned long long current_ctx_id() {
    using GetCurrent = CUresult (*)(CUcontext*);
    using GetId = CUresult (*)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}
NoAllocDevice g_noalloc[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

int noalloc_slot(int G) { return G == 16 ? 0 : (G == 32 ? 1 : (G == 64 ? 2 : 3)); }

// Once per device, with that device current: resolve the device addresses of
// the file-scope arrays (their names are host-side stand-ins in host code),
// upload the twiddle tables and set the kernels' shared-memory attributes.
int noalloc_setup(int dev) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    NoAllocDevice& d = g_noalloc[dev];
    void* p = nullptr;
    // resolving a symbol also makes the device's context current, which the ID needs
    if (SD_CUDA(cudaGetSymbolAddress(&p, g_noalloc_spec))) return SD_E_CUDA;
    const unsigned long long ctx = current_ctx_id();
    if (d.ready && ctx == d.ctx_id) return SD_OK;
    d.ready = false;
    d.ctx_id = ctx;
    d.spec = static_cast<float2*>(p);
    if (SD_CUDA(cudaGetSymbolAddress(&p, g_noalloc_tw))) return SD_E_CUDA;
    d.tw = static_cast<float2*>(p);
    if (SD_CUDA(cudaGetSymbolAddress(&p, g_noalloc_gexp))) return SD_E_CUDA;
    d.gexp = static_cast<float*>(p);
    std::vector<float2> tw((size_t)4 * kNoAllocMaxGrid, make_float2(0.f, 0.f));
    const double two_pi = 6.283185307179586476925286766559;
    for (int G = 16; G <= kNoAllocMaxGrid; G *= 2) {
        float2* row = tw.data() + (size_t)noalloc_slot(G) * kNoAllocMaxGrid;
        for (int m = 0; m < G; ++m) {
            const double a = -two_pi * (double)m / (double)G;
            row[m] = make_float2((float)cos(a), (float)sin(a));
        }
        if (int rc = poisson_configure(G)) return rc;
    }
    if (SD_CUDA(cudaMemcpy(d.tw, tw.data(), sizeof(float2) * tw.size(), cudaMemcpyHostToDevice))) return SD_E_CUDA;
    d.ready = true;
    return SD_OK;
}

}  // namespace

}  // namespace sd

extern "C" int sd_poisson_noalloc(const float* rho, int grid_size, float softening_cells, float* phi, void* stream) {
    using namespace sd;
    const int G = grid_size;
    if (!rho || !phi) return fail(SD_E_ARG, "sd_poisson_noalloc: null rho or phi");
    if (G < 16 || G > kNoAllocMaxGrid || (G & (G - 1)))
        return fail(SD_E_ARG,
                    "sd_poisson_noalloc: grid_size %d is not a power of two in [16, %d]; its fixed workspace holds "
                    "the spectrum of a %d^3 grid at most (use sd_poisson with a caller workspace for larger grids)",
                    G, kNoAllocMaxGrid, kNoAllocMaxGrid);
    int dev = 0;
    if (SD_CUDA(cudaGetDevice(&dev))) return SD_E_CUDA;
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(SD_E_ARG, "sd_poisson_noalloc: device %d unsupported", dev);
    if (int rc = noalloc_setup(dev)) return rc;
    const NoAllocDevice& d = g_noalloc[dev];
    cudaStream_t st = (cudaStream_t)stream;
    // the exponent table depends on the softening: rebuilt by every call
    if (int rc = fill_gexp(d.gexp, G, softening_cells, st)) return rc;
    PoissonPlan plan;
    plan.G = G;
    plan.soft = softening_cells;
    plan.tw = d.tw + (size_t)noalloc_slot(G) * kNoAllocMaxGrid;
    plan.gexp = d.gexp;
    plan.scale = (float)(1.0 / (4.0 * 3.14159265358979323846 * 3.14159265358979323846 * (double)G * G * G));
    // pass A writes every spectrum element (padding columns as zeros), so the
    // shared workspace needs no clearing between calls
    const int rc = launch_poisson(plan, nullptr, rho, nullptr, d.spec, phi, st);
    plan.tw = nullptr;  // static storage: the plan does not own it
    plan.gexp = nullptr;
    return rc;
}

