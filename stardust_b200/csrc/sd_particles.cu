// sd_particles.cu -- per-particle kernels: CIC deposit, gather + kick + drift,
// momentum sums, speed, energy and small grid reductions.
//
// Reference counterparts: kScatter (Sim.cu:503-521), kGridAccel (Sim.cu:589-611),
// sampleAcc and kIntegrate (Sim.cu:614-629, 685-906), kMaxSpeed (Sim.cu:2923-2930),
// kMomentumAccum / kSubtractMeanVelDev (Sim.cu:2252-2291).
//
// Design points:
//  * The deposit rounds each CIC weight once to a multiple of 2^-32 and adds it to
//    an int64 grid. Integer addition is associative, so the density is the same
//    whatever order the atomics land in: bit-exact run to run, and bit-exact
//    against the oracle's fixed-point deposit.
//  * No force grid is stored. The gather reads the potential and forms the
//    reference's central difference for each of the 8 CIC corners with the
//    reference's arithmetic; given the same phi the kick is bit-identical to the
//    reference's accG route (kGridAccel then sampleAcc), and it saves writing and
//    re-reading a float4 grid (32 B per cell).
//  * Momentum zeroing is deferred: the kernel that writes the new velocities also
//    sums them (FP64 per block, then a fixed-order final sum), and the mean is
//    subtracted as the next consumer loads each velocity. The float arithmetic
//    (v - (float)(sum/count)) is the reference's.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "sd_common.cuh"
#include "sd_internal.h"

namespace sd {

namespace {

constexpr int kGatherThreads = 256;
constexpr int kGatherMaxBlocks = 4096;
constexpr int kKeysPlain = 0, kKeysCounts = 1, kKeysChanged = 2;  // the gather's KEYS modes

// 16-byte global -> shared copy that does not hold registers while in flight
// (L2 only); copy groups and the wait until at most N of this thread's most
// recent groups are pending.
__device__ __forceinline__ void cp_async16(float4* smem, const float4* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// records (pos, vel) of the gather's next particles in flight ahead of the one in use
constexpr int kAhead = 1;

__global__ void __launch_bounds__(256) k_deposit_fixed(const float4* __restrict__ pos, int n, int G,
                                                       unsigned long long* __restrict__ acc, int periodic) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (p.x < 0.f) return;
    int ix, iy, iz;
    float fx, fy, fz;
    cic_axis(p.x, G, ix, fx);
    cic_axis(p.y, G, iy, fy);
    cic_axis(p.z, G, iz, fz);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int cx = cic_cell(ix + (k & 1), G, periodic);
        const int cy = cic_cell(iy + ((k >> 1) & 1), G, periodic);
        const int cz = cic_cell(iz + ((k >> 2) & 1), G, periodic);
        const long long q = fixed_weight(cic_weight(k, fx, fy, fz));
        atomicAdd(acc + ((size_t)cz * G + cy) * G + cx, (unsigned long long)q);
    }
}

__global__ void k_fixed_to_float(long long* __restrict__ acc, size_t cells, float* __restrict__ rho, int clear) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    rho[i] = fixed_to_float(acc[i]);
    if (clear) acc[i] = 0;
}

__global__ void k_clear_u64(unsigned long long* __restrict__ a, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = 0ull;
}

// CIC-interpolated central-difference gradient of phi at p: the reference's
// kGridAccel values (Sim.cu:604-610) sampled with sampleAcc's weights and FMA
// order (Sim.cu:614-629). The 8 corners' 48 potential reads touch 32 distinct
// cells; each is loaded once:
//   A[oy][oz][d]  rows (iy+oy, iz+oz), x = ix-1+d, d < 4
//   Y[e][oz][ox]  rows (iy-1+3e, iz+oz), x = ix+ox
//   Z[e][oy][ox]  rows (iy+oy, iz-1+3e), x = ix+ox
__device__ __forceinline__ float3 gather_accel(const float* __restrict__ phi, int G, float h, float4 p,
                                               float* phi_at = nullptr) {
    int ix, iy, iz;
    float fx, fy, fz;
    cic_axis(p.x, G, ix, fx);
    cic_axis(p.y, G, iy, fy);
    cic_axis(p.z, G, iz, fz);
    const int m = G - 1;
    const size_t G2 = (size_t)G * G;
    int xs[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) xs[d] = (ix - 1 + d) & m;
    size_t ys[4], zs[4];
#pragma unroll
    for (int d = 0; d < 4; ++d) {
        ys[d] = (size_t)((iy - 1 + d) & m) * G;
        zs[d] = (size_t)((iz - 1 + d) & m) * G2;
    }
    float A[2][2][4], Y[2][2][2], Z[2][2][2];
#pragma unroll
    for (int oy = 0; oy < 2; ++oy)
#pragma unroll
        for (int oz = 0; oz < 2; ++oz)
#pragma unroll
            for (int d = 0; d < 4; ++d) A[oy][oz][d] = __ldg(phi + zs[1 + oz] + ys[1 + oy] + xs[d]);
#pragma unroll
    for (int e = 0; e < 2; ++e)
#pragma unroll
        for (int o = 0; o < 2; ++o)
#pragma unroll
            for (int ox = 0; ox < 2; ++ox) {
                Y[e][o][ox] = __ldg(phi + zs[1 + o] + ys[3 * e] + xs[1 + ox]);
                Z[e][o][ox] = __ldg(phi + zs[3 * e] + ys[1 + o] + xs[1 + ox]);
            }
    float3 a = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int ox = k & 1, oy = (k >> 1) & 1, oz = (k >> 2) & 1;
        const float w = cic_weight(k, fx, fy, fz);
        const float xp = A[oy][oz][ox + 2], xm = A[oy][oz][ox];
        const float yp = oy ? Y[1][oz][ox] : A[1][oz][ox + 1];
        const float ym = oy ? A[0][oz][ox + 1] : Y[0][oz][ox];
        const float zp = oz ? Z[1][oy][ox] : A[oy][1][ox + 1];
        const float zm = oz ? A[oy][0][ox + 1] : Z[0][oy][ox];
        const float gx = __fmul_rn(-__fsub_rn(xp, xm), h);
        const float gy = __fmul_rn(-__fsub_rn(yp, ym), h);
        const float gz = __fmul_rn(-__fsub_rn(zp, zm), h);
        a.x = __fmaf_rn(gx, w, a.x);
        a.y = __fmaf_rn(gy, w, a.y);
        a.z = __fmaf_rn(gz, w, a.z);
    }
    if (phi_at) {  // CIC-interpolated potential: the corners are A[oy][oz][1 + ox]
        float f = 0.f;
#pragma unroll
        for (int k = 0; k < 8; ++k)
            f = __fmaf_rn(cic_weight(k, fx, fy, fz), A[(k >> 1) & 1][(k >> 2) & 1][1 + (k & 1)], f);
        *phi_at = f;
    }
    return a;
}

// Isolated boundary (kGridAccel/sampleAcc with clamped indices, Sim.cu:589-629):
// the potential lives in the low G^3 corner of an S^3 box (rows S apart); every
// corner cell and its gradient neighbours are clamped to [0, G). The 8 corners'
// 48 reads are not merged (edge clamping makes them differ); this path is not
// the benchmark's.
__device__ __forceinline__ float3 gather_accel_iso(const float* __restrict__ phi, int G, int S, float h, float4 p,
                                                   float* phi_at = nullptr) {
    int ix, iy, iz;
    float fx, fy, fz;
    cic_axis(p.x, G, ix, fx);
    cic_axis(p.y, G, iy, fy);
    cic_axis(p.z, G, iz, fz);
    auto at = [&](int x, int y, int z) { return __ldg(phi + ((size_t)z * S + y) * S + x); };
    float3 a = make_float3(0.f, 0.f, 0.f);
    float f = 0.f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int cx = cic_cell(ix + (k & 1), G, false);
        const int cy = cic_cell(iy + ((k >> 1) & 1), G, false);
        const int cz = cic_cell(iz + ((k >> 2) & 1), G, false);
        const int xm = max(cx - 1, 0), xp = min(cx + 1, G - 1);
        const int ym = max(cy - 1, 0), yp = min(cy + 1, G - 1);
        const int zm = max(cz - 1, 0), zp = min(cz + 1, G - 1);
        const float w = cic_weight(k, fx, fy, fz);
        const float gx = __fmul_rn(-__fsub_rn(at(xp, cy, cz), at(xm, cy, cz)), h);
        const float gy = __fmul_rn(-__fsub_rn(at(cx, yp, cz), at(cx, ym, cz)), h);
        const float gz = __fmul_rn(-__fsub_rn(at(cx, cy, zp), at(cx, cy, zm)), h);
        a.x = __fmaf_rn(gx, w, a.x);
        a.y = __fmaf_rn(gy, w, a.y);
        a.z = __fmaf_rn(gz, w, a.z);
        if (phi_at) f = __fmaf_rn(w, at(cx, cy, cz), f);
    }
    if (phi_at) *phi_at = f;
    return a;
}

// Acceleration at p: periodic grid (S == 0) or the isolated box of side S.
template <bool ISO>
__device__ __forceinline__ float3 accel_at(const float* __restrict__ phi, int G, int S, float h, float4 p,
                                           float* phi_at = nullptr) {
    return ISO ? gather_accel_iso(phi, G, S, h, p, phi_at) : gather_accel(phi, G, h, p, phi_at);
}

// FP64 block sums of K values into partials[blockIdx.x*K + j], fixed tree order.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double* partials) {
    __shared__ double red[K][kGatherThreads / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < K; ++j)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[j] += __shfl_down_sync(0xffffffffu, v[j], o);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < K; ++j) red[j][w] = v[j];
    __syncthreads();
    if (threadIdx.x < K) {
        double s = 0.0;
        for (int j = 0; j < kGatherThreads / 32; ++j) s += red[threadIdx.x][j];
        partials[(size_t)blockIdx.x * K + threadIdx.x] = s;
    }
}

// One thread per particle, grid-stride over at most kGatherMaxBlocks blocks so the
// per-block FP64 partials stay few; the block-to-particle assignment depends only
// on n, so the sums are deterministic.
//
// With perm != nullptr the kernel also performs the sort's reorder
// (kReorder, Sim.cu:2488-2495): slot i takes particle perm[i] of the input
// arrays and the results go to separate output arrays. keys_out (optional)
// receives the order key of each new position for the next step's sort.
//
// DIAG: the FP64 partials also carry sum |v|^2 of the kicked velocities and sum
// phi(x) at the step-start positions (the potential the kick used), for the
// per-step energy record written by the finalize kernel.
//
// ISO: isolated boundary (potential box of side S, clamped sampling, and the
// reference's wall at [0.002, 0.998] that stops a particle and returns a quarter
// of its speed, Sim.cu:895-903) instead of the periodic wrap.
// CIC sample of a G^3 float4 field at p (sampleAcc, Sim.cu:614-629): cell-centred
// weights (wx wy) wz, corners wrapped (periodic) or clamped (isolated).
template <bool ISO>
__device__ __forceinline__ float3 sample_field(const float4* __restrict__ f, int G, float4 p) {
    int ix, iy, iz;
    float fx, fy, fz;
    cic_axis(p.x, G, ix, fx);
    cic_axis(p.y, G, iy, fy);
    cic_axis(p.z, G, iz, fz);
    float3 a = make_float3(0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int cx = cic_cell(ix + (k & 1), G, !ISO), cy = cic_cell(iy + ((k >> 1) & 1), G, !ISO),
                  cz = cic_cell(iz + ((k >> 2) & 1), G, !ISO);
        const float w = cic_weight(k, fx, fy, fz);
        const float4 g = f[((size_t)cz * G + cy) * G + cx];
        a.x = __fmaf_rn(g.x, w, a.x);
        a.y = __fmaf_rn(g.y, w, a.y);
        a.z = __fmaf_rn(g.z, w, a.z);
    }
    return a;
}

// PRESS: gas particles (pos.w <= 0, not dark matter) also take the CIC sample of
// the pressure acceleration grid `press` (G^3; kIntegrate, Sim.cu:740-743).
//
// KEYS: what the gather leaves for the next step's sort besides keys_out --
// kKeysPlain nothing, kKeysCounts the first pass's tile counts (tile_counts),
// kKeysChanged the change bits (chg_words). Each instantiation holds only its own
// bookkeeping: the gather runs at its register limit, and code that a launch
// never executes still costs it.
template <bool DIAG, bool ISO, bool PRESS, int KEYS>
__global__ void __launch_bounds__(kGatherThreads, 3) k_gather_kick_drift(
    const float* __restrict__ phi, int G, float h, const float4* pos_in, const float4* vel_in,
    const int* __restrict__ perm, float4* pos_out, float4* vel_out, uint32_t* __restrict__ keys_out, int order, int n,
    float dt_kick, float dt_drift, float c2, const float* __restrict__ mean_vel, double* __restrict__ partials,
    const float4* __restrict__ extra, int S, unsigned* __restrict__ tile_counts, int count_bits,
    const float4* __restrict__ press, unsigned* __restrict__ chg_words) {
    // Per-thread FP64 sums (momentum, count; with DIAG |v|^2 and phi), each in the
    // thread's own shared-memory slot: held in registers they crowd out the stencil's
    // loads at the kernel's register limit. The summation order is the same.
    __shared__ double acc[6][kGatherThreads];
    // Software pipeline over the grid-stride loop: the records (pos, vel) of this
    // thread's next kAhead particles are in flight into its own shared-memory slots
    // (cp.async, one copy group per particle), and the permutation index of the
    // particle after them is loaded, so the dependent perm -> record loads overlap
    // the stencils of the particles before them instead of preceding each one.
    // kAhead + 1 slots rotate; each thread reads and fills only its own, so no
    // barrier is involved.
    __shared__ float4 rec[kAhead + 1][2][kGatherThreads];
    const int me = threadIdx.x;
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q][me] = 0.0;
    const unsigned cmask = (1u << count_bits) - 1u;
    const float mx = mean_vel ? mean_vel[0] : 0.f, my = mean_vel ? mean_vel[1] : 0.f,
                mz = mean_vel ? mean_vel[2] : 0.f;
    const int stride = gridDim.x * blockDim.x;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    // prologue: the records of this thread's first kAhead particles, one copy group
    // each, and the permutation index of the particle after them
#pragma unroll
    for (int q = 0; q < kAhead; ++q) {
        const int iq = i + q * stride;
        if (iq < n) {
            const int jq = perm ? perm[iq] : iq;
            cp_async16(&rec[q][0][me], pos_in + jq);
            cp_async16(&rec[q][1][me], vel_in + jq);
        }
        cp_async_commit();
    }
    int jn = 0;
    if (i + kAhead * stride < n) jn = perm ? perm[i + kAhead * stride] : i + kAhead * stride;
    for (int slot = 0; i < n; i += stride, slot = (slot == kAhead) ? 0 : slot + 1) {
        uint32_t key = 0u;      // the order key written for output i (0: empty or lost)
        uint32_t key_old = 0u;  // the key of the step-start position (the one output i was sorted by)
        cp_async_wait_group<kAhead - 1>();  // this thread's copies of particle i
        float4 p = rec[slot][0][me];
        float4 v = rec[slot][1][me];
        {
            const int ia = i + kAhead * stride;  // the particle whose record goes in flight now
            const int sa = (slot == 0) ? kAhead : slot - 1;
            if (ia < n) {
                cp_async16(&rec[sa][0][me], pos_in + jn);
                cp_async16(&rec[sa][1][me], vel_in + jn);
                if (ia + stride < n) jn = perm ? perm[ia + stride] : ia + stride;
            }
            cp_async_commit();
        }
        do {
            if (p.x < 0.f) {
                if (perm) {
                    pos_out[i] = p;
                    vel_out[i] = v;
                }
                if (keys_out) keys_out[i] = 0u;
                break;
            }
            if (mean_vel) {
                v.x = __fsub_rn(v.x, mx);
                v.y = __fsub_rn(v.y, my);
                v.z = __fsub_rn(v.z, mz);
            }
            float phi_p = 0.f;
            float3 a = accel_at<ISO>(phi, G, S, h, p, DIAG ? &phi_p : nullptr);
            if (extra) {  // learned correction, indexed like the outputs
                const float4 e = extra[i];
                a.x = __fadd_rn(a.x, e.x);
                a.y = __fadd_rn(a.y, e.y);
                a.z = __fadd_rn(a.z, e.z);
            }
            if (PRESS && p.w <= 0.f && v.w >= -50.f) {
                const float3 pr = sample_field<ISO>(press, G, p);
                a.x = __fadd_rn(a.x, pr.x);
                a.y = __fadd_rn(a.y, pr.y);
                a.z = __fadd_rn(a.z, pr.z);
            }
            v.x = __fmaf_rn(a.x, dt_kick, v.x);
            v.y = __fmaf_rn(a.y, dt_kick, v.y);
            v.z = __fmaf_rn(a.z, dt_kick, v.z);
            {  // light-speed clamp (Sim.cu:834-840)
                const float sp2 = __fmaf_rn(v.z, v.z, __fmaf_rn(v.y, v.y, __fmul_rn(v.x, v.x)));
                if (sp2 > c2) {
                    const float k = sqrtf(__fdiv_rn(c2, sp2));
                    v.x = __fmul_rn(v.x, k);
                    v.y = __fmul_rn(v.y, k);
                    v.z = __fmul_rn(v.z, k);
                }
            }
            // taken here rather than at the load: nothing holds it across the stencil loads
            if (KEYS == kKeysChanged) key_old = order_key(p, G, order);
            p.x = __fmaf_rn(v.x, dt_drift, p.x);
            p.y = __fmaf_rn(v.y, dt_drift, p.y);
            p.z = __fmaf_rn(v.z, dt_drift, p.z);
            if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z) || !isfinite(v.x) || !isfinite(v.y) ||
                !isfinite(v.z)) {
                pos_out[i] = make_float4(-1.f, -1.f, -1.f, 0.f);
                vel_out[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (keys_out) keys_out[i] = 0u;
                break;
            }
            if (ISO) {
                if (p.x < 0.002f) { p.x = 0.002f; v.x = __fmul_rn(fabsf(v.x), 0.25f); }
                if (p.x > 0.998f) { p.x = 0.998f; v.x = -__fmul_rn(fabsf(v.x), 0.25f); }
                if (p.y < 0.002f) { p.y = 0.002f; v.y = __fmul_rn(fabsf(v.y), 0.25f); }
                if (p.y > 0.998f) { p.y = 0.998f; v.y = -__fmul_rn(fabsf(v.y), 0.25f); }
                if (p.z < 0.002f) { p.z = 0.002f; v.z = __fmul_rn(fabsf(v.z), 0.25f); }
                if (p.z > 0.998f) { p.z = 0.998f; v.z = -__fmul_rn(fabsf(v.z), 0.25f); }
            } else {
                p.x = __fsub_rn(p.x, floorf(p.x));
                p.y = __fsub_rn(p.y, floorf(p.y));
                p.z = __fsub_rn(p.z, floorf(p.z));
            }
            pos_out[i] = p;
            vel_out[i] = v;
            if (keys_out) {
                key = order_key(p, G, order);
                keys_out[i] = key;
            }
            acc[0][me] += v.x;
            acc[1][me] += v.y;
            acc[2][me] += v.z;
            acc[3][me] += 1.0;
            if (DIAG) {
                acc[4][me] += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z;
                acc[5][me] += (double)phi_p;
            }
        } while (0);
        // The change bit of output i for the next step's merge sort: one word per
        // warp (a warp's outputs are 32 consecutive, aligned indices).
        if (KEYS == kKeysChanged) {
            const unsigned act = __activemask();
            const unsigned b = __ballot_sync(act, key != key_old);
            if (b && (int)(threadIdx.x & 31) == __ffs(act) - 1) atomicOr(chg_words + (i >> 5), b);
        }
        // First sort pass's digit counts of the keys just written: the lanes that
        // share (sort tile, digit) add once. A warp's outputs are consecutive, so
        // they fall in one tile and, the particles being sorted, carry few digits.
        if (KEYS == kKeysCounts) {
            const unsigned pair = (((unsigned)i >> kSortTileShift) << count_bits) | (key & cmask);
            const unsigned peers = __match_any_sync(__activemask(), pair);
            if ((peers & lanemask_lt()) == 0u) atomicAdd(tile_counts + pair, (unsigned)__popc(peers));
        }
    }
    if (partials) {
        if (DIAG) {
            double v6[6] = {acc[0][me], acc[1][me], acc[2][me], acc[3][me], acc[4][me], acc[5][me]};
            block_sum<6>(v6, partials);
        } else {
            double v4[4] = {acc[0][me], acc[1][me], acc[2][me], acc[3][me]};
            block_sum<4>(v4, partials);
        }
    }
}

// Fixed-order sum of the per-block partials; mean = (float)(sum / count).
// With K = 6 it also appends one record to the diagnostics ring rec[cap][8]:
//   {step, kinetic, potential, px, py, pz, live, mean removed |mu|}
// kinetic = sum 1/2 m |v - mu|^2 of the zeroed velocities (from sum |v|^2, sum v
// and the float mean mu actually subtracted), potential = 1/2 m pot_scale sum phi
// at the step-start positions, momentum = m (sum v - live mu), m = 1/N.
template <int K>
__global__ void __launch_bounds__(256) k_finalize_mean(const double* __restrict__ partials, int blocks,
                                                       double* __restrict__ mom_out, float* __restrict__ mean_out,
                                                       double* __restrict__ rec, unsigned long long* __restrict__ rec_n,
                                                       int cap, double mass, double pot_scale) {
    __shared__ double red[K][256];
    double s[K];
#pragma unroll
    for (int j = 0; j < K; ++j) s[j] = 0.0;
    for (int b = threadIdx.x; b < blocks; b += 256)
#pragma unroll
        for (int j = 0; j < K; ++j) s[j] += partials[(size_t)b * K + j];
#pragma unroll
    for (int j = 0; j < K; ++j) red[j][threadIdx.x] = s[j];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o)
#pragma unroll
            for (int j = 0; j < K; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double c = red[3][0];
        float mu[3];
        for (int j = 0; j < 3; ++j) mu[j] = (c >= 1.0) ? (float)(red[j][0] / c) : 0.f;
        if (mom_out)
            for (int j = 0; j < 4; ++j) mom_out[j] = red[j][0];
        if (mean_out)
            for (int j = 0; j < 3; ++j) mean_out[j] = mu[j];
        if (K == 6 && rec) {
            const unsigned long long idx = *rec_n;
            *rec_n = idx + 1;
            double* r = rec + (size_t)(idx % (unsigned long long)cap) * 8;
            double mv = 0.0, mu2 = 0.0;
            for (int j = 0; j < 3; ++j) {
                mv += (double)mu[j] * red[j][0];
                mu2 += (double)mu[j] * mu[j];
            }
            r[0] = (double)idx;
            r[1] = 0.5 * mass * (red[K - 2][0] - 2.0 * mv + c * mu2);
            r[2] = 0.5 * mass * pot_scale * red[K - 1][0];
            for (int j = 0; j < 3; ++j) r[3 + j] = mass * (red[j][0] - c * (double)mu[j]);
            r[6] = c;
            r[7] = sqrt(mu2);
        }
    }
}

__global__ void __launch_bounds__(256) k_interpolate_accel(const float* __restrict__ phi, int G, float h,
                                                           const float4* __restrict__ pos, float4* __restrict__ acc,
                                                           int n, const float4* __restrict__ extra, int S) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (p.x < 0.f) {
        acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    float3 a = S ? gather_accel_iso(phi, G, S, h, p) : gather_accel(phi, G, h, p);
    if (extra) {
        const float4 e = extra[i];
        a.x = __fadd_rn(a.x, e.x);
        a.y = __fadd_rn(a.y, e.y);
        a.z = __fadd_rn(a.z, e.z);
    }
    acc[i] = make_float4(a.x, a.y, a.z, 0.f);
}

__global__ void k_apply_mean(float4* __restrict__ vel, const float4* __restrict__ pos, int n,
                             const float* __restrict__ mean_vel) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || pos[i].x < 0.f) return;
    float4 v = vel[i];
    v.x = __fsub_rn(v.x, mean_vel[0]);
    v.y = __fsub_rn(v.y, mean_vel[1]);
    v.z = __fsub_rn(v.z, mean_vel[2]);
    vel[i] = v;
}

__global__ void k_max_speed(const float4* __restrict__ pos, const float4* __restrict__ vel, int n,
                            const float* __restrict__ mean_vel, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float s = 0.f;
    if (i < n && pos[i].x >= 0.f) {
        float4 v = vel[i];
        if (mean_vel) {
            v.x = __fsub_rn(v.x, mean_vel[0]);
            v.y = __fsub_rn(v.y, mean_vel[1]);
            v.z = __fsub_rn(v.z, mean_vel[2]);
        }
        s = sqrtf(__fmaf_rn(v.z, v.z, __fmaf_rn(v.y, v.y, __fmul_rn(v.x, v.x))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s = fmaxf(s, __shfl_down_sync(0xffffffffu, s, o));
    if ((threadIdx.x & 31) == 0 && s > 0.f) atomicMax(reinterpret_cast<int*>(out), __float_as_int(s));
}

// Kinetic and potential energy and momentum, FP64, two-level fixed order.
// partials: 8 doubles per block: KE, PE, px, py, pz, count, -, -.
__global__ void __launch_bounds__(kGatherThreads) k_energy(const float* __restrict__ phi, int G,
                                                           const float4* __restrict__ pos,
                                                           const float4* __restrict__ vel, int n,
                                                           const float* __restrict__ mean_vel,
                                                           double* __restrict__ partials, int S) {
    double ke = 0.0, pe = 0.0, px = 0.0, py = 0.0, pz = 0.0, c = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        if (p.x < 0.f) continue;
        float4 v = vel[i];
        if (mean_vel) {
            v.x = __fsub_rn(v.x, mean_vel[0]);
            v.y = __fsub_rn(v.y, mean_vel[1]);
            v.z = __fsub_rn(v.z, mean_vel[2]);
        }
        ke += 0.5 * ((double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z);
        px += v.x;
        py += v.y;
        pz += v.z;
        c += 1.0;
        if (phi) {
            int ix, iy, iz;
            float fx, fy, fz;
            cic_axis(p.x, G, ix, fx);
            cic_axis(p.y, G, iy, fy);
            cic_axis(p.z, G, iz, fz);
            const bool per = S == 0;
            const int R = per ? G : S;  // row stride of the potential
            double f = 0.0;
            for (int k = 0; k < 8; ++k) {
                const int cx = cic_cell(ix + (k & 1), G, per), cy = cic_cell(iy + ((k >> 1) & 1), G, per),
                          cz = cic_cell(iz + ((k >> 2) & 1), G, per);
                f += (double)cic_weight(k, fx, fy, fz) * (double)phi[((size_t)cz * R + cy) * R + cx];
            }
            pe += 0.5 * f;
        }
    }
    __shared__ double red[6][kGatherThreads / 32];
    double vals[6] = {ke, pe, px, py, pz, c};
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < 6; ++j)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) vals[j] += __shfl_down_sync(0xffffffffu, vals[j], o);
    if (lane == 0)
#pragma unroll
        for (int j = 0; j < 6; ++j) red[j][w] = vals[j];
    __syncthreads();
    if (threadIdx.x < 8) {
        double s = 0.0;
        if (threadIdx.x < 6)
            for (int k = 0; k < kGatherThreads / 32; ++k) s += red[threadIdx.x][k];
        partials[(size_t)blockIdx.x * 8 + threadIdx.x] = s;
    }
}

__global__ void __launch_bounds__(256) k_finalize8(const double* __restrict__ partials, int blocks,
                                                   double* __restrict__ out) {
    __shared__ double red[8][256];
    double s[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) s[j] = 0.0;
    for (int b = threadIdx.x; b < blocks; b += 256)
#pragma unroll
        for (int j = 0; j < 8; ++j) s[j] += partials[(size_t)b * 8 + j];
#pragma unroll
    for (int j = 0; j < 8; ++j) red[j][threadIdx.x] = s[j];
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o)
#pragma unroll
            for (int j = 0; j < 8; ++j) red[j][threadIdx.x] += red[j][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 8) out[threadIdx.x] = red[threadIdx.x][0];
}

// op 0: sum, 1: max. Grid-stride, 8 partial doubles per block slot (only [0] used).
__global__ void __launch_bounds__(256) k_reduce_grid(const float* __restrict__ a, size_t n, int op,
                                                     double* __restrict__ partials) {
    double acc = (op == 1) ? -INFINITY : 0.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double v = (op == 2) ? (a[i] > 1e-6f ? 1.0 : 0.0) : (double)a[i];
        acc = (op == 1) ? fmax(acc, v) : acc + v;
    }
    __shared__ double red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = (op == 1) ? fmax(red[threadIdx.x], red[threadIdx.x + o])
                                                          : red[threadIdx.x] + red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

__global__ void k_reduce_final(const double* __restrict__ partials, int blocks, int op, double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    double acc = (op == 1) ? -INFINITY : 0.0;
    for (int b = 0; b < blocks; ++b) acc = (op == 1) ? fmax(acc, partials[b]) : acc + partials[b];
    *out = acc;
}

// Per-block sums of x, y and the count of live particles (pos.x >= 0), then one
// thread adds the block sums in block order: the result does not depend on timing.
__global__ void __launch_bounds__(256) k_centroid(const float4* __restrict__ pos, int n, double* __restrict__ partials) {
    double sx = 0.0, sy = 0.0, c = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 p = pos[i];
        if (p.x < 0.f) continue;
        sx += (double)p.x;
        sy += (double)p.y;
        c += 1.0;
    }
    __shared__ double red[3][256];
    red[0][threadIdx.x] = sx;
    red[1][threadIdx.x] = sy;
    red[2][threadIdx.x] = c;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o)
            for (int k = 0; k < 3; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x < 3) partials[3 * blockIdx.x + threadIdx.x] = red[threadIdx.x][0];
}

__global__ void k_centroid_final(const double* __restrict__ partials, int blocks, double* __restrict__ out) {
    if (threadIdx.x >= 3) return;
    double acc = 0.0;
    for (int b = 0; b < blocks; ++b) acc += partials[3 * b + threadIdx.x];
    out[threadIdx.x] = acc;
}

__global__ void k_hide_range(float4* __restrict__ pos, float4* __restrict__ vel, int from, int to) {
    const int i = from + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= to) return;
    pos[i] = make_float4(-1.f, -1.f, -1.f, 0.f);
    vel[i] = make_float4(0.f, 0.f, 0.f, 0.f);
}

}  // namespace

size_t deposit_workspace_bytes(int G) { return align_up(sizeof(long long) * (size_t)G * G * G, 256); }

int launch_deposit_fixed(const float4* pos, int n, int G, long long* acc, cudaStream_t s, int periodic) {
    if (n <= 0) return SD_OK;
    k_deposit_fixed<<<(n + 255) / 256, 256, 0, s>>>(pos, n, G, reinterpret_cast<unsigned long long*>(acc),
                                                     periodic);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_clear_u64(long long* a, size_t n, cudaStream_t s) {
    k_clear_u64<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(reinterpret_cast<unsigned long long*>(a), n);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_fixed_to_float(const long long* acc, int G, float* rho, int clear, cudaStream_t s) {
    const size_t cells = (size_t)G * G * G;
    k_fixed_to_float<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(const_cast<long long*>(acc), cells, rho, clear);
    SD_LAUNCHED(s);
    return SD_OK;
}

size_t gather_partials(int n) {
    const int b = (n + kGatherThreads - 1) / kGatherThreads;
    return (size_t)(b < 1 ? 1 : (b > kGatherMaxBlocks ? kGatherMaxBlocks : b));
}

// Gather CTAs that are resident at once on each device (one full wave): the
// default grid, so every CTA runs the grid-stride loop from start to end with
// no partial last wave. Filled by gather_prepare outside any stream capture.
namespace {
int g_gather_wave[64] = {0};
}

int gather_prepare(int device) {
    if (device < 0 || device >= 64) return SD_OK;
    if (g_gather_wave[device] > 0) return SD_OK;
    int sms = 0, per_sm = 0, per_sm_diag = 0;
    if (SD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) ||
        SD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, k_gather_kick_drift<false, false, false, kKeysChanged>, kGatherThreads, 0)) ||
        SD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm_diag, k_gather_kick_drift<true, false, false, kKeysChanged>, kGatherThreads, 0)))
        return SD_E_CUDA;
    const int w = sms * (per_sm < per_sm_diag ? per_sm : per_sm_diag);
    g_gather_wave[device] = w > 0 ? w : kGatherMaxBlocks;
    return SD_OK;
}

static int gather_wave() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64 || g_gather_wave[dev] <= 0) return kGatherMaxBlocks;
    return g_gather_wave[dev];
}

int launch_gather_kick_drift(const float* phi, int G, float pot_scale, const float4* pos_in, const float4* vel_in,
                             const int* perm, float4* pos_out, float4* vel_out, uint32_t* keys_out, int order, int n,
                             float dt_kick, float dt_drift, float c2, const float* mean_vel, double* partials,
                             double* mom_out, float* mean_out, cudaStream_t s, const float4* extra,
                             int max_blocks, const DiagRecord* diag, int iso_S, unsigned* tile_counts,
                             int count_bits, const float4* press, unsigned* chg_words) {
    if (n <= 0) return SD_OK;
    // particle records are read and written as float4
    if (((uintptr_t)pos_in | (uintptr_t)vel_in | (uintptr_t)pos_out | (uintptr_t)vel_out) & 15u)
        return fail(SD_E_ARG, "gather: pos and vel must be 16-byte aligned");
    const float h = (0.5f * (float)G) * pot_scale;  // Sim.cu:604
    int blocks = (int)gather_partials(n);
    const int cap = max_blocks > 0 ? max_blocks : gather_wave();
    if (blocks > cap) blocks = cap;
    const bool dg = diag && partials;
    // change bits serve the merge sort of the periodic tiled order only
    if (chg_words && (iso_S || tile_counts || !keys_out))
        return fail(SD_E_ARG, "gather: change bits need keys, no tile counts and the periodic box");
    const int keys_mode = chg_words ? kKeysChanged : (tile_counts ? kKeysCounts : kKeysPlain);
#define SD_GATHER(D, I, P, K)                                                                              \
    k_gather_kick_drift<D, I, P, K><<<blocks, kGatherThreads, 0, s>>>(                                         \
        phi, G, h, pos_in, vel_in, perm, pos_out, vel_out, keys_out, order, n, dt_kick, dt_drift, c2, mean_vel, \
        partials, extra, iso_S, tile_counts, count_bits, press, chg_words)
#define SD_GATHER_K(D, I, P)                                          \
    if (keys_mode == kKeysCounts) SD_GATHER(D, I, P, kKeysCounts);    \
    else if (!I && keys_mode == kKeysChanged) SD_GATHER(D, false, P, kKeysChanged); \
    else SD_GATHER(D, I, P, kKeysPlain)
#define SD_GATHER_P(D, I)                \
    if (press) { SD_GATHER_K(D, I, true); } \
    else { SD_GATHER_K(D, I, false); }
    if (iso_S) {
        if (dg) { SD_GATHER_P(true, true); }
        else { SD_GATHER_P(false, true); }
    } else {
        if (dg) { SD_GATHER_P(true, false); }
        else { SD_GATHER_P(false, false); }
    }
#undef SD_GATHER_P
#undef SD_GATHER_K
#undef SD_GATHER
    SD_LAUNCHED(s);
    if (dg) {
        k_finalize_mean<6><<<1, 256, 0, s>>>(partials, blocks, mom_out, mean_out, diag->rec, diag->count, diag->cap,
                                            diag->mass, (double)pot_scale);
        SD_LAUNCHED(s);
    } else if (partials && (mom_out || mean_out)) {
        k_finalize_mean<4><<<1, 256, 0, s>>>(partials, blocks, mom_out, mean_out, nullptr, nullptr, 1, 0.0, 0.0);
        SD_LAUNCHED(s);
    }
    return SD_OK;
}

int launch_interpolate_accel(const float* phi, int G, float pot_scale, const float4* pos, float4* acc, int n,
                             cudaStream_t s, const float4* extra, int iso_S) {
    if (n <= 0) return SD_OK;
    const float h = (0.5f * (float)G) * pot_scale;
    k_interpolate_accel<<<(n + 255) / 256, 256, 0, s>>>(phi, G, h, pos, acc, n, extra, iso_S);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_apply_mean(float4* vel, const float4* pos, int n, const float* mean_vel, cudaStream_t s) {
    if (n <= 0) return SD_OK;
    k_apply_mean<<<(n + 255) / 256, 256, 0, s>>>(vel, pos, n, mean_vel);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_max_speed(const float4* pos, const float4* vel, int n, const float* mean_vel, float* out,
                     cudaStream_t s) {
    if (SD_CUDA(cudaMemsetAsync(out, 0, sizeof(float), s)) != SD_OK) return SD_E_CUDA;
    if (n <= 0) return SD_OK;
    k_max_speed<<<(n + 255) / 256, 256, 0, s>>>(pos, vel, n, mean_vel, out);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_energy(const float* phi, int G, const float4* pos, const float4* vel, int n, const float* mean_vel,
                  double* partials, double* out8, cudaStream_t s, int iso_S) {
    if (n <= 0) return SD_OK;
    const int blocks = (int)gather_partials(n);  // partials hold 8 doubles per block
    k_energy<<<blocks, kGatherThreads, 0, s>>>(phi, G, pos, vel, n, mean_vel, partials, iso_S);
    SD_LAUNCHED(s);
    k_finalize8<<<1, 256, 0, s>>>(partials, blocks, out8);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_reduce_grid(const float* a, size_t cells, int op, double* partials, double* out, cudaStream_t s) {
    const int blocks = 296;
    k_reduce_grid<<<blocks, 256, 0, s>>>(a, cells, op, partials);
    SD_LAUNCHED(s);
    k_reduce_final<<<1, 32, 0, s>>>(partials, blocks, op, out);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_centroid(const float4* pos, int n, double* partials, double* out3, cudaStream_t s) {
    const int blocks = 296;
    k_centroid<<<blocks, 256, 0, s>>>(pos, n, partials);
    SD_LAUNCHED(s);
    k_centroid_final<<<1, 32, 0, s>>>(partials, blocks, out3);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_hide_range(float4* pos, float4* vel, int from, int to, cudaStream_t s) {
    if (to <= from) return SD_OK;
    k_hide_range<<<(to - from + 255) / 256, 256, 0, s>>>(pos, vel, from, to);
    SD_LAUNCHED(s);
    return SD_OK;
}

}  // namespace sd
