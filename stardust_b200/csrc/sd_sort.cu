// sd_sort.cu -- cell keys, stable LSD radix sort and particle reorder.
//
// Replaces kCellKey (Sim.cu:2476-2486), cub::DeviceRadixSort::SortPairs
// (Sim.cu:3659-3667) and kReorder (Sim.cu:2488-2495).
//
// The sort is a classic stable LSD radix sort with 8- to 10-bit digits (the key
// width is split into the fewest passes of at most 10 bits), written for
// sm_100a, in three steps per digit pass:
//   1. digit counts per 2048-key tile, count[t][d]: for the first pass
//      k_digit_counts counts each tile in shared memory and writes one coalesced
//      row; every later pass gets its counts from the scatter before it, which
//      knows where each key lands and adds one count per (tile, digit) run of a
//      warp into a zeroed buffer, so the keys are not read an extra time;
//   2. a column scan over tiles (chunk sums, a per-digit scan of the chunk sums
//      plus the digit bases, a rescan of each chunk) turns the rows into, for
//      every (tile, digit), the global output offset: all keys of smaller digits
//      plus the same digit's keys in earlier tiles, which is what makes the
//      result stable across tiles. Counts from k_digit_counts or added by a
//      scatter bring their chunk sums with them; counts added by the gather that
//      wrote the keys have their chunks summed;
//   3. k_digit_scatter: each tile ranks its keys stably (per warp, in input order,
//      with __match_any_sync on the digit), stages them digit-sorted in shared
//      memory and writes each digit run contiguously; it then clears its row of
//      the offsets, so both count buffers are zero again when the sort ends.
// No kernel waits on another block, so nothing can spin. Keys are key+1 as
// uint32, so the empty slot (reference key -1) sorts first, as CUB does with the
// reference's signed keys.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "sd_common.cuh"
#include "sd_internal.h"

namespace sd {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;  // 2048 keys per tile
static_assert(kSortTile == 1 << kSortTileShift, "sort tile size");
constexpr int kMaxRadixBits = 10;
constexpr int kWarps = kSortThreads / 32;
constexpr int kColChunk = 1 << kSortChunkShift;  // tiles per column-scan chunk
constexpr int kColThreads = 256;
constexpr int kColSegs = kColThreads / 32;  // 8 segments of a column per CTA

__global__ void __launch_bounds__(256) k_cell_keys(const float4* __restrict__ pos, int n, int G, int order,
                                                   uint32_t* __restrict__ keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = order_key(pos[i], G, order);
}

// Inclusive warp scan.
__device__ __forceinline__ unsigned warp_inclusive(unsigned v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan across a 256-thread block; *total receives the block sum.
__device__ __forceinline__ unsigned block_exclusive(unsigned v, unsigned* warp_sums, unsigned* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned inc = warp_inclusive(v);
    if (lane == 31) warp_sums[w] = inc;
    __syncthreads();
    if (w == 0) {
        const unsigned s = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0u;
        const unsigned si = warp_inclusive(s);
        if (lane < (int)(blockDim.x >> 5)) warp_sums[lane] = si - s;
        if (lane == 31) warp_sums[32] = si;
    }
    __syncthreads();
    const unsigned r = warp_sums[w] + inc - v;
    if (total) *total = warp_sums[32];
    __syncthreads();
    return r;
}

template <int BITS>
__global__ void __launch_bounds__(kSortThreads) k_digit_counts(const uint32_t* __restrict__ keys, int n, int shift,
                                                               unsigned* __restrict__ counts,
                                                               unsigned* __restrict__ chunk_sums,
                                                               const int* __restrict__ n_dev) {
    constexpr int kRadix = 1 << BITS;
    constexpr unsigned mask = kRadix - 1;
    __shared__ unsigned hist[kRadix];
    if (n_dev) n = *n_dev;  // a count made on the device; the grid covers at most the capacity
    const int ntiles = (n + kSortTile - 1) / kSortTile;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        for (int d = threadIdx.x; d < kRadix; d += kSortThreads) hist[d] = 0u;
        __syncthreads();
        const int base = tile * kSortTile;
        // Nearly sorted keys put few distinct digits in a warp: one shared add per
        // digit and warp (of the number of lanes holding it) instead of one per key.
        unsigned dd[kSortItems];
#pragma unroll
        for (int it = 0; it < kSortItems; ++it) {
            const int idx = base + it * kSortThreads + threadIdx.x;
            dd[it] = (idx < n) ? ((keys[idx] >> shift) & mask) : 0xffffffffu;
        }
        const unsigned lt = lanemask_lt();
#pragma unroll
        for (int it = 0; it < kSortItems; ++it) {
            const unsigned d = dd[it];
            const unsigned peers = __match_any_sync(0xffffffffu, d);
            if ((peers & lt) == 0u && d != 0xffffffffu) atomicAdd(&hist[d], (unsigned)__popc(peers));
        }
        __syncthreads();
        // tile-major rows: one coalesced row of kRadix counts per tile; with chunk_sums
        // (zero at the start of a sort) each tile also adds into its chunk's sums, so
        // the column scan needs no separate summing pass
        for (int d = threadIdx.x; d < kRadix; d += kSortThreads) {
            const unsigned c = hist[d];
            counts[(size_t)tile * kRadix + d] = c;
            if (chunk_sums && c) atomicAdd(chunk_sums + (size_t)(tile >> kSortChunkShift) * kRadix + d, c);
        }
        __syncthreads();
    }
}

// Shared memory of one scatter tile.
template <int BITS>
struct ScatterSmem {
    // per-warp digit counts fit 16 bits (a warp ranks at most 32 * kSortItems keys)
    unsigned short warp_cnt[kWarps][1 << BITS];
    unsigned local_start[1 << BITS];
    unsigned dst_base[1 << BITS];  // global start of the digit's run minus its local start
    unsigned scan_tmp[33];
    uint32_t skeys[kSortTile];
    int32_t svals[kSortTile];
};

// One tile of k_digit_scatter (n keys in all).
template <int BITS>
__device__ __forceinline__ void scatter_tile(ScatterSmem<BITS>& sm, int tile, const uint32_t* __restrict__ keys_in,
                                             const int32_t* __restrict__ vals_in, uint32_t* __restrict__ keys_out,
                                             int32_t* __restrict__ vals_out, int n, int shift,
                                             unsigned* __restrict__ offsets, unsigned* __restrict__ next_counts,
                                             unsigned* __restrict__ next_sums, int next_shift) {
    constexpr int kRadix = 1 << BITS;
    constexpr unsigned mask = kRadix - 1;
    constexpr int DPT = (kRadix + kSortThreads - 1) / kSortThreads;  // digits per thread
    auto& warp_cnt = sm.warp_cnt;
    auto& local_start = sm.local_start;
    auto& dst_base = sm.dst_base;
    auto& skeys = sm.skeys;
    auto& svals = sm.svals;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kWarps * kRadix; i += kSortThreads) (&warp_cnt[0][0])[i] = 0;
    __syncthreads();

    const int tile0 = tile * kSortTile;
    const unsigned lt = lanemask_lt();
    uint32_t k[kSortItems];
    int32_t v[kSortItems];
    unsigned rank[kSortItems];
    // Each warp owns a contiguous run of 32*kSortItems inputs, visited in order.
    // All of a thread's loads are issued before the ranking, which synchronises
    // the warp after every item.
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int idx = tile0 + w * 32 * kSortItems + it * 32 + lane;
        const bool valid = idx < n;
        k[it] = valid ? keys_in[idx] : 0u;
        v[it] = valid ? (vals_in ? vals_in[idx] : idx) : 0;
    }
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int idx = tile0 + w * 32 * kSortItems + it * 32 + lane;
        const bool valid = idx < n;
        const unsigned d = (k[it] >> shift) & mask;
        const unsigned vmask = __ballot_sync(0xffffffffu, valid);
        unsigned before = 0u, peers = 0u;
        if (valid) {
            peers = __match_any_sync(vmask, d);
            before = warp_cnt[w][d];
        }
        __syncwarp();
        if (valid) {
            rank[it] = before + __popc(peers & lt);
            if ((peers & lt) == 0u) warp_cnt[w][d] = (unsigned short)(before + __popc(peers));
        }
        __syncwarp();
    }
    __syncthreads();

    // Per digit: exclusive scan over warps, then the block-local digit starts.
    unsigned dtot[DPT];
    unsigned tsum = 0u;
#pragma unroll
    for (int j = 0; j < DPT; ++j) {
        const int d = threadIdx.x * DPT + j;
        unsigned run = 0u;
        if (d < kRadix) {
#pragma unroll
            for (int ww = 0; ww < kWarps; ++ww) {
                const unsigned c = warp_cnt[ww][d];
                warp_cnt[ww][d] = (unsigned short)run;
                run += c;
            }
        }
        dtot[j] = run;
        tsum += run;
    }
    __syncthreads();
    {
        unsigned tot;
        unsigned ex = block_exclusive(tsum, sm.scan_tmp, &tot);
#pragma unroll
        for (int j = 0; j < DPT; ++j) {
            const int d = threadIdx.x * DPT + j;
            if (d < kRadix) {
                local_start[d] = ex;
                dst_base[d] = offsets[(size_t)tile * kRadix + d] - ex;
            }
            ex += dtot[j];
        }
    }
    __syncthreads();
    // this tile's row of offsets is consumed: clear it for the next sort
    for (int d = threadIdx.x; d < kRadix; d += kSortThreads) offsets[(size_t)tile * kRadix + d] = 0u;

#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int idx = tile0 + w * 32 * kSortItems + it * 32 + lane;
        if (idx < n) {
            const unsigned d = (k[it] >> shift) & mask;
            const unsigned lp = local_start[d] + warp_cnt[w][d] + rank[it];
            skeys[lp] = k[it];
            svals[lp] = v[it];
        }
    }
    __syncthreads();

    // Digit runs go out contiguously. With next_counts, the next pass's digit of
    // each key is counted for the tile its output position falls in: lanes that
    // share (output tile, next digit) add once, by their lowest lane.
    const int count = min(kSortTile, n - tile0);
#pragma unroll
    for (int it = 0; it < kSortItems; ++it) {
        const int i = it * kSortThreads + threadIdx.x;
        unsigned pair = 0xffffffffu;  // (output tile << BITS | next digit); never all ones
        if (i < count) {
            const uint32_t key = skeys[i];
            const unsigned d = (key >> shift) & mask;
            const unsigned dst = dst_base[d] + (unsigned)i;
            keys_out[dst] = key;
            vals_out[dst] = svals[i];
            pair = ((dst / (unsigned)kSortTile) << BITS) | ((key >> next_shift) & mask);
        }
        if (next_counts) {
            const unsigned peers = __match_any_sync(0xffffffffu, pair);
            if (pair != 0xffffffffu && (peers & lt) == 0u) {
                const unsigned c = (unsigned)__popc(peers), t = pair >> BITS, d = pair & mask;
                atomicAdd(next_counts + (size_t)t * kRadix + d, c);
                atomicAdd(next_sums + (size_t)(t >> kSortChunkShift) * kRadix + d, c);
            }
        }
    }
}

// LOOP: the key count comes from the device (n_dev) and the grid loops over the
// tiles in use; otherwise one CTA per tile (no loop state held across tiles).
template <int BITS, bool LOOP>
__global__ void __launch_bounds__(kSortThreads) k_digit_scatter(const uint32_t* __restrict__ keys_in,
                                                                const int32_t* __restrict__ vals_in,
                                                                uint32_t* __restrict__ keys_out,
                                                                int32_t* __restrict__ vals_out, int n, int shift,
                                                                unsigned* __restrict__ offsets,
                                                                unsigned* __restrict__ next_counts,
                                                                unsigned* __restrict__ next_sums, int next_shift,
                                                                const int* __restrict__ n_dev) {
    __shared__ ScatterSmem<BITS> sm;
    if (!LOOP) {
        scatter_tile<BITS>(sm, blockIdx.x, keys_in, vals_in, keys_out, vals_out, n, shift, offsets, next_counts,
                           next_sums, next_shift);
        return;
    }
    n = *n_dev;  // a count made on the device; the grid covers at most the capacity
    const int ntiles = (n + kSortTile - 1) / kSortTile;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        scatter_tile<BITS>(sm, tile, keys_in, vals_in, keys_out, vals_out, n, shift, offsets, next_counts, next_sums,
                           next_shift);
        __syncthreads();  // the tile's shared memory is read to the end before the next one
    }
}

// Exclusive offsets of the tile-major digit counts counts[tile][digit]:
//   offset(t, d) = base(d) + sum_{t' < t} counts[t'][d],  base(d) = sum_{d' < d} total(d'),
// over chunks of kColChunk tiles and slabs of 32 digits, so every global access
// is a coalesced 128-byte row piece and every chain of dependent adds is short:
//   k_col_sums   S[c][d] = chunk sums (first pass only)
//   k_col_prefix S[c][d] -> exclusive prefix over chunks, T[d] = digit totals;
//                the last CTA to finish turns T into the digit bases base(d)
//   k_col_apply  counts[t][d] -> base(d) + S[c][d] + prefix within the chunk,
//                and clears S, ready for the adds of the next counts

// Tiles holding n keys (n from the device when n_dev is set: the grids cover the capacity).
__device__ __forceinline__ int tiles_of(int tiles, const int* n_dev) {
    return n_dev ? (*n_dev + kSortTile - 1) / kSortTile : tiles;
}

__global__ void __launch_bounds__(kColThreads) k_col_sums(const unsigned* __restrict__ counts, int tiles, int radix,
                                                          unsigned* __restrict__ S, const int* __restrict__ n_dev) {
    const int d = blockIdx.y * kColThreads + threadIdx.x;
    tiles = tiles_of(tiles, n_dev);
    if (d >= radix) return;
    for (int c = blockIdx.x; c * kColChunk < tiles; c += gridDim.x) {
        const int t0 = c * kColChunk, t1 = min(tiles, t0 + kColChunk);
        unsigned s = 0u;
#pragma unroll 8
        for (int t = t0; t < t1; ++t) s += counts[(size_t)t * radix + d];
        S[(size_t)c * radix + d] = s;
    }
}

// CTA per 32-digit slab: thread (seg, lane) owns digit slab*32 + lane and a
// contiguous run of chunks; two sweeps (sum, rewrite) around a scan of the runs.
__global__ void __launch_bounds__(kColThreads) k_col_prefix(unsigned* __restrict__ S, int chunks, int radix,
                                                            unsigned* __restrict__ T, unsigned* __restrict__ done,
                                                            const int* __restrict__ n_dev) {
    __shared__ unsigned seg_sum[kColSegs][32];
    __shared__ unsigned scan_tmp[33];
    __shared__ bool last;
    if (n_dev) chunks = (tiles_of(0, n_dev) + kColChunk - 1) / kColChunk;
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5;
    const int d = blockIdx.x * 32 + lane;
    const int per = (chunks + kColSegs - 1) / kColSegs;
    const int c0 = seg * per, c1 = min(chunks, c0 + per);
    unsigned sum = 0u;
    if (d < radix) {
#pragma unroll 8
        for (int c = c0; c < c1; ++c) sum += S[(size_t)c * radix + d];
    }
    seg_sum[seg][lane] = sum;
    __syncthreads();
    unsigned run = 0u, tot = 0u;
    for (int j = 0; j < kColSegs; ++j) {
        const unsigned v = seg_sum[j][lane];
        if (j < seg) run += v;
        tot += v;
    }
    if (d < radix) {
        for (int cb = c0; cb < c1; cb += 8) {
            unsigned v[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = (cb + j < c1) ? S[(size_t)(cb + j) * radix + d] : 0u;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                if (cb + j < c1) S[(size_t)(cb + j) * radix + d] = run;
                run += v[j];
            }
        }
        if (seg == 0) T[d] = tot;
    }
    // The last CTA to finish (counted on `done`, which it resets) sees every
    // total and replaces them by their exclusive scan over the digits.
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    constexpr int kPer = (1 << kMaxRadixBits) / kColThreads;
    unsigned v[kPer], mine = 0u;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int dd = threadIdx.x * kPer + j;
        v[j] = (dd < radix) ? __ldcg(T + dd) : 0u;
        mine += v[j];
    }
    unsigned ex = block_exclusive(mine, scan_tmp, nullptr);
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int dd = threadIdx.x * kPer + j;
        if (dd < radix) T[dd] = ex;
        ex += v[j];
    }
    if (threadIdx.x == 0) *done = 0u;
}

// CTA per (chunk, 32-digit slab): the chunk's 64 x 32 counts staged in shared
// memory, scanned down each column in 8 segments of 8 tiles.
__global__ void __launch_bounds__(kColThreads) k_col_apply(unsigned* __restrict__ counts, int tiles, int radix,
                                                           unsigned* __restrict__ S,
                                                           const unsigned* __restrict__ T,
                                                           const int* __restrict__ n_dev) {
    __shared__ unsigned tile[kColChunk][33];
    __shared__ unsigned seg_sum[kColSegs][32];
    const int lane = threadIdx.x & 31, seg = threadIdx.x >> 5;
    const int d = blockIdx.y * 32 + lane;
    tiles = tiles_of(tiles, n_dev);
    for (int c = blockIdx.x; c * kColChunk < tiles; c += gridDim.x) {
        const int t0 = c * kColChunk, rows = min(tiles - t0, kColChunk);
        constexpr int kRowsPerSeg = kColChunk / kColSegs;
#pragma unroll
        for (int j = 0; j < kRowsPerSeg; ++j) {
            const int r = seg + j * kColSegs;
            tile[r][lane] = (r < rows && d < radix) ? counts[(size_t)(t0 + r) * radix + d] : 0u;
        }
        __syncthreads();
        unsigned sum = 0u;
#pragma unroll
        for (int j = 0; j < kRowsPerSeg; ++j) sum += tile[seg * kRowsPerSeg + j][lane];
        seg_sum[seg][lane] = sum;
        __syncthreads();
        unsigned run = (d < radix) ? T[d] + S[(size_t)c * radix + d] : 0u;
        for (int j = 0; j < seg; ++j) run += seg_sum[j][lane];
        __syncthreads();  // every segment has read S[c][d] and seg_sum
        if (seg == 0 && d < radix) S[(size_t)c * radix + d] = 0u;
#pragma unroll
        for (int j = 0; j < kRowsPerSeg; ++j) {
            const int r = seg * kRowsPerSeg + j;
            const unsigned v = tile[r][lane];
            tile[r][lane] = run;
            run += v;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kRowsPerSeg; ++j) {
            const int r = seg + j * kColSegs;
            if (r < rows && d < radix) counts[(size_t)(t0 + r) * radix + d] = tile[r][lane];
        }
        __syncthreads();  // the staged chunk is written out before the next one is loaded
    }
}

__global__ void __launch_bounds__(256) k_reorder(const float4* __restrict__ pos_in, const float4* __restrict__ vel_in,
                                                 const int32_t* __restrict__ perm, float4* __restrict__ pos_out,
                                                 float4* __restrict__ vel_out, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int j = perm[i];
    pos_out[i] = pos_in[j];
    vel_out[i] = vel_in[j];
}

__global__ void k_copy_keys(const uint32_t* __restrict__ kin, const int32_t* __restrict__ vin,
                            uint32_t* __restrict__ kout, int32_t* __restrict__ vout, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    kout[i] = kin[i];
    vout[i] = vin ? vin[i] : i;
}

// Sorted row keys (tiled order: key = row, below `rows`) -> row_start[r] = first
// position whose key is >= r, r = 0..rows (row_start[rows] = n). Thread per
// position i in [0, n]: the rows r in (key[i-1], key[i]] start at i (position 0
// takes the rows up to key[0], position n the rows after key[n-1]). One coalesced
// pass over the keys instead of a lower-bound search per row (a chain of dependent
// loads): a short run of empty rows is written by its own thread, a longer one is
// queued and written by the whole CTA, so no thread walks a long empty stretch of
// a clustered scene alone. Above 2^20 keys the CTAs of this pass outnumber a few
// waves and a lower-bound search per row (k_row_bounds) is faster (4M keys of the
// two-galaxy scene on 256^3: search 0.013 ms, this pass 0.017 ms; 262,144 keys of
// the disk on 64^3: search 0.011 ms, this pass 0.007 ms).
constexpr int kRowShortRun = 8;
__global__ void __launch_bounds__(256) k_row_marks(const uint32_t* __restrict__ keys, int n, int rows,
                                                   int* __restrict__ row_start) {
    __shared__ int q_lo[256], q_hi[256], q_val[256];
    __shared__ int q_count;
    if (threadIdx.x == 0) q_count = 0;
    __syncthreads();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i <= n) {
        const int prev = (i == 0) ? -1 : (int)__ldg(keys + i - 1);
        const int cur = (i == n) ? rows : (int)__ldg(keys + i);
        const int run = cur - prev;  // rows prev + 1 .. cur
        if (run > kRowShortRun) {
            const int slot = atomicAdd(&q_count, 1);
            q_lo[slot] = prev + 1;
            q_hi[slot] = cur;
            q_val[slot] = i;
        } else {
            for (int r = prev + 1; r <= cur; ++r) row_start[r] = i;
        }
    }
    __syncthreads();
    for (int q = 0; q < q_count; ++q)
        for (int r = q_lo[q] + (int)threadIdx.x; r <= q_hi[q]; r += blockDim.x) row_start[r] = q_val[q];
}

// One thread per row: a lower-bound search over the keys.
__global__ void k_row_bounds(const uint32_t* __restrict__ keys, int n, int rows, int* __restrict__ row_start) {
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r > rows) return;
    int lo = 0, len = n;
    while (len > 0) {
        const int half = len >> 1;
        if (__ldg(keys + lo + half) < (uint32_t)r) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    row_start[r] = lo;
}

}  // namespace

int launch_row_bounds(const uint32_t* keys, int n, int rows, int* row_start, cudaStream_t s) {
    if (n <= (1 << 20))
        k_row_marks<<<(n + 1 + 255) / 256, 256, 0, s>>>(keys, n, rows, row_start);
    else
        k_row_bounds<<<(rows + 1 + 255) / 256, 256, 0, s>>>(keys, n, rows, row_start);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_cell_keys(const float4* pos, int n, int G, int order, uint32_t* keys, cudaStream_t s) {
    if (n <= 0) return SD_OK;
    k_cell_keys<<<(n + 255) / 256, 256, 0, s>>>(pos, n, G, order, keys);
    SD_LAUNCHED(s);
    return SD_OK;
}

static int col_chunks(int tiles) { return (tiles + kColChunk - 1) / kColChunk; }

// Grid of a tile- or chunk-looping kernel: one CTA per unit for a count known on
// the host; for a count on the device (at most `units`), at most `cap` CTAs.
static int loop_grid(int units, const int* n_dev, int cap) { return n_dev ? std::min(units, cap) : units; }
constexpr int kNumSMs = 148;

// Workspace: two count buffers of tiles x radix (the pass being scattered and
// the next pass's counts), the chunk sums S[chunks][radix], the digit totals /
// bases T[radix] and the column scan's finish counter.
struct SortWs {
    unsigned* cnt[2];
    unsigned* S;
    unsigned* T;
    unsigned* done;
};

static size_t counts_bytes(int tiles) {
    return align_up(((size_t)1 << kMaxRadixBits) * tiles * sizeof(unsigned), 256);
}
static size_t sums_bytes(int tiles) {
    return align_up(((size_t)1 << kMaxRadixBits) * col_chunks(tiles) * sizeof(unsigned), 256);
}

static SortWs sort_ws_layout(void* ws, int n) {
    const int tiles = std::max(1, (n + kSortTile - 1) / kSortTile);
    char* b = (char*)ws;
    SortWs w;
    w.cnt[0] = (unsigned*)b;
    w.cnt[1] = (unsigned*)(b + counts_bytes(tiles));
    w.S = (unsigned*)(b + 2 * counts_bytes(tiles));
    w.T = (unsigned*)(b + 2 * counts_bytes(tiles) + sums_bytes(tiles));
    w.done = w.T + ((size_t)1 << kMaxRadixBits);
    return w;
}

size_t sort_workspace_bytes(int n) {
    const int tiles = std::max(1, (n + kSortTile - 1) / kSortTile);
    return 2 * counts_bytes(tiles) + sums_bytes(tiles) +
           align_up(((size_t)1 << kMaxRadixBits) * sizeof(unsigned) + sizeof(unsigned), 256);
}

static int col_sums(const unsigned* counts, int tiles, int radix, unsigned* S, cudaStream_t s, const int* n_dev) {
    k_col_sums<<<dim3(loop_grid(col_chunks(tiles), n_dev, kNumSMs), (radix + kColThreads - 1) / kColThreads),
                 kColThreads, 0, s>>>(
        counts, tiles, radix, S, n_dev);
    SD_LAUNCHED(s);
    return SD_OK;
}

// counts[tiles][radix] (tile-major) with their chunk sums in w.S -> exclusive
// global offsets, in place; leaves w.S zero.
static int scan_offsets(unsigned* counts, int tiles, int radix, const SortWs& w, cudaStream_t s, const int* n_dev) {
    const int chunks = col_chunks(tiles);
    const int slabs = (radix + 31) / 32;
    k_col_prefix<<<slabs, kColThreads, 0, s>>>(w.S, chunks, radix, w.T, w.done, n_dev);
    SD_LAUNCHED(s);
    k_col_apply<<<dim3(loop_grid(chunks, n_dev, kNumSMs), slabs), kColThreads, 0, s>>>(counts, tiles, radix, w.S,
                                                                                          w.T, n_dev);
    SD_LAUNCHED(s);
    return SD_OK;
}

int sort_digit_bits(int key_bits) {
    // fewest passes of at most kMaxRadixBits bits, then the even digit width (8, 9 or 10)
    const int passes = (key_bits + kMaxRadixBits - 1) / kMaxRadixBits;
    if (passes <= 0) return 0;
    const int even = (key_bits + passes - 1) / passes;
    return even <= 8 ? 8 : even;
}

unsigned* sort_first_counts(void* ws) { return (unsigned*)ws; }

int launch_sort_first_counts(const uint32_t* keys, int n, int key_bits, void* ws, size_t ws_bytes, cudaStream_t s) {
    const int bits = sort_digit_bits(key_bits);
    if (n <= 0 || bits == 0) return SD_OK;
    if (!keys || !ws || ws_bytes < sort_workspace_bytes(n)) return fail(SD_E_ARG, "sort counts: bad workspace");
    const int tiles = (n + kSortTile - 1) / kSortTile;
    const SortWs w = sort_ws_layout(ws, n);
    switch (bits) {
        case 8: k_digit_counts<8><<<tiles, kSortThreads, 0, s>>>(keys, n, 0, w.cnt[0], nullptr, nullptr); break;
        case 9: k_digit_counts<9><<<tiles, kSortThreads, 0, s>>>(keys, n, 0, w.cnt[0], nullptr, nullptr); break;
        default: k_digit_counts<10><<<tiles, kSortThreads, 0, s>>>(keys, n, 0, w.cnt[0], nullptr, nullptr); break;
    }
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_sort_pairs(const uint32_t* keys_in, const int32_t* vals_in, uint32_t* keys_out, int32_t* vals_out,
                      uint32_t* keys_tmp, int32_t* vals_tmp, int n, int key_bits, void* ws, size_t ws_bytes,
                      cudaStream_t s, bool ws_zeroed, bool first_counts_ready, const int* n_dev) {
    if (n < 0 || key_bits < 0 || key_bits > 32) return fail(SD_E_ARG, "sort: bad n=%d or key_bits=%d", n, key_bits);
    if (n == 0) return SD_OK;
    if (!keys_in || !keys_out || !vals_out || !keys_tmp || !vals_tmp || !ws)
        return fail(SD_E_ARG, "sort: null buffer");
    if (ws_bytes < sort_workspace_bytes(n)) return fail(SD_E_ARG, "sort: workspace too small");
    if (keys_in == keys_out || (vals_in && vals_in == vals_out))
        return fail(SD_E_ARG, "sort: input and output buffers must differ");
    // fewest passes of at most kMaxRadixBits bits
    const int passes = (key_bits + kMaxRadixBits - 1) / kMaxRadixBits;
    if (passes == 0) {
        k_copy_keys<<<(n + 255) / 256, 256, 0, s>>>(keys_in, vals_in, keys_out, vals_out, n);
        SD_LAUNCHED(s);
        return SD_OK;
    }
    const int bits = sort_digit_bits(key_bits);
    const int tiles = (n + kSortTile - 1) / kSortTile;
    const SortWs w = sort_ws_layout(ws, n);
    unsigned* const* cnt = w.cnt;
    // a count on the device: grids of about one wave that loop over the tiles in use
    const int count_grid = loop_grid(tiles, n_dev, kNumSMs * 8);
    const int scatter_grid = loop_grid(tiles, n_dev, kNumSMs * 4);
    // The count kernel and the scatters add chunk sums into w.S and the scatters add
    // the next pass's counts into the second buffer, so both must start at zero, and
    // the column scan counts its CTAs on w.done; a sort leaves all three zero, so a
    // workspace that only ever serves this sort is cleared once.
    if (!ws_zeroed && (SD_CUDA(cudaMemsetAsync(cnt[1], 0, sizeof(unsigned) * ((size_t)tiles << bits), s)) ||
                       SD_CUDA(cudaMemsetAsync(w.S, 0, sizeof(unsigned) * ((size_t)col_chunks(tiles) << bits), s)) ||
                       SD_CUDA(cudaMemsetAsync(w.done, 0, sizeof(unsigned), s))))
        return SD_E_CUDA;

    const uint32_t* kin = keys_in;
    const int32_t* vin = vals_in;
    for (int p = 0; p < passes; ++p) {
        const int shift = p * bits;  // passes * bits >= key_bits
        // the last pass lands in *_out; earlier passes alternate so that holds
        const bool to_out = ((passes - 1 - p) % 2) == 0;
        uint32_t* kout = to_out ? keys_out : keys_tmp;
        int32_t* vout = to_out ? vals_out : vals_tmp;
        int rc = SD_OK;
        unsigned* counts = cnt[p & 1];
        unsigned* next = (p + 1 < passes) ? cnt[(p + 1) & 1] : nullptr;
        const int next_shift = (p + 1) * bits;
        // key bits above key_bits are zero, so a last digit reaching past them is exact
        if (p == 0 && !first_counts_ready) {
            const int g = count_grid;
            switch (bits) {
                case 8: k_digit_counts<8><<<g, kSortThreads, 0, s>>>(kin, n, shift, counts, w.S, n_dev); break;
                case 9: k_digit_counts<9><<<g, kSortThreads, 0, s>>>(kin, n, shift, counts, w.S, n_dev); break;
                default: k_digit_counts<10><<<g, kSortThreads, 0, s>>>(kin, n, shift, counts, w.S, n_dev); break;
            }
            SD_LAUNCHED(s);
        }
        // first-pass counts made elsewhere (the gather, launch_sort_first_counts) still
        // need their chunk sums; the count kernel above and the scatters add theirs
        if (p == 0 && first_counts_ready && (rc = col_sums(counts, tiles, 1 << bits, w.S, s, n_dev))) return rc;
        if ((rc = scan_offsets(counts, tiles, 1 << bits, w, s, n_dev))) return rc;
#define SD_SCATTER(B, L)                                                                                   \
    k_digit_scatter<B, L><<<scatter_grid, kSortThreads, 0, s>>>(kin, vin, kout, vout, n, shift, counts, next, w.S, \
                                                                next_shift, n_dev)
#define SD_SCATTER_B(B)        \
    if (n_dev) SD_SCATTER(B, true); \
    else SD_SCATTER(B, false)
        switch (bits) {
            case 8: SD_SCATTER_B(8); break;
            case 9: SD_SCATTER_B(9); break;
            default: SD_SCATTER_B(10); break;
        }
#undef SD_SCATTER_B
#undef SD_SCATTER
        SD_LAUNCHED(s);
        kin = kout;
        vin = vout;
    }
    return SD_OK;
}

int launch_reorder(const float4* pos_in, const float4* vel_in, const int32_t* perm, float4* pos_out,
                   float4* vel_out, int n, cudaStream_t s) {
    if (n <= 0) return SD_OK;
    k_reorder<<<(n + 255) / 256, 256, 0, s>>>(pos_in, vel_in, perm, pos_out, vel_out, n);
    SD_LAUNCHED(s);
    return SD_OK;
}

}  // namespace sd
