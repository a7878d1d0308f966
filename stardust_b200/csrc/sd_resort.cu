// sd_resort.cu -- the step's sort as a merge, for the tiled order.
//
// Between two steps a particle's row key changes only when it crosses a row:
// a fraction of a percent of the particles on the 16M/512^3 field. The previous
// step left the particles sorted by their old keys, its row table
// (row_start[r] = first position with old key >= r) and, from its gather, the
// new key of every position plus a bit per position saying whether it changed.
// The stable sort of the new keys is then the merge of
//   U  the unchanged positions, already in (key, position) order, and
//   C  the changed ones, radix-sorted by key (stable, so in position order
//      within a key),
// ordered by (key, position) -- exactly the stable sort's order. Every output
// slot follows from counts, with no search over the whole array:
//   changed  (k, i) at rank r in C:  r + #U before it, where the unchanged
//            positions before it are those below row_start[k] plus those in
//            [row_start[k], row_start[k+1]) below i, less the changed ones
//            among them (prefix counts of the change bits);
//   unchanged (k, j):  j - #changed below j + #C with key < k (a row table of
//            the sorted C) + #C with key k and position < j.
// The new row table needs no pass over the keys either: the positions below
// row r are the unchanged ones below the old row_start[r] plus the changed
// ones with key < r. The permutation is the one the radix sort gives; the
// sorted keys themselves are not written (the row table is all the step reads).
// Every formula holds for any set of marked positions that contains the changed
// ones: a marked position whose key did not change simply goes through C, so
// bits left over from a step whose merge never ran cost time, not correctness.
//
// Kernels, in order (the size of C stays on the device throughout):
//   k_chg_count      changed positions per chunk of 512 words
//   k_chg_compact    per word: changed positions before it; C in position order
//   (radix sort of C by key, on grids of about one wave looping over its tiles)
//   k_merge_changed  output slot of every C entry
//   k_rows           row table of C (a galloping search per row) and the new row table
//   k_merge_unchanged output slot of every unchanged position; clears the bits
#include <cuda_runtime.h>
#include <stdint.h>

#include "sd_common.cuh"
#include "sd_internal.h"

namespace sd {
namespace {

constexpr int kChgThreads = 64;
constexpr int kChgWordsPer = 8;                          // words per thread, two 16-byte loads
constexpr int kChunkWords = kChgThreads * kChgWordsPer;  // 512 words = 16,384 positions
constexpr int kMergeThreads = 256;
constexpr int kMergeWordsPerWarp = 8;                            // 256 positions per warp
constexpr int kMergeWords = (kMergeThreads / 32) * kMergeWordsPerWarp;  // words per CTA

__device__ __forceinline__ unsigned block_sum(unsigned v, unsigned* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[w] = v;
    __syncthreads();
    unsigned t = 0u;
#pragma unroll
    for (int k = 0; k < kChgThreads / 32; ++k) t += red[k];
    __syncthreads();
    return t;
}

// Exclusive scan across the block; *total receives the block sum.
__device__ __forceinline__ unsigned block_exclusive(unsigned v, unsigned* red, unsigned* total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned inc = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned t = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += t;
    }
    if (lane == 31) red[w] = inc;
    __syncthreads();
    unsigned before = 0u, tot = 0u;
#pragma unroll
    for (int k = 0; k < kChgThreads / 32; ++k) {
        const unsigned s = red[k];
        if (k < w) before += s;
        tot += s;
    }
    __syncthreads();
    *total = tot;
    return before + inc - v;
}

__device__ __forceinline__ void load_words8(const unsigned* __restrict__ p, unsigned (&w)[8]) {
    const uint4 a = *reinterpret_cast<const uint4*>(p);
    const uint4 b = *reinterpret_cast<const uint4*>(p + 4);
    w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
    w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
}

// Changed positions in each chunk of kChunkWords words (the word buffers are
// padded to whole chunks, and the padding stays zero).
__global__ void __launch_bounds__(kChgThreads) k_chg_count(const unsigned* __restrict__ words,
                                                           unsigned* __restrict__ chunk_cnt) {
    __shared__ unsigned red[kChgThreads / 32];
    unsigned w[8];
    load_words8(words + (size_t)blockIdx.x * kChunkWords + threadIdx.x * kChgWordsPer, w);
    unsigned c = 0u;
#pragma unroll
    for (int q = 0; q < 8; ++q) c += __popc(w[q]);
    c = block_sum(c, red);
    if (threadIdx.x == 0) chunk_cnt[blockIdx.x] = c;
}

// CTA per chunk: the changed positions before each word (word_pre) and C =
// (new key, position) of the changed positions, in position order. The last
// CTA writes the size of C.
__global__ void __launch_bounds__(kChgThreads) k_chg_compact(const unsigned* __restrict__ words,
                                                             const unsigned* __restrict__ chunk_cnt,
                                                             const uint32_t* __restrict__ keys,
                                                             unsigned* __restrict__ word_pre, uint32_t* __restrict__ ck,
                                                             int32_t* __restrict__ ci, int* __restrict__ n_changed) {
    __shared__ unsigned red[kChgThreads / 32];
    unsigned before = 0u;  // changed positions in the chunks before this one
    for (int c0 = 0; c0 < (int)blockIdx.x; c0 += 8 * kChgThreads) {  // eight loads in flight per thread
        unsigned v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int c = c0 + q * kChgThreads + threadIdx.x;
            v[q] = (c < (int)blockIdx.x) ? chunk_cnt[c] : 0u;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) before += v[q];
    }
    before = block_sum(before, red);
    const size_t w0 = (size_t)blockIdx.x * kChunkWords + threadIdx.x * kChgWordsPer;
    unsigned w[8];
    load_words8(words + w0, w);
    unsigned c[8], tsum = 0u;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        c[q] = __popc(w[q]);
        tsum += c[q];
    }
    unsigned total;
    unsigned base = before + block_exclusive(tsum, red, &total);
    uint4 pa, pb;
    pa.x = base; pa.y = pa.x + c[0]; pa.z = pa.y + c[1]; pa.w = pa.z + c[2];
    pb.x = pa.w + c[3]; pb.y = pb.x + c[4]; pb.z = pb.y + c[5]; pb.w = pb.z + c[6];
    *reinterpret_cast<uint4*>(word_pre + w0) = pa;
    *reinterpret_cast<uint4*>(word_pre + w0 + 4) = pb;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        unsigned b = w[q];
        while (b) {
            const int pos = (int)((w0 + q) * 32) + __ffs(b) - 1;
            b &= b - 1u;
            ck[base] = keys[pos];
            ci[base] = pos;
            ++base;
        }
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) *n_changed = (int)(before + total);
}

// Changed positions below x (0 <= x <= n; the padding words are zero).
__device__ __forceinline__ unsigned changed_below(const unsigned* __restrict__ words,
                                                  const unsigned* __restrict__ word_pre, int x) {
    const unsigned m = (1u << (x & 31)) - 1u;
    return word_pre[x >> 5] + __popc(words[x >> 5] & m);
}

__global__ void k_merge_changed(const uint32_t* __restrict__ ck, const int32_t* __restrict__ ci,
                                const int* __restrict__ n_changed, const int* __restrict__ row_start_old,
                                const unsigned* __restrict__ words, const unsigned* __restrict__ word_pre,
                                int32_t* __restrict__ vals_out) {
    const int nc = *n_changed;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nc; r += gridDim.x * blockDim.x) {
        const uint32_t k = ck[r];
        const int i = ci[r];
        const int lb = row_start_old[k], ub = row_start_old[k + 1];
        const unsigned cl = changed_below(words, word_pre, lb);
        unsigned u = (unsigned)lb - cl;
        if (i > lb) {
            const int m = min(ub, i);
            u += (unsigned)(m - lb) - (changed_below(words, word_pre, m) - cl);
        }
        vals_out[r + u] = i;
    }
}

// Thread per row r in [0, rows]: c_rows[r] = first rank of C with key >= r, and
// the new row start = unchanged positions below the old one + c_rows[r]. The
// search starts where r would fall if C were spread evenly over the rows and
// gallops outwards to a bracket, which a few steps find for an even spread.
__global__ void k_rows(const uint32_t* __restrict__ ck, const int* __restrict__ n_changed, int rows,
                       const unsigned* __restrict__ words, const unsigned* __restrict__ word_pre,
                       int* __restrict__ c_rows, int* __restrict__ row_start) {
    const int nc = *n_changed;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r <= rows; r += gridDim.x * blockDim.x) {
        // bracket [lo, hi] with ck[lo - 1] < r <= ck[hi] (ck[-1] = -inf, ck[nc] = +inf)
        const int g = (int)(((long long)r * nc) / (rows > 0 ? rows : 1));
        int lo, hi;
        if (g < nc && ck[g] < (uint32_t)r) {  // the answer lies above g
            int step = 1;
            lo = g + 1;
            hi = g + 1;
            while (hi < nc && ck[hi] < (uint32_t)r) {
                lo = hi + 1;
                hi = min(nc, hi + step);
                step <<= 1;
            }
        } else {  // at or below g
            int step = 1;
            hi = g;
            lo = g;
            while (lo > 0 && ck[lo - 1] >= (uint32_t)r) {
                hi = lo - 1;
                lo = max(0, lo - step);
                step <<= 1;
            }
        }
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (ck[mid] < (uint32_t)r) lo = mid + 1;
            else hi = mid;
        }
        c_rows[r] = lo;
        const int rs = row_start[r];
        row_start[r] = rs - (int)changed_below(words, word_pre, rs) + lo;
    }
}

// Warp per 8 words (256 positions, lane-major: position = base + 32 q + lane), all
// loads issued before use. The changed positions were placed by k_merge_changed.
// Clears the change bits for the next gather.
__global__ void __launch_bounds__(kMergeThreads) k_merge_unchanged(const uint32_t* __restrict__ keys,
                                                                   unsigned* __restrict__ words,
                                                                   const unsigned* __restrict__ word_pre,
                                                                   const int* __restrict__ c_rows,
                                                                   const int32_t* __restrict__ ci, int n,
                                                                   int32_t* __restrict__ vals_out) {
    const int lane = threadIdx.x & 31;
    const size_t wb = (size_t)blockIdx.x * kMergeWords + (threadIdx.x >> 5) * kMergeWordsPerWarp;
    const int base = (int)(wb * 32);
    if (base >= n) return;
    unsigned bits[8], pre[8];
    load_words8(words + wb, bits);
    load_words8(word_pre + wb, pre);
    uint32_t k[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int j = base + q * 32 + lane;
        k[q] = (j < n) ? keys[j] : 0u;
    }
    int lo[8], hi[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        lo[q] = c_rows[k[q]];
        hi[q] = c_rows[k[q] + 1];
    }
    const unsigned lt = lanemask_lt();
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        const int j = base + q * 32 + lane;
        if (j < n && !((bits[q] >> lane) & 1u)) {
            // C entries with key k lie at ranks [c_rows[k], c_rows[k+1]) in position order
            int a = lo[q], b = hi[q];
            while (a < b) {  // first rank whose position is above j
                const int mid = (a + b) >> 1;
                if (ci[mid] < j) a = mid + 1;
                else b = mid;
            }
            vals_out[j - (int)(pre[q] + __popc(bits[q] & lt)) + a] = j;
        }
    }
    __syncwarp();
    if (lane < kMergeWordsPerWarp) words[wb + lane] = 0u;  // every lane has used them
}

// Words for n positions plus one (changed_below(n) reads word n / 32), in whole chunks.
size_t padded_words(int n) {
    const size_t w = (size_t)n / 32 + 1;
    return (w + kChunkWords - 1) / kChunkWords * kChunkWords;
}

}  // namespace

size_t resort_words(int n) { return padded_words(n); }

size_t resort_bytes(int n, int G) {
    const size_t words = padded_words(n), chunks = words / kChunkWords;
    return align_up(sizeof(unsigned) * words, 256) * 2 + align_up(sizeof(unsigned) * chunks, 256) +
           align_up(sizeof(int32_t) * ((size_t)G * G + 1), 256) + align_up(sizeof(int), 256) +
           3 * align_up(sizeof(uint32_t) * (size_t)n, 256);
}

ResortBufs resort_layout(void* base, int n, int G, uint32_t* spare_k0, int32_t* spare_v0, uint32_t* spare_k1) {
    const size_t words = padded_words(n), chunks = words / kChunkWords;
    char* b = (char*)base;
    ResortBufs r;
    r.words = (unsigned*)b;
    b += align_up(sizeof(unsigned) * words, 256);
    r.word_pre = (unsigned*)b;
    b += align_up(sizeof(unsigned) * words, 256);
    r.chunk_cnt = (unsigned*)b;
    b += align_up(sizeof(unsigned) * chunks, 256);
    r.c_rows = (int*)b;
    b += align_up(sizeof(int32_t) * ((size_t)G * G + 1), 256);
    r.n_changed = (int*)b;
    b += align_up(sizeof(int), 256);
    r.ck_out = (uint32_t*)b;
    b += align_up(sizeof(uint32_t) * (size_t)n, 256);
    r.ci_out = (int32_t*)b;
    b += align_up(sizeof(int32_t) * (size_t)n, 256);
    r.ci_tmp = (int32_t*)b;
    r.ck_in = spare_k0;
    r.ci_in = spare_v0;
    r.ck_tmp = spare_k1;
    return r;
}

int launch_resort(const ResortBufs& r, const uint32_t* keys, int n, int G, int key_bits, int* row_start,
                  int32_t* vals_out, void* sort_ws, size_t sort_ws_bytes, cudaStream_t s) {
    if (n <= 0) return SD_OK;
    const int chunks = (int)(padded_words(n) / kChunkWords);
    const int rows = G * G;
    k_chg_count<<<chunks, kChgThreads, 0, s>>>(r.words, r.chunk_cnt);
    SD_LAUNCHED(s);
    k_chg_compact<<<chunks, kChgThreads, 0, s>>>(r.words, r.chunk_cnt, keys, r.word_pre, r.ck_in, r.ci_in,
                                                 r.n_changed);
    SD_LAUNCHED(s);
    // C by key, stable: the radix sort with the count on the device
    int rc = launch_sort_pairs(r.ck_in, r.ci_in, r.ck_out, r.ci_out, r.ck_tmp, r.ci_tmp, n, key_bits, sort_ws,
                               sort_ws_bytes, s, true, false, r.n_changed);
    if (rc) return rc;
    k_merge_changed<<<148 * 4, 256, 0, s>>>(r.ck_out, r.ci_out, r.n_changed, row_start, r.words, r.word_pre,
                                            vals_out);
    SD_LAUNCHED(s);
    k_rows<<<(rows + 1 + 255) / 256, 256, 0, s>>>(r.ck_out, r.n_changed, rows, r.words, r.word_pre, r.c_rows,
                                                   row_start);
    SD_LAUNCHED(s);
    const int warps = (n + 255) / 256;
    k_merge_unchanged<<<(warps + kMergeThreads / 32 - 1) / (kMergeThreads / 32), kMergeThreads, 0, s>>>(
        keys, r.words, r.word_pre, r.c_rows, r.ci_out, n, vals_out);
    SD_LAUNCHED(s);
    return SD_OK;
}

}  // namespace sd
