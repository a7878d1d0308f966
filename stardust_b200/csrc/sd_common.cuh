// sd_common.cuh -- device helpers shared by the PM kernels (sm_100a).
//
// The CIC arithmetic below is written with explicit __fmaf_rn / __fmul_rn so the
// result of each expression is fixed by the source: the CPU oracle in oracle/
// uses the same forms with fmaf(), which is what makes keys, the fixed-point
// density and the kick bit-comparable between the two.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define SD_FIXED_ONE 4294967296.0f           // 2^32: fixed-point scale of one deposit weight
#define SD_FIXED_INV 2.3283064365386963e-10f  // 2^-32

namespace sd {

// CIC base cell and fraction along one axis: g = p*G - 1/2 (kScatter, Sim.cu:509-511).
__device__ __forceinline__ void cic_axis(float p, int G, int& i, float& f) {
    const float g = __fmaf_rn(p, (float)G, -0.5f);
    const float fl = floorf(g);
    i = (int)fl;
    f = __fsub_rn(g, fl);
}

// Cell index of a CIC corner: wrapped (periodic) or clamped to the edge cell
// (isolated; gidx3, Sim.cu:96-100 -- weights past the edge land on it).
__device__ __forceinline__ int cic_cell(int i, int G, bool periodic) {
    return periodic ? (i & (G - 1)) : min(max(i, 0), G - 1);
}

// Weight of corner k = ox | oy<<1 | oz<<2, as (wx*wy)*wz (Sim.cu:515).
__device__ __forceinline__ float cic_weight(int k, float fx, float fy, float fz) {
    const float wx = (k & 1) ? fx : __fsub_rn(1.f, fx);
    const float wy = (k & 2) ? fy : __fsub_rn(1.f, fy);
    const float wz = (k & 4) ? fz : __fsub_rn(1.f, fz);
    return __fmul_rn(__fmul_rn(wx, wy), wz);
}

__device__ __forceinline__ long long fixed_weight(float w) {
    return __float2ll_rn(__fmul_rn(w, SD_FIXED_ONE));
}

__device__ __forceinline__ float fixed_to_float(long long s) {
    return __fmul_rn(__ll2float_rn(s), SD_FIXED_INV);
}

__device__ __forceinline__ uint32_t part1by2(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Order keys (see sd_cell_keys in stardust_pm.h). Row-major and Morton: key + 1,
// 0 = empty slot. Tiled: the row index itself (G^2 values, log2(G^2) bits), with
// empty slots sharing row 0 (the fused deposit skips them).
__device__ __forceinline__ uint32_t order_key(float4 p, int G, int order) {
    if (p.x < 0.f) return 0u;
    if (order == 2) {  // tile rows of the CIC base cell
        int iy, iz; float f;
        cic_axis(p.y, G, iy, f);
        cic_axis(p.z, G, iz, f);
        iy &= (G - 1); iz &= (G - 1);
        const int tiles = G >> 2;
        const int tile = (iz >> 2) * tiles + (iy >> 2);
        return (uint32_t)(tile * 16 + (iz & 3) * 4 + (iy & 3));
    }
    // containing cell, clamped (kCellKey, Sim.cu:2482-2485)
    const int cx = min(max((int)__fmul_rn(p.x, (float)G), 0), G - 1);
    const int cy = min(max((int)__fmul_rn(p.y, (float)G), 0), G - 1);
    const int cz = min(max((int)__fmul_rn(p.z, (float)G), 0), G - 1);
    if (order == 1)
        return (part1by2((uint32_t)cx) | (part1by2((uint32_t)cy) << 1) | (part1by2((uint32_t)cz) << 2)) + 1u;
    return (uint32_t)((cz * G + cy) * G + cx) + 1u;
}

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

}  // namespace sd
