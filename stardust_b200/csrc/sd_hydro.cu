// sd_hydro.cu -- the grid hydrodynamics add-ons of the reference's step: cooling
// toward the cell-mean velocity and a pressure force from the velocity
// dispersion (Sim::Impl::doCooling, Sim.cu:3732-3868; kAccumCellVel, kCoolCell,
// kPressure, Sim.cu:1212-1415; the pressure kick in kIntegrate, Sim.cu:740-743).
//
// Per cooling step (every 2 steps with pressure, every 8 without; dt scaled by
// the period, Sim.cu:3737-3739):
//   k_cell_velocity  sum v and count over the containing cell of every live gas
//                    or star particle with a finite velocity (not dark matter);
//   k_cool           per particle: dv = cell mean - v (cells with >= 2 members);
//                    with pressure, dv_d^2 and a count into the dispersion grids;
//                    gas velocities move k dv toward the mean, k = min(60 rate dt, 1/2).
// Every step with pressure (computeAccel, Sim.cu:3620-3631):
//   k_pressure       a_d = -(disp_d[+1] - disp_d[-1]) * (G/2) * pressureK / count,
//                    clamped to +-5, in cells holding dispersion (0 elsewhere);
//                    the gather adds its CIC sample to gas particles.
//
// The per-cell sums are 64-bit fixed point (2^-24 units) instead of float
// atomics, so they do not depend on the order of the adds. Pending momentum
// corrections are applied by k_cool as it reads each velocity (it writes the
// corrected, cooled velocity back), so the gather of a cooling step reads the
// velocities as they are.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "sd_internal.h"

namespace sd {
namespace {

constexpr float kFix = 16777216.f;          // 2^24
constexpr double kFixInv = 1.0 / 16777216.0;
constexpr float kMaxPressureAcc = 5.0f;     // computeAccel's cap (Sim.cu:3627)

__device__ __forceinline__ unsigned long long fix(float v) {
    return (unsigned long long)__float2ll_rn(v * kFix);
}
__device__ __forceinline__ float unfix(long long v) { return (float)((double)v * kFixInv); }

// Containing cell (not the CIC base): clamp((int)(p G), 0, G-1) per axis
// (Sim.cu:1227-1230); the hydro grids are G^3 for both boundaries.
__device__ __forceinline__ int cell_of(float4 p, int G) {
    const int cx = min(max((int)(p.x * G), 0), G - 1);
    const int cy = min(max((int)(p.y * G), 0), G - 1);
    const int cz = min(max((int)(p.z * G), 0), G - 1);
    return (cz * G + cy) * G + cx;
}

__device__ __forceinline__ float4 load_vel(const float4* vel, int i, const float* mean) {
    float4 v = vel[i];
    if (mean) {
        v.x = __fsub_rn(v.x, mean[0]);
        v.y = __fsub_rn(v.y, mean[1]);
        v.z = __fsub_rn(v.z, mean[2]);
    }
    return v;
}

__device__ __forceinline__ bool finite3(float4 v) { return isfinite(v.x) && isfinite(v.y) && isfinite(v.z); }

__global__ void k_cell_velocity(const float4* __restrict__ pos, const float4* __restrict__ vel, int n, int G,
                                const float* __restrict__ mean, long long* __restrict__ sx,
                                long long* __restrict__ sy, long long* __restrict__ sz, unsigned* __restrict__ cnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (p.x < 0.f) return;
    const float4 v = load_vel(vel, i, mean);
    if (!finite3(v) || v.w < -50.f) return;  // dark matter does not cool (vel.w = -100)
    const int c = cell_of(p, G);
    atomicAdd(reinterpret_cast<unsigned long long*>(sx + c), fix(v.x));
    atomicAdd(reinterpret_cast<unsigned long long*>(sy + c), fix(v.y));
    atomicAdd(reinterpret_cast<unsigned long long*>(sz + c), fix(v.z));
    atomicAdd(cnt + c, 1u);
}

__global__ void k_cool(const float4* __restrict__ pos, float4* __restrict__ vel, int n, int G,
                       const float* __restrict__ mean, const long long* __restrict__ sx,
                       const long long* __restrict__ sy, const long long* __restrict__ sz,
                       const unsigned* __restrict__ cnt, float k, long long* __restrict__ dx,
                       long long* __restrict__ dy, long long* __restrict__ dz, unsigned* __restrict__ dcnt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (p.x < 0.f) return;  // empty slots take no correction
    float4 v = load_vel(vel, i, mean);
    if (v.w >= -50.f && finite3(v)) {
        const int c = cell_of(p, G);
        const unsigned nc = cnt[c];
        if (nc >= 2u) {
            const float inv = 1.f / (float)nc;
            const float dvx = unfix(sx[c]) * inv - v.x;
            const float dvy = unfix(sy[c]) * inv - v.y;
            const float dvz = unfix(sz[c]) * inv - v.z;
            if (dcnt) {
                atomicAdd(reinterpret_cast<unsigned long long*>(dx + c), fix(dvx * dvx));
                atomicAdd(reinterpret_cast<unsigned long long*>(dy + c), fix(dvy * dvy));
                atomicAdd(reinterpret_cast<unsigned long long*>(dz + c), fix(dvz * dvz));
                atomicAdd(dcnt + c, 1u);
            }
            if (p.w <= 0.f) {  // stars keep their velocity (Sim.cu:1302)
                v.x = v.x + k * dvx;
                v.y = v.y + k * dvy;
                v.z = v.z + k * dvz;
            }
        }
    }
    vel[i] = v;  // corrected by the pending mean, and cooled
}

__global__ void k_pressure(const long long* __restrict__ dx, const long long* __restrict__ dy,
                           const long long* __restrict__ dz, const unsigned* __restrict__ dcnt, int G, int periodic,
                           float pk, float4* __restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G * G * G) return;
    const int x = i % G, y = (i / G) % G, z = i / (G * G);
    const float rho = (float)dcnt[i];
    if (rho < 1e-6f) {
        acc[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    int xm, xp, ym, yp, zm, zp;
    if (periodic) {
        xm = (x - 1) & (G - 1), xp = (x + 1) & (G - 1);
        ym = (y - 1) & (G - 1), yp = (y + 1) & (G - 1);
        zm = (z - 1) & (G - 1), zp = (z + 1) & (G - 1);
    } else {
        xm = max(x - 1, 0), xp = min(x + 1, G - 1);
        ym = max(y - 1, 0), yp = min(y + 1, G - 1);
        zm = max(z - 1, 0), zp = min(z + 1, G - 1);
    }
    const float h = 0.5f * (float)G * pk / rho;
    float ax = -(unfix(dx[(z * G + y) * G + xp]) - unfix(dx[(z * G + y) * G + xm])) * h;
    float ay = -(unfix(dy[(z * G + yp) * G + x]) - unfix(dy[(z * G + ym) * G + x])) * h;
    float az = -(unfix(dz[(zp * G + y) * G + x]) - unfix(dz[(zm * G + y) * G + x])) * h;
    ax = fminf(fmaxf(ax, -kMaxPressureAcc), kMaxPressureAcc);
    ay = fminf(fmaxf(ay, -kMaxPressureAcc), kMaxPressureAcc);
    az = fminf(fmaxf(az, -kMaxPressureAcc), kMaxPressureAcc);
    acc[i] = make_float4(ax, ay, az, 0.f);
}

}  // namespace

size_t hydro_bytes(int G) {
    const size_t cells = (size_t)G * G * G;
    return cells * (6 * sizeof(long long) + 2 * sizeof(unsigned) + sizeof(float4));
}

int hydro_alloc(HydroGrids& h, int G) {
    const size_t cells = (size_t)G * G * G;
    void* p = nullptr;
    if (cudaMalloc(&p, hydro_bytes(G)) != cudaSuccess) {
        cudaGetLastError();
        return fail(SD_E_NOMEM, "cudaMalloc of the hydro grids failed");
    }
    char* b = (char*)p;
    h.base = p;
    h.acc = (float4*)b;
    b += sizeof(float4) * cells;
    for (int d = 0; d < 3; ++d, b += sizeof(long long) * cells) h.vsum[d] = (long long*)b;
    for (int d = 0; d < 3; ++d, b += sizeof(long long) * cells) h.disp[d] = (long long*)b;
    h.cnt = (unsigned*)b;
    b += sizeof(unsigned) * cells;
    h.dcnt = (unsigned*)b;
    h.G = G;
    // the dispersion and the pressure field start empty (Sim.cu:3483-3497)
    return SD_CUDA(cudaMemset(p, 0, hydro_bytes(G)));
}

void hydro_free(HydroGrids& h) {
    if (h.base) cudaFree(h.base);
    h = HydroGrids{};
}

int launch_pressure(const HydroGrids& h, int periodic, float pressure_k, cudaStream_t s) {
    const int cells = h.G * h.G * h.G;
    k_pressure<<<(cells + 255) / 256, 256, 0, s>>>(h.disp[0], h.disp[1], h.disp[2], h.dcnt, h.G, periodic, pressure_k,
                                                   h.acc);
    SD_LAUNCHED(s);
    return SD_OK;
}

int launch_cooling(const HydroGrids& h, const float4* pos, float4* vel, int n, const float* mean, float rate,
                   float dt, bool pressure, cudaStream_t s) {
    if (n <= 0) return SD_OK;
    const size_t cells = (size_t)h.G * h.G * h.G;
    // cleared each cooling step: the velocity sums and counts, and (with pressure) the
    // dispersion grids (Sim.cu:3770-3790)
    if (SD_CUDA(cudaMemsetAsync(h.vsum[0], 0, 3 * sizeof(long long) * cells, s)) ||
        SD_CUDA(cudaMemsetAsync(h.cnt, 0, sizeof(unsigned) * cells, s)))
        return SD_E_CUDA;
    if (pressure && (SD_CUDA(cudaMemsetAsync(h.disp[0], 0, 3 * sizeof(long long) * cells, s)) ||
                     SD_CUDA(cudaMemsetAsync(h.dcnt, 0, sizeof(unsigned) * cells, s))))
        return SD_E_CUDA;
    const int blocks = (n + 255) / 256;
    k_cell_velocity<<<blocks, 256, 0, s>>>(pos, vel, n, h.G, mean, h.vsum[0], h.vsum[1], h.vsum[2], h.cnt);
    SD_LAUNCHED(s);
    float k = rate * dt * 60.0f;  // the ash factor is 1: no star formation on this path
    if (k > 0.5f) k = 0.5f;
    k_cool<<<blocks, 256, 0, s>>>(pos, vel, n, h.G, mean, h.vsum[0], h.vsum[1], h.vsum[2], h.cnt, k,
                                  pressure ? h.disp[0] : nullptr, pressure ? h.disp[1] : nullptr,
                                  pressure ? h.disp[2] : nullptr, pressure ? h.dcnt : nullptr);
    SD_LAUNCHED(s);
    return SD_OK;
}

}  // namespace sd
