// sd_scene.cu -- the particles a reset lays down: Sim::reset's placement path
// (Sim.cu:4160-4238) for the presets of this path.
//
//   k_place            kPlace (Sim.cu:281-407): the Filament preset (a uniform
//                      ball of radius 0.5 displaced by three crossed sine modes,
//                      clamped to the sphere, optionally shrunk about the centre;
//                      a hashed fraction marked dark matter, vel.w = -100) and the
//                      Empty preset (all slots empty, except that a dark-matter
//                      fraction still lands in a halo, as in the reference);
//   k_initial_velocity kAddSpin, kAddHubble, kAddDispersion (Sim.cu:2406-2476),
//                      applied in the reference's order;
//   centre-of-mass stop kMomentumAccum + kSubtractMeanVel (Sim.cu:2099-2104,
//                      2252-2266, reset at Sim.cu:4218-4235): the mean velocity
//                      over the active count, in FP64 with a fixed summation order.
//
// Random numbers are the reference's: a PCG hash of a per-particle seed
// (pcgHash / rnd01, Sim.cu:78-86), so the same configuration lays down the same
// particles. Angles use the fast intrinsics the reference uses.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "sd_internal.h"

namespace sd {
namespace {

constexpr unsigned kPlaceSeed = 12345u;       // placeInitial's seed (Sim.cu:3642)
constexpr unsigned kDispersionSeed = 24680u;  // reset's kAddDispersion seed (Sim.cu:4213)
constexpr float kTwoPi = 6.2831853f;

__device__ __forceinline__ unsigned pcg(unsigned v) {
    const unsigned st = v * 747796405u + 2891336453u;
    const unsigned w = ((st >> ((st >> 28u) + 4u)) ^ st) * 277803737u;
    return (w >> 22u) ^ w;
}

// uniform in [0, 1): the hash as a float times 2^-32
__device__ __forceinline__ float u01(unsigned s) { return (float)pcg(s) * 2.3283064365386963e-10f; }

// A direction uniform on the sphere from two hashes of s: cos theta, sin theta, phi.
struct Dir {
    float cz, sz, ph;
};
__device__ __forceinline__ Dir sphere_dir(unsigned s) {
    Dir d;
    d.cz = u01(s * 3u + 1u) * 2.0f - 1.0f;
    d.sz = sqrtf(fmaxf(1.0f - d.cz * d.cz, 0.0f));
    d.ph = u01(s * 7u + 5u) * kTwoPi;
    return d;
}

// The point at radius r in direction d, each component as (r sin theta) cos phi etc.
__device__ __forceinline__ float3 at_radius(float r, Dir d) {
    return make_float3(r * d.sz * __cosf(d.ph), r * d.sz * __sinf(d.ph), r * d.cz);
}

// Uniform in the ball of radius R: r = R u^(1/3) (ballPoint, Sim.cu:194-200).
__device__ __forceinline__ float3 ball_point(float R, unsigned s) {
    return at_radius(R * cbrtf(fmaxf(u01(s), 1e-9f)), sphere_dir(s));
}

// Centrally concentrated: r = R u^2 (bulgePoint, Sim.cu:228-236).
__device__ __forceinline__ float3 bulge_point(float R, unsigned s) {
    const float u = u01(s);
    return at_radius(R * u * u, sphere_dir(s));
}

__global__ void k_place(float4* __restrict__ pos, float4* __restrict__ vel, int n, int preset, float dark_frac,
                        float shrink) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const unsigned s = (unsigned)i * 2654435761u + kPlaceSeed;
    float vel_w = 0.f;
    if (dark_frac > 0.f && u01(s * 13u + 7u) < dark_frac) {
        if (preset == SD_PRESET_FILAMENT) {
            vel_w = -100.f;  // dark matter, placed with the same displacement as the gas
        } else {
            const float3 h = bulge_point(0.42f, s ^ 0x2545F491u);  // a halo about the centre
            pos[i] = make_float4(0.5f + h.x, 0.5f + h.y, 0.5f + h.z, 0.f);
            vel[i] = make_float4(0.f, 0.f, 0.f, -100.f);
            return;
        }
    }
    if (preset != SD_PRESET_FILAMENT) {
        pos[i] = make_float4(-1.f, -1.f, -1.f, 0.f);
        vel[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        return;
    }
    const float3 b = ball_point(0.5f, s ^ 0x6C8E9CF5u);
    const float x = 0.5f + b.x, y = 0.5f + b.y, z = 0.5f + b.z;
    // three crossed modes of 2, 4 and 6 wavelengths per box, amplitude 0.16/(1+m),
    // evaluated at the undisplaced point
    float dx = 0.f, dy = 0.f, dz = 0.f;
#pragma unroll
    for (int m = 0; m < 3; ++m) {
        const float fm = (float)m;
        const float k = kTwoPi * (2.0f + fm * 2.0f);
        const float amp = 0.16f / (1.0f + fm);
        dx += amp * __sinf(k * (y + 0.13f * fm)) * __cosf(k * (z + 0.29f));
        dy += amp * __sinf(k * (z + 0.19f * fm)) * __cosf(k * (x + 0.37f));
        dz += amp * __sinf(k * (x + 0.23f * fm)) * __cosf(k * (y + 0.11f));
    }
    float px = x + dx, py = y + dy, pz = z + dz;
    {  // pushed outside the sphere: back onto its surface
        const float rx = px - 0.5f, ry = py - 0.5f, rz = pz - 0.5f;
        const float rr = sqrtf(rx * rx + ry * ry + rz * rz);
        if (rr > 0.5f) {
            const float q = 0.5f / rr;
            px = 0.5f + rx * q;
            py = 0.5f + ry * q;
            pz = 0.5f + rz * q;
        }
    }
    if (shrink > 0.f) {
        px = 0.5f + (px - 0.5f) * shrink;
        py = 0.5f + (py - 0.5f) * shrink;
        pz = 0.5f + (pz - 0.5f) * shrink;
    }
    pos[i] = make_float4(px, py, pz, 0.f);
    vel[i] = make_float4(0.f, 0.f, 0.f, vel_w);
}

// Rigid rotation about the z axis through the centre, radial Hubble flow, then an
// isotropic random velocity of mean size vrms, on every live particle.
__global__ void k_initial_velocity(const float4* __restrict__ pos, float4* __restrict__ vel, int n, float spin,
                                   float hubble, float vrms) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (p.x < 0.f) return;
    float4 v = vel[i];
    if (spin != 0.f) {
        const float rx = p.x - 0.5f, ry = p.y - 0.5f;
        v.x += -spin * ry;
        v.y += spin * rx;
    }
    if (hubble != 0.f) {
        v.x += hubble * (p.x - 0.5f);
        v.y += hubble * (p.y - 0.5f);
        v.z += hubble * (p.z - 0.5f);
    }
    if (vrms > 0.f) {
        const unsigned s = (unsigned)i * 2654435761u + kDispersionSeed;
        const Dir d = sphere_dir(s);
        // size: the sum of three uniforms over 1.5, so its mean is 1
        const float g = (u01(s * 11u + 3u) + u01(s * 13u + 7u) + u01(s * 17u + 9u)) / 1.5f;
        v.x += vrms * g * d.sz * __cosf(d.ph);
        v.y += vrms * g * d.sz * __sinf(d.ph);
        v.z += vrms * g * d.cz;
    }
    vel[i] = v;
}

// mean[j] = (float)(sum_j / alive) from the momentum sums out8[2..4] of launch_energy
__global__ void k_com_mean(const double* __restrict__ out8, double alive, float* __restrict__ mean) {
    if (threadIdx.x < 3) mean[threadIdx.x] = (float)(out8[2 + threadIdx.x] / alive);
}

}  // namespace

int launch_place_preset(float4* pos, float4* vel, int n, const sd_config& cfg, double* partials, double* out8,
                        float* mean, cudaStream_t s) {
    if (n <= 0) return SD_OK;
    const int blocks = (n + 255) / 256;
    const bool filament = cfg.preset == SD_PRESET_FILAMENT;
    k_place<<<blocks, 256, 0, s>>>(pos, vel, n, cfg.preset, cfg.dark_matter_fraction,
                                   filament ? cfg.big_bang_shrink : 0.f);
    SD_LAUNCHED(s);
    if (cfg.spin != 0.f || cfg.hubble != 0.f || cfg.vel_dispersion > 0.f) {
        k_initial_velocity<<<blocks, 256, 0, s>>>(pos, vel, n, cfg.spin, cfg.hubble, cfg.vel_dispersion);
        SD_LAUNCHED(s);
    }
    // centre-of-mass stop over the active count: all slots for Filament, none for
    // Empty (whose dark halo, if any, keeps its momentum, as in the reference)
    if (!filament) return SD_OK;
    if (int rc = launch_energy(nullptr, 16, pos, vel, n, nullptr, partials, out8, s, 0)) return rc;
    k_com_mean<<<1, 32, 0, s>>>(out8, (double)n, mean);
    SD_LAUNCHED(s);
    return launch_apply_mean(vel, pos, n, mean, s);
}

}  // namespace sd
