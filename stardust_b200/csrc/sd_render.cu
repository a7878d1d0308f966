// sd_render.cu -- headless point render of the particle buffers into an RGBA
// image in device memory: the reference's kSplatPoints -> kAccumToRGBA path
// (src/gfx/RenderField.cu:318-735) for the particles of the PM path (gas, w = 0),
// coloured by density or speed, without the OpenGL texture it feeds there.
//
// Differences by design: the accumulation buffer holds 64-bit fixed-point sums
// (2^-24 units per channel) instead of float atomics, so the image is the same
// bit for bit whatever order the particles land in; star light, black-hole
// disks and the ash map (colour modes 3 and 4) belong to features outside the
// PM path and are not drawn.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "sd_internal.h"

namespace sd {
namespace {

constexpr float kAccumOne = 16777216.f;  // 2^24: fixed-point unit of the accumulation

// Colour maps (RenderField.cu:14-35, 96-102).
__device__ __forceinline__ float3 cmap_astro(float t) {
    t = fminf(fmaxf(t, 0.f), 1.f);
    const float3 c[7] = {{0.00f, 0.00f, 0.00f}, {0.05f, 0.06f, 0.19f}, {0.16f, 0.14f, 0.47f},
                         {0.47f, 0.27f, 0.67f}, {0.88f, 0.55f, 0.27f}, {1.00f, 0.84f, 0.51f},
                         {1.00f, 1.00f, 0.94f}};
    const float stops[7] = {0.00f, 0.18f, 0.38f, 0.58f, 0.76f, 0.90f, 1.00f};
    for (int i = 0; i < 6; ++i) {
        if (t <= stops[i + 1]) {
            const float f = (t - stops[i]) / (stops[i + 1] - stops[i]);
            return make_float3(c[i].x + (c[i + 1].x - c[i].x) * f, c[i].y + (c[i + 1].y - c[i].y) * f,
                               c[i].z + (c[i + 1].z - c[i].z) * f);
        }
    }
    return c[6];
}

__device__ __forceinline__ float3 cmap_thermal(float t) {
    t = fminf(fmaxf(t, 0.f), 1.f);
    return make_float3(fminf(t * 2.2f, 1.f), fminf(fmaxf((t - 0.32f) * 1.9f, 0.f), 1.f),
                       fminf(fmaxf((t - 0.70f) * 3.2f, 0.f), 1.f));
}

__device__ __forceinline__ float3 cmap(int kind, float t) {
    return (kind == 1) ? make_float3(t, t, t) : (kind == 2) ? cmap_thermal(t) : cmap_astro(t);
}

__device__ __forceinline__ void add_px(unsigned long long* acc, int W, int x, int y, float3 c) {
    unsigned long long* a = acc + 3 * ((size_t)y * W + x);
    atomicAdd(a + 0, (unsigned long long)__float2ll_rn(c.x * kAccumOne));
    atomicAdd(a + 1, (unsigned long long)__float2ll_rn(c.y * kAccumOne));
    atomicAdd(a + 2, (unsigned long long)__float2ll_rn(c.z * kAccumOne));
}

// One particle per thread: project (projectPoint, ViewRot.h:76-96), frame with
// zoom / pan / aspect, pick the colour and the footprint (a point, 3x3 or 5x5
// binomial weights, capped by how many particles are visible), accumulate.
__global__ void k_splat(const float4* __restrict__ pos, const float4* __restrict__ vel, int n, sd_view v, int W, int H,
                        unsigned long long* __restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (p.x < 0.f) return;
    // gas only: stars, remnants and explosions (w != 0) are drawn by the star-light mode
    if (p.w != 0.f) return;
    const float fx = p.x - v.center[0], fy = p.y - v.center[1], fz = p.z - v.center[2];
    const float xc = v.rot[0] * fx + v.rot[1] * fy + v.rot[2] * fz;
    const float yc = v.rot[3] * fx + v.rot[4] * fy + v.rot[5] * fz;
    float px, py, depth = 1.f;
    if (v.fly) {
        const float zc = v.rot[6] * fx + v.rot[7] * fy + v.rot[8] * fz;
        if (zc < 1e-3f) return;
        const float k = 0.5f / (zc * v.tan_half_fov);
        px = xc * k + 0.5f;
        py = yc * k + 0.5f;
        depth = zc;
    } else {
        px = xc + 0.5f;
        py = yc + 0.5f;
    }
    float u, w;
    if (v.fly) {
        u = px;
        w = py;
    } else {
        u = (px - 0.5f + v.pan_x) * v.zoom + 0.5f;
        w = (py - 0.5f + v.pan_y) * v.zoom + 0.5f;
    }
    const float aspect = (float)W / (float)H;
    if (aspect > 1.f) u = (u - 0.5f) / aspect + 0.5f;
    else w = (w - 0.5f) * aspect + 0.5f;
    if (u < 0.f || u >= 1.f || w < 0.f || w >= 1.f) return;
    const int x = (int)(u * W), y = (int)((1.f - w) * H);  // rows top-down
    if (x < 0 || x >= W || y < 0 || y >= H) return;

    float3 c;
    if (v.color_by == 0) {  // density: one colour, overlap makes brightness
        c = (v.cmap == 1) ? make_float3(1.f, 1.f, 1.f)
            : (v.cmap == 2) ? cmap_thermal(0.62f)
                            : make_float3(0.55f, 0.42f, 0.85f);
    } else {
        float t = 0.5f;
        if (v.color_by == 2) {  // speed, all three components
            const float4 q = vel[i];
            t = fminf(sqrtf(q.x * q.x + q.y * q.y + q.z * q.z) * 0.25f, 1.f);
        }
        c = cmap(v.cmap, t);
    }
    const float visible = (float)n / fmaxf(v.zoom * v.zoom, 1.0f);
    const int cap = (visible > 8.0e6f) ? 0 : ((visible > 2.0e6f) ? 1 : 2);
    const float grow = v.fly ? fminf(0.35f / fmaxf(depth, 1e-3f), 6.0f) : fminf(sqrtf(fmaxf(v.zoom, 1.0f)), 4.0f);
    const float rr = v.size_px * grow;
    int rad = (rr < 2.0f) ? 0 : ((rr < 4.0f) ? 1 : 2);
    if (rad > cap) rad = cap;
    if (rad == 0) {
        add_px(acc, W, x, y, c);
        return;
    }
    const float k3[3] = {0.25f, 0.5f, 0.25f};
    const float k5[5] = {0.0625f, 0.25f, 0.375f, 0.25f, 0.0625f};
    const float* kk = (rad == 1) ? k3 : k5;
    for (int dy = -rad; dy <= rad; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= H) continue;
        const float wy = kk[dy + rad];
        for (int dx = -rad; dx <= rad; ++dx) {
            const int xx = x + dx;
            if (xx < 0 || xx >= W) continue;
            const float f = wy * kk[dx + rad];
            add_px(acc, W, xx, yy, make_float3(c.x * f, c.y * f, c.z * f));
        }
    }
}

// Accumulation -> RGBA (kAccumToRGBA, RenderField.cu:687-735); clears the sums.
__global__ void k_tonemap(unsigned long long* __restrict__ acc, uchar4* __restrict__ out, int npx, sd_view v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npx) return;
    unsigned long long* a = acc + 3 * (size_t)i;
    const float ax = (float)(double)(long long)a[0] * (1.f / kAccumOne);
    const float ay = (float)(double)(long long)a[1] * (1.f / kAccumOne);
    const float az = (float)(double)(long long)a[2] * (1.f / kAccumOne);
    a[0] = a[1] = a[2] = 0ull;
    const float lum = (ax + ay + az) * 0.3333f;
    float r, g, b;
    if (v.use_cmap) {
        const float t = __powf(fminf(__logf(1.f + lum * v.bright) * 0.42f, 1.f), v.inv_gamma);
        const float3 c = cmap(v.cmap, t);
        r = c.x;
        g = c.y;
        b = c.z;
    } else {
        float tone;
        if (v.reinhard) {
            const float x = fmaxf(__logf(1.f + lum * v.bright) * 0.42f, 0.f);
            tone = __powf(x / (1.f + x), v.inv_gamma);
        } else {
            tone = __powf(fminf(__logf(1.f + lum * v.bright) * 0.42f, 1.f), v.inv_gamma);
        }
        const float s = (lum > 1e-6f) ? tone / lum : 0.f;
        r = fminf(ax * s, 1.f);
        g = fminf(ay * s, 1.f);
        b = fminf(az * s, 1.f);
    }
    out[i] = make_uchar4((unsigned char)(fminf(r, 1.f) * 255.f), (unsigned char)(fminf(g, 1.f) * 255.f),
                         (unsigned char)(fminf(b, 1.f) * 255.f), 255);
}

}  // namespace
}  // namespace sd

using namespace sd;

extern "C" {

void sd_view_default(sd_view* v) {
    if (!v) return;
    *v = sd_view{};
    v->rot[0] = v->rot[4] = v->rot[8] = 1.f;
    v->center[0] = v->center[1] = v->center[2] = 0.5f;
    v->tan_half_fov = 0.5773503f;  // 60 degree field of view
    v->zoom = 1.f;
    v->size_px = 1.f;
    v->color_by = 0;
    v->cmap = 0;
    v->bright = 1.f;
    v->inv_gamma = 1.f;
    v->use_cmap = 1;
}

size_t sd_render_workspace_bytes(int width, int height) {
    if (width <= 0 || height <= 0) return 0;
    return align_up(sizeof(unsigned long long) * 3 * (size_t)width * height, 256);
}

int sd_render_points(const float* pos, const float* vel, int n, const sd_view* view, int width, int height,
                     void* workspace, size_t workspace_bytes, void* rgba_out, void* stream) {
    if (!view || !rgba_out || !workspace || n < 0 || (n > 0 && (!pos || !vel)) || width <= 0 || height <= 0 ||
        width > 16384 || height > 16384)
        return fail(SD_E_ARG, "render_points: bad arguments");
    if (workspace_bytes < sd_render_workspace_bytes(width, height))
        return fail(SD_E_ARG, "render_points: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const int npx = width * height;
    // the sums start at zero: the workspace is cleared here and by every tone map
    if (SD_CUDA(cudaMemsetAsync(workspace, 0, sizeof(unsigned long long) * 3 * (size_t)npx, st))) return SD_E_CUDA;
    auto* acc = reinterpret_cast<unsigned long long*>(workspace);
    if (n > 0) {
        k_splat<<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float4*>(pos),
                                                 reinterpret_cast<const float4*>(vel), n, *view, width, height, acc);
        SD_LAUNCHED(st);
    }
    k_tonemap<<<(npx + 255) / 256, 256, 0, st>>>(acc, reinterpret_cast<uchar4*>(rgba_out), npx, *view);
    SD_LAUNCHED(st);
    return SD_OK;
}

}  // extern "C"
