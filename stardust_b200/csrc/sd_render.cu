// sd_render.cu -- headless renders into an RGBA image in device memory, without
// the OpenGL texture they feed in the reference:
//   points: kSplatPoints -> kAccumToRGBA (src/gfx/RenderField.cu:318-735) for the
//           particles of the PM path (gas, w = 0), coloured by density or speed;
//   grid:   the field view -- Sim::fieldDevicePtr's projections (kProjectXY,
//           kScatterDispersion + kDivideInto, Sim.cu:2526-2570, 2701-2707,
//           5229-5296), the top-5 % brightness reference of a log histogram
//           (kHistLog and its percentile, RenderField.cu:125-137, 930-1000), and
//           kShade (RenderField.cu:158-316).
//
// Differences by design: sums that the reference makes with float atomics are
// 64-bit fixed point here (2^-24 units), so an image is the same bit for bit
// whatever order its inputs land in; star light, black-hole disks, the ash map
// and the star-temperature colouring belong to features outside the PM path and
// are not drawn; the frame-to-frame blending of the interactive view
// (kBlendGrid) and its slow brightness follower do not apply to a single image,
// which takes the first-frame values.
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

// Black body, red -> white -> blue-white, dimmed at the dark end (RenderField.cu:60-82).
__device__ __forceinline__ float3 cmap_blackbody(float t) {
    t = fminf(fmaxf(t, 0.f), 1.f);
    float r, g, b;
    if (t < 0.5f) {
        const float u = t * 2.0f;
        r = 1.0f;
        g = 0.32f + 0.68f * u;
        b = 0.08f + 0.80f * u * u;
    } else {
        const float u = (t - 0.5f) * 2.0f;
        r = 1.0f - 0.38f * u;
        g = 1.0f - 0.30f * u;
        b = 1.0f;
    }
    const float dim = fminf(t * 3.2f, 1.0f);
    return make_float3(r * dim, g * dim, b * dim);
}

__device__ __forceinline__ float3 cmap(int kind, float t) {
    return (kind == 1)   ? make_float3(t, t, t)
           : (kind == 2) ? cmap_thermal(t)
           : (kind == 3) ? cmap_blackbody(t)
                         : cmap_astro(t);
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

// ---- grid view -------------------------------------------------------------

constexpr int kHistBins = 64;  // log bins of 1e-4 .. 1e8 (kHistLog)

__device__ __forceinline__ long long to_fixed24(float v) { return __float2ll_rn(v * kAccumOne); }

// rotPoint (ViewRot.h:25-31): the orthographic image of a point, inside [0,1)^2?
__device__ __forceinline__ bool rot_point(float px, float py, float pz, const sd_view& v, float& ox, float& oy) {
    const float fx = px - v.center[0], fy = py - v.center[1], fz = pz - v.center[2];
    ox = v.rot[0] * fx + v.rot[1] * fy + v.rot[2] * fz + 0.5f;
    oy = v.rot[3] * fx + v.rot[4] * fy + v.rot[5] * fz + 0.5f;
    return ox >= 0.f && ox < 1.f && oy >= 0.f && oy < 1.f;
}

// kProjectXY without rotation: each screen cell sums its z column, in z order.
__global__ void k_project_columns(const float* __restrict__ rho, int G, float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= G * G) return;
    const size_t plane = (size_t)G * G;
    float s = 0.f;
    for (int z = 0; z < G; ++z) s += rho[z * plane + i];
    out[i] = s;
}

// kProjectXY with rotation (rotCell, Sim.cu:2514-2524): each non-empty cell's
// centre to the screen cell it falls in, summed in fixed point.
__global__ void k_project_rotated(const float* __restrict__ rho, int G, sd_view v, long long* __restrict__ acc) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)G * G * G) return;
    const float val = rho[i];
    if (val == 0.f) return;
    const int x = (int)(i % G), y = (int)((i / G) % G), z = (int)(i / ((size_t)G * G));
    const float inv = 1.0f / (float)G;
    float ox, oy;
    if (!rot_point((x + 0.5f) * inv, (y + 0.5f) * inv, (z + 0.5f) * inv, v, ox, oy)) return;
    const int sx = (int)(ox * (float)G), sy = (int)(oy * (float)G);
    if (sx < 0 || sx >= G || sy < 0 || sy >= G) return;
    atomicAdd(reinterpret_cast<unsigned long long*>(acc + sy * G + sx), (unsigned long long)to_fixed24(val));
}

// kScatterDispersion (Sim.cu:2548-2570): per particle, w |v|^2 and w onto the 4
// bilinear screen cells (edge-clamped) of its (rotated) image.
__global__ void k_scatter_dispersion(const float4* __restrict__ pos, const float4* __restrict__ vel, int n, int G,
                                     sd_view v, long long* __restrict__ num, long long* __restrict__ den) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i];
    if (p.x < 0.f) return;
    const float4 q = vel[i];
    const float v2 = q.x * q.x + q.y * q.y + q.z * q.z;
    float ux = p.x, uy = p.y;
    if (v.rot_on && !rot_point(p.x, p.y, p.z, v, ux, uy)) return;
    const float gx = ux * G - 0.5f, gy = uy * G - 0.5f;
    const int ix = (int)floorf(gx), iy = (int)floorf(gy);
    const float fx = gx - ix, fy = gy - iy;
    for (int k = 0; k < 4; ++k) {
        const int ox = k & 1, oy = (k >> 1) & 1;
        const int cx = min(max(ix + ox, 0), G - 1), cy = min(max(iy + oy, 0), G - 1);
        const float w = (ox ? fx : 1.f - fx) * (oy ? fy : 1.f - fy);
        atomicAdd(reinterpret_cast<unsigned long long*>(num + cy * G + cx), (unsigned long long)to_fixed24(w * v2));
        atomicAdd(reinterpret_cast<unsigned long long*>(den + cy * G + cx), (unsigned long long)to_fixed24(w));
    }
}

// fixed -> float; with den: kDivideInto (Sim.cu:2701-2707), the rms speed of the cell
__global__ void k_finish_field(const long long* __restrict__ num, const long long* __restrict__ den, int cells,
                               float* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const float a = (float)((double)num[i] * (1.0 / kAccumOne));
    if (!den) {
        out[i] = a;
        return;
    }
    const float d = (float)((double)den[i] * (1.0 / kAccumOne));
    out[i] = (d > 1e-6f) ? sqrtf(fmaxf(a / d, 0.f)) : 0.f;
}

// kHistLog (RenderField.cu:125-137)
__global__ void k_hist_log(const float* __restrict__ g, int n, int* __restrict__ hist) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float val = g[i];
    if (val <= 0.f) return;
    const float t = (__logf(val) + 9.21f) / (18.42f + 9.21f);
    int b = (int)(t * (float)kHistBins);
    b = min(max(b, 0), kHistBins - 1);
    atomicAdd(&hist[b], 1);
}

// The brightness factor of kShade (RenderField.cu:930-1012): for the density, the
// view brightness over the value 5 % from the top of the histogram (interpolated
// inside its bin; the mean density per screen cell when the field is empty); for
// the dispersion, 60 times the view brightness.
__global__ void k_brightness(const int* __restrict__ hist, float mean_rho, float brightness, int normalise,
                             float* __restrict__ bright) {
    if (threadIdx.x != 0) return;
    if (!normalise) {
        *bright = brightness * 60.0f;
        return;
    }
    float norm = mean_rho;
    int total = 0;
    for (int b = 0; b < kHistBins; ++b) total += hist[b];
    if (total > 0) {
        const int want = (int)(total * 0.05f) + 1;
        int acc = 0, hit = kHistBins - 1;
        for (int b = kHistBins - 1; b >= 0; --b) {
            acc += hist[b];
            if (acc >= want) {
                hit = b;
                break;
            }
        }
        const int below = acc - hist[hit];
        const float need = (float)(want - below);
        const float frac = (hist[hit] > 0) ? fminf(fmaxf(need / (float)hist[hit], 0.f), 1.f) : 0.5f;
        const float t = ((float)hit + 1.0f - frac) / (float)kHistBins;
        const float m = expf(t * (18.42f + 9.21f) - 9.21f);
        if (m > 1e-6f) norm = m;
    }
    *bright = brightness / fmaxf(norm, 1e-6f);
}

// kShade (RenderField.cu:158-316): bilinear sample of the G x G field under each
// pixel (square view on the short side, zoom and pan about the centre), log and
// x/(1+x) tone curve, colour map; rows bottom-up as the reference's texture.
__global__ void k_shade(const float* __restrict__ g, int G, uchar4* __restrict__ out, int W, int H,
                        const float* __restrict__ bright_p, float inv_gamma, int cmap_kind, float zoom, float pan_x,
                        float pan_y) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= W || y >= H) return;
    const float aspect = (float)W / (float)H;
    float u = (x + 0.5f) / W, v = (y + 0.5f) / H;
    if (aspect > 1.f) u = (u - 0.5f) * aspect + 0.5f;
    else v = (v - 0.5f) / aspect + 0.5f;
    u = (u - 0.5f) / zoom + 0.5f - pan_x;
    v = (v - 0.5f) / zoom + 0.5f - pan_y;
    uchar4 px = make_uchar4(0, 0, 0, 255);
    if (u >= 0.f && u < 1.f && v >= 0.f && v < 1.f) {
        const float gfx = u * G - 0.5f, gfy = v * G - 0.5f;
        int x0 = (int)floorf(gfx), y0 = (int)floorf(gfy);
        const float tx = gfx - x0, ty = gfy - y0;
        int x1 = x0 + 1, y1 = y0 + 1;
        x0 = min(max(x0, 0), G - 1);
        x1 = min(max(x1, 0), G - 1);
        y0 = min(max(y0, 0), G - 1);
        y1 = min(max(y1, 0), G - 1);
        const float d = g[y0 * G + x0] * (1.f - tx) * (1.f - ty) + g[y0 * G + x1] * tx * (1.f - ty) +
                        g[y1 * G + x0] * (1.f - tx) * ty + g[y1 * G + x1] * tx * ty;
        const float xl = fmaxf(__logf(1.f + d * *bright_p) * 0.60f, 0.f);
        const float t = __powf(xl / (1.f + xl), inv_gamma);
        const float3 c = cmap(cmap_kind, t);
        px = make_uchar4((unsigned char)(c.x * 255.f), (unsigned char)(c.y * 255.f), (unsigned char)(c.z * 255.f),
                         255);
    }
    out[(size_t)(H - 1 - y) * W + x] = px;
}

struct FieldWs {
    float* field;     // G^2
    long long* num;   // G^2
    long long* den;   // G^2
    int* hist;        // kHistBins
    float* bright;    // 1
};

FieldWs field_ws(void* ws, int G) {
    const size_t cells = (size_t)G * G;
    char* b = (char*)ws;
    FieldWs w;
    w.field = (float*)b;
    b += align_up(sizeof(float) * cells, 256);
    w.num = (long long*)b;
    b += align_up(sizeof(long long) * cells, 256);
    w.den = (long long*)b;
    b += align_up(sizeof(long long) * cells, 256);
    w.hist = (int*)b;
    w.bright = (float*)(b + sizeof(int) * kHistBins);
    return w;
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

size_t sd_render_field_workspace_bytes(int grid_size) {
    if (grid_size <= 0) return 0;
    const size_t cells = (size_t)grid_size * grid_size;
    return align_up(sizeof(float) * cells, 256) + 2 * align_up(sizeof(long long) * cells, 256) +
           align_up(sizeof(int) * kHistBins + sizeof(float), 256);
}

int sd_render_field(int field, const float* density, int grid_size, const float* pos, const float* vel, int n,
                    const sd_view* view, int width, int height, void* workspace, size_t workspace_bytes,
                    void* rgba_out, void* stream) {
    const int G = grid_size;
    if (!view || !rgba_out || !workspace || G < 1 || G > 1024 || width <= 0 || height <= 0 || width > 16384 ||
        height > 16384 || n < 0)
        return fail(SD_E_ARG, "render_field: bad arguments");
    if (field == SD_FIELD_DENSITY && !density) return fail(SD_E_ARG, "render_field: density grid missing");
    if (field == SD_FIELD_DISPERSION && n > 0 && (!pos || !vel))
        return fail(SD_E_ARG, "render_field: particles missing");
    if (field != SD_FIELD_DENSITY && field != SD_FIELD_DISPERSION) return fail(SD_E_ARG, "render_field: bad field");
    if (workspace_bytes < sd_render_field_workspace_bytes(G)) return fail(SD_E_ARG, "render_field: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const FieldWs w = field_ws(workspace, G);
    const int cells = G * G;
    const int cb = (cells + 255) / 256;
    if (field == SD_FIELD_DENSITY && !view->rot_on) {
        k_project_columns<<<cb, 256, 0, st>>>(density, G, w.field);
        SD_LAUNCHED(st);
    } else {
        const bool disp = field == SD_FIELD_DISPERSION;
        if (SD_CUDA(cudaMemsetAsync(w.num, 0, sizeof(long long) * cells, st)) ||
            (disp && SD_CUDA(cudaMemsetAsync(w.den, 0, sizeof(long long) * cells, st))))
            return SD_E_CUDA;
        if (disp) {
            if (n > 0) {
                k_scatter_dispersion<<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<const float4*>(pos),
                                                                      reinterpret_cast<const float4*>(vel), n, G,
                                                                      *view, w.num, w.den);
                SD_LAUNCHED(st);
            }
        } else {
            const size_t all = (size_t)G * G * G;
            k_project_rotated<<<(unsigned)((all + 255) / 256), 256, 0, st>>>(density, G, *view, w.num);
            SD_LAUNCHED(st);
        }
        k_finish_field<<<cb, 256, 0, st>>>(w.num, disp ? w.den : nullptr, cells, w.field);
        SD_LAUNCHED(st);
    }
    const bool normalise = field == SD_FIELD_DENSITY;
    if (normalise) {
        if (SD_CUDA(cudaMemsetAsync(w.hist, 0, sizeof(int) * kHistBins, st))) return SD_E_CUDA;
        k_hist_log<<<cb, 256, 0, st>>>(w.field, cells, w.hist);
        SD_LAUNCHED(st);
    }
    // the mean density per screen cell when nothing is in the field (meanRho)
    k_brightness<<<1, 32, 0, st>>>(w.hist, (float)n / (float)cells, view->bright, normalise ? 1 : 0, w.bright);
    SD_LAUNCHED(st);
    const dim3 blk(16, 16), grd((width + 15) / 16, (height + 15) / 16);
    k_shade<<<grd, blk, 0, st>>>(w.field, G, reinterpret_cast<uchar4*>(rgba_out), width, height, w.bright,
                                 view->inv_gamma, view->cmap, view->zoom, view->pan_x, view->pan_y);
    SD_LAUNCHED(st);
    return SD_OK;
}

}  // extern "C"
