/*
 * pm_oracle.c -- CPU restatement of the reference's periodic particle-mesh step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA kernels in
 * stardust_b200/csrc and the timed CPU baseline of bench.py. Nothing in the
 * product path links, loads or calls it; the product fails loudly when its CUDA
 * library is missing instead of falling back here.
 *
 * Every function restates one piece of the reference (chdnl0420-svg/stardust,
 * src/sim/Sim.cu) in plain C with OpenMP. Floating-point expressions that nvcc
 * contracts into fused multiply-adds in the reference are written here with an
 * explicit fmaf(), and the build passes -ffp-contract=off, so that the result of
 * every expression is fixed by the source text alone. The CUDA kernels of this
 * project use the same explicit forms, which is what makes the fixed-point
 * density, the cell keys and the sort permutation comparable bit for bit.
 *
 * Conventions shared with the kernels:
 *   - particles are float4 (x, y, z, w) in box units [0,1); an empty slot has x < 0;
 *   - grids are G^3, G a power of two, index (z*G + y)*G + x;
 *   - density is in "count units" (each particle deposits total weight 1).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct { float x, y, z, w; } f4;
typedef struct { float re, im; } c32;

#define OR_FIXED_ONE 4294967296.0f          /* 2^32: fixed-point scale of a deposit weight */
#define OR_FIXED_INV 2.3283064365386963e-10f /* 2^-32 */

/* ------------------------------------------------------------------------- */
/* Cell keys.                                                                  */
/* ------------------------------------------------------------------------- */

/* Key modes. 0 = the reference's row-major key of the containing cell
 * (kCellKey, Sim.cu:2476-2486). 1 = 30-bit Morton code of the containing cell.
 * 2 = tile-row key of the CIC base cell: rows (y,z) of the base cell grouped in
 * 4x4 tiles, tile-major, 16 rows per tile (this project's deposit/gather order). */
enum { OR_KEY_ROWMAJOR = 0, OR_KEY_MORTON = 1, OR_KEY_TILEROW = 2 };

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static inline uint32_t part1by2(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000ffu;
    v = (v | (v << 8)) & 0x0300f00fu;
    v = (v | (v << 4)) & 0x030c30c3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

/* CIC base cell and fraction along one axis: g = p*G - 1/2 (Sim.cu:509-511). */
static inline void cic_axis(float p, int G, int* i, float* f) {
    const float g = fmaf(p, (float)G, -0.5f);
    const float fl = floorf(g);
    *i = (int)fl;
    *f = g - fl;
}

int32_t or_key_one(f4 p, int G, int mode) {
    if (p.x < 0.f) return -1;
    if (mode == OR_KEY_TILEROW) {
        int iy, iz; float f;
        cic_axis(p.y, G, &iy, &f);
        cic_axis(p.z, G, &iz, &f);
        iy &= (G - 1); iz &= (G - 1);
        const int tiles = G >> 2;
        const int tile = (iz >> 2) * tiles + (iy >> 2);
        return tile * 16 + (iz & 3) * 4 + (iy & 3);
    }
    const int cx = clampi((int)(p.x * (float)G), 0, G - 1);
    const int cy = clampi((int)(p.y * (float)G), 0, G - 1);
    const int cz = clampi((int)(p.z * (float)G), 0, G - 1);
    if (mode == OR_KEY_MORTON)
        return (int32_t)(part1by2((uint32_t)cx) | (part1by2((uint32_t)cy) << 1) |
                         (part1by2((uint32_t)cz) << 2));
    return (cz * G + cy) * G + cx;
}

void or_cell_keys(const f4* pos, int n, int G, int mode, int32_t* keys) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) keys[i] = or_key_one(pos[i], G, mode);
}

/* ------------------------------------------------------------------------- */
/* Stable sort of signed keys (the reference calls cub::DeviceRadixSort::      */
/* SortPairs over all 32 bits, Sim.cu:3659-3667: stable, and -1 sorts first).  */
/* LSD radix over (key + 1) as unsigned, 8 bits per pass, per-thread counts.   */
/* ------------------------------------------------------------------------- */
void or_stable_sort_perm(const int32_t* keys, int n, int key_bits, int32_t* perm) {
    uint32_t* k0 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    uint32_t* k1 = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)n);
    int32_t* v1 = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    for (int i = 0; i < n; ++i) { k0[i] = (uint32_t)(keys[i] + 1); perm[i] = i; }
    int32_t* v0 = perm;
    int nthreads = 1;
#ifdef _OPENMP
    nthreads = omp_get_max_threads();
#endif
    size_t* counts = (size_t*)malloc(sizeof(size_t) * 256 * (size_t)nthreads);
    int passes = 0;
    for (int shift = 0; shift < key_bits; shift += 8) {
        const int bits = (key_bits - shift) < 8 ? (key_bits - shift) : 8;
        const uint32_t mask = (1u << bits) - 1u;
        const int nb = 1 << bits;
        memset(counts, 0, sizeof(size_t) * 256 * (size_t)nthreads);
#pragma omp parallel num_threads(nthreads)
        {
            int t = 0;
#ifdef _OPENMP
            t = omp_get_thread_num();
#endif
            const int lo = (int)(((long long)n * t) / nthreads);
            const int hi = (int)(((long long)n * (t + 1)) / nthreads);
            size_t* c = counts + 256 * (size_t)t;
            for (int i = lo; i < hi; ++i) c[(k0[i] >> shift) & mask]++;
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (int d = 0; d < nb; ++d)
                    for (int tt = 0; tt < nthreads; ++tt) {
                        const size_t x = counts[256 * (size_t)tt + d];
                        counts[256 * (size_t)tt + d] = run;
                        run += x;
                    }
            }
            for (int i = lo; i < hi; ++i) {
                const size_t dst = c[(k0[i] >> shift) & mask]++;
                k1[dst] = k0[i];
                v1[dst] = v0[i];
            }
        }
        { uint32_t* t = k0; k0 = k1; k1 = t; }
        { int32_t* t = v0; v0 = v1; v1 = t; }
        ++passes;
    }
    if (v0 != perm) memcpy(perm, v0, sizeof(int32_t) * (size_t)n);
    free(counts);
    free(k0);
    free(k1);
    free(v0 == perm ? v1 : v0);
}

/* kReorder (Sim.cu:2488-2495): dst[i] = src[order[i]]. */
void or_reorder(const f4* src, const int32_t* order, int n, f4* dst) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) dst[i] = src[order[i]];
}

/* ------------------------------------------------------------------------- */
/* CIC deposit (kScatter, Sim.cu:503-521).                                     */
/* ------------------------------------------------------------------------- */

/* Weight of corner k = ox | oy<<1 | oz<<2, multiplied left to right as in the
 * reference: (wx * wy) * wz. */
static inline float cic_weight(int k, float fx, float fy, float fz) {
    const float wx = (k & 1) ? fx : 1.f - fx;
    const float wy = (k & 2) ? fy : 1.f - fy;
    const float wz = (k & 4) ? fz : 1.f - fz;
    return (wx * wy) * wz;
}

/* Deterministic deposit: each weight is rounded once to a multiple of 2^-32 and
 * summed exactly in int64, so the sum does not depend on the order of the adds.
 * acc must be zeroed by the caller (G^3 entries). */
void or_deposit_fixed(const f4* pos, int n, int G, int64_t* acc) {
    const int m = G - 1;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const f4 p = pos[i];
        if (p.x < 0.f) continue;
        int ix, iy, iz; float fx, fy, fz;
        cic_axis(p.x, G, &ix, &fx);
        cic_axis(p.y, G, &iy, &fy);
        cic_axis(p.z, G, &iz, &fz);
        for (int k = 0; k < 8; ++k) {
            const int cx = (ix + (k & 1)) & m;
            const int cy = (iy + ((k >> 1) & 1)) & m;
            const int cz = (iz + ((k >> 2) & 1)) & m;
            const float w = cic_weight(k, fx, fy, fz);
            const int64_t q = llrintf(w * OR_FIXED_ONE);
            int64_t* dst = acc + ((size_t)cz * G + cy) * G + cx;
#pragma omp atomic
            *dst += q;
        }
    }
}

void or_fixed_to_float(const int64_t* acc, size_t cells, float* rho) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < cells; ++i) rho[i] = (float)acc[i] * OR_FIXED_INV;
}

/* The reference's float accumulation, in particle index order (sequential). */
void or_deposit_float(const f4* pos, int n, int G, float* rho) {
    const int m = G - 1;
    for (int i = 0; i < n; ++i) {
        const f4 p = pos[i];
        if (p.x < 0.f) continue;
        int ix, iy, iz; float fx, fy, fz;
        cic_axis(p.x, G, &ix, &fx);
        cic_axis(p.y, G, &iy, &fy);
        cic_axis(p.z, G, &iz, &fz);
        for (int k = 0; k < 8; ++k) {
            const int cx = (ix + (k & 1)) & m;
            const int cy = (iy + ((k >> 1) & 1)) & m;
            const int cz = (iz + ((k >> 2) & 1)) & m;
            rho[((size_t)cz * G + cy) * G + cx] += cic_weight(k, fx, fy, fz);
        }
    }
}

/* ------------------------------------------------------------------------- */
/* FFT (project-written; the reference uses cuFFT, a closed library).           */
/* Iterative radix-2 complex transform with a twiddle table built in double.     */
/* ------------------------------------------------------------------------- */
typedef struct {
    int n;
    int logn;
    c32* tw;     /* tw[k] = exp(-2 pi i k / n), k < n/2 */
    int* rev;
} fft_plan;

static void plan_init(fft_plan* p, int n) {
    p->n = n;
    p->logn = 0;
    while ((1 << p->logn) < n) ++p->logn;
    p->tw = (c32*)malloc(sizeof(c32) * (size_t)(n / 2 > 0 ? n / 2 : 1));
    p->rev = (int*)malloc(sizeof(int) * (size_t)n);
    for (int k = 0; k < n / 2; ++k) {
        const double a = -2.0 * 3.14159265358979323846 * (double)k / (double)n;
        p->tw[k].re = (float)cos(a);
        p->tw[k].im = (float)sin(a);
    }
    for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int b = 0; b < p->logn; ++b) r |= ((i >> b) & 1) << (p->logn - 1 - b);
        p->rev[i] = r;
    }
}

static void plan_free(fft_plan* p) { free(p->tw); free(p->rev); }

/* In-place transform of a contiguous line; inverse = conjugate twiddles, no scaling. */
static void fft_line(const fft_plan* p, c32* a, int inverse) {
    const int n = p->n;
    for (int i = 0; i < n; ++i) {
        const int r = p->rev[i];
        if (r > i) { const c32 t = a[i]; a[i] = a[r]; a[r] = t; }
    }
    for (int len = 2; len <= n; len <<= 1) {
        const int half = len >> 1, step = n / len;
        for (int s = 0; s < n; s += len) {
            for (int j = 0; j < half; ++j) {
                c32 w = p->tw[j * step];
                if (inverse) w.im = -w.im;
                const c32 u = a[s + j], v = a[s + j + half];
                const c32 t = { v.re * w.re - v.im * w.im, v.re * w.im + v.im * w.re };
                a[s + j].re = u.re + t.re;  a[s + j].im = u.im + t.im;
                a[s + j + half].re = u.re - t.re;  a[s + j + half].im = u.im - t.im;
            }
        }
    }
}

/* Real line of length n -> n/2+1 complex bins, through one n/2-point complex
 * transform of z[m] = x[2m] + i x[2m+1]. tw_n holds exp(-2 pi i k / n). */
static void r2c_line(const fft_plan* half, const c32* tw_n, const float* x, c32* out, c32* work) {
    const int M = half->n;
    for (int m = 0; m < M; ++m) { work[m].re = x[2 * m]; work[m].im = x[2 * m + 1]; }
    fft_line(half, work, 0);
    for (int k = 0; k <= M; ++k) {
        const c32 zk = work[k % M];
        const c32 zc = work[(M - k) % M];   /* Z[M-k], to be conjugated */
        const float er = 0.5f * (zk.re + zc.re), ei = 0.5f * (zk.im - zc.im);
        const float orr = 0.5f * (zk.im + zc.im), oi = -0.5f * (zk.re - zc.re);
        const c32 w = tw_n[k];               /* exp(-2 pi i k / n), k <= n/2 */
        out[k].re = er + (w.re * orr - w.im * oi);
        out[k].im = ei + (w.re * oi + w.im * orr);
    }
}

/* n/2+1 Hermitian bins -> real line of length n (unnormalised inverse). The
 * imaginary parts of bins 0 and n/2 are ignored. */
static void c2r_line(const fft_plan* half, const c32* tw_n, const c32* in, float* x, c32* work) {
    const int M = half->n;
    for (int k = 0; k < M; ++k) {
        c32 a = in[k], b = in[M - k];
        if (k == 0) { a.im = 0.f; b.im = 0.f; }
        /* E = X[k] + conj(X[M-k]);  O = (X[k] - conj(X[M-k])) * exp(+2 pi i k / n) */
        const float er = a.re + b.re, ei = a.im - b.im;
        const float dr = a.re - b.re, di = a.im + b.im;
        const c32 w = tw_n[k];
        const float orr = dr * w.re + di * w.im, oi = di * w.re - dr * w.im;
        work[k].re = er - oi;
        work[k].im = ei + orr;
    }
    fft_line(half, work, 1);
    for (int m = 0; m < M; ++m) { x[2 * m] = work[m].re; x[2 * m + 1] = work[m].im; }
}

/* Periodic Poisson solve with the reference's Green's function
 * (kPoissonPeriodic Sim.cu:528-557, scale Sim.cu:3590-3595), in float with
 * this file's FFT: phi = IFFT( FFT(rho) * -scale/k^2 * exp(-k^2 s^2 / 2) ). */
void or_poisson_periodic(const float* rho, int G, float soft_cells, float* phi) {
    const int H = G / 2, P = H + 1;
    const size_t rows = (size_t)G * G;
    c32* spec = (c32*)malloc(sizeof(c32) * rows * P);
    fft_plan ph, pg;
    plan_init(&ph, H);
    plan_init(&pg, G);
    c32* twn = (c32*)malloc(sizeof(c32) * (size_t)(H + 1));
    for (int k = 0; k <= H; ++k) {
        const double a = -2.0 * 3.14159265358979323846 * (double)k / (double)G;
        twn[k].re = (float)cos(a);
        twn[k].im = (float)sin(a);
    }
    /* x lines */
#pragma omp parallel
    {
        c32* work = (c32*)malloc(sizeof(c32) * (size_t)G);
#pragma omp for schedule(static)
        for (long r = 0; r < (long)rows; ++r) r2c_line(&ph, twn, rho + (size_t)r * G, spec + (size_t)r * P, work);
        free(work);
    }
    /* y then z lines (forward), Green's multiply, z then y (inverse) */
    const float norm = 1.0f / (float)((double)G * G * G);
    const float scale = norm / (4.0f * 3.14159265f * 3.14159265f);
    const float s = 6.2831853f * soft_cells / (float)G;
    for (int pass = 0; pass < 2; ++pass) {
        /* y lines: fixed (z, kx) */
#pragma omp parallel
        {
            c32* line = (c32*)malloc(sizeof(c32) * (size_t)G);
#pragma omp for schedule(static)
            for (long t = 0; t < (long)G * P; ++t) {
                const int z = (int)(t / P), kx = (int)(t % P);
                for (int y = 0; y < G; ++y) line[y] = spec[((size_t)z * G + y) * P + kx];
                fft_line(&pg, line, pass);
                for (int y = 0; y < G; ++y) spec[((size_t)z * G + y) * P + kx] = line[y];
            }
            free(line);
        }
        if (pass == 1) break;
        /* z lines: fixed (y, kx); forward, multiply, inverse */
#pragma omp parallel
        {
            c32* line = (c32*)malloc(sizeof(c32) * (size_t)G);
#pragma omp for schedule(static)
            for (long t = 0; t < (long)G * P; ++t) {
                const int y = (int)(t / P), kx = (int)(t % P);
                for (int z = 0; z < G; ++z) line[z] = spec[((size_t)z * G + y) * P + kx];
                fft_line(&pg, line, 0);
                const int ky = (y <= G / 2) ? y : y - G;
                for (int z = 0; z < G; ++z) {
                    const int kz = (z <= G / 2) ? z : z - G;
                    const float k2 = (float)(kx * kx + ky * ky + kz * kz);
                    if (k2 < 1e-6f) { line[z].re = 0.f; line[z].im = 0.f; continue; }
                    float m = -scale / k2;
                    if (soft_cells > 0.f) m *= expf(-0.5f * k2 * s * s);
                    line[z].re *= m; line[z].im *= m;
                }
                fft_line(&pg, line, 1);
                for (int z = 0; z < G; ++z) spec[((size_t)z * G + y) * P + kx] = line[z];
            }
            free(line);
        }
    }
#pragma omp parallel
    {
        c32* work = (c32*)malloc(sizeof(c32) * (size_t)G);
#pragma omp for schedule(static)
        for (long r = 0; r < (long)rows; ++r) c2r_line(&ph, twn, spec + (size_t)r * P, phi + (size_t)r * G, work);
        free(work);
    }
    free(twn);
    plan_free(&ph);
    plan_free(&pg);
    free(spec);
}

/* ------------------------------------------------------------------------- */
/* Gradient, gather, kick, drift.                                              */
/* ------------------------------------------------------------------------- */

/* kGridAccel, periodic branch (Sim.cu:589-611): a = -(phi[+1] - phi[-1]) * h,
 * h = 0.5 * G * potScale. Output float4 per cell (w = 0). */
void or_grid_accel(const float* phi, int G, float pot_scale, f4* acc) {
    const int m = G - 1;
    const float h = (0.5f * (float)G) * pot_scale;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < G; ++z)
        for (int y = 0; y < G; ++y)
            for (int x = 0; x < G; ++x) {
                const int xm = (x - 1) & m, xp = (x + 1) & m;
                const int ym = (y - 1) & m, yp = (y + 1) & m;
                const int zm = (z - 1) & m, zp = (z + 1) & m;
                f4 a;
                a.x = -(phi[((size_t)z * G + y) * G + xp] - phi[((size_t)z * G + y) * G + xm]) * h;
                a.y = -(phi[((size_t)z * G + yp) * G + x] - phi[((size_t)z * G + ym) * G + x]) * h;
                a.z = -(phi[((size_t)zp * G + y) * G + x] - phi[((size_t)zm * G + y) * G + x]) * h;
                a.w = 0.f;
                acc[((size_t)z * G + y) * G + x] = a;
            }
}

/* sampleAcc (Sim.cu:614-629): CIC read of the cell accelerations. */
static inline f4 sample_acc(const f4* acc, f4 p, int G) {
    const int m = G - 1;
    int ix, iy, iz; float fx, fy, fz;
    cic_axis(p.x, G, &ix, &fx);
    cic_axis(p.y, G, &iy, &fy);
    cic_axis(p.z, G, &iz, &fz);
    f4 a = { 0.f, 0.f, 0.f, 0.f };
    for (int k = 0; k < 8; ++k) {
        const float w = cic_weight(k, fx, fy, fz);
        const int cx = (ix + (k & 1)) & m;
        const int cy = (iy + ((k >> 1) & 1)) & m;
        const int cz = (iz + ((k >> 2) & 1)) & m;
        const f4 g = acc[((size_t)cz * G + cy) * G + cx];
        a.x = fmaf(g.x, w, a.x);
        a.y = fmaf(g.y, w, a.y);
        a.z = fmaf(g.z, w, a.z);
    }
    return a;
}

/* The plain-PM part of kIntegrate (Sim.cu:685-906) on a periodic box: gather,
 * kick by dt_kick, light-speed clamp (Sim.cu:834-840), drift by dt_drift, NaN
 * to empty slot (Sim.cu:846-851), periodic wrap (Sim.cu:853-854). The reference
 * has dt_kick == dt_drift; a leapfrog opening step uses dt_kick = dt/2. */
void or_integrate(const f4* acc, f4* pos, f4* vel, int n, int G, float dt_kick, float dt_drift, float c2) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        f4 p = pos[i];
        if (p.x < 0.f) continue;
        f4 v = vel[i];
        const f4 a = sample_acc(acc, p, G);
        v.x = fmaf(a.x, dt_kick, v.x);
        v.y = fmaf(a.y, dt_kick, v.y);
        v.z = fmaf(a.z, dt_kick, v.z);
        {
            const float sp2 = fmaf(v.z, v.z, fmaf(v.y, v.y, v.x * v.x));
            if (sp2 > c2) {
                const float k = sqrtf(c2 / sp2);
                v.x *= k; v.y *= k; v.z *= k;
            }
        }
        p.x = fmaf(v.x, dt_drift, p.x);
        p.y = fmaf(v.y, dt_drift, p.y);
        p.z = fmaf(v.z, dt_drift, p.z);
        if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z) ||
            !isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) {
            const f4 e = { -1.f, -1.f, -1.f, 0.f }, z = { 0.f, 0.f, 0.f, 0.f };
            pos[i] = e; vel[i] = z;
            continue;
        }
        p.x -= floorf(p.x); p.y -= floorf(p.y); p.z -= floorf(p.z);
        pos[i] = p; vel[i] = v;
    }
}

/* kMomentumAccum + kSubtractMeanVelDev (Sim.cu:2252-2291): sums over live
 * particles with finite velocity, in double; subtract (float)(sum/count).
 * out[0..3] receives (sum vx, sum vy, sum vz, count). */
void or_momentum_zero(const f4* pos, f4* vel, int n, double* out) {
    double sx = 0, sy = 0, sz = 0, c = 0;
    for (int i = 0; i < n; ++i) {
        if (pos[i].x < 0.f) continue;
        const f4 v = vel[i];
        if (!isfinite(v.x) || !isfinite(v.y) || !isfinite(v.z)) continue;
        sx += v.x; sy += v.y; sz += v.z; c += 1.0;
    }
    if (out) { out[0] = sx; out[1] = sy; out[2] = sz; out[3] = c; }
    if (c < 1.0) return;
    const float mx = (float)(sx / c), my = (float)(sy / c), mz = (float)(sz / c);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        if (pos[i].x < 0.f) continue;
        vel[i].x -= mx; vel[i].y -= my; vel[i].z -= mz;
    }
}

/* kMaxSpeed (Sim.cu:2923-2930). */
float or_max_speed(const f4* pos, const f4* vel, int n) {
    float vmax = 0.f;
#pragma omp parallel for reduction(max : vmax) schedule(static)
    for (int i = 0; i < n; ++i) {
        if (pos[i].x < 0.f) continue;
        const f4 v = vel[i];
        const float s = sqrtf(fmaf(v.z, v.z, fmaf(v.y, v.y, v.x * v.x)));
        if (s > vmax) vmax = s;
    }
    return vmax;
}

/* ------------------------------------------------------------------------- */
/* One whole step in the reference's order (Sim::step, Sim.cu:4240-4525, with   */
/* cooling, pressure, contact, black holes and stars off): sort every call,     */
/* deposit, Poisson, gradient, integrate, momentum zeroing.                     */
/* deterministic != 0 deposits in fixed point (this project's density); 0 uses  */
/* the reference's float accumulation. Scratch buffers are allocated per call.  */
/* ------------------------------------------------------------------------- */
int or_step(f4* pos, f4* vel, int n, int G, float gravity, float soft_cells, float dt_kick,
            float dt_drift, float c2, int key_mode, int deterministic, float* rho_out, double* mom_out) {
    const size_t cells = (size_t)G * G * G;
    int32_t* keys = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* order = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    f4* tmp = (f4*)malloc(sizeof(f4) * (size_t)n);
    float* rho = (float*)malloc(sizeof(float) * cells);
    float* phi = (float*)malloc(sizeof(float) * cells);
    f4* acc = (f4*)malloc(sizeof(f4) * cells);
    if (!keys || !order || !tmp || !rho || !phi || !acc) return -1;

    int key_bits = 0;
    {
        /* largest shifted key (key + 1): G^3 for row-major and Morton codes, G^2 for tile rows */
        const long long top = (key_mode == OR_KEY_TILEROW) ? (long long)G * G : (long long)cells;
        while ((1ll << key_bits) < top + 1) ++key_bits;
    }
    or_cell_keys(pos, n, G, key_mode, keys);
    or_stable_sort_perm(keys, n, key_bits, order);
    or_reorder(pos, order, n, tmp); memcpy(pos, tmp, sizeof(f4) * (size_t)n);
    or_reorder(vel, order, n, tmp); memcpy(vel, tmp, sizeof(f4) * (size_t)n);

    if (deterministic) {
        int64_t* q = (int64_t*)calloc(cells, sizeof(int64_t));
        or_deposit_fixed(pos, n, G, q);
        or_fixed_to_float(q, cells, rho);
        free(q);
    } else {
        memset(rho, 0, sizeof(float) * cells);
        or_deposit_float(pos, n, G, rho);
    }
    if (rho_out) memcpy(rho_out, rho, sizeof(float) * cells);
    or_poisson_periodic(rho, G, soft_cells, phi);
    or_grid_accel(phi, G, gravity / (float)n, acc);
    or_integrate(acc, pos, vel, n, G, dt_kick, dt_drift, c2);
    or_momentum_zero(pos, vel, n, mom_out);

    free(keys); free(order); free(tmp); free(rho); free(phi); free(acc);
    return 0;
}

int or_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
