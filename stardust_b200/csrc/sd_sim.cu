// sd_sim.cu -- the simulation handle and the C ABI (include/stardust_pm.h).
//
// Reference counterpart: class Sim and Sim::Impl (src/sim/Sim.h:854-1135,
// src/sim/Sim.cu:2937-3168, 3895-4525, 4985-5120). One handle owns its device
// buffers and a stream; all work is issued on that stream with no host
// synchronisation inside a step (the reference syncs twice per step: the vmax
// read and the end-of-step event; sd_step_auto keeps the vmax read).
//
// Step pipeline (periodic, plain PM):
//   [sort]    keys -> stable LSD radix sort -> reorder pos/vel (ping-pong buffers)
//   deposit   int64 fixed-point CIC into `acc`
//   Poisson   pass A (reads and clears acc) .. pass E -> phi
//   gather    gradient of phi at the 8 corners + kick + clamp + drift + wrap,
//             FP64 momentum partials -> mean, subtracted at the next load
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <cmath>
#include <mutex>
#include <utility>
#include <vector>

#include "sd_internal.h"
#include "sd_sim_impl.h"

// ---------------------------------------------------------------------------
// sticky error record and launch accounting
// ---------------------------------------------------------------------------
namespace sd {
namespace {
std::mutex g_err_mu;
bool g_failed = false;
char g_msg[512] = {0};
std::atomic<long long> g_launches{0};
}  // namespace

int fail(int code, const char* fmt, ...) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    if (!g_failed) {
        g_failed = true;
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
        va_end(ap);
    }
    return code;
}

int check_cuda(cudaError_t e, const char* what, const char* file, int line) {
    if (e == cudaSuccess) return SD_OK;
    const char* base = strrchr(file, '/');
    fail(e == cudaErrorMemoryAllocation ? SD_E_NOMEM : SD_E_CUDA, "%s: %s (%s:%d)", what, cudaGetErrorString(e),
         base ? base + 1 : file, line);
    return e == cudaErrorMemoryAllocation ? SD_E_NOMEM : SD_E_CUDA;
}

void count_launch(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launches() { return g_launches.load(std::memory_order_relaxed); }
}  // namespace sd

using namespace sd;

namespace sdsim {

DeviceGuard::DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) cudaSetDevice(dev);
}
DeviceGuard::~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
}

int ceil_pow2_clamp(int g, int cap) {
    if (g <= 0) g = 64;
    if (g > cap) g = cap;
    if (g < 16) g = 16;
    int p = 16;
    while (p * 2 <= g) p *= 2;  // round down to a power of two (Sim.cu:4081-4086)
    return p;
}

float light_speed_sq(float length_scale, float time_unit_scale) {
    // lightSpeedSqFor (Sim.h:133-148): c = (1e7 * tus) / (1e5 * ls)
    const double L = 1.0e5 * (double)(length_scale > 1e-6f ? length_scale : 1e-6f);
    const double T = 1.0e7 * (double)(time_unit_scale > 1e-6f ? time_unit_scale : 1e-6f);
    const float c = (float)(T / (L > 1e-30 ? L : 1e-30));
    return c * c;
}

float dt_scale_for(float ts) {  // dtScaleFor (Sim.h:89-93)
    if (ts <= 1.0f) return ts;
    return (ts <= 3.0f) ? 1.0f : (ts / 3.0f);
}

int key_bits_for(int G, int order) {
    // largest key: G^2 - 1 (tiled rows) or G^3 (row-major / Morton key + 1)
    const long long top = (order == SD_ORDER_TILED) ? (long long)G * G - 1 : (long long)G * G * G;
    int b = 0;
    while ((1ll << b) < top + 1) ++b;
    return b;
}

bool isolated(const sd_sim* s) { return s->cfg.boundary == SD_BOUNDARY_ISOLATED; }

// Side of the Poisson transform box: G (periodic) or 2G (isolated, Sim.cu:3100).
int box_of(int G, int boundary) { return boundary == SD_BOUNDARY_ISOLATED ? 2 * G : G; }

float pot_scale_of(const sd_sim* s) {
    const double n = (double)(s->N > 0 ? s->N : 1);
    if (s->cfg.units == SD_UNITS_NEWTON) {
        // periodic: the spectral Green's function carries 1/(4 pi^2) in box units (factor
        // 4 pi G^3); isolated: -1/r in cell units (factor G)
        const double f = isolated(s) ? (double)s->G : 4.0 * 3.14159265358979323846 * (double)s->G * s->G * s->G;
        return (float)(f * (double)s->cfg.gravity / n);
    }
    return s->cfg.gravity / (float)(s->N > 0 ? s->N : 1);  // potScale (Sim.cu:3107-3109)
}

// Isolated-boundary options of a Poisson solve on this handle (nullptr: periodic).
const PoissonIso* iso_opts(const sd_sim* s, PoissonIso& o) {
    if (!isolated(s)) return nullptr;
    const int S = 2 * s->G;
    o.src_g = s->G;
    o.table = s->green;
    o.table_scale = (float)(1.0 / ((double)S * S * S));  // kMulSpec's FFT normalisation (Sim.cu:3590-3599)
    return &o;
}

template <class T>
void free_dev(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

void free_buffers(sd_sim* s) {
    free_dev(s->pos); free_dev(s->vel); free_dev(s->pos2); free_dev(s->vel2);
    free_dev(s->stage_pos); free_dev(s->stage_vel);
    s->stage_free = nullptr;
    free_dev(s->keys); free_dev(s->keys2); free_dev(s->keys3);
    free_dev(s->vals); free_dev(s->vals2);
    if (s->sort_ws) cudaFree(s->sort_ws);
    s->sort_ws = nullptr;
    s->sort_ws_bytes = 0;
    free_dev(s->acc); free_dev(s->row_start); free_dev(s->dep_ints); free_dev(s->spec); free_dev(s->phi);
    free_dev(s->rho);
    free_dev(s->green);
    hydro_free(s->hydro);
    if (s->rs_base) cudaFree(s->rs_base);
    s->rs_base = nullptr;
    free_dev(s->partials); free_dev(s->mom); free_dev(s->mean);
    free_dev(s->mlp_out);
    free_dev(s->diag_rec);
    free_dev(s->diag_count);
    poisson_plan_free(s->plan);
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    s->configured = false;
}

template <class T>
int alloc_dev(T*& p, size_t count) {
    if (cudaMalloc((void**)&p, sizeof(T) * (count > 0 ? count : 1)) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        return fail(SD_E_NOMEM, "cudaMalloc of %zu bytes failed", sizeof(T) * count);
    }
    return SD_OK;
}

size_t estimate_bytes(int n, int G, int boundary) {
    const size_t N = (size_t)(n > 0 ? n : 1), cells = (size_t)G * G * G;
    const int S = box_of(G, boundary);
    const size_t box = (size_t)S * S * S;
    size_t b = 0;
    b += sizeof(float4) * N * 4;                       // pos, vel, pos2, vel2
    b += (sizeof(uint32_t) * 3 + sizeof(int32_t) * 2) * N;
    b += sort_workspace_bytes((int)N);
    b += sizeof(long long) * cells;                    // fixed-point deposit
    b += sizeof(int) * deposit_work_ints(G);           // the fused deposit's work plan
    b += sizeof(float2) * poisson_spectrum_elems(S);
    b += sizeof(float) * (box + cells);                // phi, kept density
    if (S != G) b += sizeof(float) * green_table_elems(S);
    b += sizeof(double) * 8 * (gather_partials((int)N) + 1024);
    if (S == G) b += resort_bytes((int)N, G);  // the merge sort (periodic box, tiled order)
    return b;
}

int allocate(sd_sim* s) {
    free_buffers(s);
    const size_t N = (size_t)s->N, cells = (size_t)s->G * s->G * s->G;
    const int S = box_of(s->G, s->cfg.boundary);
    const size_t box = (size_t)S * S * S;
    int rc = SD_OK;
    rc = rc ? rc : alloc_dev(s->pos, N);
    rc = rc ? rc : alloc_dev(s->vel, N);
    rc = rc ? rc : alloc_dev(s->pos2, N);
    rc = rc ? rc : alloc_dev(s->vel2, N);
    rc = rc ? rc : alloc_dev(s->keys, N);
    rc = rc ? rc : alloc_dev(s->keys2, N);
    rc = rc ? rc : alloc_dev(s->keys3, N);
    rc = rc ? rc : alloc_dev(s->vals, N);
    rc = rc ? rc : alloc_dev(s->vals2, N);
    s->sort_ws_bytes = sort_workspace_bytes(s->N);
    if (!rc && cudaMalloc(&s->sort_ws, s->sort_ws_bytes) != cudaSuccess) {
        cudaGetLastError();
        rc = fail(SD_E_NOMEM, "cudaMalloc of sort workspace failed");
    }
    // the sort's count buffers start zero and every sort leaves them zero
    if (!rc && SD_CUDA(cudaMemset(s->sort_ws, 0, s->sort_ws_bytes))) rc = SD_E_CUDA;
    rc = rc ? rc : alloc_dev(s->acc, cells);
    rc = rc ? rc : alloc_dev(s->row_start, (size_t)s->G * s->G + 1);
    rc = rc ? rc : alloc_dev(s->dep_ints, deposit_work_ints(s->G));
    rc = rc ? rc : alloc_dev(s->spec, poisson_spectrum_elems(S));
    rc = rc ? rc : alloc_dev(s->phi, box);
    if (!rc && isolated(s)) rc = alloc_dev(s->green, green_table_elems(S));
    if (!rc && (s->cfg.keep_density || s->mlp_on)) rc = alloc_dev(s->rho, cells);
    if (!rc && s->mlp_on) rc = alloc_dev(s->mlp_out, N);
    s->partials_count = 8 * (gather_partials(s->N) + 1024);
    rc = rc ? rc : alloc_dev(s->partials, s->partials_count);
    rc = rc ? rc : alloc_dev(s->mom, 8);
    rc = rc ? rc : alloc_dev(s->mean, 4);
    rc = rc ? rc : alloc_dev(s->diag_rec, (size_t)kDiagCap * 8);
    rc = rc ? rc : alloc_dev(s->diag_count, 1);
    if (rc) {
        free_buffers(s);
        return rc;
    }
    rc = poisson_plan_build(s->plan, S, s->cfg.softening_cells);
    // the isolated Green spectrum, with phi and the spectrum as scratch (buildGreen, Sim.cu:3569-3576)
    if (!rc && isolated(s)) rc = build_green_table(s->plan, s->cfg.softening_cells, s->phi, s->spec, s->green, s->stream);
    if (rc) {
        free_buffers(s);
        return rc;
    }
    // zeroed state: empty slots, clear fixed-point grid, no pending mean
    if (SD_CUDA(cudaMemsetAsync(s->acc, 0, sizeof(long long) * cells, s->stream)) ||
        SD_CUDA(cudaMemsetAsync(s->dep_ints, 0, sizeof(int) * deposit_work_ints(s->G), s->stream)) ||
        SD_CUDA(cudaMemsetAsync(s->mean, 0, sizeof(float) * 4, s->stream)) ||
        SD_CUDA(cudaMemsetAsync(s->mom, 0, sizeof(double) * 8, s->stream)) ||
        SD_CUDA(cudaMemsetAsync(s->diag_count, 0, sizeof(unsigned long long), s->stream)) ||
        SD_CUDA(cudaMemsetAsync(s->phi, 0, sizeof(float) * box, s->stream))) {
        free_buffers(s);
        return SD_E_CUDA;
    }
    rc = launch_hide_range(s->pos, s->vel, 0, s->N, s->stream);
    if (rc) return rc;
    s->configured = true;
    return SD_OK;
}

int validate_config(const sd_config* c) {
    if (!c) return fail(SD_E_ARG, "config: null");
    if (c->particle_count <= 0 || c->particle_count > 400000000)
        return fail(SD_E_ARG, "config: particle_count %d out of range", c->particle_count);
    if (c->boundary != SD_BOUNDARY_PERIODIC && c->boundary != SD_BOUNDARY_ISOLATED)
        return fail(SD_E_ARG, "config: bad boundary %d", c->boundary);
    if (c->order < SD_ORDER_ROWMAJOR || c->order > SD_ORDER_TILED) return fail(SD_E_ARG, "config: bad order");
    if (c->full_sort < -1 || c->full_sort > 1) return fail(SD_E_ARG, "config: full_sort must be -1, 0 or 1");
    if (c->integrator != SD_INT_KD && c->integrator != SD_INT_KDK) return fail(SD_E_ARG, "config: bad integrator");
    if (c->units != SD_UNITS_REFERENCE && c->units != SD_UNITS_NEWTON) return fail(SD_E_ARG, "config: bad units");
    if (c->preset != SD_PRESET_FILAMENT && c->preset != SD_PRESET_EMPTY) return fail(SD_E_ARG, "config: bad preset");
    if (!std::isfinite(c->pressure_k) || !std::isfinite(c->cooling_rate))
        return fail(SD_E_ARG, "config: non-finite pressure_k or cooling_rate");
    return SD_OK;
}

bool hydro_on(const sd_sim* s) { return s->cfg.pressure_enabled || (s->cfg.cooling_enabled && s->cfg.cooling_rate > 0.f); }

// doCooling's period (Sim.cu:3737): every 2 steps with pressure, every 8 without.
int cooling_period(const sd_sim* s) { return s->cfg.pressure_enabled ? 2 : 8; }

// The hydro grids exist while either add-on is on (zeroed when made, as the
// reference's are at allocation); toggling does not touch the particles.
int ensure_hydro(sd_sim* s) {
    if (!hydro_on(s)) {
        hydro_free(s->hydro);
        return SD_OK;
    }
    if (s->hydro.base && s->hydro.G == s->G) return SD_OK;
    hydro_free(s->hydro);
    return hydro_alloc(s->hydro, s->G);
}

// The keys no longer describe the particles (loaded, moved or reordered outside
// a step): no sort counts, no merge sort until a full one.
void invalidate_keys(sd_sim* s) {
    s->keys_valid = false;
    s->counts_valid = false;
    s->incr_ready = false;
}

bool incr_possible(const sd_sim* s) {
    return s->allow_incr && s->cfg.full_sort != 1 && s->cfg.order == SD_ORDER_TILED && !isolated(s);
}

// Above this share of changed keys the full radix sort is cheaper than the merge
// (4M particles on 256^3 with a third of the keys changing: merge 0.146 ms, full
// sort with its row table 0.093 ms; 16M on 512^3 with 0.8 % changing: merge
// 0.12 ms, full sort 0.23 ms). Below kMergeMinParticles the merge's dozen launches
// cost more than a full sort whatever changes (262,144 particles on 64^3 with 9 %
// changing: merge 0.107 ms, full sort and row table 0.05 ms).
constexpr double kMergeMaxFraction = 0.10;
constexpr int kMergeProbe = 64;
constexpr int kMergeMinParticles = 1 << 22;

// The next sorted step leaves change bits for a merge (otherwise first-pass counts).
bool merge_next(const sd_sim* s) {
    if (!s->rs_base || !incr_possible(s)) return false;
    return s->cfg.full_sort == -1 || (!s->merge_off && s->N >= kMergeMinParticles);
}

// Read the share of keys the last merge found changed (written to pinned memory
// by the device, possibly a step or more behind) and choose merge or full sort.
void update_merge_policy(sd_sim* s) {
    if (!s->rs_base || !s->chg_host) return;
    if (s->cfg.full_sort == -1) s->merge_off = false;  // merges asked for whatever changes
    const int c = *reinterpret_cast<volatile int*>(s->chg_host);
    if (c >= 0 && s->N > 0) s->chg_frac = (double)c / (double)s->N;
    if (!s->merge_off) {
        if (c >= 0 && s->chg_frac > kMergeMaxFraction) {
            s->merge_off = true;
            s->merge_probe_at = s->step_count + kMergeProbe;
        }
    } else if (s->step_count >= s->merge_probe_at) {
        // probe: merge again, and decide on the share that merge measures
        s->merge_off = false;
        *reinterpret_cast<volatile int*>(s->chg_host) = -1;
    }
}

// Merge-sort buffers exist while the configuration can merge-sort (zeroed when made).
int ensure_resort(sd_sim* s) {
    if (!incr_possible(s)) {
        if (s->rs_base) cudaFree(s->rs_base);
        s->rs_base = nullptr;
        s->incr_ready = s->chg_dirty = false;
        return SD_OK;
    }
    if (s->rs_base) return SD_OK;
    if (!s->chg_host) {
        if (cudaHostAlloc((void**)&s->chg_host, sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            s->chg_host = nullptr;
            return fail(SD_E_NOMEM, "cudaHostAlloc of the changed-key count failed");
        }
        *s->chg_host = -1;
    }
    s->chg_frac = -1.0;
    s->merge_off = false;
    const size_t b = resort_bytes(s->N, s->G);
    if (cudaMalloc(&s->rs_base, b) != cudaSuccess) {
        cudaGetLastError();
        s->rs_base = nullptr;
        return fail(SD_E_NOMEM, "cudaMalloc of the merge-sort buffers failed");
    }
    // the full sort's scratch (sorted keys, temporaries) is idle while a merge runs
    s->rs = resort_layout(s->rs_base, s->N, s->G, s->keys2, s->vals2, s->keys3);
    s->incr_ready = s->chg_dirty = false;
    return SD_CUDA(cudaMemset(s->rs_base, 0, b));
}

// placeInitial + reset's velocity and centre-of-mass passes (Sim.cu:3635-3649,
// 4160-4238): the configured preset in every slot. The mean buffer serves as
// scratch and is left zero (no correction pending).
int place_initial(sd_sim* s) {
    int rc = launch_place_preset(s->pos, s->vel, s->N, s->cfg, s->partials, s->mom, s->mean, s->stream);
    if (!rc && SD_CUDA(cudaMemsetAsync(s->mean, 0, sizeof(float) * 4, s->stream))) rc = SD_E_CUDA;
    s->active = (s->cfg.preset == SD_PRESET_FILAMENT) ? s->N : 0;
    s->mean_pending = false;
    s->rho_valid = false;
    invalidate_keys(s);
    return rc;
}

int sim_error(sd_sim* s, int rc) {
    if (rc == SD_E_CUDA) s->cuda_failed = true;
    return rc;
}

// Apply the pending mean-velocity subtraction to the stored velocities.
int materialize(sd_sim* s) {
    if (!s->mean_pending) return SD_OK;
    int rc = launch_apply_mean(s->vel, s->pos, s->N, s->mean, s->stream);
    if (rc) return sim_error(s, rc);
    if (SD_CUDA(cudaMemsetAsync(s->mean, 0, sizeof(float) * 3, s->stream))) return sim_error(s, SD_E_CUDA);
    s->mean_pending = false;
    return SD_OK;
}

int ensure_events(sd_sim* s) {
    if (s->ev[0]) return SD_OK;
    for (auto& e : s->ev)
        if (SD_CUDA(cudaEventCreate(&e))) return SD_E_CUDA;
    for (auto& e : s->pev)
        if (SD_CUDA(cudaEventCreate(&e))) return SD_E_CUDA;
    return SD_OK;
}

bool keeps_rho(const sd_sim* s) { return s->rho && (s->cfg.keep_density || s->mlp_on); }

// Learned correction of the particles pos[perm[i]] from the density just kept.
int mlp_correction(sd_sim* s, const int32_t* perm) {
    const float inv_mean = (float)((double)s->G * s->G * s->G / (double)(s->N > 0 ? s->N : 1));
    return launch_mlp_infer(s->mlp_params, s->pos, perm, s->N, s->rho, s->G, inv_mean, s->mlp_scale, s->mlp_out,
                            s->stream);
}

// Keys and first-pass sort counts for the current order, where the last step's
// gather has not left them.
int ensure_sort_inputs(sd_sim* s) {
    int rc = SD_OK;
    if (!s->keys_valid) {
        if ((rc = launch_cell_keys(s->pos, s->N, s->G, s->cfg.order, s->keys, s->stream))) return rc;
        s->keys_valid = true;
        s->counts_valid = s->incr_ready = false;
    }
    if (!s->counts_valid && !s->incr_ready) {  // a merge sort needs no counts
        if ((rc = launch_sort_first_counts(s->keys, s->N, key_bits_for(s->G, s->cfg.order), s->sort_ws,
                                           s->sort_ws_bytes, s->stream)))
            return rc;
        s->counts_valid = true;
    }
    return SD_OK;
}

// Sort + reorder (sortParticles, Sim.cu:3656-3671).
int do_sort(sd_sim* s, int32_t* perm_out_dev) {
    int rc = launch_cell_keys(s->pos, s->N, s->G, s->cfg.order, s->keys, s->stream);
    if (rc) return rc;
    rc = launch_sort_pairs(s->keys, nullptr, s->keys2, s->vals, s->keys3, s->vals2, s->N,
                           key_bits_for(s->G, s->cfg.order), s->sort_ws, s->sort_ws_bytes, s->stream, true);
    if (rc) return rc;
    rc = launch_reorder(s->pos, s->vel, s->vals, s->pos2, s->vel2, s->N, s->stream);
    if (rc) return rc;
    if (perm_out_dev &&
        SD_CUDA(cudaMemcpyAsync(perm_out_dev, s->vals, sizeof(int32_t) * s->N, cudaMemcpyDeviceToDevice, s->stream)))
        return SD_E_CUDA;
    std::swap(s->pos, s->pos2);
    std::swap(s->vel, s->vel2);
    invalidate_keys(s);
    return SD_OK;
}

// Field for the current positions: deposit + Poisson -> phi (computeAccel, Sim.cu:3605-3633).
int do_field(sd_sim* s, bool keep) {
    int rc = launch_deposit_fixed(s->pos, s->N, s->G, s->acc, s->stream, isolated(s) ? 0 : 1);
    if (rc) return rc;
    PoissonIso io;
    rc = launch_poisson_ex(s->plan, s->acc, nullptr, nullptr, nullptr, nullptr, keep ? s->rho : nullptr, s->spec,
                           s->phi, s->stream, nullptr, iso_opts(s, io));
    if (rc) return rc;
    if (keep) s->rho_valid = true;
    return SD_OK;
}

int do_step(sd_sim* s, float dt, bool sort, bool timed) {
    if (!s->configured) return fail(SD_E_STATE, "step: not initialised");
    if (s->cuda_failed) return SD_E_CUDA;
    float dt_kick = dt, dt_drift = dt;
    if (s->cfg.integrator == SD_INT_KDK) {
        dt_kick = s->lf_open ? 0.5f * (s->lf_dt_prev + dt) : 0.5f * dt;
        s->lf_open = true;
        s->lf_dt_prev = dt;
    }
    int rc = SD_OK;
    if (timed && (rc = ensure_events(s))) return sim_error(s, rc);
    if (timed) cudaEventRecord(s->ev[0], s->stream);
    // Sort (sortParticles, Sim.cu:3656-3671): keys come from the previous step's
    // gather; the permutation is applied by the deposit and gather reads, so no
    // separate reorder pass runs.
    const int32_t* perm = nullptr;
    // After a sorted step whose gather marked the changed keys, the sort is a merge
    // of those few into the rest (sd_resort.cu); otherwise the full radix sort.
    const bool incr_next = sort && merge_next(s);
    bool merged = false;  // the merge also left the new row table
    if (sort) {
        if (s->incr_ready && s->keys_valid && s->rs_base) {
            rc = launch_resort(s->rs, s->keys, s->N, s->G, key_bits_for(s->G, s->cfg.order), s->row_start, s->vals,
                               s->sort_ws, s->sort_ws_bytes, s->stream);
            if (rc) return sim_error(s, rc);
            // the share of changed keys, for the choice between merge and full sort
            if (s->chg_host && SD_CUDA(cudaMemcpyAsync(s->chg_host, s->rs.n_changed, sizeof(int),
                                                       cudaMemcpyDeviceToHost, s->stream)))
                return sim_error(s, SD_E_CUDA);
            s->chg_dirty = false;  // consumed and cleared
            merged = true;
        } else {
            if ((rc = ensure_sort_inputs(s))) return sim_error(s, rc);
            rc = launch_sort_pairs(s->keys, nullptr, s->keys2, s->vals, s->keys3, s->vals2, s->N,
                                   key_bits_for(s->G, s->cfg.order), s->sort_ws, s->sort_ws_bytes, s->stream, true,
                                   true);
            if (rc) return sim_error(s, rc);
        }
        s->counts_valid = false;  // the sort consumed and cleared them
        perm = s->vals;
    }
    // change bits written by an earlier gather and never merged are cleared first
    if (incr_next && s->chg_dirty) {
        if (SD_CUDA(cudaMemsetAsync(s->rs.words, 0, sizeof(unsigned) * resort_words(s->N), s->stream)))
            return sim_error(s, SD_E_CUDA);
        s->chg_dirty = false;
    }
    if (timed) cudaEventRecord(s->ev[1], s->stream);
    const bool keep = keeps_rho(s);
    // Tiled order right after a sort: the first FFT pass deposits the particles
    // itself from the row table. Otherwise: int64 atomics (any particle order).
    // (The isolated boundary always takes the atomic deposit, which clamps corners
    // onto the edge cells.)
    const bool fused = sort && s->cfg.order == SD_ORDER_TILED && !isolated(s);
    if (fused) {
        if (!merged && (rc = launch_row_bounds(s->keys2, s->N, s->G * s->G, s->row_start, s->stream)))
            return sim_error(s, rc);
    } else if ((rc = launch_deposit_fixed(s->pos, s->N, s->G, s->acc, s->stream, isolated(s) ? 0 : 1))) {
        return sim_error(s, rc);
    }
    if (timed) cudaEventRecord(s->ev[2], s->stream);
    PoissonIso io;
    DepositWork dw;
    dw.acc = s->acc;
    dw.ints = s->dep_ints;
    dw.split = s->dep_split > 0 ? s->dep_split : deposit_split(s->N, s->G);
    if ((rc = launch_poisson_ex(s->plan, fused ? nullptr : s->acc, nullptr, fused ? s->pos : nullptr, perm,
                                s->row_start, keep ? s->rho : nullptr, s->spec, s->phi, s->stream,
                                timed ? s->pev : nullptr, iso_opts(s, io), &dw)))
        return sim_error(s, rc);
    if (keep) s->rho_valid = true;
    if (timed) cudaEventRecord(s->ev[3], s->stream);
    if (s->mlp_on && (rc = mlp_correction(s, perm))) return sim_error(s, rc);
    // Grid hydrodynamics (computeAccel's kPressure, then doCooling, Sim.cu:3620-3631,
    // 3732-3868): the pressure field comes from the dispersion of the last cooling
    // step; a cooling step then corrects and cools the velocities in place, so the
    // gather reads them without the pending mean.
    const float* mean_in = s->mean;
    const bool press = s->hydro.base && s->cfg.pressure_enabled;
    // velocities still arriving on the offload stream (sd_step_host): nothing
    // before this point reads them
    if (s->vel_wait) {
        if (SD_CUDA(cudaStreamWaitEvent(s->stream, s->vel_wait, 0))) return sim_error(s, SD_E_CUDA);
        s->vel_wait = nullptr;
    }
    if (press && (rc = launch_pressure(s->hydro, isolated(s) ? 0 : 1, s->cfg.pressure_k, s->stream)))
        return sim_error(s, rc);
    if (s->hydro.base && (s->step_count % cooling_period(s)) == 0) {
        const float rate = (s->cfg.cooling_enabled && s->cfg.cooling_rate > 0.f) ? s->cfg.cooling_rate : 0.f;
        if ((rc = launch_cooling(s->hydro, s->pos, s->vel, s->N, s->mean, rate, dt * (float)cooling_period(s),
                                 s->cfg.pressure_enabled != 0, s->stream)))
            return sim_error(s, rc);
        mean_in = nullptr;
    }
    const float c2 = light_speed_sq(s->cfg.length_scale, s->cfg.time_unit_scale);
    // The mean written last step is read here as the correction for the loaded
    // velocities; the finalize kernel then overwrites it with this step's mean.
    float4* pos_out = perm ? s->pos2 : s->pos;
    float4* vel_out = perm ? s->vel2 : s->vel;
    // FP64 energy and momentum of every step, accumulated by the gather itself
    DiagRecord diag;
    diag.rec = s->diag_rec;
    diag.count = s->diag_count;
    diag.cap = kDiagCap;
    diag.mass = 1.0 / (double)(s->N > 0 ? s->N : 1);
    rc = launch_gather_kick_drift(s->phi, s->G, pot_scale_of(s), s->pos, s->vel, perm, pos_out, vel_out, s->keys,
                                  s->cfg.order, s->N, dt_kick, dt_drift, c2, mean_in, s->partials, s->mom, s->mean,
                                  s->stream, s->mlp_on ? s->mlp_out : nullptr, s->gather_blocks,
                                  s->cfg.diagnostics ? &diag : nullptr, isolated(s) ? 2 * s->G : 0,
                                  (sort && !incr_next) ? sort_first_counts(s->sort_ws) : nullptr,
                                  sort_digit_bits(key_bits_for(s->G, s->cfg.order)), press ? s->hydro.acc : nullptr,
                                  incr_next ? s->rs.words : nullptr);
    if (rc) return sim_error(s, rc);
    if (perm) {
        std::swap(s->pos, s->pos2);
        std::swap(s->vel, s->vel2);
    }
    s->keys_valid = true;
    // after a sort the counts buffer was zero, and the gather counted the new keys --
    // or, when the next sort can merge, marked the changed ones
    s->counts_valid = sort && !incr_next;
    s->incr_ready = incr_next;
    // bits stay dirty until a merge or the clear above consumes them (a step that
    // does not sort leaves them as they are)
    if (incr_next) s->chg_dirty = true;
    s->mean_pending = true;
    if (timed) cudaEventRecord(s->ev[4], s->stream);
    s->ev_valid = timed;
    s->sim_time += dt;
    ++s->step_count;
    return SD_OK;
}

bool sort_due(const sd_sim* s) {
    return s->cfg.sort_interval > 0 && (s->step_count % s->cfg.sort_interval) == 0;
}

int copy_in(void* dst, const void* src, size_t bytes, int where, cudaStream_t st) {
    const cudaMemcpyKind k = (where == SD_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    return SD_CUDA(cudaMemcpyAsync(dst, src, bytes, k, st));
}

int copy_out(void* dst, const void* src, size_t bytes, int where, cudaStream_t st) {
    const cudaMemcpyKind k = (where == SD_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    int rc = SD_CUDA(cudaMemcpyAsync(dst, src, bytes, k, st));
    if (rc == SD_OK && where == SD_HOST) rc = SD_CUDA(cudaStreamSynchronize(st));
    return rc;
}

// Free device memory for the VRAM clamp (Sim::deviceFreeBytes, Sim.cu:3921-3925), or
// the value a test set with sd_set_device_free_bytes_override.
std::atomic<size_t> g_free_override{0};

size_t device_free_bytes() {
    const size_t o = g_free_override.load();
    if (o) return o;
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return f;
}

constexpr int kMaxParticles = 400000000;  // validate_config's limit

// Device bytes that grow with the particle count, from the allocation model.
size_t per_particle_bytes(int G, int boundary) {
    const int step = 1 << 20;
    const size_t a = estimate_bytes(1, G, boundary), b = estimate_bytes(step + 1, G, boundary);
    return (b - a + step - 1) / step;
}

// Sim::maxParticlesFor (Sim.cu:4057-4066): the grid takes its share first, then 80 %
// of the rest holds particles (the other 20 % stays for the driver and other users).
int max_particles_for(int G, int boundary, size_t free_bytes) {
    const size_t grid_part = estimate_bytes(1, G, boundary);
    if (free_bytes <= grid_part) return 0;
    const size_t usable = (size_t)((double)(free_bytes - grid_part) * 0.8);
    const size_t n = usable / per_particle_bytes(G, boundary);
    return n > (size_t)kMaxParticles ? kMaxParticles : (int)n;
}

// Sim::reconfigure (Sim.cu:4074-4152). A request is structural when its count, grid
// or boundary differs from the last structural request (not from the clamped
// count, so repeating a clamped request changes nothing). A structural request
// that keeps the grid and boundary and asks for no more slots than the kernels
// run over only narrows that range: buffers, particles and time stay (the
// shrink-only path, Sim.cu:4108-4116). Any other structural request clamps the
// count to the device's free memory (Sim.cu:4123-4134; a grid that leaves no room
// fails with SD_E_NOMEM and changes nothing), reallocates and lays down the preset.
int reconfigure(sd_sim* s, const sd_config* c) {
    int rc = validate_config(c);
    if (rc) return rc;
    const int G = ceil_pow2_clamp(c->grid_size, sd_max_grid_size(c->boundary));
    const bool requested = !s->configured || c->particle_count != s->req_n || G != s->req_g ||
                           c->boundary != s->req_boundary;
    const bool shrink =
        requested && s->configured && G == s->G && c->boundary == s->req_boundary && c->particle_count <= s->N;
    int n = c->particle_count;
    if (requested && !shrink) {
        size_t avail = device_free_bytes();
        if (avail > 0) {
            // what this handle holds now is freed before the new allocation
            if (s->pos && s->capacity > 0 && s->req_boundary >= 0)
                avail += estimate_bytes(s->capacity, s->G, s->req_boundary);
            const int cap = max_particles_for(G, c->boundary, avail);
            if (cap <= 0)
                return fail(SD_E_NOMEM, "reconfigure: a %d^3 grid (%s boundary) does not fit this device (%zu bytes free)",
                            G, c->boundary == SD_BOUNDARY_ISOLATED ? "isolated" : "periodic", avail);
            if (n > cap) n = cap;
        }
    }
    const bool soft_changed = c->softening_cells != s->cfg.softening_cells;
    if (c->order != s->cfg.order) invalidate_keys(s);
    s->cfg = *c;
    s->cfg.grid_size = G;
    if (!requested || shrink) {
        if (shrink) {
            s->req_n = c->particle_count;
            s->N = c->particle_count;
            if (s->active > s->N) s->active = s->N;
            s->rho_valid = false;
            invalidate_keys(s);  // the sort covers a shorter range
            // change bits of slots past the new range must not reach a merge
            if (s->rs_base &&
                SD_CUDA(cudaMemsetAsync(s->rs.words, 0, sizeof(unsigned) * resort_words(s->capacity), s->stream)))
                return sim_error(s, SD_E_CUDA);
            s->chg_dirty = false;
        }
        if (s->graph) cudaGraphExecDestroy(s->graph);
        s->graph = nullptr;
        if (c->keep_density && !s->rho && (rc = alloc_dev(s->rho, (size_t)s->G * s->G * s->G))) return rc;
        if ((rc = ensure_hydro(s)) || (rc = ensure_resort(s))) return rc;
        if (!soft_changed) return SD_OK;
        rc = poisson_plan_build(s->plan, box_of(s->G, s->cfg.boundary), s->cfg.softening_cells);
        if (!rc && isolated(s))
            rc = build_green_table(s->plan, s->cfg.softening_cells, s->phi, s->spec, s->green, s->stream);
        return rc;
    }
    s->req_n = c->particle_count;
    s->req_g = G;
    s->req_boundary = c->boundary;
    s->N = s->capacity = n;
    s->G = G;
    rc = allocate(s);
    if (rc) {
        s->req_n = s->req_g = s->req_boundary = -1;
        s->capacity = 0;
        return rc;
    }
    if ((rc = ensure_hydro(s)) || (rc = ensure_resort(s))) return rc;
    // the reference's init / structural reconfigure ends in reset() (Sim.cu:4151)
    if ((rc = place_initial(s))) return sim_error(s, rc);
    s->sim_time = 0.0;
    s->step_count = 0;
    s->mean_pending = false;
    s->lf_open = false;
    s->rho_valid = false;
    invalidate_keys(s);
    s->cuda_failed = false;
    return SD_OK;
}

// STARDUST v1/v2 header (Sim.cu:4985-4997), byte-compatible.
struct StateHeader {
    char magic[8];
    int32_t version;
    int32_t count;
    int32_t gridSize;
    int32_t preset;
    int32_t boundary;
    float gravity;
    float simTime;
    float bhX, bhY, bhRs, bhMass;
    int32_t bhActive;
    int32_t reserved[5];
};
static_assert(sizeof(StateHeader) == 76, "STARDUST header layout");
constexpr size_t kBlackHoleRecord = 48;  // sizeof(BlackHoleState) (Sim.h:813-825)

// Wait for queued offload steps (sd_step_host_async) before any other use of the
// handle: their uploads, steps and downloads run on three streams, and the other
// entry points assume the handle's buffers are at rest between calls.
int settle(sd_sim* s) {
    if (!s->async_pending) return SD_OK;
    s->async_pending = false;
    int rc = SD_OK;
    if (s->up_stream && SD_CUDA(cudaStreamSynchronize(s->up_stream))) rc = SD_E_CUDA;
    if (s->io_stream && SD_CUDA(cudaStreamSynchronize(s->io_stream))) rc = SD_E_CUDA;
    if (SD_CUDA(cudaStreamSynchronize(s->stream))) rc = SD_E_CUDA;
    s->stage_free = nullptr;
    return rc ? sim_error(s, rc) : SD_OK;
}

}  // namespace sdsim

using namespace sdsim;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int sd_abi_version(void) { return SD_ABI_VERSION; }

int sd_device_available(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0 ? 1 : 0;
}

int sd_failed(void) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    return g_failed ? 1 : 0;
}

const char* sd_last_error(void) { return g_msg; }

void sd_clear_error(void) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_failed = false;
    g_msg[0] = 0;
}

int sd_config_default(sd_config* c) {
    if (!c) return fail(SD_E_ARG, "config_default: null");
    memset(c, 0, sizeof(*c));
    c->particle_count = 2000000;  // Sim.h:166
    c->grid_size = 128;           // Sim.h:167
    c->boundary = SD_BOUNDARY_PERIODIC;
    c->gravity = 1.0f;
    c->softening_cells = 3.0f;    // Sim.h:315
    c->time_scale = 1.0f;         // Sim.h:316
    c->sort_interval = 1;
    c->length_scale = 1.0f;       // Sim.h:172
    c->time_unit_scale = 1.0f;    // Sim.h:180
    c->order = SD_ORDER_ROWMAJOR;
    c->integrator = SD_INT_KD;
    c->units = SD_UNITS_REFERENCE;
    c->diagnostics = 0;
    c->keep_density = 1;
    c->preset = SD_PRESET_FILAMENT;  // Sim.h:277
    c->pressure_k = 0.45f;           // Sim.h:320 (pressure itself off: the PM path)
    c->cooling_rate = 0.08f;         // Sim.h:345 (cooling itself off)
    return SD_OK;
}

int sd_max_grid_size(int boundary) { return boundary == SD_BOUNDARY_ISOLATED ? 256 : 512; }

size_t sd_estimate_bytes(int particle_count, int grid_size, int boundary) {
    const int G = ceil_pow2_clamp(grid_size, sd_max_grid_size(boundary));
    return estimate_bytes(particle_count, G, boundary);
}

int sd_max_particles_for(int grid_size, int boundary, size_t free_bytes) {
    if (boundary != SD_BOUNDARY_PERIODIC && boundary != SD_BOUNDARY_ISOLATED) return 0;
    const int G = ceil_pow2_clamp(grid_size, sd_max_grid_size(boundary));
    return max_particles_for(G, boundary, free_bytes);
}

size_t sd_device_free_bytes(void) { return device_free_bytes(); }

void sd_set_device_free_bytes_override(size_t bytes) { g_free_override.store(bytes); }

double sd_device_bandwidth_gbs(void) {
    // Sim::deviceBandwidthGBs (Sim.cu:4003-4012): memory clock x bus width x 2 (DDR)
    int khz = 0, bits = 0, dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&khz, cudaDevAttrMemoryClockRate, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&bits, cudaDevAttrGlobalMemoryBusWidth, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0.0;
    }
    if (khz <= 0 || bits <= 0) return 0.0;
    return (double)khz * 1000.0 * ((double)bits / 8.0) * 2.0 / 1.0e9;
}

double sd_estimate_step_ms(int particle_count, int grid_size, int boundary) {
    // Sim::estimateStepMs (Sim.cu:4022-4055) with this build's costs: the byte model
    // of a step, 184 B per particle + 40 B per cell of the transform box, at 55 % of
    // the memory bandwidth (a 16M / 512^3 step runs at about 0.66 of the measured
    // copy bandwidth), plus 0.02 ms of launch overhead. A scene whose particles
    // crowd a few rows costs more than the model says.
    const double bw = sd_device_bandwidth_gbs();
    if (bw <= 0.0) return 0.0;
    if (boundary != SD_BOUNDARY_PERIODIC && boundary != SD_BOUNDARY_ISOLATED) return 0.0;
    const double G = (double)ceil_pow2_clamp(grid_size, sd_max_grid_size(boundary));
    const double S = (boundary == SD_BOUNDARY_ISOLATED) ? 2.0 * G : G;
    const double n = (double)(particle_count > 0 ? particle_count : 0);
    const double bytes = 184.0 * n + 40.0 * S * S * S;
    return bytes / (0.55 * bw * 1.0e9) * 1.0e3 + 0.02;
}

int sd_device_multiprocessors(void) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return sms;
}

int sd_device_name(char* out, int capacity) {
    if (!out || capacity <= 0) return fail(SD_E_ARG, "device_name: no buffer");
    int dev = 0;
    cudaDeviceProp p{};
    const char* name = "unknown";
    if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&p, dev) == cudaSuccess)
        name = p.name;
    else
        cudaGetLastError();
    snprintf(out, (size_t)capacity, "%s", name);
    return SD_OK;
}

int sd_device_driver(char* out, int capacity) {
    // the CUDA version the driver supports (Sim::deviceDriver, Sim.cu:3912-3920)
    if (!out || capacity <= 0) return fail(SD_E_ARG, "device_driver: no buffer");
    int v = 0;
    out[0] = 0;
    if (cudaDriverGetVersion(&v) != cudaSuccess || v <= 0) {
        cudaGetLastError();
        return SD_OK;
    }
    snprintf(out, (size_t)capacity, "CUDA %d.%d", v / 1000, (v % 1000) / 10);
    return SD_OK;
}

int sd_create(sd_sim** out, int device) {
    if (!out) return fail(SD_E_ARG, "create: null out");
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
        cudaGetLastError();
        return fail(SD_E_CUDA, "create: no CUDA device %d", device);
    }
    sd_sim* s = new sd_sim();
    s->device = device;
    DeviceGuard g(device);
    if (SD_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking))) {
        delete s;
        return SD_E_CUDA;
    }
    s->own_stream = true;
    sd_config_default(&s->cfg);
    if (int rc = gather_prepare(device)) {
        cudaStreamDestroy(s->stream);
        delete s;
        return rc;
    }
    *out = s;
    return SD_OK;
}

int sd_destroy(sd_sim* s) {
    if (!s) return SD_OK;
    DeviceGuard g(s->device);
    settle(s);
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_buffers(s);
    free_dev(s->mlp_params);
    for (auto& e : s->up_ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : s->down_ev)
        if (e) cudaEventDestroy(e);
    if (s->out_ev) cudaEventDestroy(s->out_ev);
    if (s->up_stream) cudaStreamDestroy(s->up_stream);
    if (s->chg_host) cudaFreeHost(s->chg_host);
    for (auto& e : s->ev)
        if (e) cudaEventDestroy(e);
    for (auto& e : s->pev)
        if (e) cudaEventDestroy(e);
    for (auto& e : s->io_ev)
        if (e) cudaEventDestroy(e);
    if (s->io_stream) {
        cudaStreamSynchronize(s->io_stream);
        cudaStreamDestroy(s->io_stream);
    }
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return SD_OK;
}

int sd_set_stream(sd_sim* s, void* stream) {
    if (!s) return fail(SD_E_ARG, "set_stream: null handle");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    cudaStreamSynchronize(s->stream);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    s->stream = (cudaStream_t)stream;
    s->own_stream = false;
    if (s->graph) cudaGraphExecDestroy(s->graph);
    s->graph = nullptr;
    return SD_OK;
}

int sd_init(sd_sim* s, const sd_config* c) {
    if (!s) return fail(SD_E_ARG, "init: null handle");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    s->configured = false;
    return reconfigure(s, c);
}

int sd_reconfigure(sd_sim* s, const sd_config* c) {
    if (!s) return fail(SD_E_ARG, "reconfigure: null handle");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    return reconfigure(s, c);
}

int sd_reset(sd_sim* s) {
    if (!s || !s->configured) return fail(SD_E_STATE, "reset: not initialised");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    s->sim_time = 0.0;
    s->step_count = 0;
    s->lf_open = false;
    if (SD_CUDA(cudaMemsetAsync(s->diag_count, 0, sizeof(unsigned long long), s->stream))) return SD_E_CUDA;
    const int rc = place_initial(s);
    return rc ? sim_error(s, rc) : SD_OK;
}

int sd_get_config(const sd_sim* s, sd_config* out) {
    if (!s || !out) return fail(SD_E_ARG, "get_config: null");
    *out = s->cfg;
    return SD_OK;
}

int sd_set_particles(sd_sim* s, const float* pos, const float* vel, int n, int where) {
    if (!s || !s->configured) return fail(SD_E_STATE, "set_particles: not initialised");
    if (!pos || !vel || n < 0 || n > s->N) return fail(SD_E_ARG, "set_particles: bad arguments (n=%d)", n);
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    int rc = copy_in(s->pos, pos, sizeof(float4) * (size_t)n, where, s->stream);
    if (!rc) rc = copy_in(s->vel, vel, sizeof(float4) * (size_t)n, where, s->stream);
    if (!rc) rc = launch_hide_range(s->pos, s->vel, n, s->N, s->stream);
    if (!rc && SD_CUDA(cudaMemsetAsync(s->mean, 0, sizeof(float) * 4, s->stream))) rc = SD_E_CUDA;
    if (!rc && where == SD_HOST) rc = SD_CUDA(cudaStreamSynchronize(s->stream));
    if (rc) return sim_error(s, rc);
    s->active = n;
    s->mean_pending = false;
    s->lf_open = false;
    s->rho_valid = false;
    invalidate_keys(s);
    return SD_OK;
}

int sd_get_particles(sd_sim* s, float* pos, float* vel, int n, int where) {
    if (!s || !s->configured) return fail(SD_E_STATE, "get_particles: not initialised");
    if (n < 0 || n > s->N) return fail(SD_E_ARG, "get_particles: bad n=%d", n);
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    int rc = materialize(s);
    if (!rc && pos) rc = copy_out(pos, s->pos, sizeof(float4) * (size_t)n, where, s->stream);
    if (!rc && vel) rc = copy_out(vel, s->vel, sizeof(float4) * (size_t)n, where, s->stream);
    return rc ? sim_error(s, rc) : SD_OK;
}

const float* sd_particle_pos_device_ptr(sd_sim* s) {
    if (!s || !s->configured) return nullptr;
    DeviceGuard g(s->device);
    settle(s);
    materialize(s);
    return reinterpret_cast<const float*>(s->pos);
}

const float* sd_particle_vel_device_ptr(sd_sim* s) {
    if (!s || !s->configured) return nullptr;
    DeviceGuard g(s->device);
    settle(s);
    materialize(s);
    return reinterpret_cast<const float*>(s->vel);
}

const float* sd_density_device_ptr(sd_sim* s) {
    if (!s || !s->configured || !s->rho || !s->rho_valid) return nullptr;
    return s->rho;
}

int sd_get_density(sd_sim* s, float* out, int where) {
    if (!s || !s->configured || !out) return fail(SD_E_STATE, "get_density: not initialised");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    if (!s->rho) return fail(SD_E_STATE, "get_density: keep_density is off");
    if (!s->rho_valid) {  // no step yet: density of the current positions
        int rc = do_field(s, true);
        if (rc) return sim_error(s, rc);
    }
    return copy_out(out, s->rho, sizeof(float) * (size_t)s->G * s->G * s->G, where, s->stream);
}

int sd_get_potential(sd_sim* s, float* out, int where) {
    if (!s || !s->configured || !out) return fail(SD_E_STATE, "get_potential: not initialised");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    if (!isolated(s)) return copy_out(out, s->phi, sizeof(float) * (size_t)s->G * s->G * s->G, where, s->stream);
    // isolated: the G^3 corner of the 2G box, one 2D copy per z plane
    const int G = s->G, S = 2 * G;
    const cudaMemcpyKind k = (where == SD_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    for (int z = 0; z < G; ++z)
        if (SD_CUDA(cudaMemcpy2DAsync(out + (size_t)z * G * G, sizeof(float) * G, s->phi + (size_t)z * S * S,
                                      sizeof(float) * S, sizeof(float) * G, G, k, s->stream)))
            return sim_error(s, SD_E_CUDA);
    return (where == SD_HOST) ? SD_CUDA(cudaStreamSynchronize(s->stream)) : SD_OK;
}

int sd_get_accel(sd_sim* s, float* out, int n, int where) {
    if (!s || !s->configured || !out) return fail(SD_E_STATE, "get_accel: not initialised");
    if (n < 0 || n > s->N) return fail(SD_E_ARG, "get_accel: bad n=%d", n);
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    int rc = do_field(s, keeps_rho(s));
    if (rc) return sim_error(s, rc);
    if (s->mlp_on && (rc = mlp_correction(s, nullptr))) return sim_error(s, rc);
    float4* dst = reinterpret_cast<float4*>(out);
    float4* tmp = nullptr;
    if (where == SD_HOST) tmp = s->pos2;  // scratch: pos2 is free between steps
    rc = launch_interpolate_accel(s->phi, s->G, pot_scale_of(s), s->pos, tmp ? tmp : dst, n, s->stream,
                                  s->mlp_on ? s->mlp_out : nullptr, isolated(s) ? 2 * s->G : 0);
    if (rc) return sim_error(s, rc);
    if (tmp) return copy_out(out, tmp, sizeof(float4) * (size_t)n, SD_HOST, s->stream);
    return SD_OK;
}

int sd_set_mlp(sd_sim* s, const float* params_device, float out_scale) {
    if (!s || !s->configured) return fail(SD_E_STATE, "set_mlp: not initialised");
    if (params_device && isolated(s)) return fail(SD_E_UNSUPPORTED, "set_mlp: the correction is trained for periodic boxes");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    if (s->graph) cudaGraphExecDestroy(s->graph);  // replays must see the new setting
    s->graph = nullptr;
    if (!params_device) {
        s->mlp_on = false;
        return SD_OK;
    }
    if (!std::isfinite(out_scale)) return fail(SD_E_ARG, "set_mlp: out_scale is not finite");
    int rc = SD_OK;
    if (!s->mlp_params) rc = alloc_dev(s->mlp_params, mlp_param_count());
    if (!rc && !s->mlp_out) rc = alloc_dev(s->mlp_out, (size_t)s->N);
    if (!rc && !s->rho) rc = alloc_dev(s->rho, (size_t)s->G * s->G * s->G);
    if (rc) return rc;
    if (SD_CUDA(cudaMemcpyAsync(s->mlp_params, params_device, sizeof(float) * mlp_param_count(),
                                cudaMemcpyDeviceToDevice, s->stream)))
        return sim_error(s, SD_E_CUDA);
    s->mlp_scale = out_scale;
    s->mlp_on = true;
    return SD_OK;
}

int sd_step(sd_sim* s, float dt) {
    if (!s) return fail(SD_E_ARG, "step: null handle");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    update_merge_policy(s);
    const bool sort = sort_due(s);
    int rc = do_step(s, dt, sort, true);
    if (rc) return rc;
    s->tm.dt_used = dt;
    s->tm.steps = 1;
    return SD_OK;
}

int sd_step_host(sd_sim* s, const float* pos_in, const float* vel_in, int n, float dt, float* pos_out,
                 float* vel_out) {
    if (!s || !s->configured) return fail(SD_E_STATE, "step_host: not initialised");
    if (!pos_in || !vel_in || !pos_out || !vel_out || n < 0 || n > s->N)
        return fail(SD_E_ARG, "step_host: bad arguments (n=%d)", n);
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    if (!s->io_stream) {
        if (SD_CUDA(cudaStreamCreateWithFlags(&s->io_stream, cudaStreamNonBlocking))) return SD_E_CUDA;
        for (auto& e : s->io_ev)
            if (SD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming))) return SD_E_CUDA;
    }
    const size_t bytes = sizeof(float4) * (size_t)n;
    cudaStream_t st = s->stream, io = s->io_stream;
    // Inputs: the positions first, at the link's full speed, on the handle's
    // stream; then the velocities on the offload stream while the step's sort,
    // deposit and Poisson solve run. The first kernel that reads velocities waits.
    int rc = SD_CUDA(cudaMemcpyAsync(s->pos, pos_in, bytes, cudaMemcpyHostToDevice, st));
    if (!rc) rc = SD_CUDA(cudaEventRecord(s->io_ev[0], st));
    if (!rc) rc = SD_CUDA(cudaStreamWaitEvent(io, s->io_ev[0], 0));
    if (!rc) rc = SD_CUDA(cudaMemcpyAsync(s->vel, vel_in, bytes, cudaMemcpyHostToDevice, io));
    if (!rc) rc = SD_CUDA(cudaEventRecord(s->io_ev[1], io));
    if (!rc) rc = launch_hide_range(s->pos, s->vel, n, s->N, st);  // slots >= n: disjoint from the copy
    if (!rc && SD_CUDA(cudaMemsetAsync(s->mean, 0, sizeof(float) * 4, st))) rc = SD_E_CUDA;
    // on any failure the call returns only after its copies stopped reading the caller's buffers
    auto drain = [&](int code) {
        cudaStreamSynchronize(io);
        cudaStreamSynchronize(st);
        return sim_error(s, code);
    };
    if (rc) return drain(rc);
    s->active = n;
    s->mean_pending = false;
    s->lf_open = false;
    s->rho_valid = false;
    invalidate_keys(s);
    s->vel_wait = s->io_ev[1];
    rc = do_step(s, dt, sort_due(s), true);
    if (s->vel_wait) {  // a step that read no velocity still owes the wait
        if (!rc) rc = SD_CUDA(cudaStreamWaitEvent(st, s->vel_wait, 0));
        s->vel_wait = nullptr;
    }
    if (rc) return drain(rc);
    s->tm.dt_used = dt;
    s->tm.steps = 1;
    // Outputs: the positions leave on the offload stream while the handle's stream
    // applies the pending momentum correction to the velocities, which follow
    // (the two downloads share the link).
    rc = SD_CUDA(cudaEventRecord(s->io_ev[0], st));
    if (!rc) rc = SD_CUDA(cudaStreamWaitEvent(io, s->io_ev[0], 0));
    if (!rc) rc = SD_CUDA(cudaMemcpyAsync(pos_out, s->pos, bytes, cudaMemcpyDeviceToHost, io));
    if (!rc) rc = materialize(s);
    if (!rc) rc = SD_CUDA(cudaMemcpyAsync(vel_out, s->vel, bytes, cudaMemcpyDeviceToHost, st));
    if (rc) return drain(rc);
    if ((rc = SD_CUDA(cudaStreamSynchronize(io))) || (rc = SD_CUDA(cudaStreamSynchronize(st)))) return drain(rc);
    return SD_OK;
}

int sd_step_host_async(sd_sim* s, const float* pos_in, const float* vel_in, int n, float dt, float* pos_out,
                       float* vel_out) {
    if (!s || !s->configured) return fail(SD_E_STATE, "step_host_async: not initialised");
    if (!pos_in || !vel_in || !pos_out || !vel_out || n < 0 || n > s->N)
        return fail(SD_E_ARG, "step_host_async: bad arguments (n=%d)", n);
    DeviceGuard g(s->device);
    if (!s->up_stream) {
        if (SD_CUDA(cudaStreamCreateWithFlags(&s->up_stream, cudaStreamNonBlocking))) return SD_E_CUDA;
        for (auto& e : s->up_ev)
            if (SD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming))) return SD_E_CUDA;
        for (auto& e : s->down_ev)
            if (SD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming))) return SD_E_CUDA;
        if (SD_CUDA(cudaEventCreateWithFlags(&s->out_ev, cudaEventDisableTiming))) return SD_E_CUDA;
    }
    if (!s->io_stream && SD_CUDA(cudaStreamCreateWithFlags(&s->io_stream, cudaStreamNonBlocking))) return SD_E_CUDA;
    // the staging set: allocated by the first call, kept with the other particle buffers
    if (!s->stage_pos) {
        int rc = settle(s);
        if (!rc) rc = alloc_dev(s->stage_pos, (size_t)s->N);
        if (!rc) rc = alloc_dev(s->stage_vel, (size_t)s->N);
        if (rc) return rc;
        s->stage_free = nullptr;
    }
    const size_t bytes = sizeof(float4) * (size_t)n;
    cudaStream_t st = s->stream, io = s->io_stream, up = s->up_stream;
    // on failure the queued work is drained before returning, so no copy still
    // reads or writes the caller's buffers
    auto drain = [&](int code) {
        s->async_pending = true;
        settle(s);
        return sim_error(s, code);
    };
    // 1. upload into the staging set once its last download (two calls ago) is done
    int rc = SD_OK;
    if (s->stage_free) rc = SD_CUDA(cudaStreamWaitEvent(up, s->stage_free, 0));
    if (!rc) rc = SD_CUDA(cudaMemcpyAsync(s->stage_pos, pos_in, bytes, cudaMemcpyHostToDevice, up));
    if (!rc) rc = SD_CUDA(cudaEventRecord(s->up_ev[0], up));
    if (!rc) rc = SD_CUDA(cudaMemcpyAsync(s->stage_vel, vel_in, bytes, cudaMemcpyHostToDevice, up));
    if (!rc) rc = SD_CUDA(cudaEventRecord(s->up_ev[1], up));
    if (rc) return drain(rc);
    // 2. rotate the three particle sets: the staged inputs become the step's input;
    // the last result, still downloading, becomes the next staging set (free once
    // its download event fires); the last input stays the step's output buffer
    float4* const last_pos = s->pos;
    float4* const last_vel = s->vel;
    s->pos = s->stage_pos;
    s->vel = s->stage_vel;
    s->stage_pos = last_pos;
    s->stage_vel = last_vel;
    s->stage_free = (s->async_calls > 0 && s->async_pending) ? s->down_ev[(s->async_calls - 1) & 1] : nullptr;
    s->async_pending = true;
    // 3. the step, on the handle's stream, after the positions arrive; the first
    // kernel that reads velocities waits for them
    rc = SD_CUDA(cudaStreamWaitEvent(st, s->up_ev[0], 0));
    if (!rc) rc = launch_hide_range(s->pos, s->vel, n, s->N, st);  // slots >= n: disjoint from the copy
    if (!rc && SD_CUDA(cudaMemsetAsync(s->mean, 0, sizeof(float) * 4, st))) rc = SD_E_CUDA;
    if (rc) return drain(rc);
    s->active = n;
    s->mean_pending = false;
    s->lf_open = false;
    s->rho_valid = false;
    invalidate_keys(s);
    s->vel_wait = s->up_ev[1];
    rc = do_step(s, dt, sort_due(s), false);
    if (s->vel_wait) {  // a step that read no velocity still owes the wait
        if (!rc) rc = SD_CUDA(cudaStreamWaitEvent(st, s->vel_wait, 0));
        s->vel_wait = nullptr;
    }
    if (!rc) rc = materialize(s);
    if (rc) return drain(rc);
    s->tm.dt_used = dt;
    s->tm.steps = 1;
    // 4. download the result on the offload stream
    const int k = (int)(s->async_calls & 1);
    rc = SD_CUDA(cudaEventRecord(s->out_ev, st));
    if (!rc) rc = SD_CUDA(cudaStreamWaitEvent(io, s->out_ev, 0));
    if (!rc) rc = SD_CUDA(cudaMemcpyAsync(pos_out, s->pos, bytes, cudaMemcpyDeviceToHost, io));
    if (!rc) rc = SD_CUDA(cudaMemcpyAsync(vel_out, s->vel, bytes, cudaMemcpyDeviceToHost, io));
    if (!rc) rc = SD_CUDA(cudaEventRecord(s->down_ev[k], io));
    if (rc) return drain(rc);
    ++s->async_calls;
    return SD_OK;
}

int sd_step_host_wait(sd_sim* s) {
    if (!s) return fail(SD_E_ARG, "step_host_wait: null handle");
    DeviceGuard g(s->device);
    return settle(s);
}

int sd_step_auto(sd_sim* s) {
    if (!s || !s->configured) return fail(SD_E_STATE, "step_auto: not initialised");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    // CFL (Sim.cu:4255-4269): vmax of the current (momentum-zeroed) velocities.
    int rc = launch_max_speed(s->pos, s->vel, s->N, s->mean_pending ? s->mean : nullptr, s->mean + 3, s->stream);
    if (rc) return sim_error(s, rc);
    float vmax = 0.f;
    rc = copy_out(&vmax, s->mean + 3, sizeof(float), SD_HOST, s->stream);
    if (rc) return sim_error(s, rc);
    const float cell = 1.0f / (float)s->G;
    float dt = 0.0016f * dt_scale_for(s->cfg.time_scale);
    const float dt_max = (vmax > 1e-6f) ? (0.8f * cell / vmax) : dt;
    if (dt > dt_max) dt = dt_max;
    rc = do_step(s, dt, sort_due(s), true);
    if (rc) return rc;
    s->tm.dt_used = dt;
    s->tm.max_speed = vmax;
    s->tm.steps = 1;
    return SD_OK;
}

int sd_steps(sd_sim* s, float dt, int nsteps) {
    if (!s || !s->configured) return fail(SD_E_STATE, "steps: not initialised");
    if (nsteps < 0) return fail(SD_E_ARG, "steps: negative count");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    // A two-step graph repeats the cooling schedule only when its period is 2.
    const bool graphable = (s->cfg.sort_interval == 0 || s->cfg.sort_interval == 1) &&
                           (!hydro_on(s) || cooling_period(s) == 2);
    int done = 0;
    update_merge_policy(s);
    // leapfrog opening kick and odd counts run eagerly
    while (done < nsteps && (!graphable || (s->cfg.integrator == SD_INT_KDK && !s->lf_open))) {
        int rc = do_step(s, dt, sort_due(s), false);
        if (rc) return rc;
        ++done;
    }
    if (done >= nsteps) return SD_OK;
    const bool sort = s->cfg.sort_interval == 1;
    while (nsteps - done >= 2) {
        // Keys and first-pass counts are made outside the graph, so replays never
        // depend on them being stale.
        if (sort) {
            int rc = ensure_sort_inputs(s);
            if (rc) return sim_error(s, rc);
        }
        const int phase = hydro_on(s) ? (s->step_count & 1) : 0;
        const bool incr_now = s->incr_ready && s->keys_valid;  // the first captured step merge-sorts
        // a full sort with change bits pending records their clearing (the merge consumes them)
        const bool dirty_now = !incr_now && s->chg_dirty;
        // A captured graph covers two steps so the pos/pos2 ping-pong returns to the
        // same buffers; it is rebuilt when dt changes, the particles sit in the other
        // buffer of the pair, the cooling phase moved, or its first step would sort
        // differently (a merge needs the last step's change bits; stale bits must be
        // cleared before the gather marks new ones).
        if (!s->graph || s->graph_dt != dt || s->graph_pos != s->pos || s->graph_phase != phase ||
            s->graph_incr != incr_now || s->graph_dirty != dirty_now || s->graph_merge_off != s->merge_off) {
            if (s->graph) cudaGraphExecDestroy(s->graph);
            s->graph = nullptr;
            cudaGraph_t graph = nullptr;
            if (SD_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal)))
                return sim_error(s, SD_E_CUDA);
            const double t0 = s->sim_time;
            const int c0 = s->step_count;
            const bool lf0 = s->lf_open;
            const float lfd = s->lf_dt_prev;
            const bool mp0 = s->mean_pending;
            const bool kv0 = s->keys_valid;
            const bool cv0 = s->counts_valid;
            const bool iv0 = s->incr_ready, dv0 = s->chg_dirty;
            const long long l0 = launches();
            int rc = do_step(s, dt, sort, false);
            if (!rc) rc = do_step(s, dt, sort, false);
            cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
            // capture only recorded the kernels; count them per replay instead
            s->graph_launches = launches() - l0;
            count_launch(-s->graph_launches);
            // capture recorded work only; restore the host-side counters
            s->sim_time = t0;
            s->step_count = c0;
            s->lf_open = lf0;
            s->lf_dt_prev = lfd;
            s->mean_pending = mp0;
            s->keys_valid = kv0;
            s->counts_valid = cv0;
            s->incr_ready = iv0;
            s->chg_dirty = dv0;
            if (rc) {
                if (graph) cudaGraphDestroy(graph);
                return rc;
            }
            if (SD_CUDA(e)) return sim_error(s, SD_E_CUDA);
            e = cudaGraphInstantiate(&s->graph, graph, 0);
            cudaGraphDestroy(graph);
            if (SD_CUDA(e)) return sim_error(s, SD_E_CUDA);
            s->graph_dt = dt;
            s->graph_pos = s->pos;
            s->graph_phase = phase;
            s->graph_incr = incr_now;
            s->graph_dirty = dirty_now;
            s->graph_merge_off = s->merge_off;
        }
        if (SD_CUDA(cudaGraphLaunch(s->graph, s->stream))) return sim_error(s, SD_E_CUDA);
        count_launch(s->graph_launches);
        s->sim_time += 2.0 * dt;
        s->step_count += 2;
        s->mean_pending = true;
        s->keys_valid = true;
        {  // the graph's last step leaves what do_step leaves after a sorted step
            const bool incr_next = sort && merge_next(s);
            s->counts_valid = sort && !incr_next;
            s->incr_ready = incr_next;
            if (incr_next) s->chg_dirty = true;
        }
        if (s->cfg.integrator == SD_INT_KDK) {
            s->lf_open = true;
            s->lf_dt_prev = dt;
        }
        done += 2;
    }
    if (done < nsteps) {
        int rc = do_step(s, dt, sort_due(s), false);
        if (rc) return rc;
    }
    s->ev_valid = false;
    return SD_OK;
}

int sd_synchronize(sd_sim* s) {
    if (!s || !s->configured) return fail(SD_E_STATE, "synchronize: not initialised");
    if (s->cfg.integrator != SD_INT_KDK || !s->lf_open) return SD_OK;
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    int rc = do_field(s, keeps_rho(s));
    if (rc) return sim_error(s, rc);
    if (s->mlp_on && (rc = mlp_correction(s, nullptr))) return sim_error(s, rc);
    const float c2 = light_speed_sq(s->cfg.length_scale, s->cfg.time_unit_scale);
    rc = launch_gather_kick_drift(s->phi, s->G, pot_scale_of(s), s->pos, s->vel, nullptr, s->pos, s->vel, s->keys,
                                  s->cfg.order, s->N, 0.5f * s->lf_dt_prev, 0.f, c2, s->mean, s->partials, s->mom,
                                  s->mean, s->stream, s->mlp_on ? s->mlp_out : nullptr, 0, nullptr,
                                  isolated(s) ? 2 * s->G : 0);
    if (rc) return sim_error(s, rc);
    s->counts_valid = s->incr_ready = false;  // keys were rewritten (a lost particle changes its key)
    s->mean_pending = true;
    s->lf_open = false;
    return SD_OK;
}

int sd_sort_only(sd_sim* s, int32_t* perm, int where) {
    if (!s || !s->configured) return fail(SD_E_STATE, "sort_only: not initialised");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    int32_t* dev_perm = nullptr;
    if (perm && where == SD_DEVICE) dev_perm = perm;
    int rc = do_sort(s, dev_perm);
    if (rc) return sim_error(s, rc);
    if (perm && where == SD_HOST) {
        // do_sort leaves the permutation in vals
        rc = copy_out(perm, s->vals, sizeof(int32_t) * (size_t)s->N, SD_HOST, s->stream);
        if (rc) return sim_error(s, rc);
    }
    s->rho_valid = false;
    return SD_OK;
}

int sd_save_state(sd_sim* s, const char* path) {
    if (!s || !s->configured || !path) return fail(SD_E_STATE, "save_state: not initialised");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    const int n = (s->active > 0) ? s->active : s->N;
    std::vector<float4> hp((size_t)n), hv((size_t)n);
    int rc = sd_get_particles(s, reinterpret_cast<float*>(hp.data()), reinterpret_cast<float*>(hv.data()), n, SD_HOST);
    if (rc) return rc;
    StateHeader h;
    memset(&h, 0, sizeof(h));
    memcpy(h.magic, "STARDUST", 8);
    h.version = 2;
    h.count = n;
    h.gridSize = s->G;
    h.preset = s->cfg.preset;  // Sim.cu:5017
    h.boundary = s->cfg.boundary;
    h.gravity = s->cfg.gravity;
    h.simTime = (float)s->sim_time;
    h.bhX = h.bhY = 0.5f;
    FILE* f = fopen(path, "wb");
    if (!f) return fail(SD_E_IO, "save_state: cannot open %s", path);
    bool ok = fwrite(&h, sizeof(h), 1, f) == 1 && fwrite(hp.data(), sizeof(float4), (size_t)n, f) == (size_t)n &&
              fwrite(hv.data(), sizeof(float4), (size_t)n, f) == (size_t)n;
    ok = (fclose(f) == 0) && ok;
    return ok ? SD_OK : fail(SD_E_IO, "save_state: write failed for %s", path);
}

int sd_load_state(sd_sim* s, const char* path) {
    if (!s || !path) return fail(SD_E_ARG, "load_state: null");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    FILE* f = fopen(path, "rb");
    if (!f) return fail(SD_E_IO, "load_state: cannot open %s", path);
    StateHeader h;
    if (fread(&h, sizeof(h), 1, f) != 1 || memcmp(h.magic, "STARDUST", 8) != 0 || (h.version != 1 && h.version != 2) ||
        h.count <= 0 || h.count > 100000000) {
        fclose(f);
        return fail(SD_E_FORMAT, "load_state: %s is not a STARDUST v1/v2 file", path);
    }
    if (h.version >= 2) {
        const int bh = h.reserved[0];
        if (bh < 0 || bh > 8) {
            fclose(f);
            return fail(SD_E_FORMAT, "load_state: bad black-hole count %d", bh);
        }
        // Black holes are outside the plain-PM path: their records are skipped.
        if (bh > 0 && fseek(f, (long)(kBlackHoleRecord * (size_t)bh), SEEK_CUR) != 0) {
            fclose(f);
            return fail(SD_E_FORMAT, "load_state: truncated black-hole records");
        }
    }
    sd_config c = s->cfg;
    c.particle_count = h.count;
    c.grid_size = h.gridSize;
    c.boundary = h.boundary;
    c.gravity = h.gravity;
    // (Preset)h.preset (Sim.cu:5082); presets other than Filament place as Empty
    c.preset = (h.preset == SD_PRESET_FILAMENT) ? SD_PRESET_FILAMENT : SD_PRESET_EMPTY;
    int rc = reconfigure(s, &c);
    if (rc) {
        fclose(f);
        return rc;
    }
    const int n = h.count < s->N ? h.count : s->N;
    std::vector<float4> hp((size_t)n), hv((size_t)n);
    // positions of every record come first, then velocities: skip the positions
    // past a clamped count
    const bool ok = fread(hp.data(), sizeof(float4), (size_t)n, f) == (size_t)n &&
                    (n == h.count || fseek(f, (long)(sizeof(float4) * (size_t)(h.count - n)), SEEK_CUR) == 0) &&
                    fread(hv.data(), sizeof(float4), (size_t)n, f) == (size_t)n;
    fclose(f);
    if (!ok) return fail(SD_E_FORMAT, "load_state: truncated particle data");
    rc = sd_set_particles(s, reinterpret_cast<const float*>(hp.data()), reinterpret_cast<const float*>(hv.data()), n,
                          SD_HOST);
    if (rc) return rc;
    s->sim_time = h.simTime;
    return SD_OK;
}

int sd_timings_get(const sd_sim* s, sd_timings* out) {
    if (!s || !out) return fail(SD_E_ARG, "timings: null");
    *out = s->tm;
    if (s->ev_valid) {
        DeviceGuard g(s->device);
        cudaEventSynchronize(s->ev[4]);
        float ms[4] = {0, 0, 0, 0}, tot = 0.f;
        for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&ms[i], s->ev[i], s->ev[i + 1]);
        cudaEventElapsedTime(&tot, s->ev[0], s->ev[4]);
        out->sort_ms = ms[0];
        out->deposit_ms = ms[1];
        out->poisson_ms = ms[2];
        out->gather_ms = ms[3];
        out->total_ms = tot;
        // kernels: sort, row table / deposit, passes A-E, gather
        cudaEvent_t seq[9] = {s->ev[0], s->ev[1], s->ev[2], s->pev[0], s->pev[1], s->pev[2], s->pev[3], s->ev[3],
                              s->ev[4]};
        for (int i = 0; i < 8; ++i) {
            float k = 0.f;
            cudaEventElapsedTime(&k, seq[i], seq[i + 1]);
            out->kernel_ms[i] = k;
        }
    }
    return SD_OK;
}

double sd_sim_time(const sd_sim* s) { return s ? s->sim_time : 0.0; }
int sd_grid_size(const sd_sim* s) { return s ? s->G : 0; }
int sd_particle_count(const sd_sim* s) { return s ? s->N : 0; }
int sd_particle_capacity(const sd_sim* s) { return s ? s->capacity : 0; }
double sd_changed_fraction(const sd_sim* s) { return s ? s->chg_frac : -1.0; }
int sd_merge_sorting(const sd_sim* s) { return (s && merge_next(s)) ? 1 : 0; }
int sd_active_count(const sd_sim* s) { return s ? s->active : 0; }
int sd_step_count(const sd_sim* s) { return s ? s->step_count : 0; }

static double reduce_rho(sd_sim* s, int op) {
    if (!s || !s->configured || !s->rho) return 0.0;
    DeviceGuard g(s->device);
    settle(s);
    if (!s->rho_valid && do_field(s, true)) return 0.0;
    double out = 0.0;
    if (launch_reduce_grid(s->rho, (size_t)s->G * s->G * s->G, op, s->partials, s->mom + 7, s->stream)) return 0.0;
    if (copy_out(&out, s->mom + 7, sizeof(double), SD_HOST, s->stream)) return 0.0;
    return out;
}

double sd_measure_total_grid_mass(sd_sim* s) { return reduce_rho(s, 0); }
double sd_measure_max_density(sd_sim* s) { return reduce_rho(s, 1); }
int sd_measure_occupied_cells(sd_sim* s) { return (int)reduce_rho(s, 2); }

int sd_measure_centroid(sd_sim* s, double* cx, double* cy) {
    if (cx) *cx = 0.5;
    if (cy) *cy = 0.5;
    if (!s || !s->configured || !cx || !cy) return fail(SD_E_ARG, "measure_centroid: not initialised or null output");
    DeviceGuard g(s->device);
    settle(s);
    double out[3] = {0.0, 0.0, 0.0};
    int rc = launch_centroid(s->pos, s->N, s->partials, s->mom + 5, s->stream);
    if (!rc) rc = copy_out(out, s->mom + 5, sizeof(double) * 3, SD_HOST, s->stream);
    if (rc) return sim_error(s, rc);
    if (out[2] > 0.0) {
        *cx = out[0] / out[2];
        *cy = out[1] / out[2];
    }
    return SD_OK;
}

double sd_measure_kinetic_energy(sd_sim* s) {
    if (!s || !s->configured) return 0.0;
    DeviceGuard g(s->device);
    settle(s);
    double out[8];
    if (launch_energy(nullptr, s->G, s->pos, s->vel, s->N, s->mean_pending ? s->mean : nullptr, s->partials, s->mom,
                      s->stream))
        return 0.0;
    if (copy_out(out, s->mom, sizeof(double) * 8, SD_HOST, s->stream)) return 0.0;
    return out[0] / (double)(s->N > 0 ? s->N : 1);  // m = 1/N (Sim.cu:5141-5149)
}

int sd_diagnostics_get(sd_sim* s, sd_diagnostics* out) {
    if (!s || !out || !s->configured) return fail(SD_E_ARG, "diagnostics: null");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    double d[8];
    // momentum sums of the last gather (before zeroing) and energies after zeroing
    int rc = launch_energy(s->phi, s->G, s->pos, s->vel, s->N, s->mean_pending ? s->mean : nullptr, s->partials,
                           s->mom, s->stream, isolated(s) ? 2 * s->G : 0);
    if (rc) return sim_error(s, rc);
    rc = copy_out(d, s->mom, sizeof(double) * 8, SD_HOST, s->stream);
    if (rc) return sim_error(s, rc);
    float mean[4] = {0, 0, 0, 0};
    rc = copy_out(mean, s->mean, sizeof(float) * 4, SD_HOST, s->stream);
    if (rc) return sim_error(s, rc);
    // a = -pot_scale grad(phi): the potential per unit mass is pot_scale * phi; m = 1/N.
    const double m = 1.0 / (double)(s->N > 0 ? s->N : 1);
    out->kinetic = d[0] * m;
    out->potential = d[1] * (double)pot_scale_of(s) * m;
    out->momentum[0] = d[2] * m;
    out->momentum[1] = d[3] * m;
    out->momentum[2] = d[4] * m;
    for (int j = 0; j < 3; ++j) out->mean_velocity_removed[j] = s->mean_pending ? mean[j] : 0.0;
    out->live_count = d[5];
    return SD_OK;
}

int sd_diagnostics_history(sd_sim* s, double* out, int max_records, int* count_out) {
    if (!s || !s->configured || !out || max_records < 0) return fail(SD_E_ARG, "diagnostics_history: bad arguments");
    DeviceGuard g(s->device);
    if (int rc_settle = settle(s)) return rc_settle;
    unsigned long long total = 0;
    if (copy_out(&total, s->diag_count, sizeof(total), SD_HOST, s->stream)) return sim_error(s, SD_E_CUDA);
    const unsigned long long avail = total < (unsigned long long)kDiagCap ? total : (unsigned long long)kDiagCap;
    const int k = (int)(avail < (unsigned long long)max_records ? avail : (unsigned long long)max_records);
    // the last k records, oldest first; the ring may wrap once inside them
    for (int i = 0; i < k; ++i) {
        const unsigned long long idx = total - (unsigned long long)k + (unsigned long long)i;
        const double* src = s->diag_rec + (size_t)(idx % (unsigned long long)kDiagCap) * 8;
        if (SD_CUDA(cudaMemcpyAsync(out + (size_t)i * 8, src, sizeof(double) * 8, cudaMemcpyDeviceToHost, s->stream)))
            return sim_error(s, SD_E_CUDA);
    }
    if (SD_CUDA(cudaStreamSynchronize(s->stream))) return sim_error(s, SD_E_CUDA);
    if (count_out) *count_out = k;
    return SD_OK;
}

long long sd_kernel_launches(const sd_sim* s) {
    (void)s;
    return launches();
}

// ---- stage entry points ----------------------------------------------------

int sd_key_bits(int grid_size, int order) { return key_bits_for(grid_size, order); }

int sd_cell_keys(const float* pos, int n, int G, int order, uint32_t* keys, void* stream) {
    if (!pos || !keys || n < 0 || G < 16 || (G & (G - 1)) || order < 0 || order > 2)
        return fail(SD_E_ARG, "cell_keys: bad arguments");
    return launch_cell_keys(reinterpret_cast<const float4*>(pos), n, G, order, keys, (cudaStream_t)stream);
}

size_t sd_sort_workspace_bytes(int n) { return sort_workspace_bytes(n); }

int sd_sort_pairs(const uint32_t* keys_in, const int32_t* vals_in, uint32_t* keys_out, int32_t* vals_out,
                  uint32_t* keys_tmp, int32_t* vals_tmp, int n, int key_bits, void* ws, size_t ws_bytes,
                  void* stream) {
    return launch_sort_pairs(keys_in, vals_in, keys_out, vals_out, keys_tmp, vals_tmp, n, key_bits, ws, ws_bytes,
                             (cudaStream_t)stream);
}

int sd_reorder(const float* pos_in, const float* vel_in, const int32_t* perm, float* pos_out, float* vel_out, int n,
               void* stream) {
    if (!pos_in || !vel_in || !perm || !pos_out || !vel_out || n < 0) return fail(SD_E_ARG, "reorder: bad arguments");
    return launch_reorder(reinterpret_cast<const float4*>(pos_in), reinterpret_cast<const float4*>(vel_in), perm,
                          reinterpret_cast<float4*>(pos_out), reinterpret_cast<float4*>(vel_out), n,
                          (cudaStream_t)stream);
}

size_t sd_deposit_workspace_bytes(int G) { return deposit_workspace_bytes(G); }

int sd_deposit(const float* pos, int n, int G, float* rho, void* ws, size_t ws_bytes, void* stream) {
    if (!pos || !rho || !ws || n < 0 || G < 16 || G > 512 || (G & (G - 1)))
        return fail(SD_E_ARG, "deposit: bad arguments");
    if (ws_bytes < deposit_workspace_bytes(G)) return fail(SD_E_ARG, "deposit: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    long long* acc = reinterpret_cast<long long*>(ws);
    int rc = launch_clear_u64(acc, (size_t)G * G * G, st);
    if (!rc) rc = launch_deposit_fixed(reinterpret_cast<const float4*>(pos), n, G, acc, st);
    if (!rc) rc = launch_fixed_to_float(acc, G, rho, 0, st);
    return rc;
}

size_t sd_poisson_workspace_bytes(int G) { return align_up(sizeof(float2) * poisson_spectrum_elems(G), 256); }

int sd_poisson(const float* rho, int G, float soft, float* phi, void* ws, size_t ws_bytes, void* stream) {
    if (!rho || !phi || !ws || G < 16 || G > 512 || (G & (G - 1))) return fail(SD_E_ARG, "poisson: bad arguments");
    if (ws_bytes < sd_poisson_workspace_bytes(G)) return fail(SD_E_ARG, "poisson: workspace too small");
    // plans are cached per (G, softening); the cache is never freed (small: G float2 + G/2 floats)
    static std::mutex mu;
    static std::vector<PoissonPlan*> cache;
    PoissonPlan* plan = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu);
        for (PoissonPlan* p : cache)
            if (p->G == G && p->soft == soft) plan = p;
        if (!plan) {
            plan = new PoissonPlan();
            int rc = poisson_plan_build(*plan, G, soft);
            if (rc) {
                delete plan;
                return rc;
            }
            cache.push_back(plan);
        }
    }
    return launch_poisson(*plan, nullptr, rho, nullptr, reinterpret_cast<float2*>(ws), phi, (cudaStream_t)stream);
}

size_t sd_gather_workspace_bytes(int n) { return sizeof(double) * 4 * gather_partials(n); }

int sd_gather_kick_drift(const float* phi, int G, float pot_scale, float* pos, float* vel, int n, float dt_kick,
                         float dt_drift, float c2, const float* mean_vel, double* mom_out, void* ws, size_t ws_bytes,
                         void* stream) {
    if (!phi || !pos || !vel || n < 0 || G < 16 || (G & (G - 1))) return fail(SD_E_ARG, "gather: bad arguments");
    if (mom_out && (!ws || ws_bytes < sd_gather_workspace_bytes(n))) return fail(SD_E_ARG, "gather: workspace too small");
    float4* p4 = reinterpret_cast<float4*>(pos);
    float4* v4 = reinterpret_cast<float4*>(vel);
    return launch_gather_kick_drift(phi, G, pot_scale, p4, v4, nullptr, p4, v4, nullptr, 0, n, dt_kick, dt_drift, c2,
                                    mean_vel, mom_out ? (double*)ws : nullptr, mom_out, nullptr, (cudaStream_t)stream);
}

int sd_interpolate_accel(const float* phi, int G, float pot_scale, const float* pos, float* acc, int n, void* stream) {
    if (!phi || !pos || !acc || n < 0 || G < 16 || (G & (G - 1))) return fail(SD_E_ARG, "interpolate: bad arguments");
    return launch_interpolate_accel(phi, G, pot_scale, reinterpret_cast<const float4*>(pos),
                                    reinterpret_cast<float4*>(acc), n, (cudaStream_t)stream);
}

}  // extern "C"
