// sd_ensemble.cu -- many independent scenes advanced together (no counterpart
// in the reference, which runs one Sim per scene).
//
// Each scene is a full sd_sim with its own buffers and stream. One step of the
// whole ensemble is ONE CUDA graph: a fork node, one branch per scene holding
// that scene's complete step (sort, fused deposit + Poisson passes, gather),
// and a join. Branches are independent, so the GPU runs small scenes side by
// side instead of one after another, and the host issues a single launch per
// step. Two graphs are kept, one per parity of the ping-pong particle buffers.
//
// The autotuner times, for every scene, each combination of
//   deposit path  : fused tiled (pass A deposits from the row table) or
//                   int64 atomics (row-major sort, separate deposit kernel)
//   deposit share : for the fused path, the window particles one CTA takes before
//                   a heavy bundle is split among several (3, 10 or 30 times the
//                   mean window)
//   gather grid   : 2, 4 or 8 CTAs per SM, or one CTA per 256 particles
// on a snapshot of the scene (restored afterwards) and keeps the fastest.
// The density of every choice is the same integer fixed-point sum, so the
// tuned ensemble's densities are bit-exact against the scene run alone.
#include <cuda_runtime.h>

#include <algorithm>
#include <utility>
#include <vector>

#include "sd_internal.h"
#include "sd_sim_impl.h"

using namespace sd;
using namespace sdsim;

namespace {

constexpr int kSmCount = 148;

struct SceneSlot {
    sd_sim* sim = nullptr;
    cudaEvent_t join = nullptr;
    // particle buffers after each parity's step (what the graph writes)
    float4* pos_after[2] = {nullptr, nullptr};
    float4* vel_after[2] = {nullptr, nullptr};
    float4* pos2_after[2] = {nullptr, nullptr};
    float4* vel2_after[2] = {nullptr, nullptr};
    sd_scene_tuning tuning{};
    // what the graphs were captured with; any difference makes them stale
    const float4* expect_pos = nullptr;
    int order = 0, gather_blocks = 0, dep_split = 0, N = 0, G = 0;
    bool mlp_on = false;
};

}  // namespace

struct sd_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaEvent_t fork = nullptr;
    std::vector<SceneSlot> scenes;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    float graph_dt = 0.f;
    int parity = 0;             // graph to launch next
    long long graph_kernels = 0;  // kernels in one step graph
};

namespace {

void drop_graphs(sd_ensemble* e) {
    for (auto& g : e->graph)
        if (g) cudaGraphExecDestroy(g);
    e->graph[0] = e->graph[1] = nullptr;
}

// Scenes with the hydro add-ons (a cooling schedule tied to the step count) run
// as solo simulations.
bool graphable(const sd_sim* s) {
    return s->configured && (s->cfg.sort_interval == 0 || s->cfg.sort_interval == 1) && !hydro_on(s);
}

struct HostCounters {
    double sim_time;
    int step_count;
    bool lf_open;
    float lf_dt_prev;
    bool mean_pending, keys_valid, counts_valid, rho_valid;
};

HostCounters save_counters(const sd_sim* s) {
    return {s->sim_time,  s->step_count,   s->lf_open,     s->lf_dt_prev,
            s->mean_pending, s->keys_valid, s->counts_valid, s->rho_valid};
}

void restore_counters(sd_sim* s, const HostCounters& c) {
    s->sim_time = c.sim_time;
    s->step_count = c.step_count;
    s->lf_open = c.lf_open;
    s->lf_dt_prev = c.lf_dt_prev;
    s->mean_pending = c.mean_pending;
    s->keys_valid = c.keys_valid;
    s->counts_valid = c.counts_valid;
    s->rho_valid = c.rho_valid;
}

// Everything a step needs that must not be inside the graph: leapfrog opening
// kicks, and keys and first-pass sort counts of unsorted buffers.
int prepare_scenes(sd_ensemble* e, float dt) {
    for (auto& sl : e->scenes) {
        sd_sim* s = sl.sim;
        if (!graphable(s))
            return fail(SD_E_STATE, "ensemble: scenes must sort every step or never, without hydro add-ons");
        if (s->cfg.integrator == SD_INT_KDK && !s->lf_open) {
            if (int rc = do_step(s, dt, sort_due(s), false)) return rc;
        }
        if (s->cfg.sort_interval == 1) {
            if (int rc = ensure_sort_inputs(s)) return sim_error(s, rc);
        }
    }
    return SD_OK;
}

// One step of every scene as one graph (fork -> scene branches -> join).
int capture_step(sd_ensemble* e, float dt, int par, cudaGraphExec_t* out) {
    if (SD_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal))) return SD_E_CUDA;
    int rc = SD_CUDA(cudaEventRecord(e->fork, e->stream));
    for (auto& sl : e->scenes) {
        if (rc) break;
        sd_sim* s = sl.sim;
        rc = SD_CUDA(cudaStreamWaitEvent(s->stream, e->fork, 0));
        if (!rc) rc = do_step(s, dt, s->cfg.sort_interval == 1, false);
        if (!rc) rc = SD_CUDA(cudaEventRecord(sl.join, s->stream));
        if (!rc) rc = SD_CUDA(cudaStreamWaitEvent(e->stream, sl.join, 0));
        sl.pos_after[par] = s->pos;
        sl.vel_after[par] = s->vel;
        sl.pos2_after[par] = s->pos2;
        sl.vel2_after[par] = s->vel2;
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(e->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (SD_CUDA(ec)) return SD_E_CUDA;
    const cudaError_t ei = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    return SD_CUDA(ei);
}

int build_graphs(sd_ensemble* e, float dt) {
    drop_graphs(e);
    std::vector<HostCounters> saved;
    for (auto& sl : e->scenes) saved.push_back(save_counters(sl.sim));
    const long long l0 = launches();
    int rc = capture_step(e, dt, 0, &e->graph[0]);
    const long long one = launches() - l0;
    if (!rc) rc = capture_step(e, dt, 1, &e->graph[1]);
    // capture only recorded the kernels: undo their launch count and host effects
    count_launch(-(launches() - l0));
    for (size_t i = 0; i < e->scenes.size(); ++i) restore_counters(e->scenes[i].sim, saved[i]);
    if (rc) {
        drop_graphs(e);
        return rc;
    }
    e->graph_kernels = one;
    e->graph_dt = dt;
    e->parity = 0;
    for (auto& sl : e->scenes) {
        const sd_sim* s = sl.sim;
        sl.expect_pos = s->pos;
        sl.order = s->cfg.order;
        sl.gather_blocks = s->gather_blocks;
        sl.dep_split = s->dep_split;
        sl.N = s->N;
        sl.G = s->G;
        sl.mlp_on = s->mlp_on;
    }
    return SD_OK;
}

bool graphs_current(const sd_ensemble* e, float dt) {
    if (!e->graph[0] || e->graph_dt != dt) return false;
    for (const auto& sl : e->scenes) {
        const sd_sim* s = sl.sim;
        if (s->pos != sl.expect_pos || s->cfg.order != sl.order || s->gather_blocks != sl.gather_blocks ||
            s->dep_split != sl.dep_split || s->N != sl.N || s->G != sl.G || s->mlp_on != sl.mlp_on || !graphable(s))
            return false;
    }
    return true;
}

// Host-side effects of one replayed step on every scene.
void after_replay(sd_ensemble* e, float dt, int par) {
    for (auto& sl : e->scenes) {
        sd_sim* s = sl.sim;
        s->pos = sl.pos_after[par];
        s->vel = sl.vel_after[par];
        s->pos2 = sl.pos2_after[par];
        s->vel2 = sl.vel2_after[par];
        s->sim_time += dt;
        ++s->step_count;
        s->mean_pending = true;
        s->keys_valid = s->cfg.sort_interval == 1;
        s->counts_valid = s->cfg.sort_interval == 1;
        s->rho_valid = s->rho && (s->cfg.keep_density || s->mlp_on);
        s->ev_valid = false;
        if (s->cfg.integrator == SD_INT_KDK) {
            s->lf_open = true;
            s->lf_dt_prev = dt;
        }
    }
}

// Device snapshot of one scene (particles and the pending mean) for the tuner.
struct Snapshot {
    float4* pos = nullptr;
    float4* vel = nullptr;
    float* mean = nullptr;
    HostCounters c{};
    int order = 0;
};

int take_snapshot(sd_sim* s, Snapshot& sn) {
    const size_t b = sizeof(float4) * (size_t)s->N;
    if (SD_CUDA(cudaMalloc(&sn.pos, b)) || SD_CUDA(cudaMalloc(&sn.vel, b)) ||
        SD_CUDA(cudaMalloc(&sn.mean, 4 * sizeof(float))))
        return SD_E_NOMEM;
    if (SD_CUDA(cudaMemcpyAsync(sn.pos, s->pos, b, cudaMemcpyDeviceToDevice, s->stream)) ||
        SD_CUDA(cudaMemcpyAsync(sn.vel, s->vel, b, cudaMemcpyDeviceToDevice, s->stream)) ||
        SD_CUDA(cudaMemcpyAsync(sn.mean, s->mean, 4 * sizeof(float), cudaMemcpyDeviceToDevice, s->stream)))
        return SD_E_CUDA;
    sn.c = save_counters(s);
    sn.order = s->cfg.order;
    return SD_OK;
}

int restore_snapshot(sd_sim* s, const Snapshot& sn) {
    const size_t b = sizeof(float4) * (size_t)s->N;
    if (SD_CUDA(cudaMemcpyAsync(s->pos, sn.pos, b, cudaMemcpyDeviceToDevice, s->stream)) ||
        SD_CUDA(cudaMemcpyAsync(s->vel, sn.vel, b, cudaMemcpyDeviceToDevice, s->stream)) ||
        SD_CUDA(cudaMemcpyAsync(s->mean, sn.mean, 4 * sizeof(float), cudaMemcpyDeviceToDevice, s->stream)))
        return SD_E_CUDA;
    restore_counters(s, sn.c);
    s->keys_valid = false;  // keys of the restored order are recomputed
    s->counts_valid = false;
    s->rho_valid = false;
    return SD_OK;
}

void free_snapshot(Snapshot& sn) {
    if (sn.pos) cudaFree(sn.pos);
    if (sn.vel) cudaFree(sn.vel);
    if (sn.mean) cudaFree(sn.mean);
    sn = Snapshot{};
}

// Median time of `reps` eager steps of one scene under its current settings.
int time_scene(sd_sim* s, float dt, int reps, cudaEvent_t a, cudaEvent_t b, float* ms_out) {
    std::vector<float> t;
    for (int r = 0; r < reps + 1; ++r) {
        if (SD_CUDA(cudaEventRecord(a, s->stream))) return SD_E_CUDA;
        if (int rc = do_step(s, dt, true, false)) return rc;
        if (SD_CUDA(cudaEventRecord(b, s->stream)) || SD_CUDA(cudaEventSynchronize(b))) return SD_E_CUDA;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (r > 0) t.push_back(ms);  // the first rep warms caches and the sort keys
    }
    std::sort(t.begin(), t.end());
    *ms_out = t[t.size() / 2];
    return SD_OK;
}

}  // namespace

extern "C" {

int sd_ensemble_create(sd_ensemble** out, int device) {
    if (!out) return fail(SD_E_ARG, "ensemble_create: null output");
    *out = nullptr;
    DeviceGuard g(device);
    sd_ensemble* e = new sd_ensemble();
    e->device = device;
    if (SD_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) ||
        SD_CUDA(cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming))) {
        if (e->stream) cudaStreamDestroy(e->stream);
        delete e;
        return SD_E_CUDA;
    }
    e->own_stream = true;
    *out = e;
    return SD_OK;
}

int sd_ensemble_destroy(sd_ensemble* e) {
    if (!e) return SD_OK;
    DeviceGuard g(e->device);
    cudaStreamSynchronize(e->stream);
    drop_graphs(e);
    for (auto& sl : e->scenes) {
        sd_destroy(sl.sim);
        if (sl.join) cudaEventDestroy(sl.join);
    }
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return SD_OK;
}

int sd_ensemble_add(sd_ensemble* e, const sd_config* cfg, const float* pos, const float* vel, int n, int where) {
    if (!e || !cfg) return fail(SD_E_ARG, "ensemble_add: null argument");
    if (cfg->boundary != SD_BOUNDARY_PERIODIC) return fail(SD_E_UNSUPPORTED, "ensemble_add: periodic scenes only");
    DeviceGuard g(e->device);
    sd_sim* s = nullptr;
    int rc = sd_create(&s, e->device);
    if (!rc) s->allow_incr = false;  // scenes sort in full: one graph per step, no per-scene merge state
    if (!rc) rc = sd_init(s, cfg);
    if (!rc && pos) rc = sd_set_particles(s, pos, vel, n, where);
    if (!rc && !graphable(s))
        rc = fail(SD_E_ARG, "ensemble_add: scenes must sort every step or never");
    SceneSlot sl;
    if (!rc) rc = SD_CUDA(cudaEventCreateWithFlags(&sl.join, cudaEventDisableTiming));
    if (rc) {
        if (s) sd_destroy(s);
        return rc;
    }
    sl.sim = s;
    sl.tuning.order = s->cfg.order;
    sl.tuning.gather_blocks = 0;
    sl.tuning.step_ms = -1.f;
    sl.tuning.deposit_split = 0;
    e->scenes.push_back(sl);
    drop_graphs(e);
    return (int)e->scenes.size() - 1;
}

int sd_ensemble_size(const sd_ensemble* e) { return e ? (int)e->scenes.size() : 0; }

sd_sim* sd_ensemble_scene(sd_ensemble* e, int index) {
    if (!e || index < 0 || index >= (int)e->scenes.size()) return nullptr;
    return e->scenes[index].sim;
}

int sd_ensemble_autotune(sd_ensemble* e, float dt, int reps) {
    if (!e) return fail(SD_E_ARG, "ensemble_autotune: null handle");
    if (reps < 1) reps = 3;
    DeviceGuard g(e->device);
    drop_graphs(e);
    cudaEvent_t a = nullptr, b = nullptr;
    if (SD_CUDA(cudaEventCreate(&a)) || SD_CUDA(cudaEventCreate(&b))) return SD_E_CUDA;
    const int orders[2] = {SD_ORDER_TILED, SD_ORDER_ROWMAJOR};
    const int caps[4] = {2 * kSmCount, 4 * kSmCount, 8 * kSmCount, 0};
    const int mults[3] = {3, 10, 30};  // deposit share: times a window's mean particle count
    int rc = SD_OK;
    for (auto& sl : e->scenes) {
        if (rc) break;
        sd_sim* s = sl.sim;
        if (s->cfg.sort_interval != 1) continue;  // the variants differ only in sorted steps
        if (s->graph) cudaGraphExecDestroy(s->graph);  // the scene's own sd_steps graph
        s->graph = nullptr;
        Snapshot sn;
        rc = take_snapshot(s, sn);
        float best = 1e30f;
        int best_order = s->cfg.order, best_cap = s->gather_blocks, best_split = s->dep_split;
        for (int o = 0; o < 2 && !rc; ++o)
            for (int m = 0; m < (orders[o] == SD_ORDER_TILED ? 3 : 1) && !rc; ++m)
                for (int c = 0; c < 4 && !rc; ++c) {
                    s->cfg.order = orders[o];
                    s->dep_split = orders[o] == SD_ORDER_TILED ? deposit_split(s->N, s->G, mults[m]) : 0;
                    s->gather_blocks = caps[c];
                    rc = restore_snapshot(s, sn);
                    float ms = 0.f;
                    if (!rc) rc = time_scene(s, dt, reps, a, b, &ms);
                    if (!rc && ms < best) {
                        best = ms;
                        best_order = orders[o];
                        best_cap = caps[c];
                        best_split = s->dep_split;
                    }
                }
        s->cfg.order = best_order;
        s->gather_blocks = best_cap;
        s->dep_split = best_split;
        if (!rc) rc = restore_snapshot(s, sn);
        if (!rc) rc = SD_CUDA(cudaStreamSynchronize(s->stream));
        free_snapshot(sn);
        sl.tuning.order = best_order;
        sl.tuning.gather_blocks = best_cap;
        sl.tuning.step_ms = best;
        sl.tuning.deposit_split = best_split;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return rc;
}

int sd_ensemble_get_tuning(const sd_ensemble* e, int index, sd_scene_tuning* out) {
    if (!e || !out || index < 0 || index >= (int)e->scenes.size()) return fail(SD_E_ARG, "ensemble_get_tuning: bad index");
    *out = e->scenes[index].tuning;
    return SD_OK;
}

int sd_ensemble_steps(sd_ensemble* e, float dt, int nsteps) {
    if (!e) return fail(SD_E_ARG, "ensemble_steps: null handle");
    if (nsteps < 0) return fail(SD_E_ARG, "ensemble_steps: negative count");
    if (e->scenes.empty() || nsteps == 0) return SD_OK;
    DeviceGuard g(e->device);
    // the graphs are stale when dt changed or a scene was stepped or changed on its own
    if (e->graph[0] && !graphs_current(e, dt)) drop_graphs(e);
    if (!e->graph[0]) {
        if (int rc = prepare_scenes(e, dt)) return rc;
    }
    // work issued on the scenes' own streams so far (particle uploads, opening
    // kicks, keys) precedes the replays
    for (auto& sl : e->scenes) {
        if (SD_CUDA(cudaEventRecord(sl.join, sl.sim->stream)) || SD_CUDA(cudaStreamWaitEvent(e->stream, sl.join, 0)))
            return SD_E_CUDA;
    }
    if (!e->graph[0]) {
        if (int rc = build_graphs(e, dt)) return rc;
    }
    for (int k = 0; k < nsteps; ++k) {
        if (SD_CUDA(cudaGraphLaunch(e->graph[e->parity], e->stream))) return SD_E_CUDA;
        count_launch(e->graph_kernels);
        after_replay(e, dt, e->parity);
        e->parity ^= 1;
    }
    for (auto& sl : e->scenes) sl.expect_pos = sl.sim->pos;
    // later per-scene calls on the scenes' own streams run after the replays
    if (SD_CUDA(cudaEventRecord(e->fork, e->stream))) return SD_E_CUDA;
    for (auto& sl : e->scenes)
        if (SD_CUDA(cudaStreamWaitEvent(sl.sim->stream, e->fork, 0))) return SD_E_CUDA;
    return SD_OK;
}

int sd_ensemble_synchronize(sd_ensemble* e) {
    if (!e) return fail(SD_E_ARG, "ensemble_synchronize: null handle");
    DeviceGuard g(e->device);
    if (SD_CUDA(cudaStreamSynchronize(e->stream))) return SD_E_CUDA;
    for (auto& sl : e->scenes)
        if (SD_CUDA(cudaStreamSynchronize(sl.sim->stream))) return SD_E_CUDA;
    return SD_OK;
}

void* sd_ensemble_stream(const sd_ensemble* e) { return e ? (void*)e->stream : nullptr; }

long long sd_ensemble_graph_kernels(const sd_ensemble* e) { return e ? e->graph_kernels : 0; }

}  // extern "C"
