// sd_sim_impl.h -- the simulation handle's state, shared by sd_sim.cu (the
// single-scene C ABI) and sd_ensemble.cu (many scenes in one graph).
#pragma once

#include <cuda_runtime.h>

#include "sd_internal.h"
#include "stardust_pm.h"

struct sd_sim {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    bool configured = false;
    bool cuda_failed = false;
    sd_config cfg{};
    int N = 0;          // slots the kernels run over (the reference's allocN)
    int G = 0;
    int capacity = 0;   // slots allocated (capacityN); N <= capacity, a shrink narrows N only
    // the last structural request (requestedN / requestedG / requestedBoundary): a
    // repeated request changes nothing even when N was clamped below it
    int req_n = -1, req_g = -1, req_boundary = -1;
    int active = 0;     // slots loaded by the last set_particles / load_state
    double sim_time = 0.0;
    int step_count = 0;

    float4 *pos = nullptr, *vel = nullptr, *pos2 = nullptr, *vel2 = nullptr;
    uint32_t *keys = nullptr, *keys2 = nullptr, *keys3 = nullptr;
    int32_t *vals = nullptr, *vals2 = nullptr;
    void* sort_ws = nullptr;
    size_t sort_ws_bytes = 0;
    long long* acc = nullptr;
    int* row_start = nullptr;    // key-space row starts of the sorted particles (tiled order)
    int* dep_ints = nullptr;     // work plan of the fused deposit (deposit_work_ints(G), zero between uses)
    float2* spec = nullptr;     // bricked spectrum, transformed in place
    float* phi = nullptr;
    float* rho = nullptr;        // kept density (keep_density)
    float* green = nullptr;      // isolated boundary: real Green spectrum of the 2G box
    sd::HydroGrids hydro;        // pressure / cooling grids, allocated while either is on
    int graph_phase = 0;         // step count parity the captured graph was made at (hydro)
    bool graph_incr = false;     // whether the captured graph's first step merge-sorts
    bool graph_dirty = false;    // whether it clears change bits left by an unmerged gather first
    double* partials = nullptr;  // gather / energy / reduction partials
    size_t partials_count = 0;
    double* mom = nullptr;       // 8 doubles: momentum sums of the last step, energy results
    float* mean = nullptr;       // 4 floats: pending mean velocity; [3] = max speed scratch
    bool mean_pending = false;
    bool rho_valid = false;
    bool keys_valid = false;     // keys hold the order keys of the current pos order
    bool counts_valid = false;   // the sort workspace holds the first-pass tile counts of keys
    bool incr_ready = false;     // the last step left change bits and its row table: merge-sort next
    bool chg_dirty = false;      // change bits written and not consumed yet (cleared before reuse)
    bool allow_incr = true;      // merge sorting allowed (ensemble members sort in full)
    // Merge or full sort, by the share of keys that changed: each merge copies its
    // changed-key count to chg_host (pinned); above kMergeMaxFraction the steps
    // run the full sort, with one probing merge every kMergeProbe steps
    int* chg_host = nullptr;
    double chg_frac = -1.0;      // the last measured share (-1: none yet)
    bool merge_off = false;
    int merge_probe_at = 0;
    bool graph_merge_off = false;  // merge_off when the sd_steps graph was captured
    void* rs_base = nullptr;     // merge-sort buffers (tiled order, periodic)
    sd::ResortBufs rs;
    sd::PoissonPlan plan;

    // leapfrog
    bool lf_open = false;
    float lf_dt_prev = 0.f;

    // timings of the last eager step: ev[0..4] phase bounds, pev[0..3] after Poisson passes A-D
    cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    cudaEvent_t pev[4] = {nullptr, nullptr, nullptr, nullptr};
    // host offload step (sd_step_host): a second stream for the copies that overlap
    // the step, its two events, and the event the step's first velocity read waits on
    cudaStream_t io_stream = nullptr;
    cudaEvent_t io_ev[2] = {nullptr, nullptr};
    cudaEvent_t vel_wait = nullptr;
    // pipelined offload (sd_step_host_async): a third particle set that stages the
    // next step's inputs, the stream that uploads into it, and the events ordering
    // uploads, steps and downloads across calls
    cudaStream_t up_stream = nullptr;
    float4 *stage_pos = nullptr, *stage_vel = nullptr;
    cudaEvent_t up_ev[2] = {nullptr, nullptr};    // this call's positions / velocities are on the device
    cudaEvent_t out_ev = nullptr;                 // this call's result is ready to download
    cudaEvent_t down_ev[2] = {nullptr, nullptr};  // downloads done, alternating between calls
    cudaEvent_t stage_free = nullptr;             // the staging set's last download (null: free)
    long long async_calls = 0;
    bool async_pending = false;                   // offload work queued and not waited for
    bool ev_valid = false;
    sd_timings tm{};
    sd_diagnostics diag{};
    bool diag_valid = false;

    // learned correction (sd_set_mlp): device copy of the parameters, per-slot output
    float* mlp_params = nullptr;
    float4* mlp_out = nullptr;
    float mlp_scale = 0.f;
    bool mlp_on = false;

    int gather_blocks = 0;   // cap of the gather grid (0: the default); set by the ensemble autotuner
    int dep_split = 0;       // window particles per CTA share of the fused deposit (0: deposit_split's default)

    // per-step FP64 diagnostics ring (cfg.diagnostics): kDiagCap records of 8 doubles
    double* diag_rec = nullptr;
    unsigned long long* diag_count = nullptr;

    // captured steps for sd_steps
    cudaGraphExec_t graph = nullptr;
    float graph_dt = 0.f;
    const float4* graph_pos = nullptr;  // particle buffer the graph's first step reads
    long long graph_launches = 0;       // kernels inside one replay
};


namespace sdsim {

constexpr int kDiagCap = 4096;

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev);
    ~DeviceGuard();
};

int sim_error(sd_sim* s, int rc);
bool sort_due(const sd_sim* s);
int ensure_sort_inputs(sd_sim* s);
void invalidate_keys(sd_sim* s);
bool incr_possible(const sd_sim* s);
bool hydro_on(const sd_sim* s);
int cooling_period(const sd_sim* s);
int key_bits_for(int G, int order);
// One step of one scene on s->stream (no host synchronisation; capturable).
int do_step(sd_sim* s, float dt, bool sort, bool timed);

}  // namespace sdsim
