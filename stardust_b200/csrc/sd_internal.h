// sd_internal.h -- host-side helpers shared by the library's translation units.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/stardust_pm.h"

namespace sd {

// Sticky process-wide error record (the reference's g_failed / g_failMsg,
// Sim.cu:52-75): the first failure's message is kept until sd_clear_error.
int fail(int code, const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what, const char* file, int line);

// Launch accounting: every kernel launch of the library goes through
// count_launch so sd_kernel_launches can report how many ran.
void count_launch(long long n = 1);
long long launches();

inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Stage launchers (defined in the .cu files). All return SD_OK or SD_E_*.
int launch_cell_keys(const float4* pos, int n, int G, int order, uint32_t* keys, cudaStream_t s);
size_t sort_workspace_bytes(int n);
int launch_sort_pairs(const uint32_t* keys_in, const int32_t* vals_in, uint32_t* keys_out, int32_t* vals_out,
                      uint32_t* keys_tmp, int32_t* vals_tmp, int n, int key_bits, void* ws, size_t ws_bytes,
                      cudaStream_t s, bool ws_zeroed = false, bool first_counts_ready = false,
                      const int* n_dev = nullptr);
// n_dev: the key count lives in device memory (made by an earlier kernel); n is
// then the capacity the grids are sized for, and keys past the count are ignored.
// ws_zeroed: the workspace's count buffers are zero, as every sort leaves them.
// first_counts_ready: the first digit pass's tile counts are already in the
// workspace (launch_sort_first_counts, or added by the gather that wrote the keys).
constexpr int kSortTileShift = 11;   // sort tiles of 2048 keys
constexpr int kSortChunkShift = 6;   // the column scan sums chunks of 64 tiles
int sort_digit_bits(int key_bits);  // digit width of the passes (0: no pass)
unsigned* sort_first_counts(void* ws);  // tile-major counts[tile][1 << digit bits] of the first pass
int launch_sort_first_counts(const uint32_t* keys, int n, int key_bits, void* ws, size_t ws_bytes, cudaStream_t s);
int launch_reorder(const float4* pos_in, const float4* vel_in, const int32_t* perm, float4* pos_out,
                   float4* vel_out, int n, cudaStream_t s);

size_t deposit_workspace_bytes(int G);
// periodic = 0: corners past the edge are clamped onto the edge cells (isolated boundary)
int launch_deposit_fixed(const float4* pos, int n, int G, long long* acc, cudaStream_t s, int periodic = 1);
int launch_clear_u64(long long* a, size_t n, cudaStream_t s);
int launch_fixed_to_float(const long long* acc, int G, float* rho, int clear, cudaStream_t s);

// Poisson plan: twiddles and Green's tables for one grid size (device memory).
struct PoissonPlan {
    int G = 0;
    float soft = -1.f;
    float2* tw = nullptr;    // W_G^m = exp(-2 pi i m / G), m < G (FP64-built, rounded)
    float* gexp = nullptr;   // exp(-(2 pi soft / G)^2 k^2 / 2), k = 0..G/2 (FP64-built)
    float scale = 0.f;       // 1 / (4 pi^2 G^3)
};
int poisson_plan_build(PoissonPlan& p, int G, float soft);
void poisson_plan_free(PoissonPlan& p);
size_t poisson_spectrum_elems(int G);  // complex elements of the (bricked, padded) spectrum buffer
// rho_fixed != nullptr: the first pass reads the int64 fixed-point grid and
// zeroes it; otherwise it reads rho_float. rho_keep (optional) receives the
// float density. The spectrum buffer is transformed in place.
int launch_poisson(const PoissonPlan& p, const long long* rho_fixed, const float* rho_float, float* rho_keep,
                   float2* spec, float* phi, cudaStream_t s);
// pos != nullptr: the first pass deposits the particles itself (SD_ORDER_TILED
// order, row_start from launch_row_bounds) instead of reading a density grid.
// ev (optional): 4 events recorded after passes A, B, C and D.
// Isolated-boundary options of the Poisson solve (Hockney-Eastwood, kGreen/kMulSpec,
// Sim.cu:563-584): the density has side src_g inside the 2 src_g transform box;
// table is the real Green spectrum (green_table_elems floats), applied with
// table_scale; forward_only stops after the forward transform (table build).
struct PoissonIso {
    int src_g = 0;
    const float* table = nullptr;
    float table_scale = 0.f;
    bool forward_only = false;
};
// Work plan of the fused deposit (pos != nullptr). A row bundle's CTA reads the
// particles of the 25 base rows whose stencils reach its 16 rows; a bundle whose
// window holds more than `split` particles is shared by several CTAs, which add
// their exact int64 partial rows into `acc` (the fixed-point grid, zero between
// uses) and the last of them to finish transforms the rows. `ints` is scratch of
// deposit_work_ints(G) ints, zeroed once when allocated and left zero by every use.
struct DepositWork {
    long long* acc = nullptr;
    int* ints = nullptr;
    int split = 0;
};
size_t deposit_work_ints(int G);
// the particles per CTA above which a window is split: mult times a window's mean count
// (mult 0: 10 where the grid has at least 1024 row bundles, 5 below)
int deposit_split(int n, int G, int mult = 0);
int launch_poisson_ex(const PoissonPlan& p, const long long* acc, const float* rho, const float4* pos,
                      const int* perm, const int* row_start, float* keep, float2* spec, float* phi, cudaStream_t s,
                      cudaEvent_t* ev = nullptr, const PoissonIso* iso = nullptr, const DepositWork* dw = nullptr);
size_t green_table_elems(int S);
// Green spectrum of the isolated boundary on an S^3 transform box (plan of size S);
// kernel_grid (S^3 floats) and spec are scratch.
int build_green_table(const PoissonPlan& p, float softening_cells, float* kernel_grid, float2* spec, float* table,
                      cudaStream_t s);
// row_start[r] = first index i with sorted row keys[i] >= r, for r in [0, rows]
int launch_row_bounds(const uint32_t* keys, int n, int rows, int* row_start, cudaStream_t s);

size_t gather_partials(int n);
// one-time per-device set-up of the gather's default grid (call outside stream capture)
int gather_prepare(int device);
// perm != nullptr: slot i takes input particle perm[i] (fused reorder) and the
// outputs must be separate arrays; otherwise pos_out/vel_out may alias the inputs.
// keys_out (optional) receives the next step's order keys (key + 1).
// extra (optional) is an acceleration added to the PM one, indexed like the outputs.
// max_blocks > 0 caps the grid (grid-stride loop); partials need gather_partials(n) blocks.
// diag (optional): per-step FP64 energy/momentum record appended to a device ring
// of `cap` records of 8 doubles; count is a device counter of records written.
struct DiagRecord {
    double* rec = nullptr;
    unsigned long long* count = nullptr;
    int cap = 0;
    double mass = 0.0;  // particle mass, 1/N
};
int launch_gather_kick_drift(const float* phi, int G, float pot_scale, const float4* pos_in, const float4* vel_in,
                             const int* perm, float4* pos_out, float4* vel_out, uint32_t* keys_out, int order, int n,
                             float dt_kick, float dt_drift, float c2, const float* mean_vel, double* partials,
                             double* mom_out, float* mean_out, cudaStream_t s, const float4* extra = nullptr,
                             int max_blocks = 0, const DiagRecord* diag = nullptr, int iso_S = 0,
                             unsigned* tile_counts = nullptr, int count_bits = 0, const float4* press = nullptr,
                             unsigned* chg_words = nullptr);
// chg_words: zeroed change bits (one per output) for the next step's merge sort
// (sd_resort.cu); a bit is set where the key written differs from the key of the
// step-start position.
// tile_counts: zeroed first-pass sort counts; the gather adds the digit (low
// count_bits bits) of every key it writes to the row of the key's sort tile.
// iso_S > 0: isolated boundary, potential box of side iso_S (= 2G), clamped sampling
int launch_interpolate_accel(const float* phi, int G, float pot_scale, const float4* pos, float4* acc, int n,
                             cudaStream_t s, const float4* extra = nullptr, int iso_S = 0);
// learned correction (sd_mlp.cu): out[i] = out_scale * MLP(features of pos[perm ? perm[i] : i])
size_t mlp_param_count();
int launch_mlp_infer(const float* params, const float4* pos, const int* perm, int n, const float* rho, int G,
                     float inv_mean, float out_scale, float4* out, cudaStream_t s);
int launch_apply_mean(float4* vel, const float4* pos, int n, const float* mean_vel, cudaStream_t s);
int launch_max_speed(const float4* pos, const float4* vel, int n, const float* mean_vel, float* out,
                     cudaStream_t s);
int launch_energy(const float* phi, int G, const float4* pos, const float4* vel, int n, const float* mean_vel,
                  double* partials, double* out8, cudaStream_t s, int iso_S = 0);
// op 0: sum, 1: max, 2: cells above 1e-6 (kCountOccupied, Sim.cu:2727-2730); fixed summation order
int launch_reduce_grid(const float* rho, size_t cells, int op, double* partials, double* out, cudaStream_t s);
// out[0..2] = sum x, sum y and count of the live particles (kCentroidAccum, Sim.cu:2733-2741),
// in a fixed summation order
int launch_centroid(const float4* pos, int n, double* partials, double* out3, cudaStream_t s);
// The step's sort as a merge of the unchanged and the changed keys (sd_resort.cu).
struct ResortBufs {
    unsigned* words = nullptr;      // change bits, one per position (zero between uses)
    unsigned* word_pre = nullptr;   // changed positions before each word
    unsigned* chunk_cnt = nullptr;  // changed positions per chunk of words
    int* c_rows = nullptr;          // row table of the sorted changed keys
    int* n_changed = nullptr;
    // the changed keys and positions, compacted, then radix-sorted (capacity n each)
    uint32_t *ck_in = nullptr, *ck_out = nullptr, *ck_tmp = nullptr;
    int32_t *ci_in = nullptr, *ci_out = nullptr, *ci_tmp = nullptr;
};
size_t resort_bytes(int n, int G);
size_t resort_words(int n);  // entries of the change-bit buffer (padded; the padding stays zero)
// Lays out resort_bytes(n, G) at base; ck_in, ci_in and ck_tmp are the three
// spare arrays of n entries given (scratch of the full sort, idle during a merge).
ResortBufs resort_layout(void* base, int n, int G, uint32_t* spare_k0, int32_t* spare_v0, uint32_t* spare_k1);
// keys: the new key of every position, positions sorted by their old keys, whose
// row table is row_start; writes the stable sort's permutation to vals_out and
// the new keys' row table over row_start.
int launch_resort(const ResortBufs& r, const uint32_t* keys, int n, int G, int key_bits, int* row_start,
                  int32_t* vals_out, void* sort_ws, size_t sort_ws_bytes, cudaStream_t s);

// Grid hydrodynamics add-ons (sd_hydro.cu): per-cell fixed-point sums for cooling
// and the velocity dispersion, and the pressure acceleration grid (G^3 each).
struct HydroGrids {
    void* base = nullptr;
    float4* acc = nullptr;              // pressure acceleration
    long long* vsum[3] = {nullptr, nullptr, nullptr};
    long long* disp[3] = {nullptr, nullptr, nullptr};
    unsigned* cnt = nullptr;            // members of each cell
    unsigned* dcnt = nullptr;           // members that entered the dispersion
    int G = 0;
};
size_t hydro_bytes(int G);
int hydro_alloc(HydroGrids& h, int G);
void hydro_free(HydroGrids& h);
int launch_pressure(const HydroGrids& h, int periodic, float pressure_k, cudaStream_t s);
int launch_cooling(const HydroGrids& h, const float4* pos, float4* vel, int n, const float* mean, float rate,
                   float dt, bool pressure, cudaStream_t s);

// Sim::reset's placement (sd_scene.cu): preset, initial velocities, centre-of-mass stop.
int launch_place_preset(float4* pos, float4* vel, int n, const sd_config& cfg, double* partials, double* out8,
                        float* mean, cudaStream_t s);
int launch_hide_range(float4* pos, float4* vel, int from, int to, cudaStream_t s);

}  // namespace sd

#define SD_CUDA(x) ::sd::check_cuda((x), #x, __FILE__, __LINE__)
#define SD_LAUNCHED(s)                                                        \
    do {                                                                      \
        ::sd::count_launch();                                                 \
        cudaError_t e_ = cudaGetLastError();                                  \
        if (e_ != cudaSuccess) return ::sd::check_cuda(e_, "launch", __FILE__, __LINE__); \
    } while (0)
