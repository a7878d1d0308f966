/*
 * stardust_pm.h -- C ABI of the B200 particle-mesh gravity step.
 *
 * This is the drop-in boundary for the reference's PM path. The reference
 * (chdnl0420-svg/stardust) exposes it as the C++ class `Sim`
 * (src/sim/Sim.h:854-1135), a Pimpl that owns every device buffer. This header
 * restates the same operations as plain C: an opaque handle, POD config,
 * plain pointers and sizes, integer status codes. No CUDA or torch types appear
 * in any signature; streams are passed as `void*` (a cudaStream_t).
 *
 * Error convention (reference: sticky g_failed / g_failMsg, Sim.cu:52-75). Every
 * call returns SD_OK (0) or a negative SD_E* code. The first failure is recorded
 * process-wide (sd_failed / sd_last_error); unlike the reference, later calls are
 * not silently skipped: they still validate and run, so one bad call does not
 * poison unrelated handles. A CUDA error inside a kernel launch marks the handle
 * failed and its later step calls return SD_E_CUDA.
 *
 * Units: positions in box units [0,1), periodic box of side 1. Densities are in
 * count units (each particle deposits total weight 1), as in the reference.
 */
#ifndef STARDUST_PM_H
#define STARDUST_PM_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 2: sd_config carries the initial conditions (preset, ...), which sd_init /
 * sd_reset lay down as the reference's init / reset do, and the hydro add-ons;
 * it grew to 32 words. */
#define SD_ABI_VERSION 2

/* ---- status codes ---------------------------------------------------------- */
enum {
    SD_OK = 0,
    SD_E_ARG = -1,        /* invalid argument (null pointer, bad size, bad enum) */
    SD_E_CUDA = -2,       /* a CUDA runtime call or kernel failed */
    SD_E_NOMEM = -3,      /* device allocation failed / does not fit */
    SD_E_STATE = -4,      /* call not valid in the current state (e.g. not initialised) */
    SD_E_IO = -5,         /* state file could not be read or written */
    SD_E_FORMAT = -6,     /* state file is not a valid STARDUST v1/v2 file */
    SD_E_UNSUPPORTED = -7 /* configuration this build does not implement */
};

/* ---- enums ----------------------------------------------------------------- */
/* Boundary (Sim.h:20 `enum class Boundary { Isolated, Periodic }`). */
enum { SD_BOUNDARY_ISOLATED = 0, SD_BOUNDARY_PERIODIC = 1 };

/* Particle order used by the sort (Sim.cu:2476-2486 is SD_ORDER_ROWMAJOR). */
enum {
    SD_ORDER_ROWMAJOR = 0, /* reference key: (cz*G+cy)*G+cx of the containing cell */
    SD_ORDER_MORTON = 1,   /* 30-bit Morton code of the containing cell */
    SD_ORDER_TILED = 2     /* CIC base-cell rows in 4x4 row tiles (fused deposit/gather) */
};

/* Time integrator. SD_INT_KD is the reference's kick-then-drift
 * (kIntegrate Sim.cu:822,842). SD_INT_KDK is leapfrog: the first step opens
 * with a half kick, later steps kick by (dt_prev + dt)/2, and sd_synchronize
 * closes with the last half kick. */
enum { SD_INT_KD = 0, SD_INT_KDK = 1 };

/* Force units. SD_UNITS_REFERENCE: a = -(gravity/N) grad(phi), lap(phi) = counts
 * (Sim.cu:3107-3109, 528-557). SD_UNITS_NEWTON: Newtonian gravity with
 * G_N = gravity and total mass 1 (each particle 1/N), i.e. the reference
 * formula scaled by 4*pi*G^3. */
enum { SD_UNITS_REFERENCE = 0, SD_UNITS_NEWTON = 1 };

/* Memory side of a pointer argument. */
enum { SD_HOST = 0, SD_DEVICE = 1 };

/* ---- configuration (SimConfig, Sim.h:157-796; plain-PM fields) ------------- */
typedef struct sd_config {
    int32_t particle_count;   /* SimConfig::particleCount (Sim.h:166) */
    int32_t grid_size;        /* SimConfig::gridSize (Sim.h:167); clamped to a power of two in [16,512] */
    int32_t boundary;         /* SimConfig::boundary (Sim.h:278) */
    float gravity;            /* SimConfig::gravity (Sim.h:280) */
    float softening_cells;    /* SimConfig::softeningCells (Sim.h:315), Gaussian in k for periodic */
    float time_scale;         /* SimConfig::timeScale (Sim.h:316): sd_step_auto dt = 0.0016*dtScaleFor(ts) */
    int32_t sort_interval;    /* SimConfig::sortInterval (Sim.h:317); 0 = never sort */
    float length_scale;       /* SimConfig::lengthScale (Sim.h:172), light-speed clamp */
    float time_unit_scale;    /* SimConfig::timeUnitScale (Sim.h:180), light-speed clamp */
    int32_t order;            /* SD_ORDER_* */
    int32_t integrator;       /* SD_INT_* */
    int32_t units;            /* SD_UNITS_* */
    int32_t diagnostics;      /* 1 = FP64 energy and momentum of every step (sd_diagnostics_history) */
    int32_t keep_density;     /* 1 = keep the step-start density for sd_density_device_ptr (4 B/cell more traffic) */
    /* Initial conditions laid down by sd_init (structural changes) and sd_reset
     * (Sim::reset, Sim.cu:4160-4238). */
    int32_t preset;              /* SimConfig::preset (Sim.h:277): SD_PRESET_FILAMENT (default) or SD_PRESET_EMPTY */
    float dark_matter_fraction;  /* SimConfig::darkMatterFraction (Sim.h:536): hashed share with vel.w = -100 */
    float big_bang_shrink;       /* SimConfig::bigBangShrink (Sim.h:214): Filament ball scaled about the centre if > 0 */
    float spin;                  /* SimConfig::spin (Sim.h:766): rigid rotation about z, v += spin * (-dy, dx, 0) */
    float hubble;                /* SimConfig::hubble (Sim.h:196): radial flow, v += hubble * (p - 0.5) */
    float vel_dispersion;        /* SimConfig::velDispersion (Sim.h:263): isotropic random speed of mean size */
    /* Grid hydrodynamics add-ons (doCooling / kPressure, Sim.cu:3605-3868). The
     * reference enables both by default; here they are off unless set, as the PM
     * path is the product. A cooling step runs every 2 steps with pressure, every
     * 8 without (then sd_steps runs eagerly and ensembles reject the scene). */
    int32_t pressure_enabled;    /* SimConfig::pressureEnabled (Sim.h:319) */
    float pressure_k;            /* SimConfig::pressureK (Sim.h:320), default 0.45 */
    int32_t cooling_enabled;     /* SimConfig::coolingEnabled (Sim.h:327) */
    float cooling_rate;          /* SimConfig::coolingRate (Sim.h:345), default 0.08 */
    int32_t full_sort;           /* the sort of a step after a sorted step (tiled order, periodic):
                                    1 always the full radix sort; 0 (default) a merge of the keys that
                                    changed into the rest for 2^22 particles or more while at most 10 %
                                    change, else the full sort; -1 the merge whenever possible.
                                    Every choice gives the same permutation. */
    int32_t reserved[7];
} sd_config;

/* SimConfig::preset (Preset, Sim.h:14-17) */
enum { SD_PRESET_FILAMENT = 0, SD_PRESET_EMPTY = 1 };

/* Per-step timings (SimTimings, Sim.h:844-852), milliseconds of device time. */
typedef struct sd_timings {
    float sort_ms;     /* key + radix sort + reorder */
    float deposit_ms;  /* CIC deposit (+ the first FFT pass where fused) */
    float poisson_ms;  /* FFT passes and Green's function */
    float gather_ms;   /* gather + kick + drift */
    float total_ms;
    float dt_used;
    float max_speed;
    int32_t steps;     /* steps covered by these numbers */
    /* per-kernel device time of the last eager step: [0] keys + sort,
     * [1] row table or atomic deposit, [2] pass A (fused deposit + x real FFT),
     * [3] pass B (y forward), [4] pass C (z forward, Green's function, z
     * inverse), [5] pass D (y inverse), [6] pass E (x complex-to-real),
     * [7] gather + kick + drift (+ momentum sums) */
    float kernel_ms[8];
} sd_timings;

/* FP64 diagnostics of the last step (computed on the device). */
typedef struct sd_diagnostics {
    double kinetic;      /* sum 1/2 m v^2, m = 1/N (after momentum zeroing) */
    double potential;    /* 1/2 sum m phi(x_i), phi in the configured units */
    double momentum[3];  /* sum m v (after zeroing: ~0) */
    double mean_velocity_removed[3];
    double live_count;
} sd_diagnostics;

typedef struct sd_sim sd_sim;  /* opaque; the reference's Sim::Impl */

/* ---- process-level --------------------------------------------------------- */
int sd_abi_version(void);
/* Sim::deviceAvailable (Sim.cu:3903-3906). Returns 1 when a CUDA device exists. */
int sd_device_available(void);
/* Sim::failed / Sim::failMessage (Sim.h:994-995). */
int sd_failed(void);
const char* sd_last_error(void);
void sd_clear_error(void);
/* Default config: the reference's SimConfig defaults for the plain-PM fields
 * (boundary periodic, gravity 1, sortInterval 1, softening 3 cells). */
int sd_config_default(sd_config* cfg);
/* Sim::maxGridSize (Sim.cu:4158): 256 isolated, 512 periodic. */
int sd_max_grid_size(int boundary);
/* Sim::estimateBytes (Sim.cu:3935-3998), for this implementation's buffers. */
size_t sd_estimate_bytes(int particle_count, int grid_size, int boundary);
/* Sim::maxParticlesFor (Sim.cu:4057-4066): the most particles a grid leaves room
 * for in free_bytes of device memory. The grid's buffers come first; 80 % of the
 * rest holds particles, at this implementation's bytes per particle. 0 when the
 * grid alone does not fit. At most 400,000,000 (the largest particle_count). */
int sd_max_particles_for(int grid_size, int boundary, size_t free_bytes);
/* Sim::estimateStepMs (Sim.cu:4022-4055): a step's time from this build's byte
 * model (184 B per particle + 40 B per transform-box cell) at 55 % of the device's
 * memory bandwidth, plus launch overhead. 0 without a device. Particles crowded
 * into a few rows cost more than the model says. */
double sd_estimate_step_ms(int particle_count, int grid_size, int boundary);
/* Sim::deviceFreeBytes (Sim.cu:3921-3925): cudaMemGetInfo's free bytes of the
 * current device, or the override below. 0 without a device. */
size_t sd_device_free_bytes(void);
/* Testing aid (no reference counterpart): when bytes > 0, sd_device_free_bytes and
 * the VRAM clamp of sd_init / sd_reconfigure see this many free bytes instead of
 * the device's; 0 restores the real query. Process-wide. */
void sd_set_device_free_bytes_override(size_t bytes);
/* Sim::deviceBandwidthGBs (Sim.cu:4003-4012): memory clock x bus width x 2, GB/s. */
double sd_device_bandwidth_gbs(void);
/* Sim::deviceMultiProcessors (Sim.cu:3926-3930). */
int sd_device_multiprocessors(void);
/* Sim::deviceName / deviceDriver (Sim.cu:3907-3920): the current device's name
 * ("unknown" without one) and the CUDA version its driver supports ("CUDA 12.9";
 * empty without a driver), NUL-terminated into out[capacity]. */
int sd_device_name(char* out, int capacity);
int sd_device_driver(char* out, int capacity);

/* ---- lifetime (Sim::Sim / ~Sim, Sim.cu:3900-3901) --------------------------- */
int sd_create(sd_sim** out, int device);
int sd_destroy(sd_sim* sim);
/* Stream for all work of this handle (default: a stream the handle creates). */
int sd_set_stream(sd_sim* sim, void* cuda_stream);

/* ---- configuration (Sim::init / reconfigure / reset, Sim.cu:4068-4238) ------ */
/* Sim::init / Sim::reconfigure (Sim.cu:4068-4152). A request is structural when
 * its particle_count, grid_size (after clamping to a power of two) or boundary
 * differs from the last structural request; repeating a request changes nothing.
 * A structural request with the same grid and boundary and no more particles than
 * the kernels run over only narrows that range: no reallocation, particles and
 * simulation time stay (the reference's shrink-only path, Sim.cu:4108-4116).
 * Other structural requests clamp particle_count to what the device's free memory
 * holds (sd_max_particles_for; Sim.cu:4123-4134), reallocate and lay down the
 * preset; SD_E_NOMEM, with nothing changed, when the grid alone does not fit.
 * sd_init always reallocates. Other fields apply in place. */
int sd_init(sd_sim* sim, const sd_config* cfg);
int sd_reconfigure(sd_sim* sim, const sd_config* cfg);
/* Sim::reset (Sim.cu:4160-4238): zero time and step count and lay down the
 * configured preset -- kPlace's Filament ball (Sim.cu:281-407; all slots live)
 * or Empty (all slots empty but a dark-matter halo, active count 0) -- then
 * spin, Hubble flow and velocity dispersion, then stop the centre of mass
 * (Filament only, as the reference divides by the active count). sd_init and
 * structural sd_reconfigure calls do the same, as the reference's init does.
 * Other scenes are loaded with sd_set_particles / sd_load_state. */
int sd_reset(sd_sim* sim);
int sd_get_config(const sd_sim* sim, sd_config* out);

/* ---- particle buffers (Sim::loadState's upload path, Sim.cu:5096-5101; ------
 * particlePosDevicePtr / particleVelDevicePtr, Sim.h:1128-1129).
 * pos, vel: float4[n] (x,y,z,w). n <= particle_count; slots >= n become empty.
 * `where` is SD_HOST or SD_DEVICE. */
int sd_set_particles(sd_sim* sim, const float* pos, const float* vel, int n, int where);
int sd_get_particles(sd_sim* sim, float* pos, float* vel, int n, int where);
/* Device pointers (float4 arrays as float*), valid until the next step or
 * reconfigure. Pending momentum corrections are applied first. */
const float* sd_particle_pos_device_ptr(sd_sim* sim);
const float* sd_particle_vel_device_ptr(sd_sim* sim);
/* Density of the step-start positions of the last step (Sim::densityDevicePtr,
 * Sim.h:1082), G^3 floats z-major. */
const float* sd_density_device_ptr(sd_sim* sim);
int sd_get_density(sd_sim* sim, float* out, int where);
/* Potential of the last force solve, G^3 floats z-major, configured units. */
int sd_get_potential(sd_sim* sim, float* out, int where);
/* Accelerations the current positions would receive (solves the field for the
 * current positions without moving particles): float4[n], w = 0. */
int sd_get_accel(sd_sim* sim, float* out, int n, int where);

/* ---- stepping (Sim::step, Sim.cu:4240-4525) -------------------------------- */
/* Advance by exactly dt (no CFL clamp). */
int sd_step(sd_sim* sim, float dt);
/* The reference's step(): dt = 0.0016*dtScaleFor(time_scale) clamped to
 * 0.8*cell/vmax (Sim.cu:4255-4269); blocks for the vmax read like the reference. */
int sd_step_auto(sd_sim* sim);
/* One offload step on host buffers: the same as sd_set_particles(pos_in, vel_in,
 * n, SD_HOST) + sd_step(dt) + sd_get_particles(pos_out, vel_out, n, SD_HOST), with
 * the velocity upload overlapping the sort, deposit and Poisson solve and the
 * position download overlapping the momentum correction. Synchronous: returns
 * when the outputs are written. Use pinned host memory for full copy speed. */
int sd_step_host(sd_sim* sim, const float* pos_in, const float* vel_in, int n, float dt, float* pos_out,
                 float* vel_out);
/* The same offload step, pipelined (no reference counterpart): the call queues
 * the upload, the step and the download and returns. Consecutive calls overlap
 * one step's download, the next step's computation and the upload after it (both
 * copy directions at once), through a third particle set the handle allocates on
 * the first call (32 bytes per slot). The outputs of the queued calls are complete
 * when sd_step_host_wait returns; until then the caller leaves pos_in and vel_in
 * unchanged and does not read pos_out or vel_out. Every other call on the handle
 * first waits for the queued ones. Each call's result is the same as
 * sd_step_host's on the same inputs. Use pinned host memory. */
int sd_step_host_async(sd_sim* sim, const float* pos_in, const float* vel_in, int n, float dt, float* pos_out,
                       float* vel_out);
int sd_step_host_wait(sd_sim* sim);
/* nsteps fixed-dt steps; replays a captured CUDA graph after the first call. */
int sd_steps(sd_sim* sim, float dt, int nsteps);
/* Leapfrog: apply the closing half kick so velocities are synchronous with
 * positions (no-op for SD_INT_KD). */
int sd_synchronize(sd_sim* sim);
/* Sort and reorder only (sortParticles, Sim.cu:3656-3671). perm (optional,
 * int32[n]) receives, for each new slot, the old slot it came from. */
int sd_sort_only(sd_sim* sim, int32_t* perm, int where);

/* ---- state (Sim::saveState / loadState, Sim.cu:4985-5120; STARDUST v2) ------- */
int sd_save_state(sd_sim* sim, const char* path);
int sd_load_state(sd_sim* sim, const char* path);

/* ---- queries and measurements ----------------------------------------------- */
int sd_timings_get(const sd_sim* sim, sd_timings* out);             /* Sim::timings */
double sd_sim_time(const sd_sim* sim);                              /* Sim::simTime */
int sd_grid_size(const sd_sim* sim);                                /* Sim::gridSize */
int sd_particle_count(const sd_sim* sim);                           /* Sim::particleCount: slots the kernels run over (allocN) */
int sd_particle_capacity(const sd_sim* sim);                        /* slots allocated (capacityN, Sim.cu:3032-3045) */
int sd_active_count(const sd_sim* sim);                             /* Sim::activeCount */
int sd_step_count(const sd_sim* sim);
/* The merge sort (tiled order, periodic; no reference counterpart) measures the
 * share of particles whose row key changed since the last sorted step. With
 * full_sort = 0, above 10 % (or below 2^22 particles) the steps run the full radix
 * sort instead (the same permutation), with one probing merge every 64 steps.
 * sd_changed_fraction: the last measured share (-1 before the first merge);
 * sd_merge_sorting: 1 while merges are chosen. */
double sd_changed_fraction(const sd_sim* sim);
int sd_merge_sorting(const sd_sim* sim);
double sd_measure_total_grid_mass(sd_sim* sim);                     /* Sim.cu:4890-4906 */
double sd_measure_max_density(sd_sim* sim);                         /* Sim.cu:4908-4924 */
double sd_measure_kinetic_energy(sd_sim* sim);                      /* Sim.cu:5141-5149 */
/* Sim::measureOccupiedCells (Sim.cu:4926-4935): density cells above 1e-6 (needs keep_density) */
int sd_measure_occupied_cells(sd_sim* sim);
/* Sim::measureCentroid (Sim.cu:4937-4950): mean x and y of the live particles, in
 * FP64 with a fixed summation order; 0.5, 0.5 when none is live. */
int sd_measure_centroid(sd_sim* sim, double* cx, double* cy);
int sd_diagnostics_get(sd_sim* sim, sd_diagnostics* out);
/* Per-step FP64 records of the steps taken with diagnostics = 1 (accumulated
 * inside the gather, no extra pass; kept in a device ring of the last 4096
 * steps; also inside sd_steps graphs). Copies the most recent min(max_records,
 * available) records, oldest first, 8 doubles each:
 *   {record index, kinetic, potential, momentum x, y, z, live count, |mean velocity removed|}
 * kinetic = sum 1/2 m |v|^2 of the step's zeroed end velocities; potential =
 * 1/2 sum m phi(x) at the step-start positions with the step's potential. */
int sd_diagnostics_history(sd_sim* sim, double* out, int max_records, int* count_out);
/* Number of kernel launches the handle issued since creation. */
long long sd_kernel_launches(const sd_sim* sim);

/* ---- stage entry points on caller buffers (device pointers) ----------------
 * Each runs one stage of the step on `stream` with caller-owned memory, so the
 * stages can be checked one at a time. Workspace sizes come from the *_bytes
 * queries; workspaces must be 256-byte aligned. */

/* kCellKey (Sim.cu:2476-2486) for order SD_ORDER_ROWMAJOR / SD_ORDER_MORTON:
 * keys_plus1[i] = key + 1 (empty slot -> 0), so an unsigned sort puts empty slots
 * first as CUB does with the reference's signed -1. SD_ORDER_TILED (no reference
 * counterpart): keys_plus1[i] = the row index of the CIC base cell in 4x4 row
 * tiles, (tile_z * G/4 + tile_y) * 16 + (iz & 3) * 4 + (iy & 3), in log2(G^2)
 * bits; empty slots get 0 and share row 0. */
int sd_cell_keys(const float* pos, int n, int grid_size, int order, uint32_t* keys_plus1, void* stream);
/* Bits a stable sort of keys_plus1 must cover for this grid and order. */
int sd_key_bits(int grid_size, int order);
/* Stable LSD radix sort of (keys, vals) over the low key_bits bits
 * (cub::DeviceRadixSort::SortPairs, Sim.cu:3659-3667). vals_in == NULL means
 * the identity 0..n-1. Results land in keys_out / vals_out; keys_tmp / vals_tmp
 * are ping-pong buffers of n entries; workspace from sd_sort_workspace_bytes. */
size_t sd_sort_workspace_bytes(int n);
int sd_sort_pairs(const uint32_t* keys_in, const int32_t* vals_in, uint32_t* keys_out, int32_t* vals_out,
                  uint32_t* keys_tmp, int32_t* vals_tmp, int n, int key_bits, void* workspace,
                  size_t workspace_bytes, void* stream);
/* kReorder (Sim.cu:2488-2495): dst[i] = src[perm[i]] for float4 pos and vel. */
int sd_reorder(const float* pos_in, const float* vel_in, const int32_t* perm, float* pos_out, float* vel_out,
               int n, void* stream);
/* Deterministic CIC deposit (kScatter Sim.cu:503-521 with int64 fixed-point
 * sums): rho[G^3] in count units. workspace: sd_deposit_workspace_bytes. */
size_t sd_deposit_workspace_bytes(int grid_size);
int sd_deposit(const float* pos, int n, int grid_size, float* rho, void* workspace, size_t workspace_bytes,
               void* stream);
/* Periodic Poisson solve rho -> phi with the reference's Green's function
 * (kPoissonPeriodic Sim.cu:528-557, cuFFT R2C/C2R Sim.cu:3592,3601).
 * workspace: sd_poisson_workspace_bytes. */
size_t sd_poisson_workspace_bytes(int grid_size);
int sd_poisson(const float* rho, int grid_size, float softening_cells, float* phi, void* workspace,
               size_t workspace_bytes, void* stream);
/* The same Poisson solve for callers that cannot allocate device memory: no
 * counterpart in the reference. Some callers cannot call cudaMalloc, or be handed
 * a workspace, on this path: code inside another component's allocation-free
 * hot loop, or under a fixed memory budget that forbids growth after start-up.
 * This entry point
 * allocates nothing: its spectrum and tables live in fixed device storage of
 * the library, which every GPU that loads the library holds (about 9 MB) until
 * the process exits. grid_size must be a power of two in [16, 128]; larger
 * grids are rejected with SD_E_ARG. The first call on a device resolves that
 * storage and uploads the twiddle tables, synchronously (it waits for the
 * device). All calls on a device share the storage: calls that overlap
 * on the GPU (different streams, no ordering between them) race and give wrong
 * results. rho and phi are caller device buffers of grid_size^3 floats. */
int sd_poisson_noalloc(const float* rho, int grid_size, float softening_cells, float* phi, void* stream);
/* Gather + kick + drift (kGridAccel Sim.cu:589-611 folded into sampleAcc /
 * kIntegrate Sim.cu:614-629, 685-906). pot_scale = gravity/N. mean_vel (3
 * floats, device, may be NULL) is subtracted from each loaded velocity (the
 * deferred momentum zeroing of the previous step). mom_out (device, 4 doubles,
 * may be NULL) receives sum vx, vy, vz and the live count of the new
 * velocities, in a fixed summation order. pos and vel must be 16-byte aligned
 * (SD_E_ARG otherwise). */
int sd_gather_kick_drift(const float* phi, int grid_size, float pot_scale, float* pos, float* vel, int n,
                         float dt_kick, float dt_drift, float c2, const float* mean_vel, double* mom_out,
                         void* workspace, size_t workspace_bytes, void* stream);
size_t sd_gather_workspace_bytes(int n);
/* Per-particle accelerations from phi (the same arithmetic as the kick). */
int sd_interpolate_accel(const float* phi, int grid_size, float pot_scale, const float* pos, float* acc_out,
                         int n, void* stream);

/* ---- learned sub-grid force correction (no counterpart in the reference) ----
 * An MLP 30 -> 64 -> 64 -> 3 (SiLU) maps a particle's coarse-grid features (the
 * 3x3x3 CIC density stencil around its cell as log(1 + rho/rho_bar) - log 2, and
 * its sub-cell offset) to a residual acceleration that is added to the PM
 * acceleration before the kick. BF16 weights and activations, FP32 accumulation
 * on the tensor cores. params: FP32 vector of sd_mlp_param_count() floats
 * (W1[32][64], b1[64], W2[64][64], b2[64], W3[64][8], b3[8]). inv_mean =
 * grid_size^3 / particle count. Outputs are scaled by out_scale. */
int sd_mlp_param_count(void);
/* features (bf16[n][32]) of pos[perm[i]] (perm may be NULL) from the density rho[G^3] */
int sd_mlp_features(const float* pos, const int32_t* perm, int n, const float* rho, int grid_size, float inv_mean,
                    void* features_bf16, void* stream);
/* residual accelerations float4[n] (w = 0; empty slots get 0). Runs on the
 * 5th-generation tensor cores (tcgen05.mma, accumulators in tensor memory). */
int sd_mlp_infer(const float* params, const float* pos, const int32_t* perm, int n, const float* rho,
                 int grid_size, float inv_mean, float out_scale, float* out, void* stream);
/* Bounded waits of the inference on tensor-core completion that gave up since the
 * library was loaded on the current device (0 unless the hardware stalled; the
 * affected outputs are NaN). Synchronises the device. */
int sd_mlp_wait_timeouts(void);
/* gradient (FP32 [params]) of the mean squared error over rows and the 3 outputs
 * of one batch (rows a multiple of 16); *sse = sum of squared errors (device) */
size_t sd_mlp_train_workspace_bytes(int rows);
int sd_mlp_loss_grad(const float* params, const void* features_bf16, const float* targets, int rows, float* grad,
                     float* sse, void* workspace, size_t workspace_bytes, void* stream);
/* one Adam step on the FP32 master parameters (device arrays m, v of the same size) */
int sd_mlp_adam(float* params, float* m, float* v, const float* grad, int step, float lr, float beta1, float beta2,
                float eps, void* stream);
/* Enable (params != NULL) or disable the correction in sd_step / sd_steps of a
 * handle; params are copied. Needs keep_density (the correction reads the
 * step-start density), which this call switches on. */
int sd_set_mlp(sd_sim* sim, const float* params_device, float out_scale);

/* ---- batched ensemble (no counterpart in the reference: one Sim per scene) --
 * Independent periodic scenes of any particle count and grid size, advanced
 * together. One step of the ensemble is one CUDA graph launch: a fork, one
 * branch per scene holding that scene's whole step, a join; scenes run side by
 * side on the GPU. Scenes are ordinary sd_sim handles owned by the ensemble
 * (sd_ensemble_scene), so every per-scene query works on them. Each scene's
 * density is the same fixed-point sum as when it runs alone (bit-exact). */
typedef struct sd_ensemble sd_ensemble;
typedef struct sd_scene_tuning {
    int order;          /* SD_ORDER_TILED (fused deposit) or SD_ORDER_ROWMAJOR (atomic deposit) */
    int gather_blocks;  /* gather grid cap in CTAs (0: one CTA per 256 particles, at most 4096) */
    float step_ms;      /* median step time of the chosen variant alone; -1 before tuning */
    int deposit_split;  /* window particles per CTA share of the fused deposit (0 with the atomic deposit) */
} sd_scene_tuning;
int sd_ensemble_create(sd_ensemble** out, int device);
int sd_ensemble_destroy(sd_ensemble* ens);
/* adds a scene (sort_interval 0 or 1); returns its index or a negative status */
int sd_ensemble_add(sd_ensemble* ens, const sd_config* cfg, const float* pos, const float* vel, int n, int where);
int sd_ensemble_size(const sd_ensemble* ens);
sd_sim* sd_ensemble_scene(sd_ensemble* ens, int index);
/* times each scene's deposit path, deposit share size and gather grid on a snapshot
 * (restored) and keeps the fastest */
int sd_ensemble_autotune(sd_ensemble* ens, float dt, int reps);
int sd_ensemble_get_tuning(const sd_ensemble* ens, int index, sd_scene_tuning* out);
/* nsteps steps of every scene: one graph launch per step, no host synchronisation */
int sd_ensemble_steps(sd_ensemble* ens, float dt, int nsteps);
int sd_ensemble_synchronize(sd_ensemble* ens);
void* sd_ensemble_stream(const sd_ensemble* ens);
long long sd_ensemble_graph_kernels(const sd_ensemble* ens);

/* ---- headless point render (kSplatPoints -> kAccumToRGBA, RenderField.cu:318-735)
 * Particle buffers to an RGBA8 image in device memory (rows top-down), without
 * OpenGL. Gas particles (pos.w == 0) only; colour by density (0) or speed (2).
 * Sums are 64-bit fixed point, so an image does not depend on particle order. */
typedef struct sd_view {
    float rot[9];        /* row-major view rotation (ViewRot.m, ViewRot.h:25-31) */
    float center[3];     /* rotation centre (ViewRot.cx/cy/cz) */
    int32_t fly;         /* 1: perspective from the centre, 0: orthographic */
    float tan_half_fov;  /* perspective only */
    float zoom, pan_x, pan_y;
    float size_px;       /* particle footprint before the visibility cap */
    int32_t color_by;    /* 0 density, 2 speed */
    int32_t cmap;        /* 0 astro, 1 gray, 2 thermal, 3 black body */
    float bright, inv_gamma;
    int32_t use_cmap;    /* 1: accumulated brightness through the colour map */
    int32_t reinhard;    /* 1: x / (1 + x) tone curve when use_cmap is 0 */
    int32_t rot_on;      /* ViewRot.on: grid views project through rot (0: straight down z) */
    int32_t reserved[3];
} sd_view;
void sd_view_default(sd_view* view); /* top-down, zoom 1, density, astro map */
size_t sd_render_workspace_bytes(int width, int height);
/* pos, vel: device float4[n]; rgba_out: device uchar4[width * height] */
int sd_render_points(const float* pos, const float* vel, int n, const sd_view* view, int width, int height,
                     void* workspace, size_t workspace_bytes, void* rgba_out, void* stream);
/* Grid view of a field (Sim::fieldDevicePtr, Sim.cu:5229-5296, drawn by kShade,
 * RenderField.cu:158-316): SD_FIELD_DENSITY projects the density grid
 * (device float[G^3], z-major) along z -- or through view->rot when
 * view->rot_on -- and scales brightness by the value 5 % from the top of its
 * log histogram (n / G^2 when empty); SD_FIELD_DISPERSION is the rms speed of
 * the particles (device float4[n]) under each screen cell. Zoom, pan, bright,
 * inv_gamma and cmap come from view; rows are bottom-up like the points image. */
enum { SD_FIELD_DENSITY = 0, SD_FIELD_DISPERSION = 1 };
size_t sd_render_field_workspace_bytes(int grid_size);
int sd_render_field(int field, const float* density, int grid_size, const float* pos, const float* vel, int n,
                    const sd_view* view, int width, int height, void* workspace, size_t workspace_bytes,
                    void* rgba_out, void* stream);

/* ---- FP64 reference forces (force-error reference; not on the step) ------------
 * Periodic Newtonian accelerations (G = 1, each source of mass 1/n_src, mean
 * density removed) of Gaussian-smoothed masses of width `softening` (box units;
 * the PM step's softening_cells / grid_size), by Ewald summation in FP64:
 * structure factors over modes 0 < |n| <= nmax and the erf-difference pair
 * kernel over all sources at their nearest image. split_b is the Ewald
 * smoothing length (b^2 > 2 softening^2, b <= 0.1); choose nmax >= 1.75 / split_b
 * so the dropped modes carry weights below 1e-12. acc_out: double[3 * n_tgt], device.
 * The reference has no force-accuracy code (its test was deleted); the metric
 * is .drive/nbody-simulator/method-search/scoring.md:38. Synchronises `stream`. */
int sd_ewald_modes(int nmax);
size_t sd_ewald_workspace_bytes(int nmax);
int sd_ewald_forces(const float* src, int n_src, const float* tgt, int n_tgt, double softening, double split_b,
                    int nmax, double* acc_out, void* workspace, size_t workspace_bytes, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* STARDUST_PM_H */
