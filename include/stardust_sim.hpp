// stardust_sim.hpp -- header-only C++ facade over the C ABI (stardust_pm.h) with
// the public surface of the reference's `class Sim` for the particle-mesh path
// (src/sim/Sim.h:854-1135), so App-style callers keep their code: the same class
// and method names, the same SimConfig field names for the PM fields, the same
// SimTimings fields, no exceptions, and a sticky process-wide failure flag
// (Sim::failed / Sim::failMessage, Sim.cu:52-75).
//
// What the reference has and this facade does not: shapes, gas physics, stars,
// black holes (not part of the PM path). init/reset lay down the Filament or
// Empty preset as the reference's do; other scenes are loaded with setParticles
// (host float4 arrays) or loadState (STARDUST v1/v2 files).
//
// Link with -lstardust_pm (stardust_b200/libstardust_pm.so).
#pragma once

#include <cstddef>
#include <string>

#include "stardust_pm.h"

namespace stardust {

enum class Boundary { Isolated = SD_BOUNDARY_ISOLATED, Periodic = SD_BOUNDARY_PERIODIC };
enum class Preset { Filament = SD_PRESET_FILAMENT, Empty = SD_PRESET_EMPTY };  // Sim.h:14-17

// The plain-PM fields of the reference's SimConfig (Sim.h:157-796), with its
// defaults, plus this build's options.
struct SimConfig {
    int particleCount = 2000000;       // Sim.h:166
    int gridSize = 128;                // Sim.h:167
    Boundary boundary = Boundary::Periodic;
    float gravity = 1.0f;              // Sim.h:280
    float softeningCells = 3.0f;       // Sim.h:315
    float timeScale = 1.0f;            // Sim.h:316
    int sortInterval = 1;              // Sim.h:317
    float lengthScale = 1.0f;          // Sim.h:172
    float timeUnitScale = 1.0f;        // Sim.h:180
    Preset preset = Preset::Filament;  // Sim.h:277
    float darkMatterFraction = 0.0f;   // Sim.h:536
    float bigBangShrink = 0.0f;        // Sim.h:214
    float spin = 0.0f;                 // Sim.h:766
    float hubble = 0.0f;               // Sim.h:196
    float velDispersion = 0.0f;        // Sim.h:263
    // grid hydrodynamics (the reference's defaults are on; off here unless set)
    bool pressureEnabled = false;      // Sim.h:319
    float pressureK = 0.45f;           // Sim.h:320
    bool coolingEnabled = false;       // Sim.h:327
    float coolingRate = 0.08f;         // Sim.h:345
    // options of this build (no reference counterpart)
    int order = SD_ORDER_ROWMAJOR;     // SD_ORDER_TILED enables the fused deposit
    int integrator = SD_INT_KD;
    int units = SD_UNITS_REFERENCE;
    bool diagnostics = false;
    bool keepDensity = true;
    bool fullSort = false;             // true: no merge sort of the keys that changed (same results)

    sd_config toC() const {
        sd_config c;
        sd_config_default(&c);
        c.particle_count = particleCount;
        c.grid_size = gridSize;
        c.boundary = static_cast<int>(boundary);
        c.gravity = gravity;
        c.softening_cells = softeningCells;
        c.time_scale = timeScale;
        c.sort_interval = sortInterval;
        c.length_scale = lengthScale;
        c.time_unit_scale = timeUnitScale;
        c.order = order;
        c.integrator = integrator;
        c.units = units;
        c.diagnostics = diagnostics ? 1 : 0;
        c.keep_density = keepDensity ? 1 : 0;
        c.full_sort = fullSort ? 1 : 0;
        c.preset = static_cast<int>(preset);
        c.dark_matter_fraction = darkMatterFraction;
        c.big_bang_shrink = bigBangShrink;
        c.spin = spin;
        c.hubble = hubble;
        c.vel_dispersion = velDispersion;
        c.pressure_enabled = pressureEnabled ? 1 : 0;
        c.pressure_k = pressureK;
        c.cooling_enabled = coolingEnabled ? 1 : 0;
        c.cooling_rate = coolingRate;
        return c;
    }
};

// SimTimings (Sim.h:844-852).
struct SimTimings {
    float scatterMs = 0.0f;
    float poissonMs = 0.0f;
    float gatherMs = 0.0f;
    float totalMs = 0.0f;
    float dtUsed = 0.0f;
    float maxSpeed = 0.0f;
};

class Sim {
  public:
    Sim() { sd_create(&h_, 0); }
    explicit Sim(int device) { sd_create(&h_, device); }
    ~Sim() { sd_destroy(h_); }
    Sim(const Sim&) = delete;
    Sim& operator=(const Sim&) = delete;

    static bool deviceAvailable() { return sd_device_available() != 0; }
    static int maxGridSize(Boundary b) { return sd_max_grid_size(static_cast<int>(b)); }
    static size_t estimateBytes(int particleCount, int gridSize, Boundary b) {
        return sd_estimate_bytes(particleCount, gridSize, static_cast<int>(b));
    }
    static int maxParticlesFor(int gridSize, Boundary b, size_t freeBytes) {
        return sd_max_particles_for(gridSize, static_cast<int>(b), freeBytes);
    }
    static double estimateStepMs(int particleCount, int gridSize, Boundary b) {
        return sd_estimate_step_ms(particleCount, gridSize, static_cast<int>(b));
    }
    static size_t deviceFreeBytes() { return sd_device_free_bytes(); }
    static double deviceBandwidthGBs() { return sd_device_bandwidth_gbs(); }
    static int deviceMultiProcessors() { return sd_device_multiprocessors(); }
    static std::string deviceName() {
        char b[256];
        sd_device_name(b, (int)sizeof(b));
        return b;
    }
    static std::string deviceDriver() {
        char b[64];
        sd_device_driver(b, (int)sizeof(b));
        return b;
    }
    static bool failed() { return sd_failed() != 0; }
    static std::string failMessage() { return sd_last_error(); }

    void init(const SimConfig& cfg) {
        cfg_ = cfg;
        const sd_config c = cfg.toC();
        sd_init(h_, &c);
        sync_config();
    }
    void reconfigure(const SimConfig& cfg) {
        cfg_ = cfg;
        const sd_config c = cfg.toC();
        sd_reconfigure(h_, &c);
        sync_config();
    }
    void reset() { sd_reset(h_); }
    // Sim::step (Sim.cu:4255-4269): dt = 0.0016 * dtScaleFor(timeScale), CFL-clamped.
    void step() { sd_step_auto(h_); }
    // Fixed time step (no reference counterpart).
    void step(float dt) { sd_step(h_, dt); }
    void steps(float dt, int n) { sd_steps(h_, dt, n); }

    // Scene init: host float4 arrays (x, y, z, w), n <= particleCount.
    bool setParticles(const float* pos, const float* vel, int n) {
        return sd_set_particles(h_, pos, vel, n, SD_HOST) == SD_OK;
    }
    bool getParticles(float* pos, float* vel, int n) { return sd_get_particles(h_, pos, vel, n, SD_HOST) == SD_OK; }

    const SimConfig& config() const { return cfg_; }
    SimTimings timings() const {
        sd_timings t{};
        SimTimings o;
        if (sd_timings_get(h_, &t) != SD_OK) return o;
        o.scatterMs = t.deposit_ms;
        o.poissonMs = t.poisson_ms;
        o.gatherMs = t.gather_ms;
        o.totalMs = t.total_ms;
        o.dtUsed = t.dt_used;
        o.maxSpeed = t.max_speed;
        return o;
    }
    double simTime() const { return sd_sim_time(h_); }
    int gridSize() const { return sd_grid_size(h_); }
    int particleCount() const { return sd_particle_count(h_); }
    int activeCount() const { return sd_active_count(h_); }

    double measureTotalGridMass() { return sd_measure_total_grid_mass(h_); }
    double measureMaxDensity() { return sd_measure_max_density(h_); }
    double measureKineticEnergy() { return sd_measure_kinetic_energy(h_); }
    int measureOccupiedCells() { return sd_measure_occupied_cells(h_); }
    void measureCentroid(double& cx, double& cy) { sd_measure_centroid(h_, &cx, &cy); }

    bool saveState(const std::string& path) { return sd_save_state(h_, path.c_str()) == SD_OK; }
    bool loadState(const std::string& path) {
        const bool ok = sd_load_state(h_, path.c_str()) == SD_OK;
        if (ok) sync_config();
        return ok;
    }

    const float* densityDevicePtr() const { return sd_density_device_ptr(h_); }
    const float* particlePosDevicePtr() const { return sd_particle_pos_device_ptr(h_); }
    const float* particleVelDevicePtr() const { return sd_particle_vel_device_ptr(h_); }

    sd_sim* handle() { return h_; }

  private:
    // the library may clamp the grid (Sim.cu:4081-4086) or take N and G from a state file
    void sync_config() {
        sd_config c;
        if (sd_get_config(h_, &c) != SD_OK) return;
        cfg_.particleCount = c.particle_count;
        cfg_.gridSize = c.grid_size;
        cfg_.gravity = c.gravity;
    }

    sd_sim* h_ = nullptr;
    SimConfig cfg_;
};

}  // namespace stardust
