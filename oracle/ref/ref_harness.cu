// ref_harness.cu -- C entry points over the reference's public Sim API.
//
// TEST INFRASTRUCTURE ONLY. Linked with the unmodified reference core
// (src/sim/Sim.cu) into oracle/_ref/libsimref.so; used on a GPU box to produce
// golden fixtures and to time the reference. It touches the reference only
// through class Sim (src/sim/Sim.h:854-1135): inputs go in through a STARDUST v2
// state file and Sim::loadState (Sim.cu:5041-5120), the only public way to hand
// the reference an arbitrary particle set; outputs come back through
// particlePosDevicePtr / particleVelDevicePtr / densityDevicePtr / timings.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "Sim.h"

// src/app/Forensics.h declares these; the reference's Forensics.cpp is
// MSVC-CRT-only, so the harness provides silent versions.
namespace fx {
void begin(const char*) {}
void line(const char*, ...) {}
void mark(const char*, ...) {}
void endOk() {}
bool lastSessionCrashed() { return false; }
const char* logDir() { return "."; }
}  // namespace fx

namespace {
// The STARDUST v2 header as the reference reads it (Sim.cu:4985-4997).
struct Header {
    char magic[8];
    int32_t version, count, gridSize, preset, boundary;
    float gravity, simTime;
    float bhX, bhY, bhRs, bhMass;
    int32_t bhActive;
    int32_t reserved[5];
};
static_assert(sizeof(Header) == 76, "header layout");

SimConfig plain_pm(int n, int G, float gravity, float soft, float time_scale, int sort_interval, Boundary b) {
    SimConfig c;  // reference defaults, then every non-gravity feature off
    c.particleCount = n;
    c.gridSize = G;
    c.boundary = b;
    c.preset = Preset::Empty;
    c.gravity = gravity;
    c.softeningCells = soft;
    c.timeScale = time_scale;
    c.sortInterval = sort_interval;
    c.pressureEnabled = false;
    c.coolingEnabled = false;
    c.starFormationEnabled = false;
    c.contactEnabled = false;
    c.blackHoleEnabled = false;
    c.strongForceEnabled = false;
    c.emForceEnabled = false;
    c.weakForceEnabled = false;
    c.collapseEnabled = false;
    c.darkEnergy = 0.f;
    c.softBoundR = 0.f;
    c.spin = 0.f;
    c.hubble = 0.f;
    c.velDispersion = 0.f;
    c.darkMatterFraction = 0.f;
    return c;
}
}  // namespace

extern "C" {

void* ref_create() { return new Sim(); }

void ref_destroy(void* h) { delete static_cast<Sim*>(h); }

int ref_failed() { return Sim::failed() ? 1 : 0; }

const char* ref_fail_message() {
    static std::string m;
    m = Sim::failMessage();
    return m.c_str();
}

// Configure plain PM (boundary 0 isolated, 1 periodic, as Sim.h's Boundary) and
// load (pos, vel) through a state file at tmp_path.
int ref_load_b(void* h, const float* pos, const float* vel, int n, int G, float gravity, float soft,
               float time_scale, int sort_interval, int boundary, const char* tmp_path) {
    const Boundary b = boundary == 0 ? Boundary::Isolated : Boundary::Periodic;
    Sim* s = static_cast<Sim*>(h);
    s->init(plain_pm(n, G, gravity, soft, time_scale, sort_interval, b));
    if (Sim::failed()) return -2;
    Header hd;
    std::memset(&hd, 0, sizeof(hd));
    std::memcpy(hd.magic, "STARDUST", 8);
    hd.version = 2;
    hd.count = n;
    hd.gridSize = G;
    hd.preset = (int)Preset::Empty;
    hd.boundary = (int)b;
    hd.gravity = gravity;
    FILE* f = std::fopen(tmp_path, "wb");
    if (!f) return -5;
    bool ok = std::fwrite(&hd, sizeof(hd), 1, f) == 1 && std::fwrite(pos, 16, (size_t)n, f) == (size_t)n &&
              std::fwrite(vel, 16, (size_t)n, f) == (size_t)n;
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return -5;
    if (!s->loadState(tmp_path)) return -6;
    cudaDeviceSynchronize();
    return Sim::failed() ? -2 : 0;
}

int ref_load(void* h, const float* pos, const float* vel, int n, int G, float gravity, float soft, float time_scale,
             int sort_interval, const char* tmp_path) {
    return ref_load_b(h, pos, vel, n, G, gravity, soft, time_scale, sort_interval, 1, tmp_path);
}

// Sim::init with the plain-PM settings and the given initial conditions; init
// ends in reset(), which lays the preset down (placeInitial, spin, Hubble flow,
// dispersion, centre-of-mass stop). preset 0 Filament, 1 Empty (Sim.h:14-17).
int ref_init_preset(void* h, int n, int G, int boundary, int preset, float dark_frac, float shrink, float spin,
                    float hubble, float disp) {
    const Boundary b = boundary == 0 ? Boundary::Isolated : Boundary::Periodic;
    SimConfig c = plain_pm(n, G, 1.f, 1.f, 1.f, 1, b);
    c.preset = preset == 0 ? Preset::Filament : Preset::Empty;
    c.darkMatterFraction = dark_frac;
    c.bigBangShrink = shrink;
    c.spin = spin;
    c.hubble = hubble;
    c.velDispersion = disp;
    Sim* s = static_cast<Sim*>(h);
    s->init(c);
    cudaDeviceSynchronize();
    return Sim::failed() ? -2 : 0;
}

// Switch the grid hydrodynamics add-ons of a configured sim (a non-structural
// reconfigure: the particles stay). Star ionisation is zeroed so pressure runs
// alone, as star formation is off.
int ref_set_hydro(void* h, int pressure, float pressure_k, int cooling, float cooling_rate) {
    Sim* s = static_cast<Sim*>(h);
    SimConfig c = s->config();
    c.pressureEnabled = pressure != 0;
    c.pressureK = pressure_k;
    c.coolingEnabled = cooling != 0;
    c.coolingRate = cooling_rate;
    c.starIonizeK = 0.f;
    s->reconfigure(c);
    return Sim::failed() ? -2 : 0;
}

int ref_step(void* h) {
    static_cast<Sim*>(h)->step();
    return Sim::failed() ? -2 : 0;
}

int ref_steps(void* h, int k) {
    Sim* s = static_cast<Sim*>(h);
    for (int i = 0; i < k; ++i) s->step();
    cudaDeviceSynchronize();
    return Sim::failed() ? -2 : 0;
}

int ref_get(void* h, float* pos, float* vel, int n) {
    Sim* s = static_cast<Sim*>(h);
    if (cudaMemcpy(pos, s->particlePosDevicePtr(), 16 * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    if (cudaMemcpy(vel, s->particleVelDevicePtr(), 16 * (size_t)n, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    return 0;
}

// The density buffer holds `side`^3 floats: G (periodic) or the 2G box (isolated).
int ref_density(void* h, float* out, int G) {
    Sim* s = static_cast<Sim*>(h);
    const size_t cells = (size_t)G * G * G;
    if (cudaMemcpy(out, s->densityDevicePtr(), 4 * cells, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    return 0;
}

// scatterMs, poissonMs, gatherMs, totalMs, dtUsed, maxSpeed (Sim.h:844-852)
int ref_timings(void* h, float* out6) {
    const SimTimings t = static_cast<Sim*>(h)->timings();
    out6[0] = t.scatterMs;
    out6[1] = t.poissonMs;
    out6[2] = t.gatherMs;
    out6[3] = t.totalMs;
    out6[4] = t.dtUsed;
    out6[5] = t.maxSpeed;
    return 0;
}

double ref_sim_time(void* h) { return static_cast<Sim*>(h)->simTime(); }

// Sim::setViewRot + Sim::fieldDevicePtr (Sim.cu:5220-5296): the G^2 screen grid of
// field 0 (the density projected along z, or through the rotation: kProjectXY) or
// field 1 (the velocity dispersion of the particles: kScatterDispersion,
// kDivideInto) for the current state. rot9 (row-major 3x3) may be null: identity.
int ref_field(void* h, int field, const float* rot9, float* out, int G) {
    Sim* s = static_cast<Sim*>(h);
    const float eye[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
    s->setViewRot(rot9 ? rot9 : eye);
    const float* p = s->fieldDevicePtr(field == 0 ? Sim::Field::Density : Sim::Field::Dispersion);
    if (cudaDeviceSynchronize() != cudaSuccess || Sim::failed()) return -2;
    if (cudaMemcpy(out, p, 4 * (size_t)G * G, cudaMemcpyDeviceToHost) != cudaSuccess) return -2;
    return 0;
}

}  // extern "C"
