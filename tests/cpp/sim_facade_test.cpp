// sim_facade_test.cpp -- the reference's sim_tests checks for the PM path
// (tests/sim_tests.cpp: mass conservation 31-52, reconfigure 97-129, long run
// 213-231, periodic softening 423-458), written against the C++ facade
// (stardust_sim.hpp) so that App-style code is shown to build and run
// unchanged. Scenes are generated here (the reference's presets are not part of
// the PM path) and loaded with setParticles. Exit status 0 = all checks passed.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "stardust_sim.hpp"

using stardust::Boundary;
using stardust::Sim;
using stardust::SimConfig;

static int g_failures = 0;

static void check(bool ok, const char* what, const std::string& detail) {
    std::printf("  [%s] %s  (%s)\n", ok ? "PASS" : "FAIL", what, detail.c_str());
    if (!ok) ++g_failures;
}

// Deterministic 64-bit LCG -> uniform floats in [0, 1).
struct Lcg {
    uint64_t s;
    explicit Lcg(uint64_t seed) : s(seed * 6364136223846793005ull + 1442695040888963407ull) {}
    float next() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return (float)((s >> 40) * (1.0 / 16777216.0));
    }
};

// A uniform ball of radius r at the box centre, at rest (float4 pos / vel).
static void cloud(int n, float r, uint64_t seed, std::vector<float>& pos, std::vector<float>& vel) {
    Lcg g(seed);
    pos.assign(4 * (size_t)n, 0.f);
    vel.assign(4 * (size_t)n, 0.f);
    for (int i = 0; i < n;) {
        const float x = 2.f * g.next() - 1.f, y = 2.f * g.next() - 1.f, z = 2.f * g.next() - 1.f;
        if (x * x + y * y + z * z > 1.f) continue;
        pos[4 * (size_t)i + 0] = 0.5f + r * x;
        pos[4 * (size_t)i + 1] = 0.5f + r * y;
        pos[4 * (size_t)i + 2] = 0.5f + r * z;
        ++i;
    }
}

// A thin rotating disk (solid-body rotation) in the z = 0.5 plane.
static void disk(int n, uint64_t seed, std::vector<float>& pos, std::vector<float>& vel) {
    Lcg g(seed);
    pos.assign(4 * (size_t)n, 0.f);
    vel.assign(4 * (size_t)n, 0.f);
    for (int i = 0; i < n; ++i) {
        const float R = 0.3f * std::sqrt(g.next()), th = 6.2831853f * g.next();
        const float dz = 0.01f * (g.next() - 0.5f);
        pos[4 * (size_t)i + 0] = 0.5f + R * std::cos(th);
        pos[4 * (size_t)i + 1] = 0.5f + R * std::sin(th);
        pos[4 * (size_t)i + 2] = 0.5f + dz;
        vel[4 * (size_t)i + 0] = -0.2f * R * std::sin(th);
        vel[4 * (size_t)i + 1] = 0.2f * R * std::cos(th);
    }
}

static std::string fmt(const char* f, double a, double b, double c) {
    char buf[200];
    std::snprintf(buf, sizeof(buf), f, a, b, c);
    return buf;
}

static void test_mass_conservation() {
    std::printf("[1] mass conservation (deposit weights sum to 1)\n");
    for (int G : {32, 64, 128}) {
        Sim sim;
        SimConfig cfg;
        cfg.particleCount = 200000;
        cfg.gridSize = G;
        sim.init(cfg);
        std::vector<float> p, v;
        disk(cfg.particleCount, 1, p, v);
        sim.setParticles(p.data(), v.data(), cfg.particleCount);
        const double m0 = sim.measureTotalGridMass();
        for (int i = 0; i < 50; ++i) sim.step();
        const double m1 = sim.measureTotalGridMass();
        const double rel = std::fabs(m1 - m0) / (m0 > 0 ? m0 : 1.0);
        check(m0 > 1.0 && rel < 1e-3, "grid mass is conserved over 50 steps", fmt("G=%g m0=%.1f rel=%.2e", G, m0, rel));
    }
}

static void test_reconfigure() {
    std::printf("[2] particle count / grid changes\n");
    Sim sim;
    SimConfig cfg;
    cfg.particleCount = 100000;
    cfg.gridSize = 128;
    cfg.gravity = 0.f;
    sim.init(cfg);
    const int cases[3][2] = {{500000, 64}, {100000, 128}, {1000000, 128}};
    for (const auto& c : cases) {
        cfg.particleCount = c[0];
        cfg.gridSize = c[1];
        sim.reconfigure(cfg);
        std::vector<float> p, v;
        disk(c[0], 2, p, v);
        sim.setParticles(p.data(), v.data(), c[0]);
        sim.step();
        const double mass = sim.measureTotalGridMass();
        const double rel = std::fabs(mass - c[0]) / c[0];
        check(sim.particleCount() == c[0] && sim.gridSize() == c[1] && rel < 1e-3,
              "mass after reconfigure matches the particle count", fmt("N=%g G=%g rel=%.2e", c[0], c[1], rel));
    }
}

static void test_long_run() {
    std::printf("[3] long run (2000 steps)\n");
    Sim sim;
    SimConfig cfg;
    cfg.particleCount = 200000;
    cfg.gridSize = 256;
    cfg.gravity = 0.6f;
    sim.init(cfg);
    std::vector<float> p, v;
    disk(cfg.particleCount, 3, p, v);
    sim.setParticles(p.data(), v.data(), cfg.particleCount);
    const double m0 = sim.measureTotalGridMass();
    for (int i = 0; i < 2000; ++i) sim.step();
    const double m1 = sim.measureTotalGridMass();
    const double rel = std::fabs(m1 - m0) / (m0 > 0 ? m0 : 1.0);
    check(m0 > 1.0 && rel < 1e-2 && !Sim::failed(), "total mass survives 2000 steps", fmt("m0=%.0f m1=%.0f rel=%.2e", m0, m1, rel));
}

static void test_periodic_softening() {
    std::printf("[4] periodic softening blunts the short-range force\n");
    auto speed_with = [](float soft) {
        Sim sim;
        SimConfig cfg;
        cfg.particleCount = 200000;
        cfg.gridSize = 128;
        cfg.boundary = Boundary::Periodic;
        cfg.softeningCells = soft;
        cfg.gravity = 3.0f;
        sim.init(cfg);
        std::vector<float> p, v;
        cloud(cfg.particleCount, 0.18f, 4, p, v);
        sim.setParticles(p.data(), v.data(), cfg.particleCount);
        for (int i = 0; i < 600; ++i) sim.step();
        return (double)sim.timings().maxSpeed;
    };
    const double sharp = speed_with(0.5f), blunt = speed_with(6.0f);
    check(sharp > 1.15 * blunt, "a larger softening gives a smaller peak speed",
          fmt("soft 0.5: %.6f  soft 6: %.6f  ratio %.2f", sharp, blunt, blunt > 0 ? sharp / blunt : 0.0));
}

static void test_state_round_trip(const std::string& dir) {
    std::printf("[5] saveState / loadState\n");
    Sim a;
    SimConfig cfg;
    cfg.particleCount = 50000;
    cfg.gridSize = 64;
    a.init(cfg);
    std::vector<float> p, v;
    disk(cfg.particleCount, 5, p, v);
    a.setParticles(p.data(), v.data(), cfg.particleCount);
    for (int i = 0; i < 5; ++i) a.step();
    const std::string path = dir + "/facade_state.bin";
    const bool saved = a.saveState(path);
    Sim b;
    b.init(cfg);
    const bool loaded = b.loadState(path);
    std::vector<float> pa(4 * (size_t)cfg.particleCount), va(pa.size()), pb(pa.size()), vb(pa.size());
    a.getParticles(pa.data(), va.data(), cfg.particleCount);
    b.getParticles(pb.data(), vb.data(), cfg.particleCount);
    check(saved && loaded && pa == pb && va == vb && b.activeCount() == cfg.particleCount,
          "particles survive a save/load round trip byte for byte", fmt("active %g of %g (%g)", b.activeCount(), cfg.particleCount, 0));
}

static void test_init_lays_down_the_preset() {
    std::printf("[7] init / reset lay down the Filament preset (Sim::reset)\n");
    Sim sim;
    SimConfig cfg;
    cfg.particleCount = 30000;
    cfg.gridSize = 32;
    cfg.spin = 0.5f;  // the reference's defaults otherwise: Filament, no shrink
    sim.init(cfg);
    std::vector<float> p(4 * (size_t)cfg.particleCount), v(p.size());
    sim.getParticles(p.data(), v.data(), cfg.particleCount);
    double rmax = 0.0, px = 0.0;
    for (int i = 0; i < cfg.particleCount; ++i) {
        const double dx = p[4 * i] - 0.5, dy = p[4 * i + 1] - 0.5, dz = p[4 * i + 2] - 0.5;
        rmax = std::max(rmax, std::sqrt(dx * dx + dy * dy + dz * dz));
        px += v[4 * i];
    }
    sim.step(1e-3f);
    sim.reset();
    std::vector<float> q(p.size()), w(p.size());
    sim.getParticles(q.data(), w.data(), cfg.particleCount);
    check(sim.activeCount() == cfg.particleCount && rmax <= 0.5 + 1e-6 && std::fabs(px) < 1e-2 * cfg.particleCount &&
              q == p && w == v && sim.simTime() == 0.0,
          "every slot filled inside the ball, momentum stopped, reset repeats it",
          fmt("active %g  r_max %.6f  sum vx %.3g", (double)sim.activeCount(), rmax, px));
}

static void test_sticky_failure() {
    std::printf("[6] sticky failure flag\n");
    sd_clear_error();
    Sim sim;
    SimConfig cfg;
    cfg.particleCount = 0;  // rejected: no particles
    cfg.gridSize = 32;
    sim.init(cfg);
    const bool f1 = Sim::failed();
    const std::string m = Sim::failMessage();
    check(f1 && !m.empty(), "an invalid configuration sets failed() with a message", m);
    sd_clear_error();
}

int main(int argc, char** argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    if (!Sim::deviceAvailable()) {
        std::printf("no CUDA device\n");
        return 2;
    }
    test_mass_conservation();
    test_reconfigure();
    test_long_run();
    test_periodic_softening();
    test_state_round_trip(dir);
    test_init_lays_down_the_preset();
    test_sticky_failure();
    std::printf("%d failure(s)\n", g_failures);
    return g_failures == 0 ? 0 : 1;
}
