// Host-side setup of the SPH step: Parameters defaults, the derived
// Simulation_config, and the scene generators (the reference's own dam break
// and world walls, and the seeded block scenes used for benchmarking).
// One-time setup code; compiled with -ffp-contract=off so every float
// operation rounds exactly as in the reference.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <random>
#include <unordered_map>
#include <vector>

#include "../../include/emerald_sph.h"
#include "engine.hpp"
#include "sph_math.cuh"

namespace emerald {

namespace {

constexpr int64_t kFlicksOneNinetieth = 7840000;  // flicks of 1/90 s

struct Box2 {
    float2 min, max;
};

// estimate_solid_box_emission_count (emerald/sph2d_box/solids.cpp:14-20).
size_t estimate_emission(Box2 const& b, float R) {
    float const sx = b.max.x - b.min.x;
    float const sy = b.max.y - b.min.y;
    size_t const nx = static_cast<size_t>(std::ceil(sx / (2.0f * R)));
    size_t const ny = static_cast<size_t>(std::ceil(sy / (std::sqrt(3.0f) * R)));
    return nx * ny;
}

// emit_solid_box: hexagonal rows, alternate rows shifted by R
// (emerald/sph2d_box/solids.cpp:22-50).
size_t emit_box(Box2 const& b, float R, size_t max_count, float2* out) {
    bool push_x = false;
    float const dx = 2.0f * R;
    float const dy = std::sqrt(3.0f) * R;
    float2 const start = mk2(b.min.x + R, b.min.y + R);
    float2 point = start;
    float2 const stop = mk2(b.max.x - R, b.max.y - R);
    size_t count = 0;
    for (; point.y <= stop.y; point.y += dy) {
        float const offset_x = R;
        point.x = push_x ? start.x : start.x + R;
        point.x += offset_x;
        for (; point.x <= stop.x; point.x += dx) {
            out[count] = point;
            ++count;
            if (count == max_count) return count;
        }
        push_x = !push_x;
    }
    return count;
}

double to_seconds(int64_t f) { return static_cast<double>(f) / 705600000.0; }

}  // namespace

void default_params(emerald_params& p) {
    p.seed = 1;
    p.time_per_step_flicks = 3 * kFlicksOneNinetieth;
    p.sub_steps = 30;
    p.length = 1.0f;
    p.support = 0.025f;
    p.gravity = 9.81f;
    p.viscosity = 0.01f;
    p.target_density = 1000.0f;
    p.iisph_max_pressure_iterations = 30;
    p.iisph_error_average_threshold = 0.005f;
    p.iisph_error_max_threshold = 0.05f;
    p.iisph_omega = 0.5f;
    p.dfsph_max_correction_iterations = 15;
    p.dfsph_density_error_average_threshold = 0.0035f;
    p.dfsph_density_error_max_threshold = 0.03f;
    p.dfsph_divergence_error_average_threshold = 0.0035f;
    p.dfsph_divergence_error_max_threshold = 0.03f;
    p.mass_per_particle = 0.0f;
    p.pressure_correction_denom = 0.0f;
    p.precision = EMERALD_PRECISION_REFERENCE;
}

// Simulation_config::Simulation_config (emerald/sph2d_box/config.cpp:16-132):
// the template sums over a hex-packed block around the point nearest the
// origin give the per-particle mass and the PCISPH denominator.
DerivedConfig derive_config(emerald_params const& p) {
    DerivedConfig c{};
    float const H = p.support;
    float const R = 0.99f * (H * 0.5f);
    c.draw_radius = R;
    float2 gsum = mk2(0.0f, 0.0f);
    float gdot = 0.0f;
    float muchness = 0.0f;
    Box2 const box{mk2(-15.0f * R, -15.0f * R), mk2(15.0f * R, 15.0f * R)};
    size_t const emit_max = estimate_emission(box, R);
    std::vector<float2> pts(emit_max);
    pts.resize(emit_max ? emit_box(box, R, emit_max, pts.data()) : 0);
    float2 best = mk2(0.0f, 0.0f);
    float best_r2 = std::numeric_limits<float>::max();
    for (auto const& q : pts) {
        float const r2 = dot2(q, q);
        if (r2 < best_r2) {
            best = q;
            best_r2 = r2;
        }
    }
    for (auto const& q : pts) {
        float2 const d = sub2(best, q);
        float const len = length2f(d);
        float const w = kernel_w(len, H);
        if (w > 0.0f) muchness += w;
        float2 const g = kernel_grad_w(d, H);
        gsum = add2(gsum, g);
        gdot += dot2(g, g);
    }
    c.mass_per_particle = p.target_density / muchness;
    c.seconds_per_sub_step =
      static_cast<float>(to_seconds(p.time_per_step_flicks / p.sub_steps));
    float const beta = 2.0f * sqrf(c.seconds_per_sub_step / muchness);
    c.pressure_correction_denom = beta * (dot2(gsum, gsum) + gdot);
    if (p.mass_per_particle > 0.0f) c.mass_per_particle = p.mass_per_particle;
    if (p.pressure_correction_denom > 0.0f) c.pressure_correction_denom = p.pressure_correction_denom;
    return c;
}

// The same template sums over an unjittered square lattice at spacing dx
// centred on a lattice point.
void lattice_config(emerald_params const& p, float dx, float dt, float& mass, float& denom) {
    float const h = p.support;
    int const reach = static_cast<int>(std::ceil(2.0 * double(h) / double(dx))) + 1;
    float muchness = 0.0f;
    float2 gsum = mk2(0.0f, 0.0f);
    float gdot = 0.0f;
    for (int j = -reach; j <= reach; ++j) {
        for (int i = -reach; i <= reach; ++i) {
            float2 const q = mk2(static_cast<float>(i) * dx, static_cast<float>(j) * dx);
            float2 const d = sub2(mk2(0.0f, 0.0f), q);
            float const w = kernel_w(length2f(d), h);
            if (w > 0.0f) muchness += w;
            float2 const g = kernel_grad_w(d, h);
            gsum = add2(gsum, g);
            gdot += dot2(g, g);
        }
    }
    mass = p.target_density / muchness;
    float const beta = 2.0f * sqrf(dt / muchness);
    denom = beta * (dot2(gsum, gsum) + gdot);
}

size_t block_scene(uint32_t nx, uint32_t ny, float dx, float x0, float y0, float jitter,
                   uint64_t seed, float* xy) {
    std::mt19937_64 gen{seed};
    std::uniform_real_distribution<float> dist{-jitter * dx, jitter * dx};
    size_t k = 0;
    for (uint32_t j = 0; j < ny; ++j) {
        for (uint32_t i = 0; i < nx; ++i) {
            float const px = x0 + (static_cast<float>(i) + 0.5f) * dx;
            float const py = y0 + (static_cast<float>(j) + 0.5f) * dx;
            float const jx = dist(gen);
            float const jy = dist(gen);
            if (xy) {
                xy[2 * k] = px + jx;
                xy[2 * k + 1] = py + jy;
            }
            ++k;
        }
    }
    return k;
}

size_t wall_scene(float dx, float length, int layers, float* xy) {
    int const n = static_cast<int>(std::lround(double(length) / double(dx)));
    size_t k = 0;
    auto put = [&](float x, float y) {
        if (xy) {
            xy[2 * k] = x;
            xy[2 * k + 1] = y;
        }
        ++k;
    };
    for (int l = 0; l < layers; ++l) {
        float const off = (static_cast<float>(l) + 0.5f) * dx;
        for (int i = -layers; i < n + layers; ++i) put((static_cast<float>(i) + 0.5f) * dx, -off);
        for (int j = 0; j < n; ++j) put(-off, (static_cast<float>(j) + 0.5f) * dx);
        for (int j = 0; j < n; ++j) put(length + off, (static_cast<float>(j) + 0.5f) * dx);
    }
    return k;
}

// world_walls_initial_solid_state (emerald/sph2d_box/solids.cpp:139-213),
// positions only (volumes follow on the device).
std::vector<float2> world_walls(emerald_params const& p) {
    float const H = p.support;
    float const R = 0.99f * (H * 0.5f);
    float const L = p.length;
    float const border = H * 3.0f;
    std::vector<Box2> boxes;
    boxes.push_back({mk2(-border, -border), mk2(0.0f, L + border)});
    boxes.push_back({mk2(L, -border), mk2(L + border, L + border)});
    boxes.push_back({mk2(-0.5f * border, -border), mk2(L + 0.5f * border, 0.0f)});
    boxes.push_back({mk2(-0.5f * border, L), mk2(L + 0.5f * border, L + border)});
    std::mt19937_64 gen{1919};
    std::uniform_real_distribution<float> dist{-0.06f, 0.06f};
    int const N = 4;
    for (int by = 0; by < N; ++by) {
        float const byf = float(by + 1) / (N + 1);
        for (int bx = 0; bx < N; ++bx) {
            float const bxf = float(bx + 1) / (N + 1);
            // Argument evaluation order of the reference's call
            // tiny_block({bxf + dist(gen), byf + dist(gen)}, dist(gen)):
            // GCC evaluates the brace-list elements left to right and the
            // second argument first (right-to-left argument order on x86-64).
            float const roff = dist(gen);
            float const ux = bxf + dist(gen);
            float const uy = byf + dist(gen);
            float const r = 0.04f + std::abs(roff);
            float2 const lo = mk2(L * (ux - r), L * (uy - r));
            float2 const hi = mk2(L * (ux + r), L * (uy + r));
            boxes.push_back({lo, hi});
        }
    }
    size_t total = 100;
    for (auto const& b : boxes) total += estimate_emission(b, R);
    std::vector<float2> pos(total);
    size_t remaining = total;
    float2* at = pos.data();
    for (auto const& b : boxes) {
        size_t const c = emit_box(b, R, remaining, at);
        remaining -= c;
        at += c;
    }
    pos.resize(total - remaining);
    return pos;
}

// dam_break_initial_state (emerald/sph2d_box/initial_state.cpp:14-97): a hex
// block with every particle closer than 2R to a boundary particle removed.
std::vector<float2> dam_break(emerald_params const& p, float2 const* solid, size_t n_solid) {
    float const H = p.support;
    float const R = 0.99f * (H * 0.5f);
    float const L = p.length;
    Box2 const box{mk2(0.0f, 0.0f), mk2(L / 2.0f, 3.25f * L / 4.0f)};
    size_t const max_count = 100 + estimate_emission(box, R);
    std::vector<float2> pos(max_count);
    pos.resize(emit_box(box, R, max_count, pos.data()));
    float const cell = 2.0f * H;
    std::unordered_map<uint64_t, std::vector<uint32_t>> grid;
    for (size_t s = 0; s < n_solid; ++s) {
        int32_t gx, gy;
        grid_coord(solid[s], cell, gx, gy);
        grid[morton2(uint32_t(gx), uint32_t(gy))].push_back(uint32_t(s));
    }
    std::vector<float2> out;
    out.reserve(pos.size());
    for (auto const& q : pos) {
        int32_t gx, gy;
        grid_coord(q, cell, gx, gy);
        bool kill = false;
        for (int32_t j = gy - 1; !kill && j <= gy + 1; ++j) {
            for (int32_t i = gx - 1; !kill && i <= gx + 1; ++i) {
                auto const it = grid.find(morton2(uint32_t(i), uint32_t(j)));
                if (it == grid.end()) continue;
                for (uint32_t s : it->second) {
                    if (length2f(sub2(solid[s], q)) < 2 * R) {
                        kill = true;
                        break;
                    }
                }
            }
        }
        if (!kill) out.push_back(q);
    }
    return out;
}

}  // namespace emerald
