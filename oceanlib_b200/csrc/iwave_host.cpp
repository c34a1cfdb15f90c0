// oceanlib-b200: host side of the iWave interaction field (see iwave_host.h).
#include "iwave_host.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <stdexcept>

namespace ocean_b200 {
namespace {

bool pow2(uint32_t v) { return v != 0 && (v & (v - 1)) == 0; }

}  // namespace

void interaction_desc_defaults(ocean_interaction_desc* d)
{
    // include/ocean/interaction.hpp:64-139 (InteractionDesc defaults)
    std::memset(d, 0, sizeof(*d));
    d->struct_size = sizeof(ocean_interaction_desc);
    d->size = 256;
    d->extent = 64.0f;
    d->kernel_radius = 6;
    d->damping = 0.20f;
    d->absorb_cells = 16;
    d->fixed_dt = 0.0f;
    d->max_substeps = 8;
    d->max_sources = 64;
    d->gravity = 9.81f;
    d->water_depth = 0.0f;
    d->obstruction = OCEAN_OBSTRUCTION_NEUMANN;
}

bool copy_interaction_desc(const ocean_interaction_desc* src, ocean_interaction_desc& dst)
{
    if (src == nullptr) return false;
    if (src->struct_size == 0 || src->struct_size > sizeof(ocean_interaction_desc)) return false;
    interaction_desc_defaults(&dst);
    std::memcpy(&dst, src, src->struct_size);
    dst.struct_size = sizeof(ocean_interaction_desc);
    return true;
}

void validate_interaction(const ocean_interaction_desc& d)
{
    // src/interaction.cpp:439-476
    if (!pow2(d.size) || d.size < 32 || d.size > 1024) throw std::invalid_argument("size");
    if (!(d.extent > 0.0f)) throw std::invalid_argument("extent");
    if (d.kernel_radius < 1 || d.kernel_radius > 12) throw std::invalid_argument("kernel_radius");
    if (2 * d.kernel_radius >= d.size) throw std::invalid_argument("kernel_radius vs size");
    if (!(d.damping >= 0.0f)) throw std::invalid_argument("damping");
    if (d.absorb_cells * 2 >= d.size) throw std::invalid_argument("absorb_cells");
    if (d.max_substeps < 1) throw std::invalid_argument("max_substeps");
    if (d.max_sources < 1) throw std::invalid_argument("max_sources");
    if (!(d.gravity > 0.0f)) throw std::invalid_argument("gravity");
    if (d.fixed_dt < 0.0f) throw std::invalid_argument("fixed_dt");
}

IWaveSetup iwave_setup(const ocean_interaction_desc& d)
{
    validate_interaction(d);
    IWaveSetup s;
    s.n = d.size;
    s.p = d.kernel_radius;
    s.cell = d.extent / static_cast<float>(d.size);
    s.cells = static_cast<size_t>(s.n) * s.n;
    s.stride = static_cast<int>((s.n + 2 * s.p + 15u) & ~15u);  // src/interaction.cpp:43-46
    s.rows = s.n + 2 * s.p;
    s.stencil = build_iwave_stencil(s.p, static_cast<double>(s.cell), static_cast<double>(d.water_depth));
    if (!s.stencil.stable())
        throw std::invalid_argument("interaction stencil has a negative symbol (unstable)");
    s.dt_limit = static_cast<float>(2.0 / std::sqrt(static_cast<double>(d.gravity) * s.stencil.max_symbol));
    s.dt = (d.fixed_dt > 0.0f) ? d.fixed_dt : std::min(1.0f / 60.0f, 0.35f * s.dt_limit);
    if (d.fixed_dt > 0.0f && d.fixed_dt > s.dt_limit)
        throw std::invalid_argument("interaction fixed_dt exceeds the stability limit");
    std::memset(&s.taps, 0, sizeof(s.taps));
    std::copy(s.stencil.taps.begin(), s.stencil.taps.end(), s.taps.t);
    return s;
}

void iwave_damping(const ocean_interaction_desc& d, const IWaveSetup& s, std::vector<float>& c1,
                   std::vector<float>& c2)
{
    // Float arithmetic as the reference's sponge.
    const float a0 = d.damping;
    const int w = static_cast<int>(d.absorb_cells);
    const float a_edge = 4.0f / std::max(s.dt * static_cast<float>(std::max(w, 1)), 1e-6f);
    const uint32_t n = s.n;
    c1.assign(s.cells, 0.0f);
    c2.assign(s.cells, 0.0f);
    for (uint32_t z = 0; z < n; ++z)
        for (uint32_t x = 0; x < n; ++x) {
            const int dx = std::min<int>(static_cast<int>(x), static_cast<int>(n - 1 - x));
            const int dz = std::min<int>(static_cast<int>(z), static_cast<int>(n - 1 - z));
            const int dd = std::min(dx, dz);
            float alpha = a0;
            if (w > 0 && dd < w) {
                const float t = static_cast<float>(w - dd) / static_cast<float>(w);
                alpha += a_edge * t * t;
            }
            const float ad = alpha * s.dt;
            const size_t i = static_cast<size_t>(z) * n + x;
            c1[i] = 1.0f / (1.0f + ad);
            c2[i] = 1.0f - ad;
        }
}

bool resolve_source(const ocean_disturbance& d, float sub_time, float scale, const IWaveSetup& g,
                    int32_t origin_x, int32_t origin_z, IWaveSource& s)
{
    const float cell = g.cell;
    const float sigma = std::max(d.radius, 0.25f * cell);
    s.inv_two_sigma2 = 1.0f / (2.0f * sigma * sigma);
    const float wx = d.world_x + d.velocity_x * sub_time;
    const float wz = d.world_z + d.velocity_z * sub_time;
    s.gx = (wx - static_cast<float>(origin_x) * cell) / cell;
    s.gz = (wz - static_cast<float>(origin_z) * cell) / cell;
    const int rad = static_cast<int>(std::ceil(4.0f * sigma / cell));
    const int n = static_cast<int>(g.n);
    s.x0 = std::max(0, static_cast<int>(std::floor(s.gx)) - rad);
    s.x1 = std::min(n - 1, static_cast<int>(std::floor(s.gx)) + rad);
    s.z0 = std::max(0, static_cast<int>(std::floor(s.gz)) - rad);
    s.z1 = std::min(n - 1, static_cast<int>(std::floor(s.gz)) + rad);
    if (s.x1 < s.x0 || s.z1 < s.z0) return false;
    s.cell = cell;
    s.disp = -d.strength * scale;
    s.vel = d.velocity_y * scale;
    s.dt = g.dt;
    s.mean = 0.0f;
    return true;
}

uint32_t IWaveClock::advance(float dt, float fixed_dt, uint32_t max_substeps)
{
    if (!(dt > 0.0f)) dt = 0.0f;
    accum += static_cast<double>(dt);
    uint32_t steps = 0;
    if (accum >= fixed_dt) steps = static_cast<uint32_t>(accum / static_cast<double>(fixed_dt));
    clamped = steps > max_substeps;
    if (clamped) {
        steps = max_substeps;
        accum = 0.0;
    } else {
        accum -= static_cast<double>(steps) * static_cast<double>(fixed_dt);
    }
    last_steps = steps;
    return steps;
}

void IWaveQueue::reset(uint32_t max_sources)
{
    items.assign(max_sources, ocean_disturbance{});
    count = 0;
}

void IWaveQueue::add(const ocean_disturbance& d)
{
    if (count >= items.size()) {
        ++dropped;
        return;
    }
    items[count++] = d;
}

void IWaveQueue::keep_impulses()
{
    uint32_t keep = 0;
    for (uint32_t i = 0; i < count; ++i)
        if (items[i].kind == OCEAN_SOURCE_IMPULSE) items[keep++] = items[i];
    count = keep;
}

void IWaveQueue::resolve_all(uint32_t steps, const IWaveSetup& g, int32_t origin_x, int32_t origin_z,
                             std::vector<IWaveSource>& out, std::vector<uint32_t>& first)
{
    first.assign(static_cast<size_t>(steps) + 1, 0);
    for (uint32_t s = 0; s < steps; ++s) {
        first[s] = static_cast<uint32_t>(out.size());
        const float sub_time = static_cast<float>(s) * g.dt;
        for (uint32_t i = 0; i < count; ++i) {
            const ocean_disturbance& d = items[i];
            const bool impulse = d.kind != OCEAN_SOURCE_CONTINUOUS;
            if (impulse && s != 0) continue;
            IWaveSource src;
            if (resolve_source(d, impulse ? 0.0f : sub_time, impulse ? 1.0f : g.dt, g, origin_x, origin_z, src))
                out.push_back(src);
        }
    }
    first[steps] = static_cast<uint32_t>(out.size());
    count = 0;
}

}  // namespace ocean_b200
