// Test-only bridge into the reference oceanlib, compiled from its own sources
// (see oracle/Makefile). Nothing in the shipped library links this: it exists so
// the parity tests and the CPU baseline can call the reference's internal
// stages (spectrum tables, evolve, FFT, finalize) and its public Ocean,
// FoamField and CascadeStack classes through a flat C interface.
//
// Every reference symbol is compiled with hidden visibility; only the oref_*
// functions below are exported, so this library can sit in the same process
// as libocean_b200.so (which exports the same ocean_* C names) without
// symbol interposition.

#include "ocean/ocean.h"
#include "ocean/ocean.hpp"
#include "ocean/foam.hpp"
#include "ocean/cascade.hpp"

#include "ocean/interaction.hpp"

#include "core/cpu_features.hpp"
#include "core/evolve.hpp"
#include "core/iwave_kernel.hpp"
#include "core/fft.hpp"
#include "core/rng.hpp"
#include "core/spectrum.hpp"
#include "half.hpp"  // examples/viewer (via -I)

#include <chrono>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#define OREF_API extern "C" __attribute__((visibility("default")))

namespace {

ocean::OceanDesc to_cpp_desc(const ocean_desc* c)
{
    // Mirrors the reference's own C->C++ translation (src/c_api.cpp:62-95).
    ocean::OceanDesc d;
    d.size = c->size;
    d.patch_length = c->patch_length;
    d.spectrum.wind_speed = c->spectrum.wind_speed;
    d.spectrum.fetch = c->spectrum.fetch;
    d.spectrum.wind_direction = c->spectrum.wind_direction;
    d.spectrum.peak_enhancement = c->spectrum.peak_enhancement;
    d.spectrum.swell = c->spectrum.swell;
    d.spectrum.small_wave_cutoff = c->spectrum.small_wave_cutoff;
    d.spectrum.gravity = c->spectrum.gravity;
    d.spectrum.depth = c->water_depth;
    d.choppiness = c->choppiness;
    d.foam_threshold = c->foam_threshold;
    d.seed = c->seed;
    d.thread_count = c->thread_count;
    d.compute_velocity = c->compute_velocity != 0;
    return d;
}

struct StageCtx {
    ocean::OceanDesc desc;
    ocean::detail::SpectrumTables tables;
    ocean::detail::FftPlan plan;
    ocean::detail::FieldSet fields;
    std::vector<float> scratch;
};

}  // namespace

// ---------------------------------------------------------------------------
// Public C ABI of the reference, re-exported under oref_ names.
// ---------------------------------------------------------------------------

OREF_API void* oref_c_create(const ocean_desc* desc, int* status)
{
    ocean_status st = OCEAN_OK;
    ocean_sim* s = ocean_create(desc, &st);
    if (status) *status = static_cast<int>(st);
    return s;
}
OREF_API void oref_c_destroy(void* sim) { ocean_destroy(static_cast<ocean_sim*>(sim)); }
OREF_API void oref_c_update(void* sim, double t) { ocean_update(static_cast<ocean_sim*>(sim), t); }
OREF_API void oref_c_get_buffers(void* sim, ocean_buffers* out)
{
    *out = ocean_get_buffers(static_cast<ocean_sim*>(sim));
}
OREF_API const float* oref_c_get_velocity(void* sim)
{
    return ocean_get_velocity(static_cast<ocean_sim*>(sim));
}
OREF_API float oref_c_height_at(void* sim, float x, float z)
{
    return ocean_height_at(static_cast<ocean_sim*>(sim), x, z);
}
OREF_API void oref_c_sample_ex(void* sim, float x, float z, ocean_surface_ex* out)
{
    ocean_sample_ex(static_cast<ocean_sim*>(sim), x, z, out);
}
OREF_API void oref_c_desc_init(ocean_desc* d) { ocean_desc_init(d); }
OREF_API const char* oref_c_force_simd_level(const char* name)
{
    return ocean_force_simd_level(name);
}
OREF_API const char* oref_c_simd_level(void) { return ocean_simd_level(); }

// Batched sample_ex over many points (a plain host loop, as a caller would
// write it against the reference API).
OREF_API void oref_c_sample_many(void* sim, const float* xz, uint64_t count,
                                 ocean_surface_ex* out)
{
    auto* s = static_cast<ocean_sim*>(sim);
    for (uint64_t i = 0; i < count; ++i) {
        ocean_sample_ex(s, xz[2 * i], xz[2 * i + 1], &out[i]);
    }
}

// ---------------------------------------------------------------------------
// Internal stages.
// ---------------------------------------------------------------------------

OREF_API void* oref_stage_create(const ocean_desc* desc)
{
    auto* c = new StageCtx();
    c->desc = to_cpp_desc(desc);
    ocean::detail::build_spectrum(c->desc, c->tables);
    c->plan = ocean::detail::FftPlan(c->desc.size, ocean::detail::SimdLevel::Scalar);
    c->fields.allocate(c->desc.size, c->desc.compute_velocity);
    c->scratch.resize(c->plan.scratch_floats());
    return c;
}
OREF_API void oref_stage_destroy(void* ctx) { delete static_cast<StageCtx*>(ctx); }

// Writes the eight spectrum tables, each N*N floats, in the order
// h0_re, h0_im, h0c_re, h0c_im, omega, kx, kz, k_inv.
OREF_API void oref_stage_tables(void* ctx, float* out)
{
    auto* c = static_cast<StageCtx*>(ctx);
    const std::size_t cells = static_cast<std::size_t>(c->desc.size) * c->desc.size;
    const float* src[8] = {c->tables.h0_re.data(), c->tables.h0_im.data(),
                           c->tables.h0c_re.data(), c->tables.h0c_im.data(),
                           c->tables.omega.data(), c->tables.kx.data(),
                           c->tables.kz.data(), c->tables.k_inv.data()};
    for (int p = 0; p < 8; ++p) std::memcpy(out + p * cells, src[p], cells * sizeof(float));
}

OREF_API void oref_stage_evolve(void* ctx, double t)
{
    auto* c = static_cast<StageCtx*>(ctx);
    ocean::detail::evolve_rows_scalar(c->tables, t, c->fields, 0, c->desc.size);
    if (c->desc.compute_velocity) {
        ocean::detail::evolve_velocity_rows(c->tables, t, c->fields, 0, c->desc.size);
    }
}

OREF_API void oref_stage_fft(void* ctx)
{
    auto* c = static_cast<StageCtx*>(ctx);
    for (int f = 0; f < c->fields.complex_fields; ++f) {
        c->plan.transform_2d(c->fields.re(f), c->fields.im(f), c->scratch.data(),
                             ocean::detail::FftSign::Inverse);
    }
}

// Planes are laid out re(0), im(0), re(1), im(1), ... (8 or 12 planes).
OREF_API int oref_stage_plane_count(void* ctx)
{
    return 2 * static_cast<StageCtx*>(ctx)->fields.complex_fields;
}
OREF_API void oref_stage_get_fields(void* ctx, float* out)
{
    auto* c = static_cast<StageCtx*>(ctx);
    std::memcpy(out, c->fields.storage.data(),
                c->fields.storage.size() * sizeof(float));
}
OREF_API void oref_stage_set_fields(void* ctx, const float* in)
{
    auto* c = static_cast<StageCtx*>(ctx);
    std::memcpy(c->fields.storage.data(), in,
                c->fields.storage.size() * sizeof(float));
}
OREF_API void oref_stage_finalize(void* ctx, float* disp, float* normal, float* vel)
{
    auto* c = static_cast<StageCtx*>(ctx);
    ocean::detail::finalize_rows(c->fields, c->desc.choppiness, c->desc.foam_threshold,
                                 disp, normal, 0, c->desc.size);
    if (c->desc.compute_velocity && vel) {
        ocean::detail::finalize_velocity_rows(c->fields, vel, 0, c->desc.size);
    }
}

// One transform of `n` points (power of two) in place, scalar kernel.
// sign: +1 inverse, -1 forward.
OREF_API void oref_fft_1d(uint32_t n, float* re, float* im, int sign)
{
    ocean::detail::FftPlan plan(n, ocean::detail::SimdLevel::Scalar);
    std::vector<float> scratch(plan.scratch_floats());
    plan.transform(re, im, 1, scratch.data(),
                   sign > 0 ? ocean::detail::FftSign::Inverse : ocean::detail::FftSign::Forward);
}
OREF_API void oref_fft_2d(uint32_t n, float* re, float* im, int sign)
{
    ocean::detail::FftPlan plan(n, ocean::detail::SimdLevel::Scalar);
    std::vector<float> scratch(plan.scratch_floats());
    plan.transform_2d(re, im, scratch.data(),
                      sign > 0 ? ocean::detail::FftSign::Inverse : ocean::detail::FftSign::Forward);
}

// PCG32 known-answer access.
OREF_API void oref_pcg32(uint64_t seed, uint64_t stream, uint32_t count, uint32_t* out)
{
    ocean::detail::Pcg32 r = ocean::detail::seed_pcg32(seed, stream);
    for (uint32_t i = 0; i < count; ++i) out[i] = ocean::detail::next_u32(r);
}
OREF_API void oref_row_gaussians(uint64_t seed, uint32_t row, uint32_t pairs, float* out)
{
    ocean::detail::Pcg32 r = ocean::detail::row_rng(seed, row);
    for (uint32_t i = 0; i < pairs; ++i) {
        const auto g = ocean::detail::next_gaussian_pair(r);
        out[2 * i] = g.a;
        out[2 * i + 1] = g.b;
    }
}

// ---------------------------------------------------------------------------
// Persistent foam (C++ only in the reference).
// ---------------------------------------------------------------------------

struct OrefFoamDesc {
    float decay, source_gain, advect_scale, wind_drift_x, wind_drift_z, fixed_dt;
    uint32_t max_substeps, thread_count;
};

OREF_API void* oref_foam_create(void* sim, const OrefFoamDesc* d, int* status)
{
    ocean::FoamDesc fd;
    fd.decay = d->decay;
    fd.source_gain = d->source_gain;
    fd.advect_scale = d->advect_scale;
    fd.wind_drift_x = d->wind_drift_x;
    fd.wind_drift_z = d->wind_drift_z;
    fd.fixed_dt = d->fixed_dt;
    fd.max_substeps = d->max_substeps;
    fd.thread_count = d->thread_count;
    try {
        auto* f = new ocean::FoamField(*reinterpret_cast<ocean::Ocean*>(sim), fd);
        if (status) *status = 0;
        return f;
    } catch (...) {
        if (status) *status = 1;
        return nullptr;
    }
}
OREF_API void oref_foam_destroy(void* f) { delete static_cast<ocean::FoamField*>(f); }
OREF_API void oref_foam_update(void* f, float dt) { static_cast<ocean::FoamField*>(f)->update(dt); }
OREF_API const float* oref_foam_data(void* f) { return static_cast<ocean::FoamField*>(f)->data(); }
OREF_API uint32_t oref_foam_last_substeps(void* f)
{
    return static_cast<ocean::FoamField*>(f)->last_substeps();
}
OREF_API double oref_foam_coverage(void* f) { return static_cast<ocean::FoamField*>(f)->coverage(); }
OREF_API float oref_foam_at(void* f, float x, float z)
{
    return static_cast<ocean::FoamField*>(f)->foam_at(x, z);
}
OREF_API void oref_foam_clear(void* f) { static_cast<ocean::FoamField*>(f)->clear(); }
OREF_API int oref_foam_set_desc(void* f, const OrefFoamDesc* d)
{
    ocean::FoamDesc fd;
    fd.decay = d->decay;
    fd.source_gain = d->source_gain;
    fd.advect_scale = d->advect_scale;
    fd.wind_drift_x = d->wind_drift_x;
    fd.wind_drift_z = d->wind_drift_z;
    fd.fixed_dt = d->fixed_dt;
    fd.max_substeps = d->max_substeps;
    fd.thread_count = d->thread_count;
    try {
        static_cast<ocean::FoamField*>(f)->set_desc(fd);
        return 0;
    } catch (...) {
        return 1;
    }
}

// ---------------------------------------------------------------------------
// Cascades (C++ only in the reference).
// ---------------------------------------------------------------------------

OREF_API void* oref_cascade_create(const ocean_desc* levels, uint32_t count, int* status)
{
    std::vector<ocean::CascadeLevel> v;
    for (uint32_t i = 0; i < count; ++i) v.push_back(to_cpp_desc(&levels[i]));
    try {
        auto* c = new ocean::CascadeStack(std::span<const ocean::CascadeLevel>(v.data(), v.size()));
        if (status) *status = 0;
        return c;
    } catch (...) {
        if (status) *status = 1;
        return nullptr;
    }
}
OREF_API void oref_cascade_destroy(void* c) { delete static_cast<ocean::CascadeStack*>(c); }
OREF_API void oref_cascade_update(void* c, double t) { static_cast<ocean::CascadeStack*>(c)->update(t); }
OREF_API void oref_cascade_sample_many(void* c, const float* xz, uint64_t count,
                                       ocean_surface_ex* out)
{
    auto* cs = static_cast<ocean::CascadeStack*>(c);
    for (uint64_t i = 0; i < count; ++i) {
        const ocean::Surface s = cs->sample_at(xz[2 * i], xz[2 * i + 1]);
        out[i] = ocean_surface_ex{s.height, s.offset_x, s.offset_z, s.normal_x, s.normal_y,
                                  s.normal_z, s.foam, s.velocity_x, s.velocity_y, s.velocity_z};
    }
}
OREF_API void oref_cascade_level_buffers(void* c, uint32_t level, ocean_buffers* out,
                                         const float** velocity)
{
    const ocean::Buffers b = static_cast<ocean::CascadeStack*>(c)->buffers(level);
    out->displacement = b.displacement;
    out->normal = b.normal;
    out->size = b.size;
    out->patch_length = b.patch_length;
    if (velocity) *velocity = b.velocity;
}

// ---------------------------------------------------------------------------
// Timing helper for the CPU baseline: `count` oceans updated in sequence for
// `frames` frames at t = t0 + i*dt, optionally with persistent foam. Returns
// the elapsed wall time in seconds (steady clock).
// ---------------------------------------------------------------------------

OREF_API double oref_time_updates(void* const* sims, void* const* foams, uint32_t count,
                                  uint32_t frames, double t0, double dt, float foam_dt)
{
    const auto start = std::chrono::steady_clock::now();
    for (uint32_t f = 0; f < frames; ++f) {
        const double t = t0 + dt * static_cast<double>(f);
        for (uint32_t i = 0; i < count; ++i) {
            ocean_update(static_cast<ocean_sim*>(sims[i]), t);
            if (foams && foams[i]) static_cast<ocean::FoamField*>(foams[i])->update(foam_dt);
        }
    }
    const auto end = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(end - start).count();
}

OREF_API uint32_t oref_hardware_concurrency(void)
{
    return std::thread::hardware_concurrency();
}

// ---------------------------------------------------------------------------
// iWave: the reference's stencil builder and its interaction C ABI.
// ---------------------------------------------------------------------------

// taps: (2P+1)^2 floats; stats: max_symbol, min_symbol, peak_relative_error.
OREF_API int oref_iwave_taps(uint32_t radius, double cell, double depth, float* taps, double* stats)
{
    try {
        ocean::detail::IWaveKernel k;
        ocean::detail::build_iwave_kernel(radius, cell, depth,
                                          ocean::detail::KernelMethod::LeastSquares, k);
        std::memcpy(taps, k.taps.data(), sizeof(float) * k.width * k.width);
        stats[0] = k.max_symbol;
        stats[1] = k.min_symbol;
        stats[2] = k.peak_relative_error;
        return 0;
    } catch (...) {
        return 1;
    }
}

OREF_API void* oref_i_create(const ocean_interaction_desc* d, int* status)
{
    ocean_status st = OCEAN_OK;
    ocean_interaction* f = ocean_interaction_create(d, &st);
    if (status) *status = static_cast<int>(st);
    return f;
}
OREF_API void oref_i_destroy(void* f) { ocean_interaction_destroy(static_cast<ocean_interaction*>(f)); }
OREF_API void oref_i_desc_init(ocean_interaction_desc* d) { ocean_interaction_desc_init(d); }
OREF_API void oref_i_add(void* f, const ocean_disturbance* d)
{
    ocean_interaction_add(static_cast<ocean_interaction*>(f), d);
}
OREF_API void oref_i_update(void* f, float dt) { ocean_interaction_update(static_cast<ocean_interaction*>(f), dt); }
OREF_API int oref_i_recenter(void* f, float x, float z)
{
    return ocean_interaction_recenter(static_cast<ocean_interaction*>(f), x, z);
}
OREF_API void oref_i_set_obstruction(void* f, const uint8_t* m)
{
    ocean_interaction_set_obstruction(static_cast<ocean_interaction*>(f), m);
}
OREF_API void oref_i_buffers(void* f, ocean_interaction_buffers* out)
{
    *out = ocean_interaction_get_buffers(static_cast<ocean_interaction*>(f));
}
OREF_API void oref_i_sample_many(void* f, const float* xz, uint64_t count, ocean_interaction_sample* out)
{
    for (uint64_t i = 0; i < count; ++i)
        ocean_interaction_sample_at(static_cast<ocean_interaction*>(f), xz[2 * i], xz[2 * i + 1], &out[i]);
}
OREF_API float oref_i_fixed_dt(void* f) { return ocean_interaction_fixed_dt(static_cast<ocean_interaction*>(f)); }
OREF_API float oref_i_dt_limit(void* f) { return ocean_interaction_dt_limit(static_cast<ocean_interaction*>(f)); }
OREF_API float oref_i_dispersion_error(void* f)
{
    return ocean_interaction_dispersion_error(static_cast<ocean_interaction*>(f));
}
OREF_API double oref_i_energy(void* f) { return reinterpret_cast<ocean::InteractionField*>(f)->energy(); }
OREF_API uint64_t oref_i_dropped(void* f) { return ocean_interaction_dropped(static_cast<ocean_interaction*>(f)); }
OREF_API void oref_sample_combined_many(void* sim, void* f, const float* xz, uint64_t count, ocean_surface_ex* out)
{
    for (uint64_t i = 0; i < count; ++i)
        ocean_sample_combined(static_cast<ocean_sim*>(sim), static_cast<ocean_interaction*>(f), xz[2 * i],
                              xz[2 * i + 1], &out[i]);
}

// Wall time of `updates` interaction updates of dt each (one disturbance set
// re-queued before every update), for the CPU baseline.
OREF_API double oref_i_time_updates(void* f, const ocean_disturbance* d, uint32_t nd, uint32_t updates, float dt)
{
    auto* h = static_cast<ocean_interaction*>(f);
    const auto start = std::chrono::steady_clock::now();
    for (uint32_t u = 0; u < updates; ++u) {
        for (uint32_t i = 0; i < nd; ++i) ocean_interaction_add(h, &d[i]);
        ocean_interaction_update(h, dt);
    }
    const auto end = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(end - start).count();
}

// The viewer's RGBA16F upload pack (examples/viewer/half.hpp:58-112), the
// scalar path, header-only: compiled from the reference's header.
OREF_API void oref_pack_rgba16(uint16_t* dst, const float* src, const float* alpha, uint64_t cells)
{
    viewer::pack_rgba16_scalar(dst, src, alpha, static_cast<std::size_t>(cells));
}
