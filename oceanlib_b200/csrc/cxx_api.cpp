// oceanlib-b200: the reference's C++ API (include/ocean/ocean.hpp, foam.hpp,
// cascade.hpp, interaction.hpp) over the library's device objects.
//
//   Ocean            - owns an ocean_sim (one-ocean batch + pinned host
//                      mirror); or, for CascadeStack::level(), a read-only
//                      view of one cascade level's device and mirror buffers.
//   FoamField        - the foam grid on the device (ping-pong), the
//                      reference's fixed-step accumulator on the host, one
//                      foam_step launch per substep, a host mirror for data().
//   CascadeStack     - an ocean_cascade (levels of one size in one launch)
//                      plus per-level host mirrors refreshed by update().
//   InteractionField - an ocean_interaction.
//   WaterSurface     - the composed query of src/interaction.cpp:863-908.
//
// Every computation is a device launch reached through the C ABI or the
// kernel launchers; this file only converts descriptors, owns buffers and
// maps failures to the reference's exceptions (constructors) or to neutral
// results (noexcept members), as the reference's noexcept API must.
#include "../../include/ocean/cascade.hpp"
#include "../../include/ocean/foam.hpp"
#include "../../include/ocean/interaction.hpp"
#include "../../include/ocean/ocean.hpp"
#include "../../include/ocean_b200.h"
#include "host_util.h"
#include "spectrum.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace ocean {
namespace {

using ocean_b200::check;
using ocean_b200::DevBuf;
using ocean_b200::HostBuf;
using ocean_b200::SurfaceEx;

[[noreturn]] void raise(ocean_status st, const char* what)
{
    switch (st) {
        case OCEAN_ERROR_INVALID_ARG: throw std::invalid_argument(std::string("ocean: invalid ") + what);
        case OCEAN_ERROR_OUT_OF_MEMORY: throw std::bad_alloc();
        default: throw std::runtime_error(std::string("ocean: ") + what + ": " + ocean_status_string(st));
    }
}

// OceanDesc -> ocean_desc (the C ABI's struct, include/ocean/ocean.h:99-137).
ocean_desc to_c(const OceanDesc& d)
{
    ocean_desc c;
    ocean_desc_init(&c);
    c.size = d.size;
    c.patch_length = d.patch_length;
    c.spectrum.wind_speed = d.spectrum.wind_speed;
    c.spectrum.fetch = d.spectrum.fetch;
    c.spectrum.wind_direction = d.spectrum.wind_direction;
    c.spectrum.peak_enhancement = d.spectrum.peak_enhancement;
    c.spectrum.swell = d.spectrum.swell;
    c.spectrum.small_wave_cutoff = d.spectrum.small_wave_cutoff;
    c.spectrum.gravity = d.spectrum.gravity;
    c.water_depth = d.spectrum.depth;
    c.choppiness = d.choppiness;
    c.foam_threshold = d.foam_threshold;
    c.seed = d.seed;
    c.parallel_for = reinterpret_cast<ocean_parallel_for_fn>(d.parallel_for);
    c.parallel_for_user = d.parallel_for_user;
    c.thread_count = d.thread_count;
    c.compute_velocity = d.compute_velocity ? 1 : 0;
    return c;
}

Surface to_surface(const ocean_surface_ex& s)
{
    Surface o;
    o.height = s.height;
    o.offset_x = s.offset_x;
    o.offset_z = s.offset_z;
    o.normal_x = s.normal_x;
    o.normal_y = s.normal_y;
    o.normal_z = s.normal_z;
    o.foam = s.foam;
    o.velocity_x = s.velocity_x;
    o.velocity_y = s.velocity_y;
    o.velocity_z = s.velocity_z;
    return o;
}

InteractionSample to_sample(const ocean_interaction_sample& e)
{
    InteractionSample o;
    o.height = e.height;
    o.slope_x = e.slope_x;
    o.slope_z = e.slope_z;
    o.velocity_y = e.velocity_y;
    return o;
}

// The composition of src/interaction.cpp:863-900: heights and vertical
// velocities add, normals compose through slopes where the FFT normal points
// up, and stay as they are inside a fold.
Surface compose(Surface s, const InteractionSample& e)
{
    s.height += e.height;
    s.velocity_y += e.velocity_y;
    if (s.normal_y > 1.0e-6f) {
        const float inv = 1.0f / s.normal_y;
        const float sx = -s.normal_x * inv + e.slope_x;
        const float sz = -s.normal_z * inv + e.slope_z;
        const float len = std::sqrt(sx * sx + sz * sz + 1.0f);
        const float il = 1.0f / len;
        s.normal_x = -sx * il;
        s.normal_y = il;
        s.normal_z = -sz * il;
    }
    return s;
}

// One-point device query scratch (a device record each way and its pinned
// host staging), allocated once.
struct PointQuery {
    DevBuf<float2> in{1};
    DevBuf<SurfaceEx> out{1};
    HostBuf<float2> host_in{1};
    HostBuf<SurfaceEx> host_out{1};
    std::mutex mutex;
};

}  // namespace

// ---------------------------------------------------------------------------
// Ocean
// ---------------------------------------------------------------------------
struct Ocean::Impl {
    OceanDesc desc;
    ocean_sim* sim = nullptr;  // owned; null for a cascade-level view

    // Cascade-level view: the level's mirrors, device buffers and the
    // stack's time (all owned by the CascadeStack, which outlives the view).
    const float* mirror[3] = {nullptr, nullptr, nullptr};
    ocean_device_buffers dev{};
    const double* stack_time = nullptr;
    std::unique_ptr<PointQuery> query;

    ~Impl()
    {
        if (sim != nullptr) ocean_destroy(sim);
    }

    ocean_device_buffers device() const
    {
        if (sim == nullptr) return dev;
        ocean_device_buffers d{};
        if (ocean_get_device_buffers(sim, &d) != OCEAN_OK) std::memset(&d, 0, sizeof(d));
        return d;
    }

    Surface sample(float x, float z) const
    {
        if (sim != nullptr) {
            ocean_surface_ex ex;
            ocean_sample_ex(sim, x, z, &ex);
            return to_surface(ex);
        }
        Surface s;
        try {
            std::lock_guard<std::mutex> lock(query->mutex);
            query->host_in.p[0] = make_float2(x, z);
            check(cudaMemcpy(query->in.p, query->host_in.p, sizeof(float2), cudaMemcpyHostToDevice), "query");
            check(ocean_b200::launch_sample(static_cast<int>(desc.size),
                                            static_cast<float>(desc.size) / desc.patch_length,
                                            reinterpret_cast<const float4*>(dev.displacement),
                                            reinterpret_cast<const float4*>(dev.normal),
                                            reinterpret_cast<const float4*>(dev.velocity), query->in.p, 1,
                                            query->out.p, nullptr),
                  "query kernel");
            check(cudaMemcpy(query->host_out.p, query->out.p, sizeof(SurfaceEx), cudaMemcpyDeviceToHost),
                  "query");
            ocean_surface_ex ex;
            static_assert(sizeof(ex) == sizeof(SurfaceEx), "layout");
            std::memcpy(&ex, query->host_out.p, sizeof(ex));
            s = to_surface(ex);
        } catch (...) {
            s = Surface{};
        }
        return s;
    }
};

Ocean::Ocean(const OceanDesc& desc) : impl_(std::make_unique<Impl>())
{
    impl_->desc = desc;
    const ocean_desc c = to_c(desc);
    ocean_status st = OCEAN_ERROR_UNKNOWN;
    impl_->sim = ocean_create(&c, &st);
    if (impl_->sim == nullptr) raise(st, "OceanDesc");
}

Ocean::Ocean(std::unique_ptr<Impl> impl) noexcept : impl_(std::move(impl)) {}
Ocean::~Ocean() = default;
Ocean::Ocean(Ocean&&) noexcept = default;
Ocean& Ocean::operator=(Ocean&&) noexcept = default;

void Ocean::update(double time) noexcept
{
    if (impl_ && impl_->sim != nullptr) ocean_update(impl_->sim, time);
}

Buffers Ocean::buffers() const noexcept
{
    Buffers b;
    if (!impl_) return b;
    b.size = impl_->desc.size;
    b.patch_length = impl_->desc.patch_length;
    if (impl_->sim != nullptr) {
        const ocean_buffers c = ocean_get_buffers(impl_->sim);
        b.displacement = c.displacement;
        b.normal = c.normal;
        b.velocity = ocean_get_velocity(impl_->sim);
    } else {
        b.displacement = impl_->mirror[0];
        b.normal = impl_->mirror[1];
        b.velocity = impl_->mirror[2];
    }
    return b;
}

float Ocean::height_at(float world_x, float world_z) const noexcept
{
    return sample_at(world_x, world_z).height;
}

Surface Ocean::sample_at(float world_x, float world_z) const noexcept
{
    if (!impl_) return Surface{};
    return impl_->sample(world_x, world_z);
}

const OceanDesc& Ocean::desc() const noexcept { return impl_->desc; }

double Ocean::time() const noexcept
{
    if (!impl_) return 0.0;
    if (impl_->sim != nullptr) return ocean_get_time(impl_->sim);
    return impl_->stack_time != nullptr ? *impl_->stack_time : 0.0;
}

void* Ocean::c_handle() const noexcept { return impl_ ? impl_->sim : nullptr; }

// ---------------------------------------------------------------------------
// FoamField (src/foam.cpp)
// ---------------------------------------------------------------------------
namespace {

void validate_foam(const FoamDesc& d)
{
    // src/foam.cpp:146-164.
    if (!(d.decay >= 0.0f)) throw std::invalid_argument("ocean: foam decay must be non-negative");
    if (!(d.source_gain >= 0.0f)) throw std::invalid_argument("ocean: foam source_gain must be non-negative");
    if (!(d.fixed_dt > 0.0f)) throw std::invalid_argument("ocean: foam fixed_dt must be positive");
    if (d.max_substeps < 1) throw std::invalid_argument("ocean: foam max_substeps must be >= 1");
    if (!std::isfinite(d.advect_scale) || !std::isfinite(d.wind_drift_x) || !std::isfinite(d.wind_drift_z))
        throw std::invalid_argument("ocean: foam drift parameters must be finite");
}

}  // namespace

struct FoamField::Impl {
    const Ocean* ocean = nullptr;
    FoamDesc desc;
    uint32_t n = 0;
    size_t cells = 0;
    float cell = 0.0f;  // metres per cell
    DevBuf<float> buf[2];
    int cur = 0;
    HostBuf<float> mirror;
    double accum = 0.0;
    uint32_t substeps_last = 0;
    cudaStream_t stream = nullptr;
    DevBuf<double> cov{1};
    HostBuf<double> host_cov{1};
    DevBuf<float2> q_in{1};
    DevBuf<float> q_out{1};
    HostBuf<float2> host_q_in{1};
    HostBuf<float> host_q_out{1};
    mutable std::mutex mutex;

    ~Impl()
    {
        if (stream != nullptr) {
            cudaStreamSynchronize(stream);
            cudaStreamDestroy(stream);
        }
    }

    // The fixed-step accumulator of FoamField::update (src/foam.cpp:218-252).
    uint32_t accumulate(float dt)
    {
        if (!(dt > 0.0f)) dt = 0.0f;
        accum += static_cast<double>(dt);
        const double step = static_cast<double>(desc.fixed_dt);
        const double eps = step * 1e-6;
        uint32_t steps = 0;
        if (accum + eps >= step) steps = static_cast<uint32_t>((accum + eps) / step);
        if (steps > desc.max_substeps) {
            steps = desc.max_substeps;
            accum = 0.0;
        } else {
            accum -= static_cast<double>(steps) * step;
            if (accum < 0.0) accum = 0.0;
        }
        substeps_last = steps;
        return steps;
    }

    void refresh_mirror()
    {
        check(cudaMemcpyAsync(mirror.p, buf[cur].p, cells * sizeof(float), cudaMemcpyDeviceToHost, stream), "copy");
        check(cudaStreamSynchronize(stream), "foam");
    }
};

FoamField::FoamField(const Ocean& ocean, const FoamDesc& desc)
{
    validate_foam(desc);
    const Buffers b = ocean.buffers();
    if (b.velocity == nullptr)
        throw std::invalid_argument("ocean: FoamField requires OceanDesc::compute_velocity to be set");
    impl_ = std::make_unique<Impl>();
    Impl& m = *impl_;
    m.ocean = &ocean;
    m.desc = desc;
    m.n = b.size;
    m.cells = static_cast<size_t>(b.size) * b.size;
    m.cell = b.patch_length / static_cast<float>(b.size);
    m.buf[0] = DevBuf<float>(m.cells);
    m.buf[1] = DevBuf<float>(m.cells);
    m.mirror = HostBuf<float>(m.cells);
    check(cudaStreamCreateWithFlags(&m.stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check(cudaMemsetAsync(m.buf[0].p, 0, m.cells * sizeof(float), m.stream), "memset");
    check(cudaMemsetAsync(m.buf[1].p, 0, m.cells * sizeof(float), m.stream), "memset");
    check(cudaStreamSynchronize(m.stream), "foam init");
}

FoamField::~FoamField() = default;
FoamField::FoamField(FoamField&&) noexcept = default;
FoamField& FoamField::operator=(FoamField&&) noexcept = default;

void FoamField::update(float dt) noexcept
{
    if (!impl_) return;
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lock(m.mutex);
    const uint32_t steps = m.accumulate(dt);
    if (steps == 0) return;
    const ocean_device_buffers d = m.ocean->impl_->device();
    if (d.velocity == nullptr) return;  // the ocean was moved from
    // Per substep, as src/foam.cpp:89-99 evaluates them (in float, host libm).
    const float fdt = m.desc.fixed_dt;
    const float decay = std::exp(-m.desc.decay * fdt);
    const float gain = m.desc.source_gain * fdt;
    const float inv_cell = 1.0f / m.cell;
    try {
        for (uint32_t s = 0; s < steps; ++s) {
            check(ocean_b200::launch_foam_step(static_cast<int>(m.n), 1,
                                               reinterpret_cast<const float4*>(d.displacement),
                                               reinterpret_cast<const float4*>(d.velocity), m.buf[m.cur].p,
                                               m.buf[1 - m.cur].p, fdt, decay, gain, m.desc.advect_scale,
                                               m.desc.wind_drift_x, m.desc.wind_drift_z, inv_cell, m.stream),
                  "foam step");
            m.cur = 1 - m.cur;
        }
        m.refresh_mirror();
    } catch (...) {
    }
}

void FoamField::clear() noexcept
{
    if (!impl_) return;
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lock(m.mutex);
    try {
        check(cudaMemsetAsync(m.buf[0].p, 0, m.cells * sizeof(float), m.stream), "memset");
        check(cudaMemsetAsync(m.buf[1].p, 0, m.cells * sizeof(float), m.stream), "memset");
        m.refresh_mirror();
    } catch (...) {
    }
    m.accum = 0.0;
}

const float* FoamField::data() const noexcept { return impl_ ? impl_->mirror.p : nullptr; }
std::uint32_t FoamField::size() const noexcept { return impl_ ? impl_->n : 0u; }
const FoamDesc& FoamField::desc() const noexcept { return impl_->desc; }

void FoamField::set_desc(const FoamDesc& d)
{
    validate_foam(d);
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lock(m.mutex);
    // src/foam.cpp:265-283: the construction-time fields stay.
    FoamDesc next = d;
    next.fixed_dt = m.desc.fixed_dt;
    next.max_substeps = m.desc.max_substeps;
    next.parallel_for = m.desc.parallel_for;
    next.parallel_for_user = m.desc.parallel_for_user;
    next.thread_count = m.desc.thread_count;
    m.desc = next;
}

std::uint32_t FoamField::last_substeps() const noexcept { return impl_ ? impl_->substeps_last : 0u; }

float FoamField::foam_at(float world_x, float world_z) const noexcept
{
    if (!impl_) return 0.0f;
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lock(m.mutex);
    const ocean_device_buffers d = m.ocean->impl_->device();
    if (d.displacement == nullptr) return 0.0f;
    try {
        m.host_q_in.p[0] = make_float2(world_x, world_z);
        check(cudaMemcpyAsync(m.q_in.p, m.host_q_in.p, sizeof(float2), cudaMemcpyHostToDevice, m.stream), "query");
        check(ocean_b200::launch_foam_at(static_cast<int>(m.n),
                                         static_cast<float>(m.n) / m.ocean->desc().patch_length, m.cell,
                                         reinterpret_cast<const float4*>(d.displacement),
                                         reinterpret_cast<const float4*>(d.normal), m.buf[m.cur].p, m.q_in.p, 1,
                                         m.q_out.p, m.stream),
              "foam_at");
        check(cudaMemcpyAsync(m.host_q_out.p, m.q_out.p, sizeof(float), cudaMemcpyDeviceToHost, m.stream), "query");
        check(cudaStreamSynchronize(m.stream), "foam_at");
        return m.host_q_out.p[0];
    } catch (...) {
        return 0.0f;
    }
}

double FoamField::coverage() const noexcept
{
    if (!impl_) return 0.0;
    Impl& m = *impl_;
    std::lock_guard<std::mutex> lock(m.mutex);
    try {
        check(ocean_b200::launch_foam_coverage(m.buf[m.cur].p, m.cells, m.cov.p, m.stream), "coverage");
        check(cudaMemcpyAsync(m.host_cov.p, m.cov.p, sizeof(double), cudaMemcpyDeviceToHost, m.stream), "copy");
        check(cudaStreamSynchronize(m.stream), "coverage");
        return m.host_cov.p[0];
    } catch (...) {
        return 0.0;
    }
}

// ---------------------------------------------------------------------------
// CascadeStack (src/cascade.cpp)
// ---------------------------------------------------------------------------
struct CascadeStack::Impl {
    ocean_cascade* cascade = nullptr;
    std::vector<OceanDesc> descs;
    std::vector<HostBuf<float>> mirrors;  // 3 per level: disp, normal, velocity
    std::vector<ocean_device_buffers> dev;
    std::vector<Ocean> views;
    double time = 0.0;

    ~Impl()
    {
        views.clear();
        if (cascade != nullptr) ocean_cascade_destroy(cascade);
    }

    void refresh()
    {
        if (ocean_cascade_synchronize(cascade) != OCEAN_OK) throw std::runtime_error("ocean: cascade update failed");
        for (size_t i = 0; i < descs.size(); ++i) {
            const size_t bytes = static_cast<size_t>(descs[i].size) * descs[i].size * sizeof(float4);
            check(cudaMemcpy(mirrors[3 * i].p, dev[i].displacement, bytes, cudaMemcpyDeviceToHost), "copy");
            check(cudaMemcpy(mirrors[3 * i + 1].p, dev[i].normal, bytes, cudaMemcpyDeviceToHost), "copy");
            if (dev[i].velocity != nullptr)
                check(cudaMemcpy(mirrors[3 * i + 2].p, dev[i].velocity, bytes, cudaMemcpyDeviceToHost), "copy");
        }
        time = ocean_cascade_get_time(cascade);
    }
};

CascadeStack::CascadeStack(std::span<const CascadeLevel> levels) : impl_(std::make_unique<Impl>())
{
    Impl& m = *impl_;
    if (levels.empty()) throw std::invalid_argument("ocean: CascadeStack needs at least one level");
    std::vector<ocean_desc> c;
    for (const CascadeLevel& l : levels) {
        m.descs.push_back(l);
        c.push_back(to_c(l));
    }
    ocean_status st = OCEAN_ERROR_UNKNOWN;
    m.cascade = ocean_cascade_create(c.data(), static_cast<uint32_t>(c.size()), &st);
    if (m.cascade == nullptr) raise(st, "cascade level");
    m.dev.resize(m.descs.size());
    for (size_t i = 0; i < m.descs.size(); ++i) {
        if (ocean_cascade_level_device_buffers(m.cascade, static_cast<uint32_t>(i), &m.dev[i]) != OCEAN_OK)
            raise(OCEAN_ERROR_UNKNOWN, "cascade level buffers");
        const size_t floats = static_cast<size_t>(m.descs[i].size) * m.descs[i].size * 4;
        m.mirrors.emplace_back(floats);
        m.mirrors.emplace_back(floats);
        m.mirrors.emplace_back(m.dev[i].velocity != nullptr ? floats : 0);
    }
    m.refresh();
    for (size_t i = 0; i < m.descs.size(); ++i) {
        auto v = std::make_unique<Ocean::Impl>();
        v->desc = m.descs[i];
        v->mirror[0] = m.mirrors[3 * i].p;
        v->mirror[1] = m.mirrors[3 * i + 1].p;
        v->mirror[2] = m.mirrors[3 * i + 2].p;
        v->dev = m.dev[i];
        v->stack_time = &m.time;
        v->query = std::make_unique<PointQuery>();
        m.views.push_back(Ocean(std::move(v)));
    }
}

CascadeStack::CascadeStack(std::initializer_list<CascadeLevel> levels)
    : CascadeStack(std::span<const CascadeLevel>(levels.begin(), levels.size()))
{
}

CascadeStack::~CascadeStack() = default;
CascadeStack::CascadeStack(CascadeStack&&) noexcept = default;
CascadeStack& CascadeStack::operator=(CascadeStack&&) noexcept = default;

void CascadeStack::update(double time) noexcept
{
    if (!impl_) return;
    if (ocean_cascade_update(impl_->cascade, time, nullptr) != OCEAN_OK) return;
    try {
        impl_->refresh();
    } catch (...) {
    }
}

std::size_t CascadeStack::level_count() const noexcept { return impl_ ? impl_->descs.size() : 0; }

Buffers CascadeStack::buffers(std::size_t level) const noexcept
{
    if (!impl_ || level >= impl_->views.size()) return Buffers{};
    return impl_->views[level].buffers();
}

const OceanDesc& CascadeStack::desc(std::size_t level) const noexcept { return impl_->descs[level]; }
const Ocean& CascadeStack::level(std::size_t level) const noexcept { return impl_->views[level]; }

float CascadeStack::height_at(float world_x, float world_z) const noexcept
{
    return sample_at(world_x, world_z).height;
}

Surface CascadeStack::sample_at(float world_x, float world_z) const noexcept
{
    if (!impl_) return Surface{};
    const float xz[2] = {world_x, world_z};
    ocean_surface_ex ex;
    if (ocean_cascade_sample_many(impl_->cascade, xz, 1, &ex, 4, 0.0f, 0, nullptr) != OCEAN_OK) return Surface{};
    return to_surface(ex);
}

double CascadeStack::time() const noexcept { return impl_ ? impl_->time : 0.0; }

// ---------------------------------------------------------------------------
// InteractionField and WaterSurface (src/interaction.cpp)
// ---------------------------------------------------------------------------
struct InteractionField::Impl {
    InteractionDesc desc;
    ocean_interaction* field = nullptr;
    ~Impl()
    {
        if (field != nullptr) ocean_interaction_destroy(field);
    }
};

InteractionField::InteractionField(const InteractionDesc& desc) : impl_(std::make_unique<Impl>())
{
    impl_->desc = desc;
    ocean_interaction_desc c;
    ocean_interaction_desc_init(&c);
    c.size = desc.size;
    c.extent = desc.extent;
    c.kernel_radius = desc.kernel_radius;
    c.damping = desc.damping;
    c.absorb_cells = desc.absorb_cells;
    c.fixed_dt = desc.fixed_dt;
    c.max_substeps = desc.max_substeps;
    c.max_sources = desc.max_sources;
    c.gravity = desc.gravity;
    c.water_depth = desc.depth;
    c.obstruction = desc.obstruction == Obstruction::Dirichlet ? OCEAN_OBSTRUCTION_DIRICHLET
                                                              : OCEAN_OBSTRUCTION_NEUMANN;
    c.parallel_for = reinterpret_cast<ocean_parallel_for_fn>(desc.parallel_for);
    c.parallel_for_user = desc.parallel_for_user;
    c.thread_count = desc.thread_count;
    ocean_status st = OCEAN_ERROR_UNKNOWN;
    impl_->field = ocean_interaction_create(&c, &st);
    if (impl_->field == nullptr) raise(st, "InteractionDesc");
}

InteractionField::~InteractionField() = default;
InteractionField::InteractionField(InteractionField&&) noexcept = default;
InteractionField& InteractionField::operator=(InteractionField&&) noexcept = default;

void InteractionField::add(const Disturbance& d) noexcept
{
    if (!impl_) return;
    ocean_disturbance c;
    c.world_x = d.world_x;
    c.world_z = d.world_z;
    c.radius = d.radius;
    c.strength = d.strength;
    c.velocity_y = d.velocity_y;
    c.velocity_x = d.velocity_x;
    c.velocity_z = d.velocity_z;
    c.kind = d.kind == SourceKind::Continuous ? OCEAN_SOURCE_CONTINUOUS : OCEAN_SOURCE_IMPULSE;
    ocean_interaction_add(impl_->field, &c);
}

std::uint64_t InteractionField::dropped_sources() const noexcept
{
    return impl_ ? ocean_interaction_dropped(impl_->field) : 0u;
}

void InteractionField::update(float dt) noexcept
{
    if (impl_) ocean_interaction_update(impl_->field, dt);
}

std::uint32_t InteractionField::last_substeps() const noexcept
{
    return impl_ ? ocean_interaction_last_substeps(impl_->field) : 0u;
}

bool InteractionField::last_update_clamped() const noexcept
{
    return impl_ && ocean_interaction_last_clamped(impl_->field) != 0;
}

void InteractionField::recenter(float world_x, float world_z) noexcept
{
    if (impl_) ocean_interaction_recenter(impl_->field, world_x, world_z);
}

bool InteractionField::recentered() const noexcept
{
    return last_shift_x() != 0 || last_shift_z() != 0;
}

std::int32_t InteractionField::last_shift_x() const noexcept
{
    int32_t dx = 0, dz = 0;
    if (impl_) ocean_interaction_last_shift(impl_->field, &dx, &dz);
    return dx;
}

std::int32_t InteractionField::last_shift_z() const noexcept
{
    int32_t dx = 0, dz = 0;
    if (impl_) ocean_interaction_last_shift(impl_->field, &dx, &dz);
    return dz;
}

void InteractionField::set_obstruction(const std::uint8_t* mask) noexcept
{
    if (impl_) ocean_interaction_set_obstruction(impl_->field, mask);
}

InteractionSample InteractionField::sample_at(float world_x, float world_z) const noexcept
{
    if (!impl_) return InteractionSample{};
    ocean_interaction_sample e;
    ocean_interaction_sample_at(impl_->field, world_x, world_z, &e);
    return to_sample(e);
}

float InteractionField::height_at(float world_x, float world_z) const noexcept
{
    return impl_ ? ocean_interaction_height_at(impl_->field, world_x, world_z) : 0.0f;
}

InteractionBuffers InteractionField::buffers() const noexcept
{
    InteractionBuffers b;
    if (!impl_) return b;
    const ocean_interaction_buffers c = ocean_interaction_get_buffers(impl_->field);
    b.field = c.field;
    b.size = c.size;
    b.extent = c.extent;
    b.origin_x = c.origin_x;
    b.origin_z = c.origin_z;
    return b;
}

const InteractionDesc& InteractionField::desc() const noexcept { return impl_->desc; }

float InteractionField::fixed_dt() const noexcept
{
    return impl_ ? ocean_interaction_fixed_dt(impl_->field) : 0.0f;
}

float InteractionField::stable_dt_limit() const noexcept
{
    return impl_ ? ocean_interaction_dt_limit(impl_->field) : 0.0f;
}

float InteractionField::kernel_dispersion_error() const noexcept
{
    return impl_ ? ocean_interaction_dispersion_error(impl_->field) : 0.0f;
}

double InteractionField::energy() const noexcept
{
    return impl_ ? ocean_interaction_energy(impl_->field) : 0.0;
}

void* InteractionField::c_handle() const noexcept { return impl_ ? impl_->field : nullptr; }

WaterSurface::WaterSurface(const Ocean& ocean, const InteractionField& field) noexcept
    : ocean_(&ocean), field_(&field)
{
}

WaterSurface::WaterSurface(const CascadeStack& stack, const InteractionField& field) noexcept
    : stack_(&stack), field_(&field)
{
}

InteractionSample WaterSurface::interaction_at(float world_x, float world_z) const noexcept
{
    return field_->sample_at(world_x, world_z);
}

Surface WaterSurface::sample_at(float world_x, float world_z) const noexcept
{
    if (ocean_ != nullptr && ocean_->c_handle() != nullptr) {
        // One device launch for the composed query (ocean_sample_combined).
        ocean_surface_ex ex;
        ocean_sample_combined(static_cast<const ocean_sim*>(ocean_->c_handle()),
                              static_cast<const ocean_interaction*>(field_->c_handle()), world_x, world_z, &ex);
        return to_surface(ex);
    }
    const Surface s = stack_ != nullptr ? stack_->sample_at(world_x, world_z) : ocean_->sample_at(world_x, world_z);
    return compose(s, field_->sample_at(world_x, world_z));
}

float WaterSurface::height_at(float world_x, float world_z) const noexcept
{
    const float base = stack_ != nullptr ? stack_->height_at(world_x, world_z) : ocean_->height_at(world_x, world_z);
    return base + field_->height_at(world_x, world_z);
}

}  // namespace ocean
