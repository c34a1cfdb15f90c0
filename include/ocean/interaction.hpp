// oceanlib-b200 - the local interaction field (iWave) and its composition
// with the FFT ocean (include/ocean/interaction.hpp of the reference). The
// field is stepped on the device; buffers() is a host mirror refreshed by
// update() and recenter().
#pragma once

#include "ocean/cascade.hpp"
#include "ocean/ocean.hpp"

#include <cstddef>
#include <cstdint>
#include <memory>

namespace ocean {

// Boundary condition at obstruction cells (include/ocean/interaction.hpp:27-35).
enum class Obstruction {
    Neumann,    // dEta/dn = 0 (hulls)
    Dirichlet,  // eta = 0
};

// include/ocean/interaction.hpp:37-120.
struct InteractionDesc {
    std::uint32_t size = 256;          // N, a power of two in [32, 1024]
    float extent = 64.0f;              // world edge, metres
    std::uint32_t kernel_radius = 6;   // P; (2P+1)^2 stencil taps
    float damping = 0.20f;             // 1/s
    std::uint32_t absorb_cells = 16;   // absorbing-layer width
    float fixed_dt = 0.0f;             // 0 = derive a stable default
    std::uint32_t max_substeps = 8;
    std::uint32_t max_sources = 64;    // queue capacity per update
    float gravity = 9.81f;
    float depth = 0.0f;                // <= 0 = deep water
    Obstruction obstruction = Obstruction::Neumann;
    ParallelForFn parallel_for = nullptr;  // accepted; the work runs on the GPU
    void* parallel_for_user = nullptr;
    std::uint32_t thread_count = 0;
};

// include/ocean/interaction.hpp:122-128.
enum class SourceKind {
    Impulse,     // one-off; strength in metres
    Continuous,  // ongoing; strength in metres per second
};

// include/ocean/interaction.hpp:130-186.
struct Disturbance {
    float world_x = 0.0f;
    float world_z = 0.0f;
    float radius = 0.35f;
    float strength = 0.25f;
    float velocity_y = 0.0f;
    float velocity_x = 0.0f;   // the source's own horizontal motion, m/s
    float velocity_z = 0.0f;
    SourceKind kind = SourceKind::Impulse;
};

// include/ocean/interaction.hpp:191-196.
struct InteractionSample {
    float height = 0.0f;
    float slope_x = 0.0f;
    float slope_z = 0.0f;
    float velocity_y = 0.0f;
};

// RGBA32F (eta, dEta/dx, dEta/dz, dEta/dt), row-major, NOT periodic
// (include/ocean/interaction.hpp:210-223).
struct InteractionBuffers {
    const float* field = nullptr;
    std::uint32_t size = 0;
    float extent = 0.0f;
    float origin_x = 0.0f;
    float origin_z = 0.0f;
};

// include/ocean/interaction.hpp:229-340. Move-only; the constructor throws
// std::invalid_argument on a malformed descriptor.
class OCEAN_CXX_API InteractionField {
public:
    explicit InteractionField(const InteractionDesc& desc);
    ~InteractionField();

    InteractionField(InteractionField&&) noexcept;
    InteractionField& operator=(InteractionField&&) noexcept;
    InteractionField(const InteractionField&) = delete;
    InteractionField& operator=(const InteractionField&) = delete;

    void add(const Disturbance& d) noexcept;
    [[nodiscard]] std::uint64_t dropped_sources() const noexcept;
    void update(float dt) noexcept;
    [[nodiscard]] std::uint32_t last_substeps() const noexcept;
    [[nodiscard]] bool last_update_clamped() const noexcept;
    void recenter(float world_x, float world_z) noexcept;
    [[nodiscard]] bool recentered() const noexcept;
    [[nodiscard]] std::int32_t last_shift_x() const noexcept;
    [[nodiscard]] std::int32_t last_shift_z() const noexcept;
    void set_obstruction(const std::uint8_t* mask) noexcept;
    [[nodiscard]] InteractionSample sample_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] float height_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] InteractionBuffers buffers() const noexcept;
    [[nodiscard]] const InteractionDesc& desc() const noexcept;
    [[nodiscard]] float fixed_dt() const noexcept;
    [[nodiscard]] float stable_dt_limit() const noexcept;
    [[nodiscard]] float kernel_dispersion_error() const noexcept;
    [[nodiscard]] double energy() const noexcept;

    // Not in the reference: the C handle behind this object (an
    // ocean_interaction* of include/ocean/ocean.h).
    [[nodiscard]] void* c_handle() const noexcept;

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

// The FFT surface (one Ocean or a CascadeStack) plus the interaction field
// (include/ocean/interaction.hpp:352-398): heights add, vertical velocities
// add, normals compose through slopes. Holds references only.
class OCEAN_CXX_API WaterSurface {
public:
    WaterSurface(const Ocean& ocean, const InteractionField& field) noexcept;
    WaterSurface(const CascadeStack& stack, const InteractionField& field) noexcept;

    [[nodiscard]] Surface sample_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] float height_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] InteractionSample interaction_at(float world_x, float world_z) const noexcept;

private:
    const Ocean* ocean_ = nullptr;
    const CascadeStack* stack_ = nullptr;
    const InteractionField* field_ = nullptr;
};

}  // namespace ocean
