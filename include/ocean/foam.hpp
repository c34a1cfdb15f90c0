// oceanlib-b200 - persistent advected foam (include/ocean/foam.hpp of the
// reference), implemented on the B200: the foam grid lives on the device, the
// semi-Lagrangian substeps are device launches, and data() is a host mirror
// refreshed after each update that stepped.
#pragma once

#include "ocean/ocean.hpp"

#include <cstddef>
#include <cstdint>
#include <memory>

namespace ocean {

// include/ocean/foam.hpp:17-86.
struct FoamDesc {
    float decay = 0.35f;              // 1/s, exponential fade
    float source_gain = 4.0f;         // Jacobian-foam injection per second
    float advect_scale = 1.0f;        // multiplier on the orbital velocity
    float wind_drift_x = 0.0f;        // extra drift, m/s
    float wind_drift_z = 0.0f;
    float fixed_dt = 1.0f / 60.0f;    // substep length, seconds
    std::uint32_t max_substeps = 4;   // backlog clamp per update
    ParallelForFn parallel_for = nullptr;  // accepted; the work runs on the GPU
    void* parallel_for_user = nullptr;
    std::uint32_t thread_count = 0;
};

// include/ocean/foam.hpp:88-142. Bound to one Ocean, which must outlive it
// and must have compute_velocity set (std::invalid_argument otherwise, as in
// the reference). update(dt) accumulates dt and runs whole fixed_dt
// substeps on the ocean's current frame, with the reference's arithmetic.
class OCEAN_CXX_API FoamField {
public:
    FoamField(const Ocean& ocean, const FoamDesc& desc);
    ~FoamField();

    FoamField(FoamField&&) noexcept;
    FoamField& operator=(FoamField&&) noexcept;
    FoamField(const FoamField&) = delete;
    FoamField& operator=(const FoamField&) = delete;

    void update(float dt) noexcept;
    void clear() noexcept;

    [[nodiscard]] const float* data() const noexcept;   // N*N floats, row-major
    [[nodiscard]] std::uint32_t size() const noexcept;
    [[nodiscard]] float foam_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] const FoamDesc& desc() const noexcept;

    // Keeps fixed_dt, max_substeps and the threading fields of the current
    // descriptor (as the reference does); throws std::invalid_argument.
    void set_desc(const FoamDesc& desc);
    [[nodiscard]] std::uint32_t last_substeps() const noexcept;
    [[nodiscard]] double coverage() const noexcept;

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

}  // namespace ocean
