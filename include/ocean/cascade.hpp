// oceanlib-b200 - cascaded patches summed at query time (include/ocean/cascade.hpp
// of the reference). Levels of equal size advance in one batched device
// launch per update; each level's Buffers are a host mirror refreshed by
// update(), and the summed query runs on the device.
#pragma once

#include "ocean/ocean.hpp"

#include <cstddef>
#include <initializer_list>
#include <memory>
#include <span>

namespace ocean {

// include/ocean/cascade.hpp:43.
using CascadeLevel = OceanDesc;

// include/ocean/cascade.hpp:45-92. At least one and at most 8 levels;
// std::invalid_argument for a malformed level or level count.
class OCEAN_CXX_API CascadeStack {
public:
    explicit CascadeStack(std::span<const CascadeLevel> levels);
    CascadeStack(std::initializer_list<CascadeLevel> levels);
    ~CascadeStack();

    CascadeStack(CascadeStack&&) noexcept;
    CascadeStack& operator=(CascadeStack&&) noexcept;
    CascadeStack(const CascadeStack&) = delete;
    CascadeStack& operator=(const CascadeStack&) = delete;

    void update(double time) noexcept;

    [[nodiscard]] std::size_t level_count() const noexcept;
    [[nodiscard]] Buffers buffers(std::size_t level) const noexcept;
    [[nodiscard]] const OceanDesc& desc(std::size_t level) const noexcept;
    // A read-only Ocean view of one level (its buffers, queries, desc, time).
    [[nodiscard]] const Ocean& level(std::size_t level) const noexcept;

    [[nodiscard]] float height_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] Surface sample_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] double time() const noexcept;

private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

}  // namespace ocean
