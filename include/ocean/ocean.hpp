// oceanlib-b200 - the C++ API of the reference (include/ocean/ocean.hpp of
// DarshanVShah/oceanlib), implemented on the B200.
//
// The same namespace, types, members, defaults and semantics as the
// reference's header, so C++ code written against it recompiles and relinks
// against libocean_b200.so unchanged. What differs is where the work runs:
// every update is device work (hand-written sm_100a kernels), and the Buffers
// an Ocean hands out are a pinned host mirror that update() refreshes, so the
// reference's "pointers valid until destruction, rewritten in place" holds.
// The thread-pool fields (parallel_for, thread_count) are accepted with the
// reference's meaning where one exists: a parallel_for hook is called exactly
// four times per update, once per device stage.
#pragma once

#include <cstddef>
#include <cstdint>
#include <memory>

#if defined(_WIN32)
#define OCEAN_CXX_API __declspec(dllexport)
#else
#define OCEAN_CXX_API __attribute__((visibility("default")))
#endif

namespace ocean {

// One unit of work over index in [0, count) (include/ocean/ocean.hpp:19).
using TaskFn = void (*)(void* ctx, std::uint32_t index);

// Blocking parallel-for hook (include/ocean/ocean.hpp:32-33): must run
// task(ctx, i) for every i in [0, count) and return only when all are done.
using ParallelForFn = void (*)(void* user, TaskFn task, void* ctx, std::uint32_t count);

// JONSWAP spectrum and directional spreading (include/ocean/ocean.hpp:41-86).
struct SpectrumDesc {
    float wind_speed = 10.0f;         // U10, m/s
    float fetch = 100000.0f;          // metres of open water
    float wind_direction = 0.0f;      // radians, 0 = +X
    float peak_enhancement = 3.3f;    // JONSWAP gamma (1 = Pierson-Moskowitz)
    float swell = 0.0f;               // 0 wind sea .. 1 narrow swell
    float small_wave_cutoff = 0.5f;   // metres; shorter waves are rolled off
    float gravity = 9.81f;
    float depth = 0.0f;               // metres; <= 0 = deep water
};

// include/ocean/ocean.hpp:88-133.
struct OceanDesc {
    std::uint32_t size = 256;         // N, a power of two in [16, 4096]
    float patch_length = 200.0f;      // tile edge, metres
    SpectrumDesc spectrum{};
    float choppiness = 1.0f;          // Tessendorf's lambda
    float foam_threshold = 0.5f;      // Jacobian below which foam appears
    std::uint64_t seed = 1337;
    ParallelForFn parallel_for = nullptr;  // called 4x per update when set
    void* parallel_for_user = nullptr;
    std::uint32_t thread_count = 0;   // accepted; the work runs on the GPU
    bool compute_velocity = false;    // orbital velocity (six transforms)
};

// Alignment the reference promises for its output buffers
// (include/ocean/ocean.hpp:141); the host mirror here is page-aligned.
inline constexpr std::size_t kBufferAlignment = 64;

// RGBA32F-shaped outputs, row-major i = z * size + x
// (include/ocean/ocean.hpp:143-171):
//   displacement = (dx, dy, dz, foam), normal = (nx, ny, nz, jacobian),
//   velocity = (vx, vy, vz, 0) or null without compute_velocity.
struct Buffers {
    const float* displacement = nullptr;
    const float* normal = nullptr;
    const float* velocity = nullptr;
    std::uint32_t size = 0;
    float patch_length = 0.0f;
};

// One world-space surface query (include/ocean/ocean.hpp:174-188).
struct Surface {
    float height = 0.0f;
    float offset_x = 0.0f;
    float offset_z = 0.0f;
    float normal_x = 0.0f;
    float normal_y = 1.0f;
    float normal_z = 0.0f;
    float foam = 0.0f;
    float velocity_x = 0.0f;
    float velocity_y = 0.0f;
    float velocity_z = 0.0f;
};

// include/ocean/ocean.hpp:194-222. Move-only. The constructor throws
// std::invalid_argument for a malformed descriptor (as the reference does),
// std::bad_alloc when device or pinned memory runs out, and
// std::runtime_error when a CUDA call fails; it leaves the ocean evaluated at
// t = 0. update(time) is a pure function of (seed, desc, time) and allocates
// nothing. Queries run on the device over the current frame.
class OCEAN_CXX_API Ocean {
public:
    explicit Ocean(const OceanDesc& desc);
    ~Ocean();

    Ocean(Ocean&&) noexcept;
    Ocean& operator=(Ocean&&) noexcept;
    Ocean(const Ocean&) = delete;
    Ocean& operator=(const Ocean&) = delete;

    void update(double time) noexcept;

    [[nodiscard]] Buffers buffers() const noexcept;
    [[nodiscard]] float height_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] Surface sample_at(float world_x, float world_z) const noexcept;
    [[nodiscard]] const OceanDesc& desc() const noexcept;
    [[nodiscard]] double time() const noexcept;

    // Not in the reference: the C handle behind this object (an ocean_sim*
    // of include/ocean/ocean.h, for the library's device-side extensions
    // such as ocean_get_device_buffers), or null for a CascadeStack level.
    [[nodiscard]] void* c_handle() const noexcept;

    struct Impl;

private:
    friend class CascadeStack;
    friend class FoamField;
    explicit Ocean(std::unique_ptr<Impl> impl) noexcept;
    std::unique_ptr<Impl> impl_;
};

}  // namespace ocean
