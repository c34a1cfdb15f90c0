// oceanlib-b200: host side of the iWave interaction field, shared by the
// single-field handle (interaction.cpp) and the serving loop (serve.cpp), so
// both resolve descriptors, damping, substep counts and sources identically.
#pragma once

#include "../../include/ocean_b200.h"
#include "iwave.h"
#include "iwave_stencil.h"

#include <cstddef>
#include <cstdint>
#include <vector>

namespace ocean_b200 {

// InteractionDesc defaults (include/ocean/interaction.hpp:64-139).
void interaction_desc_defaults(ocean_interaction_desc* d);
// struct_size-aware copy; false for a bad struct_size.
bool copy_interaction_desc(const ocean_interaction_desc* src, ocean_interaction_desc& dst);
// Throws std::invalid_argument as src/interaction.cpp:439-476 does.
void validate_interaction(const ocean_interaction_desc& d);

// What the reference derives from the descriptor at construction
// (src/interaction.cpp:43-46, :439-497): grid geometry, the fitted stencil,
// the stability limit and the fixed substep.
struct IWaveSetup {
    uint32_t n = 0, p = 0, rows = 0;
    int stride = 0;
    size_t cells = 0;
    float cell = 0.0f, dt = 0.0f, dt_limit = 0.0f;
    IWaveStencil stencil;
    IWaveTaps taps{};
};
IWaveSetup iwave_setup(const ocean_interaction_desc& d);  // validates; throws when unstable

// The absorbing sponge tables c1, c2 (src/interaction.cpp:212-241).
void iwave_damping(const ocean_interaction_desc& d, const IWaveSetup& s, std::vector<float>& c1,
                   std::vector<float>& c2);

// A disturbance resolved to grid units at `sub_time` into the update
// (src/interaction.cpp:322-356); false when its clipped box is empty.
bool resolve_source(const ocean_disturbance& d, float sub_time, float scale, const IWaveSetup& s,
                    int32_t origin_x, int32_t origin_z, IWaveSource& out);

// The fixed-step accumulator of InteractionField::update
// (src/interaction.cpp:531-549).
struct IWaveClock {
    double accum = 0.0;
    uint32_t last_steps = 0;
    bool clamped = false;
    uint32_t advance(float dt, float fixed_dt, uint32_t max_substeps);
};

// The pending-source queue: add() drops beyond max_sources; after an update
// with no substep only impulses stay queued (src/interaction.cpp:551-560).
struct IWaveQueue {
    std::vector<ocean_disturbance> items;
    uint32_t count = 0;
    uint64_t dropped = 0;
    void reset(uint32_t max_sources);
    void add(const ocean_disturbance& d);
    void keep_impulses();
    // Resolves every substep's sources in submission order into `out`
    // (first[s] .. first[s+1] for substep s), then empties the queue.
    void resolve_all(uint32_t steps, const IWaveSetup& s, int32_t origin_x, int32_t origin_z,
                     std::vector<IWaveSource>& out, std::vector<uint32_t>& first);
};

}  // namespace ocean_b200
