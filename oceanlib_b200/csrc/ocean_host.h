// oceanlib-b200: host helpers shared by the ocean handles (host.cpp) and the
// serving loop (serve.cpp): descriptor defaults and checks, the spectrum
// parameters and the per-stage twiddle tables.
#pragma once

#include "../../include/ocean_b200.h"
#include "spectrum.h"

#include <cstdint>
#include <vector>

namespace ocean_b200 {

// The reference's OceanDesc defaults (include/ocean/ocean.hpp:39-130).
void desc_defaults(ocean_desc* d);
// struct_size-aware copy (src/c_api.cpp:46-60); false for a bad struct_size.
bool copy_desc(const ocean_desc* src, ocean_desc& dst);
// Throws std::invalid_argument as the reference's constructor would
// (src/ocean.cpp:28-59): N a power of two in [16, 4096], and so on.
void validate(const ocean_desc& d);
// Largest N of the persistent frame kernel (frame.cu); 2048 and 4096 run
// the three-pass schedule of frame_large.cu.
constexpr uint32_t kMaxPersistentSize = 1024;
int ilog2u(uint32_t v);
// Per-stage inverse twiddles, N - 1 entries (src/core/fft.cpp:24-33).
std::vector<float2> stage_twiddles(uint32_t n);
SpectrumParams spectrum_params(const ocean_desc& d);
// The kernel form ocean_force_simd_level selected (ocean_fft_form).
int current_form();

}  // namespace ocean_b200
