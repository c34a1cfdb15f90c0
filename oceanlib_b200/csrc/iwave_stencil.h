// oceanlib-b200: iWave convolution stencil, built on the host at creation.
#pragma once

#include <cstdint>
#include <vector>

namespace ocean_b200 {

// A (2P+1)^2 D4-symmetric stencil whose discrete Fourier symbol matches the
// dispersion symbol S(k) = k tanh(k h) (k in deep water) over the resolved
// band, and the statistics of the symbol it actually realises.
struct IWaveStencil {
    uint32_t radius = 0;
    uint32_t width = 0;
    float cell = 0.0f;
    std::vector<float> taps;   // row-major over (j, i), width*width
    double max_symbol = 0.0;
    double min_symbol = 0.0;
    double band_low = 0.0;
    double peak_relative_error = 0.0;

    bool stable() const { return min_symbol >= -1e-3 * max_symbol && max_symbol > 0.0; }
};

// Weighted least-squares fit (reference: src/core/iwave_kernel.cpp:177-437,
// the LeastSquares method). Throws std::invalid_argument for a radius outside
// [1, 12], a non-positive cell or a singular fit.
IWaveStencil build_iwave_stencil(uint32_t radius, double cell, double depth,
                                 uint32_t fit_samples = 96, double band_low_frac = 0.125);

}  // namespace ocean_b200
