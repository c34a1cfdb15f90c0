// oceanlib-b200: iWave interaction field - device interface.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "spectrum.h"

namespace ocean_b200 {

// One field's two time levels (with a P-cell zero halo; cur/old point at
// interior cell (0, 0)), damping, output and step constants.
struct IWaveField {
    float* cur;
    float* old;
    const float* c1;
    const float* c2;
    float4* out;
    int32_t n;
    int32_t stride;
    float gdt2;          // g * dt^2
    float inv_two_cell;  // 0.5 / cell
    float inv_dt;        // 1 / dt (float, as finalize uses it)
    double inv_dt_d;     // 1 / dt (double, as the energy uses it)
};

// The stencil taps, passed by value (kernel parameter space): (2P+1)^2 <= 625.
struct IWaveTaps {
    float t[625];
};

// One queued disturbance at one substep, resolved to grid units on the host
// (src/interaction.cpp:322-356); `mean` is filled by launch_source_mean.
struct IWaveSource {
    float gx, gz;            // centre in cells
    float inv_two_sigma2;
    float cell;
    float disp, vel, dt;     // -strength*scale, velocity_y*scale, substep dt
    float mean;
    int32_t x0, x1, z0, z1;  // clipped box (inclusive)
};

cudaError_t launch_iwave_step(int p, const IWaveField* fields, int count, int max_n,
                              const IWaveTaps& taps, cudaStream_t st);
cudaError_t launch_iwave_finalize(const IWaveField* fields, int count, int max_n, cudaStream_t st);
cudaError_t launch_source_mean(IWaveSource* sources, int count, cudaStream_t st);
cudaError_t launch_source_apply(const IWaveField& f, const IWaveSource* sources, int count,
                                cudaStream_t st);
// `count` fields at once; field k adds sources [ranges[k].x, +ranges[k].y)
// (ranges on the device, means already filled).
cudaError_t launch_source_apply_batch(const IWaveField* fields, const int2* ranges,
                                      const IWaveSource* sources, int count, int max_n, cudaStream_t st);
cudaError_t launch_obstruction(const IWaveField& f, const uint32_t* solid, const uint32_t* nearest,
                               uint32_t count, bool dirichlet, cudaStream_t st);
cudaError_t launch_shift(const float* src, float* dst, int n, int stride, int dx, int dz,
                         cudaStream_t st);
cudaError_t launch_interaction_sample(const float4* out, int n, float cell, float origin_x,
                                      float origin_z, const float2* xz, uint64_t count,
                                      float4* res, cudaStream_t st);
cudaError_t launch_combine(const SurfaceEx* ocean_s, const float4* e, uint64_t count, SurfaceEx* out,
                           cudaStream_t st);
// The obstruction tables from a device mask of n*n bytes (non-zero =
// solid): solid cells in index order and the nearest-fluid index of every
// cell, as the reference's multi-source BFS assigns them
// (src/interaction.cpp:255-292). Waits for the stream; *solid_count is host.
cudaError_t build_obstruction_tables(const uint8_t* mask, int n, uint32_t* solid, uint32_t* nearest,
                                     uint32_t* solid_count, cudaStream_t st);
cudaError_t launch_energy_rows(const IWaveField& f, const float* taps, int p, double* row_kin,
                               double* row_pot, cudaStream_t st);

}  // namespace ocean_b200
