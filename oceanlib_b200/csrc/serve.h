// oceanlib-b200: device interface of the serving loop's batched queries.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ocean_b200 {

// One height_at request of one session: the combined surface height
// (WaterSurface::height_at, src/interaction.cpp:903-908) at `count` points.
struct QueryJob {
    const float4* disp;      // ocean displacement [n*n]
    const float4* normal;    // ocean normal [n*n]
    const float2* xz;        // [count] world points
    float* out;              // [count] heights
    const float4* field;     // interaction output [fn*fn], or null (ocean alone)
    int32_t n;
    float inv_cell;          // n / patch_length
    int32_t fn;
    float cell;              // interaction cell size
    float origin_x, origin_z;
    uint32_t count;
    uint32_t pad;
};

// Every job of a batch in one launch (blockIdx.y = job).
cudaError_t launch_serve_queries(const QueryJob* jobs, int count, uint32_t max_points,
                                 cudaStream_t st);

}  // namespace ocean_b200
