// oceanlib-b200: the serving loop's batched height queries.
//
// One launch answers every height_at request of a batch, whatever session it
// belongs to: block row y is request y, each thread one point. A point runs
// the ocean's fixed-point displacement inversion (4 steps, as
// Ocean::height_at -> sample_at, src/ocean.cpp:370-452) and adds the
// interaction field's bilinear height (InteractionField::height_at,
// src/interaction.cpp:775-778), exactly as WaterSurface::height_at
// (src/interaction.cpp:903-908) composes them. The arithmetic is the shared
// query code, so each height is bit-identical to a single-session query.
#include "query_device.cuh"
#include "serve.h"

namespace ocean_b200 {
namespace {

constexpr int kQueryThreads = 256;

__global__ void __launch_bounds__(kQueryThreads) serve_query_kernel(const QueryJob* __restrict__ jobs)
{
    const QueryJob& j = jobs[blockIdx.y];
    const uint32_t i = blockIdx.x * kQueryThreads + threadIdx.x;
    if (i >= j.count) return;
    const float2 p = j.xz[i];
    const SurfaceEx s = qdev::sample_one(j.n, j.inv_cell, j.disp, j.normal, nullptr, p, 4, 0.0f);
    float h = s.height;
    if (j.field != nullptr) {
        bool inside;
        const float4 e = qdev::interaction_tap(j.field, j.fn, j.cell, j.origin_x, j.origin_z, p.x, p.y, inside);
        h = h + e.x;
    }
    j.out[i] = h;
}

}  // namespace

cudaError_t launch_serve_queries(const QueryJob* jobs, int count, uint32_t max_points, cudaStream_t st)
{
    if (count == 0 || max_points == 0) return cudaSuccess;
    if (count > 65535) return cudaErrorInvalidValue;
    dim3 grid((max_points + kQueryThreads - 1) / kQueryThreads, static_cast<unsigned>(count));
    serve_query_kernel<<<grid, kQueryThreads, 0, st>>>(jobs);
    return cudaGetLastError();
}

}  // namespace ocean_b200
