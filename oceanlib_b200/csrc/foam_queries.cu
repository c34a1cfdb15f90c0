// oceanlib-b200: queries on the persistent foam field.
//
//   foam_at_kernel        FoamField::foam_at (src/foam.cpp:291-305): the
//                         ocean's fixed-point inversion (sample_one, the same
//                         as Ocean::sample_at) gives the parameter position of
//                         the water at a world point; the foam grid is then
//                         sampled there with the periodic bilinear fetch of
//                         src/foam.cpp:22-41. One thread per point.
//   foam_coverage_kernel  FoamField::coverage (src/foam.cpp:307-313): the mean
//                         of the field in double. One CTA; every thread sums a
//                         fixed strided subset and a fixed tree combines them,
//                         so the result is deterministic. It differs from the
//                         reference's sequential sum by rounding only.
#include "frame_cells.cuh"
#include "query_device.cuh"
#include "spectrum.h"

namespace ocean_b200 {
namespace {

__global__ void foam_at_kernel(int n, float inv_cell, float cell, const float4* __restrict__ disp,
                               const float4* __restrict__ normal, const float* __restrict__ foam,
                               const float2* __restrict__ xz, uint64_t count, float* __restrict__ out)
{
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float2 p = xz[i];
    // Only the offsets are used: no velocity taps.
    const SurfaceEx s = qdev::sample_one(n, inv_cell, disp, normal, nullptr, p, 4, 0.0f);
    const float u = (p.x - s.offset_x) / cell;
    const float v = (p.y - s.offset_z) / cell;
    auto get = [&](int z, int x) { return __ldg(&foam[static_cast<size_t>(z) * n + x]); };
    out[i] = foam_blend(foam_fetch(u, v, n, get));
}

constexpr int kCoverageThreads = 1024;

__global__ void __launch_bounds__(kCoverageThreads)
foam_coverage_kernel(const float* __restrict__ foam, uint64_t cells, double* __restrict__ out)
{
    __shared__ double part[kCoverageThreads];
    double sum = 0.0;
    for (uint64_t i = threadIdx.x; i < cells; i += kCoverageThreads) sum += static_cast<double>(foam[i]);
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int w = kCoverageThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = part[0] / static_cast<double>(cells);
}

}  // namespace

cudaError_t launch_foam_at(int n, float inv_cell, float cell, const float4* disp, const float4* normal,
                           const float* foam, const float2* xz, uint64_t count, float* out,
                           cudaStream_t stream)
{
    if (count == 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
    foam_at_kernel<<<blocks, 256, 0, stream>>>(n, inv_cell, cell, disp, normal, foam, xz, count, out);
    return cudaGetLastError();
}

cudaError_t launch_foam_coverage(const float* foam, uint64_t cells, double* out, cudaStream_t stream)
{
    foam_coverage_kernel<<<1, kCoverageThreads, 0, stream>>>(foam, cells, out);
    return cudaGetLastError();
}

}  // namespace ocean_b200
