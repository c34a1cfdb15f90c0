// oceanlib-b200: RGBA16F packing of the RGBA32F outputs on the device.
//
// The reference's viewer narrows every output to half floats before the
// upload, and substitutes the persistent foam for the displacement's alpha
// during the same pass (examples/viewer/half.hpp:58-125,
// examples/viewer/ocean_view.cpp:830-862). Here the same conversion runs on
// the GPU, so a host that wants half floats copies half the bytes.
// Rounding: IEEE round-to-nearest-even, overflow to infinity, NaN kept as a
// quiet NaN (sign | 0x7E00) - the reference's float_to_half, bit for bit.
#include <cuda_fp16.h>
#include <cstdint>

#include "spectrum.h"

namespace ocean_b200 {
namespace {

__device__ __forceinline__ uint16_t to_half(float v)
{
    if (isnan(v)) return static_cast<uint16_t>(((__float_as_uint(v) >> 16) & 0x8000u) | 0x7E00u);
    return __half_as_ushort(__float2half_rn(v));
}

// One texel per thread: RGB from src, A from alpha (or src's own A).
__global__ void pack_rgba16_kernel(const float4* __restrict__ src, const float* __restrict__ alpha,
                                   uint64_t cells, ushort4* __restrict__ dst)
{
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const float4 v = __ldcs(&src[i]);
    const float a = alpha != nullptr ? __ldcs(&alpha[i]) : v.w;
    __stcs(&dst[i], make_ushort4(to_half(v.x), to_half(v.y), to_half(v.z), to_half(a)));
}

}  // namespace

cudaError_t launch_pack_rgba16(const float4* src, const float* alpha, uint64_t cells, ushort4* dst,
                               cudaStream_t st)
{
    if (cells == 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((cells + 255) / 256);
    pack_rgba16_kernel<<<blocks, 256, 0, st>>>(src, alpha, cells, dst);
    return cudaGetLastError();
}

}  // namespace ocean_b200
