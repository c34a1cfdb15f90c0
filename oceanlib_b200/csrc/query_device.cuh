// oceanlib-b200: device-side surface queries shared by the query kernels.
//
//   sample_one        - one ocean's surface at a world position: the
//                       fixed-point displacement inversion and the final
//                       periodic bilinear taps (src/ocean.cpp:322-452);
//   interaction_tap   - the interaction field's (eta, d/dx, d/dz, d/dt) at a
//                       world position, bilinear, zero outside the grid
//                       (src/interaction.cpp:729-770).
// Compiled with -fmad=false like every other kernel, so each product and sum
// rounds as the reference's does.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "spectrum.h"

namespace ocean_b200 {
namespace qdev {

struct Tap {
    uint32_t i00, i10, i01, i11;
    float w00, w10, w01, w11;
};

__device__ __forceinline__ uint32_t wrap_index(int i, int n)
{
    i %= n;
    if (i < 0) i += n;
    return static_cast<uint32_t>(i);
}

__device__ __forceinline__ Tap make_tap(float u, float v, int n, float inv_cell)
{
    const float gu = u * inv_cell;
    const float gv = v * inv_cell;
    const float fu = floorf(gu);
    const float fv = floorf(gv);
    const uint32_t x0 = wrap_index(__float2int_rz(fu), n);
    const uint32_t z0 = wrap_index(__float2int_rz(fv), n);
    const uint32_t x1 = (x0 + 1u) % static_cast<uint32_t>(n);
    const uint32_t z1 = (z0 + 1u) % static_cast<uint32_t>(n);
    const float tu = gu - fu;
    const float tv = gv - fv;
    Tap t;
    t.i00 = z0 * n + x0;
    t.i10 = z0 * n + x1;
    t.i01 = z1 * n + x0;
    t.i11 = z1 * n + x1;
    t.w00 = (1.0f - tu) * (1.0f - tv);
    t.w10 = tu * (1.0f - tv);
    t.w01 = (1.0f - tu) * tv;
    t.w11 = tu * tv;
    return t;
}

struct Texels {
    float4 a, b, c, d;
};

__device__ __forceinline__ Texels load_texels(const float4* __restrict__ buf, const Tap& t)
{
    return Texels{__ldg(&buf[t.i00]), __ldg(&buf[t.i10]), __ldg(&buf[t.i01]), __ldg(&buf[t.i11])};
}

// buf[i00+c]*w00 + buf[i10+c]*w10 + buf[i01+c]*w01 + buf[i11+c]*w11, in that order.
#define OCEAN_FETCH(T, t, C) ((T).a.C * (t).w00 + (T).b.C * (t).w10 + (T).c.C * (t).w01 + (T).d.C * (t).w11)

// One ocean's surface at world (x, z): `iters` fixed-point steps of the
// displacement inversion (the reference takes 4, src/ocean.cpp:366), stopping
// early once both parameter coordinates move by <= tol (tol = 0: never), then
// the final bilinear taps and the renormalised normal.
__device__ __forceinline__ SurfaceEx sample_one(int n, float inv_cell,
                                                const float4* __restrict__ disp,
                                                const float4* __restrict__ normal,
                                                const float4* __restrict__ vel, float2 p,
                                                int iters, float tol)
{
    float u = p.x, v = p.y;
    for (int it = 0; it < iters; ++it) {
        const Tap t = make_tap(u, v, n, inv_cell);
        const Texels d = load_texels(disp, t);
        const float un = p.x - OCEAN_FETCH(d, t, x);
        const float vn = p.y - OCEAN_FETCH(d, t, z);
        const bool done = tol > 0.0f && fabsf(un - u) <= tol && fabsf(vn - v) <= tol;
        u = un;
        v = vn;
        if (done) break;
    }
    const Tap t = make_tap(u, v, n, inv_cell);
    const Texels d = load_texels(disp, t);
    SurfaceEx s;
    s.offset_x = OCEAN_FETCH(d, t, x);
    s.height = OCEAN_FETCH(d, t, y);
    s.offset_z = OCEAN_FETCH(d, t, z);
    s.foam = OCEAN_FETCH(d, t, w);
    const Texels nm = load_texels(normal, t);
    float nx = OCEAN_FETCH(nm, t, x);
    float ny = OCEAN_FETCH(nm, t, y);
    float nz = OCEAN_FETCH(nm, t, z);
    const float len2 = nx * nx + ny * ny + nz * nz;
    if (len2 > 0.0f) {
        const float inv = 1.0f / sqrtf(len2);
        nx *= inv;
        ny *= inv;
        nz *= inv;
    } else {
        nx = 0.0f;
        ny = 1.0f;
        nz = 0.0f;
    }
    s.normal_x = nx;
    s.normal_y = ny;
    s.normal_z = nz;
    if (vel != nullptr) {
        const Texels vv = load_texels(vel, t);
        s.velocity_x = OCEAN_FETCH(vv, t, x);
        s.velocity_y = OCEAN_FETCH(vv, t, y);
        s.velocity_z = OCEAN_FETCH(vv, t, z);
    } else {
        s.velocity_x = s.velocity_y = s.velocity_z = 0.0f;
    }
    return s;
}

// Bilinear, zero outside the grid (src/interaction.cpp:729-770).
__device__ __forceinline__ float4 interaction_tap(const float4* __restrict__ out, int n, float cell,
                                                  float origin_x, float origin_z, float wx, float wz,
                                                  bool& inside)
{
    const float gx = (wx - origin_x) / cell - 0.5f;
    const float gz = (wz - origin_z) / cell - 0.5f;
    inside = !(gx < 0.0f || gz < 0.0f || gx >= static_cast<float>(n - 1) ||
               gz >= static_cast<float>(n - 1));
    if (!inside) return make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    const int x0 = static_cast<int>(gx);
    const int z0 = static_cast<int>(gz);
    const float tx = gx - static_cast<float>(x0);
    const float tz = gz - static_cast<float>(z0);
    const size_t i00 = static_cast<size_t>(z0) * n + x0;
    const float4 a = out[i00], b = out[i00 + 1], c = out[i00 + n], d = out[i00 + n + 1];
    const float w00 = (1.0f - tx) * (1.0f - tz);
    const float w10 = tx * (1.0f - tz);
    const float w01 = (1.0f - tx) * tz;
    const float w11 = tx * tz;
    return make_float4(a.x * w00 + b.x * w10 + c.x * w01 + d.x * w11,
                       a.y * w00 + b.y * w10 + c.y * w01 + d.y * w11,
                       a.z * w00 + b.z * w10 + c.z * w01 + d.z * w11,
                       a.w * w00 + b.w * w10 + c.w * w01 + d.w * w11);
}

}  // namespace qdev
}  // namespace ocean_b200
