// oceanlib-b200: per-cell arithmetic of the frame - evolve, finalize and the
// persistent-foam substep - shared by the persistent frame kernel and the
// passes for sizes above 1024. Compiled with -fmad=false like everything else,
// so each operation rounds where the reference's scalar code rounds.
#pragma once

#include "ocean_device.cuh"

namespace ocean_b200 {

// The evolved spectra of one cell (src/core/evolve.cpp:28-121, and :123-184
// for the velocity fields): h0(k) = av, h0(-k) = bm (conjugated here), the
// cell's (omega, 1/|k|) = wk and wavenumbers kx, kz, at t / 2pi = top. The
// eight real spectra are packed two per complex field (A + iB) into p[0..3],
// the velocity spectra into p[4..5] when NF = 6.
template <int NF>
__device__ __forceinline__ void evolve_cell(float2 av, float2 bm, float2 wk, float kx, float kz, double top,
                                            float2 (&p)[NF])
{
    const float b_re = bm.x, b_im = -bm.y;
    float s, c;
    sincos_poly(fold_phase(wk.x, top), s, c);
    const float fwd_re = av.x * c - av.y * s;
    const float fwd_im = av.x * s + av.y * c;
    const float bwd_re = b_re * c + b_im * s;
    const float bwd_im = b_im * c - b_re * s;
    const float hr = fwd_re + bwd_re;
    const float hi = fwd_im + bwd_im;
    const float ki = wk.y;
    const float sx = kx * ki;
    const float sz = kz * ki;
    const float dx_re = sx * hi, dx_im = -sx * hr;
    const float dz_re = sz * hi, dz_im = -sz * hr;
    const float hx_re = -kx * hi, hx_im = kx * hr;
    const float hz_re = -kz * hi, hz_im = kz * hr;
    const float jxx = kx * sx, jzz = kz * sz, jxz = kx * sz;
    const float jxx_re = jxx * hr, jxx_im = jxx * hi;
    const float jzz_re = jzz * hr, jzz_im = jzz * hi;
    const float jxz_re = jxz * hr, jxz_im = jxz * hi;

    p[0] = make_float2(hr - dx_im, hi + dx_re);
    p[1] = make_float2(dz_re - hx_im, dz_im + hx_re);
    p[2] = make_float2(hz_re - jxx_im, hz_im + jxx_re);
    p[3] = make_float2(jzz_re - jxz_im, jzz_im + jxz_re);
    if constexpr (NF == 6) {
        const float dr = fwd_re - bwd_re;
        const float di = fwd_im - bwd_im;
        const float w = wk.x;
        const float wsx = w * sx, wsz = w * sz;
        const float ux_re = -wsx * dr, ux_im = -wsx * di;
        const float uz_re = -wsz * dr, uz_im = -wsz * di;
        const float uy_re = -w * di, uy_im = w * dr;
        p[4] = make_float2(ux_re - uy_im, ux_im + uy_re);
        p[5] = make_float2(uz_re, uz_im);
    }
}

// Displacement (lambda Dx, h, lambda Dz, foam) and normal (n, Jacobian) of one
// cell from its four transformed fields (src/core/evolve.cpp:238-327).
struct CellOut {
    float4 disp;
    float4 normal;
};

__device__ __forceinline__ CellOut finalize_cell(float2 f0, float2 f1, float2 f2, float2 f3, float lambda,
                                                 float foam_threshold, float inv_threshold)
{
    const float h = f0.x, d_x = f0.y, d_z = f1.x, hx = f1.y;
    const float hz = f2.x, jxx = f2.y, jzz = f3.x, jxz = f3.y;

    const float disp_x = lambda * d_x;
    const float disp_z = lambda * d_z;
    const float axx = 1.0f + lambda * jxx;
    const float azz = 1.0f + lambda * jzz;
    const float axz = lambda * jxz;
    const float jac = axx * azz - axz * axz;
    float nx = -(hx * azz - axz * hz);
    float ny = jac;
    float nz = -(axx * hz - hx * axz);
    const float len2 = nx * nx + ny * ny + nz * nz;
    const float inv_len = (len2 > 0.0f) ? 1.0f / sqrtf(len2) : 0.0f;
    nx *= inv_len;
    ny *= inv_len;
    nz *= inv_len;
    float foam = (foam_threshold - jac) * inv_threshold;
    if (foam < 0.0f) foam = 0.0f;
    if (foam > 1.0f) foam = 1.0f;
    return {make_float4(disp_x, h, disp_z, foam), make_float4(nx, ny, nz, jac)};
}

// Periodic bilinear fetch from one channel grid (src/foam.cpp:22-41): the
// four taps come from `get(z, x)`, so a caller can serve them from a staged
// shared-memory window or from global memory with the same arithmetic.
struct FoamTaps {
    float fa, fb, fc, fd, tu, tv;
};

template <typename Get>
__device__ __forceinline__ FoamTaps foam_fetch(float u, float v, int n, Get&& get)
{
    FoamTaps t;
    const float fu = floorf(u), fv = floorf(v);
    t.tu = u - fu;
    t.tv = v - fv;
    int x0 = __float2int_rz(fu) % n;
    if (x0 < 0) x0 += n;
    int z0 = __float2int_rz(fv) % n;
    if (z0 < 0) z0 += n;
    const int x1 = (x0 + 1) % n;
    const int z1 = (z0 + 1) % n;
    t.fa = get(z0, x0);
    t.fb = get(z0, x1);
    t.fc = get(z1, x0);
    t.fd = get(z1, x1);
    return t;
}

__device__ __forceinline__ float foam_blend(const FoamTaps& t)
{
    const float tu = t.tu, tv = t.tv;
    return t.fa * (1.0f - tu) * (1.0f - tv) + t.fb * tu * (1.0f - tv) + t.fc * (1.0f - tu) * tv +
           t.fd * tu * tv;
}

// The backtraced sample point of cell (x, z) and the taps there
// (src/foam.cpp:89-139, first half).
template <typename Get>
__device__ __forceinline__ FoamTaps foam_taps(int n, int x, int z, float velx, float velz, float dt, float scale,
                                              float drift_x, float drift_z, float inv_cell, Get&& get)
{
    const float vx = velx * scale + drift_x;
    const float vz = velz * scale + drift_z;
    const float su = static_cast<float>(x) - vx * dt * inv_cell;
    const float sv = static_cast<float>(z) - vz * dt * inv_cell;
    return foam_fetch(su, sv, n, get);
}

// Decay, source and clamp of the sampled foam (second half).
__device__ __forceinline__ float foam_finish(const FoamTaps& t, float src, float decay, float gain)
{
    float f = foam_blend(t);
    f = f * decay + src * gain;
    if (f > 1.0f) f = 1.0f;
    if (f < 0.0f) f = 0.0f;
    return f;
}

// One persistent-foam substep for cell (x, z) (src/foam.cpp:89-139).
__device__ __forceinline__ float foam_cell(const float* cur, int n, int x, int z, float velx,
                                           float velz, float src, float dt, float decay,
                                           float gain, float scale, float drift_x,
                                           float drift_z, float inv_cell)
{
    auto get = [&](int zz, int xx) { return cur[static_cast<size_t>(zz) * n + xx]; };
    return foam_finish(foam_taps(n, x, z, velx, velz, dt, scale, drift_x, drift_z, inv_cell, get), src, decay,
                       gain);
}

}  // namespace ocean_b200
