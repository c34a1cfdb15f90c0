// oceanlib-b200: init-time spectrum tables, built on the device.
//
// h0(k) for every cell comes from the reference's own generator chain,
// restated for one thread per cell:
//   PCG32 XSH-RR per row, seeded by SplitMix64 (src/core/rng.hpp:27-97),
//   jumped ahead 2*x draws with the LCG's closed-form advance;
//   double Box-Muller (src/core/rng.cpp:7-17);
//   JONSWAP * Hasselmann spreading in double (src/core/spectrum.cpp:27-244);
//   amp = 0.5 * sqrt(Psi) * dk (src/core/spectrum.cpp:296-322).
// Compiled with -fmad=false so the double arithmetic rounds like the
// reference's (which is built with -ffp-contract=off). The only possible
// source of difference is the last-ulp behaviour of the double math
// functions (log, cos, sin, pow, exp, cbrt, lgamma, atan2, tanh) between
// CUDA's device library and the host's libm; tests count such cells.
#include "ocean_device.cuh"
#include "spectrum.h"

#include <cmath>

namespace ocean_b200 {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kTwoPi = 6.28318530717958647692;
constexpr uint64_t kPcgMult = 6364136223846793005ULL;

struct Pcg {
    uint64_t state, inc;
};

__device__ __forceinline__ uint32_t pcg_next(Pcg& r)
{
    const uint64_t old = r.state;
    r.state = old * kPcgMult + r.inc;
    const uint32_t xs = static_cast<uint32_t>(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = static_cast<uint32_t>(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

__device__ __forceinline__ Pcg pcg_seed(uint64_t seed, uint64_t stream)
{
    Pcg r{0u, (stream << 1u) | 1u};
    pcg_next(r);
    r.state += seed;
    pcg_next(r);
    return r;
}

// Jump the LCG ahead by `delta` steps in O(log delta): the composition of
// `delta` affine maps s -> a*s + c is again affine (Brown, "Random number
// generation with arbitrary strides", 1994; the same construction PCG's
// reference implementation uses for pcg_advance).
__device__ __forceinline__ void pcg_advance(Pcg& r, uint64_t delta)
{
    uint64_t acc_mult = 1u, acc_plus = 0u;
    uint64_t cur_mult = kPcgMult, cur_plus = r.inc;
    while (delta > 0) {
        if (delta & 1u) {
            acc_mult *= cur_mult;
            acc_plus = acc_plus * cur_mult + cur_plus;
        }
        cur_plus = (cur_mult + 1u) * cur_plus;
        cur_mult *= cur_mult;
        delta >>= 1u;
    }
    r.state = acc_mult * r.state + acc_plus;
}

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

__device__ __forceinline__ double open01(Pcg& r)
{
    return (static_cast<double>(pcg_next(r)) + 0.5) * (1.0 / 4294967296.0);
}

__device__ __forceinline__ double wrap_angle(double a)
{
    a = fmod(a + kPi, kTwoPi);
    if (a < 0.0) a += kTwoPi;
    return a - kPi;
}

__device__ __forceinline__ double omega_of(double g, double k, double depth)
{
    if (!(k > 0.0)) return 0.0;
    if (depth <= 0.0) return sqrt(g * k);
    return sqrt(g * k * tanh(k * depth));
}

__device__ double domega_dk(double g, double k, double omega, double depth)
{
    if (!(omega > 0.0)) return 0.0;
    if (depth <= 0.0) return g / (2.0 * omega);
    const double kh = k * depth;
    const double th = tanh(kh);
    const double sech2 = 1.0 - th * th;
    return g * (th + kh * sech2) / (2.0 * omega);
}

__device__ double peak_omega(const SpectrumParams& d)
{
    const double g = d.gravity;
    const double u = static_cast<double>(d.wind_speed);
    const double f = static_cast<double>(d.fetch);
    if (u <= 0.0 || f <= 0.0) return 0.0;
    return 22.0 * cbrt(g * g / (u * f));
}

__device__ double jonswap_alpha(const SpectrumParams& d)
{
    const double g = d.gravity;
    const double u = static_cast<double>(d.wind_speed);
    const double f = static_cast<double>(d.fetch);
    if (u <= 0.0 || f <= 0.0) return 0.0;
    const double xt = g * f / (u * u);
    return 0.076 * pow(xt, -0.22);
}

__device__ double jonswap(const SpectrumParams& d, double omega)
{
    if (!(omega > 0.0)) return 0.0;
    const double g = d.gravity;
    const double wp = peak_omega(d);
    if (!(wp > 0.0)) return 0.0;
    const double alpha = jonswap_alpha(d);
    const double gamma = static_cast<double>(d.peak_enhancement);
    const double ratio = wp / omega;
    const double w2 = omega * omega;
    const double w4 = w2 * w2;
    const double pm = (alpha * g * g / (w4 * omega)) * exp(-1.25 * pow(ratio, 4.0));
    const double sigma = (omega <= wp) ? 0.07 : 0.09;
    const double dw = omega - wp;
    const double r = exp(-(dw * dw) / (2.0 * sigma * sigma * wp * wp));
    return pm * pow(gamma, r);
}

__device__ double spreading(const SpectrumParams& d, double omega, double theta)
{
    const double wp = peak_omega(d);
    if (!(omega > 0.0) || !(wp > 0.0)) return 0.0;
    const double g = d.gravity;
    const double u = static_cast<double>(d.wind_speed);
    const double ratio = omega / wp;
    double s;
    if (ratio < 1.0) {
        s = 6.97 * pow(ratio, 4.06);
    } else {
        const double mu = -2.33 - 1.45 * ((u * wp / g) - 1.17);
        s = 9.77 * pow(ratio, mu);
    }
    const double swell = static_cast<double>(d.swell);
    if (swell > 0.0) s += 16.0 * tanh(wp / omega) * swell * swell;
    if (s < 0.0) s = 0.0;
    const double dtheta = wrap_angle(theta - static_cast<double>(d.wind_direction));
    const double c = cos(0.5 * dtheta);
    if (c <= 0.0) return 0.0;
    const double q = exp(lgamma(s + 1.0) - lgamma(s + 0.5)) / (2.0 * sqrt(kPi));
    return q * pow(c, 2.0 * s);
}

__device__ double wave_density(const SpectrumParams& d, double kx, double kz)
{
    const double k2 = kx * kx + kz * kz;
    if (!(k2 > 0.0)) return 0.0;
    const double k = sqrt(k2);
    const double g = d.gravity;
    const double depth = static_cast<double>(d.depth);
    const double omega = omega_of(g, k, depth);
    const double s_omega = jonswap(d, omega);
    if (!(s_omega > 0.0)) return 0.0;
    const double dwdk = domega_dk(g, k, omega, depth);
    const double theta = atan2(kz, kx);
    const double sp = spreading(d, omega, theta);
    double psi = s_omega * dwdk * sp / k;
    const double l = static_cast<double>(d.small_wave_cutoff) / kTwoPi;
    psi *= exp(-k2 * l * l);
    return psi;
}

// Signed wavenumber of grid index i (src/core/spectrum.hpp:85-92).
__device__ __forceinline__ float wave_component(uint32_t i, uint32_t n, float L)
{
    const int si = (i < n / 2) ? static_cast<int>(i) : static_cast<int>(i) - static_cast<int>(n);
    return 6.28318530717958647692f * static_cast<float>(si) / L;
}

__global__ void h0_kernel(SpectrumParams p, float2* __restrict__ h0)
{
    const uint32_t n = p.n;
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= static_cast<uint64_t>(n) * n) return;
    const uint32_t y = static_cast<uint32_t>(i / n);
    const uint32_t x = static_cast<uint32_t>(i % n);

    Pcg rng = pcg_seed(mix64(p.seed ^ (0x9E3779B97F4A7C15ULL * static_cast<uint64_t>(y + 1u))), 0);
    pcg_advance(rng, 2ull * x);

    const float kz = wave_component(y, n, p.patch_length);
    const float kx = wave_component(x, n, p.patch_length);
    const double dk = kTwoPi / static_cast<double>(p.patch_length);
    const double psi = wave_density(p, kx, kz);
    const double amp = 0.5 * sqrt(psi) * dk;

    const double u1 = open01(rng);
    const double u2 = open01(rng);
    const double radius = sqrt(-2.0 * log(u1));
    const double theta = 6.283185307179586476925286766559 * u2;
    const float ga = static_cast<float>(radius * cos(theta));
    const float gb = static_cast<float>(radius * sin(theta));
    h0[i] = make_float2(static_cast<float>(ga * amp), static_cast<float>(gb * amp));
}

// Per-cell (omega, 1/|k|) and per-index signed wavenumbers; these depend only
// on (N, L, g, depth), so oceans sharing a grid geometry share one table.
__global__ void geometry_kernel(SpectrumParams p, float2* __restrict__ omega_kinv,
                                float* __restrict__ kvec)
{
    const uint32_t n = p.n;
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) kvec[i] = wave_component(static_cast<uint32_t>(i), n, p.patch_length);
    if (i >= static_cast<uint64_t>(n) * n) return;
    const uint32_t y = static_cast<uint32_t>(i / n);
    const uint32_t x = static_cast<uint32_t>(i % n);
    const float kz = wave_component(y, n, p.patch_length);
    const float kx = wave_component(x, n, p.patch_length);
    const double k2 = static_cast<double>(kx) * kx + static_cast<double>(kz) * kz;
    const double k = sqrt(k2);
    const float omega = static_cast<float>(omega_of(static_cast<double>(p.gravity), k,
                                                    static_cast<double>(p.depth)));
    const float kinv = (k > 0.0) ? static_cast<float>(1.0 / k) : 0.0f;
    omega_kinv[i] = make_float2(omega, kinv);
}

}  // namespace

cudaError_t launch_h0(const SpectrumParams& p, float2* h0, cudaStream_t stream)
{
    const uint64_t cells = static_cast<uint64_t>(p.n) * p.n;
    const unsigned blocks = static_cast<unsigned>((cells + 255) / 256);
    h0_kernel<<<blocks, 256, 0, stream>>>(p, h0);
    return cudaGetLastError();
}

cudaError_t launch_geometry(const SpectrumParams& p, float2* omega_kinv, float* kvec,
                            cudaStream_t stream)
{
    const uint64_t cells = static_cast<uint64_t>(p.n) * p.n;
    const unsigned blocks = static_cast<unsigned>((cells + 255) / 256);
    geometry_kernel<<<blocks, 256, 0, stream>>>(p, omega_kinv, kvec);
    return cudaGetLastError();
}

}  // namespace ocean_b200
