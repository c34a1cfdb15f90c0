/* Test infrastructure: plain-C restatement of oceanlib's per-frame path.
 *
 * The checker for the CUDA library; never linked into it. Compiled with
 * -ffp-contract=off -fno-fast-math so every float/double operation rounds
 * exactly where the reference's does. Citations are to the reference project
 * (DarshanVShah/oceanlib) by path:line.
 */
#include "ocean_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* PCG32 XSH-RR and SplitMix64 row seeding: src/core/rng.hpp:27-97           */
/* ------------------------------------------------------------------------ */

static const uint64_t kMult = 6364136223846793005ULL;

uint32_t or_pcg32_next(or_pcg32* r)
{
    /* src/core/rng.hpp:35-47 */
    uint64_t old = r->state;
    r->state = old * kMult + r->inc;
    uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xs >> rot) | (xs << ((32u - rot) & 31u));
}

or_pcg32 or_pcg32_seed(uint64_t seed, uint64_t stream)
{
    /* src/core/rng.hpp:53-62 */
    or_pcg32 r;
    r.state = 0u;
    r.inc = (stream << 1u) | 1u;
    or_pcg32_next(&r);
    r.state += seed;
    or_pcg32_next(&r);
    return r;
}

void or_pcg32_fill(uint64_t seed, uint64_t stream, uint32_t count, uint32_t* out)
{
    or_pcg32 r = or_pcg32_seed(seed, stream);
    for (uint32_t i = 0; i < count; ++i) out[i] = or_pcg32_next(&r);
}

uint64_t or_mix64(uint64_t x)
{
    /* src/core/rng.hpp:83-89 */
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

static or_pcg32 row_rng(uint64_t seed, uint32_t row)
{
    /* src/core/rng.hpp:94-97 */
    return or_pcg32_seed(or_mix64(seed ^ (0x9E3779B97F4A7C15ULL * (uint64_t)(row + 1u))), 0);
}

static double open01(or_pcg32* r)
{
    /* src/core/rng.hpp:68-71 */
    return ((double)or_pcg32_next(r) + 0.5) * (1.0 / 4294967296.0);
}

static void gaussian_pair(or_pcg32* r, float* a, float* b)
{
    /* src/core/rng.cpp:7-17 */
    double u1 = open01(r);
    double u2 = open01(r);
    double radius = sqrt(-2.0 * log(u1));
    double theta = 6.283185307179586476925286766559 * u2;
    *a = (float)(radius * cos(theta));
    *b = (float)(radius * sin(theta));
}

void or_row_gaussians(uint64_t seed, uint32_t row, uint32_t pairs, float* out)
{
    or_pcg32 r = row_rng(seed, row);
    for (uint32_t i = 0; i < pairs; ++i) gaussian_pair(&r, &out[2 * i], &out[2 * i + 1]);
}

/* ------------------------------------------------------------------------ */
/* JONSWAP + spreading: src/core/spectrum.cpp:27-244                          */
/* ------------------------------------------------------------------------ */

static const double kPi = 3.14159265358979323846;
static const double kTwoPi = 6.28318530717958647692;

static double wrap_angle(double a)
{
    /* src/core/spectrum.cpp:14-19 */
    a = fmod(a + kPi, kTwoPi);
    if (a < 0.0) a += kTwoPi;
    return a - kPi;
}

static double disp_omega(double g, double k, double depth)
{
    /* src/core/spectrum.cpp:27-32 */
    if (!(k > 0.0)) return 0.0;
    if (depth <= 0.0) return sqrt(g * k);
    return sqrt(g * k * tanh(k * depth));
}

static double disp_domega_dk(double g, double k, double omega, double depth)
{
    /* src/core/spectrum.cpp:34-44 */
    if (!(omega > 0.0)) return 0.0;
    if (depth <= 0.0) return g / (2.0 * omega);
    double kh = k * depth;
    double th = tanh(kh);
    double sech2 = 1.0 - th * th;
    return g * (th + kh * sech2) / (2.0 * omega);
}

static double peak_omega(const or_desc* d)
{
    /* src/core/spectrum.cpp:61-74 */
    double g = d->gravity;
    double u = (double)d->wind_speed;
    double f = (double)d->fetch;
    if (u <= 0.0 || f <= 0.0) return 0.0;
    return 22.0 * cbrt(g * g / (u * f));
}

static double alpha_of(const or_desc* d)
{
    /* src/core/spectrum.cpp:76-85 */
    double g = d->gravity;
    double u = (double)d->wind_speed;
    double f = (double)d->fetch;
    if (u <= 0.0 || f <= 0.0) return 0.0;
    double xt = g * f / (u * u);
    return 0.076 * pow(xt, -0.22);
}

static double jonswap(const or_desc* d, double omega)
{
    /* src/core/spectrum.cpp:87-123 */
    if (!(omega > 0.0)) return 0.0;
    double g = d->gravity;
    double wp = peak_omega(d);
    if (!(wp > 0.0)) return 0.0;
    double alpha = alpha_of(d);
    double gamma = (double)d->peak_enhancement;
    double ratio = wp / omega;
    double w2 = omega * omega;
    double w4 = w2 * w2;
    double pm = (alpha * g * g / (w4 * omega)) * exp(-1.25 * pow(ratio, 4.0));
    double sigma = (omega <= wp) ? 0.07 : 0.09;
    double dw = omega - wp;
    double r = exp(-(dw * dw) / (2.0 * sigma * sigma * wp * wp));
    return pm * pow(gamma, r);
}

static double spread(const or_desc* d, double omega, double theta)
{
    /* src/core/spectrum.cpp:129-192 */
    double wp = peak_omega(d);
    if (!(omega > 0.0) || !(wp > 0.0)) return 0.0;
    double g = d->gravity;
    double u = (double)d->wind_speed;
    double ratio = omega / wp;
    double s;
    if (ratio < 1.0) {
        s = 6.97 * pow(ratio, 4.06);
    } else {
        double mu = -2.33 - 1.45 * ((u * wp / g) - 1.17);
        s = 9.77 * pow(ratio, mu);
    }
    double swell = (double)d->swell;
    if (swell > 0.0) s += 16.0 * tanh(wp / omega) * swell * swell;
    if (s < 0.0) s = 0.0;
    double dtheta = wrap_angle(theta - (double)d->wind_direction);
    double c = cos(0.5 * dtheta);
    if (c <= 0.0) return 0.0;
    double q = exp(lgamma(s + 1.0) - lgamma(s + 0.5)) / (2.0 * sqrt(kPi));
    return q * pow(c, 2.0 * s);
}

static double density(const or_desc* d, double kx, double kz)
{
    /* src/core/spectrum.cpp:198-244 */
    double k2 = kx * kx + kz * kz;
    if (!(k2 > 0.0)) return 0.0;
    double k = sqrt(k2);
    double g = d->gravity;
    double depth = (double)d->depth;
    double omega = disp_omega(g, k, depth);
    double s_omega = jonswap(d, omega);
    if (!(s_omega > 0.0)) return 0.0;
    double dwdk = disp_domega_dk(g, k, omega, depth);
    double theta = atan2(kz, kx);
    double sp = spread(d, omega, theta);
    double psi = s_omega * dwdk * sp / k;
    double l = (double)d->small_wave_cutoff / kTwoPi;
    psi *= exp(-k2 * l * l);
    return psi;
}

static float wave_component(uint32_t i, uint32_t n, float L)
{
    /* src/core/spectrum.hpp:85-92 */
    const float two_pi = 6.28318530717958647692f;
    int si = (i < n / 2) ? (int)i : (int)i - (int)n;
    return two_pi * (float)si / L;
}

void or_build_spectrum(const or_desc* d, float* tables)
{
    /* src/core/spectrum.cpp:264-339 */
    const uint32_t n = d->n;
    const size_t cells = (size_t)n * n;
    float* h0_re = tables + 0 * cells;
    float* h0_im = tables + 1 * cells;
    float* h0c_re = tables + 2 * cells;
    float* h0c_im = tables + 3 * cells;
    float* omega = tables + 4 * cells;
    float* kxt = tables + 5 * cells;
    float* kzt = tables + 6 * cells;
    float* kinv = tables + 7 * cells;
    const double dk = kTwoPi / (double)d->patch_length;

    for (uint32_t y = 0; y < n; ++y) {
        or_pcg32 rng = row_rng(d->seed, y);
        float kz = wave_component(y, n, d->patch_length);
        for (uint32_t x = 0; x < n; ++x) {
            size_t i = (size_t)y * n + x;
            float kx = wave_component(x, n, d->patch_length);
            kxt[i] = kx;
            kzt[i] = kz;
            double k2 = (double)kx * kx + (double)kz * kz;
            double k = sqrt(k2);
            omega[i] = (float)disp_omega((double)d->gravity, k, (double)d->depth);
            kinv[i] = (k > 0.0) ? (float)(1.0 / k) : 0.0f;
            double psi = density(d, kx, kz);
            double amp = 0.5 * sqrt(psi) * dk;
            float ga, gb;
            gaussian_pair(&rng, &ga, &gb);
            h0_re[i] = (float)(ga * amp);
            h0_im[i] = (float)(gb * amp);
        }
    }
    for (uint32_t y = 0; y < n; ++y) {
        uint32_t my = (n - y) % n;
        for (uint32_t x = 0; x < n; ++x) {
            uint32_t mx = (n - x) % n;
            size_t i = (size_t)y * n + x;
            size_t m = (size_t)my * n + mx;
            h0c_re[i] = h0_re[m];
            h0c_im[i] = -h0_im[m];
        }
    }
}

/* ------------------------------------------------------------------------ */
/* Phase fold and sincos: src/core/trig.hpp:33-129                            */
/* ------------------------------------------------------------------------ */

static float reduced_phase(float omega, double t_over_2pi)
{
    /* src/core/trig.hpp:76-80 */
    double d = (double)omega * t_over_2pi;
    return (float)((d - floor(d)) * 6.28318530717958647692);
}

static void sincos32(float x, float* so, float* co)
{
    /* src/core/trig.hpp:87-129 */
    const float two_over_pi = 0.636619772367581343076f;
    const float pa = 1.5707963705062866f;
    const float pb = -4.3711388286737929e-8f;
    const float s0 = -1.9515295891e-4f, s1 = 8.3321608736e-3f, s2 = -1.6666654611e-1f;
    const float c0 = 2.443315711809948e-5f, c1 = -1.388731625493765e-3f,
                c2 = 4.166664568298827e-2f;
    float qf = floorf(x * two_over_pi + 0.5f);
    int32_t q = (int32_t)qf;
    float y = x - qf * pa;
    y = y - qf * pb;
    float z = y * y;
    float sy = y + ((s0 * z + s1) * z + s2) * z * y;
    float cy = 1.0f - 0.5f * z + ((c0 * z + c1) * z + c2) * z * z;
    int32_t quad = q & 3;
    int swap = (quad & 1) != 0;
    float bs = swap ? cy : sy;
    float bc = swap ? sy : cy;
    *so = ((quad & 2) != 0) ? -bs : bs;
    *co = (((quad + 1) & 2) != 0) ? -bc : bc;
}

/* ------------------------------------------------------------------------ */
/* Evolve: src/core/evolve.cpp:28-121 and velocity :123-184                   */
/* ------------------------------------------------------------------------ */

void or_evolve(const or_desc* d, const float* tables, double t, float* fields)
{
    const uint32_t n = d->n;
    const size_t cells = (size_t)n * n;
    const float* h0_re = tables + 0 * cells;
    const float* h0_im = tables + 1 * cells;
    const float* h0c_re = tables + 2 * cells;
    const float* h0c_im = tables + 3 * cells;
    const float* omega = tables + 4 * cells;
    const float* kxt = tables + 5 * cells;
    const float* kzt = tables + 6 * cells;
    const float* kinv = tables + 7 * cells;
    const double top = t * 0.159154943091895335769;

    for (size_t i = 0; i < cells; ++i) {
        float ph = reduced_phase(omega[i], top);
        float s, c;
        sincos32(ph, &s, &c);
        float a_re = h0_re[i], a_im = h0_im[i], b_re = h0c_re[i], b_im = h0c_im[i];
        float fwd_re = a_re * c - a_im * s;
        float fwd_im = a_re * s + a_im * c;
        float bwd_re = b_re * c + b_im * s;
        float bwd_im = b_im * c - b_re * s;
        float hr = fwd_re + bwd_re;
        float hi = fwd_im + bwd_im;
        float kx = kxt[i], kz = kzt[i], ki = kinv[i];
        float sx = kx * ki, sz = kz * ki;
        float dx_re = sx * hi, dx_im = -sx * hr;
        float dz_re = sz * hi, dz_im = -sz * hr;
        float hx_re = -kx * hi, hx_im = kx * hr;
        float hz_re = -kz * hi, hz_im = kz * hr;
        float jxx = kx * sx, jzz = kz * sz, jxz = kx * sz;
        float jxx_re = jxx * hr, jxx_im = jxx * hi;
        float jzz_re = jzz * hr, jzz_im = jzz * hi;
        float jxz_re = jxz * hr, jxz_im = jxz * hi;
        fields[0 * cells + i] = hr - dx_im;
        fields[1 * cells + i] = hi + dx_re;
        fields[2 * cells + i] = dz_re - hx_im;
        fields[3 * cells + i] = dz_im + hx_re;
        fields[4 * cells + i] = hz_re - jxx_im;
        fields[5 * cells + i] = hz_im + jxx_re;
        fields[6 * cells + i] = jzz_re - jxz_im;
        fields[7 * cells + i] = jzz_im + jxz_re;

        if (d->velocity) {
            float dr = fwd_re - bwd_re;
            float di = fwd_im - bwd_im;
            float w = omega[i];
            float wsx = w * sx, wsz = w * sz;
            float ux_re = -wsx * dr, ux_im = -wsx * di;
            float uz_re = -wsz * dr, uz_im = -wsz * di;
            float uy_re = -w * di, uy_im = w * dr;
            fields[8 * cells + i] = ux_re - uy_im;
            fields[9 * cells + i] = ux_im + uy_re;
            fields[10 * cells + i] = uz_re;
            fields[11 * cells + i] = uz_im;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* FFT: src/core/fft.cpp:11-82 and src/core/fft_kernel_scalar.cpp:5-35        */
/* ------------------------------------------------------------------------ */

static void twiddles(uint32_t n, int sign, float* twr, float* twi)
{
    /* src/core/fft.cpp:24-33: angle = 2*pi*j/n in double, narrowed. */
    for (uint32_t j = 0; j < n / 2; ++j) {
        double a = 6.283185307179586476925286766559 * (double)j / (double)n;
        twr[j] = (float)cos(a);
        twi[j] = sign > 0 ? (float)sin(a) : (float)(-sin(a));
    }
}

static void fft_seq(uint32_t n, float* re, float* im, size_t stride, const float* twr,
                    const float* twi, float* work)
{
    float* xr = work;
    float* xi = work + n;
    float* yr = work + 2 * (size_t)n;
    float* yi = work + 3 * (size_t)n;
    for (uint32_t j = 0; j < n; ++j) {
        xr[j] = re[j * stride];
        xi[j] = im[j * stride];
    }
    for (uint32_t len = n, s = 1; len > 1; len >>= 1, s <<= 1) {
        uint32_t m = len >> 1;
        for (uint32_t p = 0; p < m; ++p) {
            float wr = twr[(size_t)p * s];
            float wi = twi[(size_t)p * s];
            for (uint32_t q = 0; q < s; ++q) {
                float ar = xr[s * p + q], ai = xi[s * p + q];
                float br = xr[s * (p + m) + q], bi = xi[s * (p + m) + q];
                yr[s * 2 * p + q] = ar + br;
                yi[s * 2 * p + q] = ai + bi;
                float dr = ar - br, di = ai - bi;
                yr[s * (2 * p + 1) + q] = dr * wr - di * wi;
                yi[s * (2 * p + 1) + q] = dr * wi + di * wr;
            }
        }
        float* t;
        t = xr; xr = yr; yr = t;
        t = xi; xi = yi; yi = t;
    }
    for (uint32_t j = 0; j < n; ++j) {
        re[j * stride] = xr[j];
        im[j * stride] = xi[j];
    }
}

void or_fft_1d(uint32_t n, float* re, float* im, int sign)
{
    float* twr = (float*)malloc(sizeof(float) * (n / 2 + 1));
    float* twi = (float*)malloc(sizeof(float) * (n / 2 + 1));
    float* work = (float*)malloc(sizeof(float) * 4 * n);
    twiddles(n, sign, twr, twi);
    fft_seq(n, re, im, 1, twr, twi, work);
    free(twr);
    free(twi);
    free(work);
}

void or_fft_2d(uint32_t n, float* re, float* im, int sign)
{
    /* src/core/fft.cpp:170-179: rows, then columns. Column batching in the
     * reference (transform_batch, :95-150) performs the same operations per
     * element as a single strided transform, so columns are done one by one. */
    float* twr = (float*)malloc(sizeof(float) * (n / 2 + 1));
    float* twi = (float*)malloc(sizeof(float) * (n / 2 + 1));
    float* work = (float*)malloc(sizeof(float) * 4 * n);
    twiddles(n, sign, twr, twi);
    for (uint32_t r = 0; r < n; ++r) fft_seq(n, re + (size_t)r * n, im + (size_t)r * n, 1, twr, twi, work);
    for (uint32_t c = 0; c < n; ++c) fft_seq(n, re + c, im + c, n, twr, twi, work);
    free(twr);
    free(twi);
    free(work);
}

/* ------------------------------------------------------------------------ */
/* Finalize: src/core/evolve.cpp:238-327 and velocity :186-203               */
/* ------------------------------------------------------------------------ */

void or_finalize(const or_desc* d, const float* fields, float* disp, float* normal,
                 float* velocity)
{
    const uint32_t n = d->n;
    const size_t cells = (size_t)n * n;
    const float lambda = d->choppiness;
    const float thr = d->foam_threshold;
    const float inv_thr = (thr > 1e-6f) ? (1.0f / thr) : 0.0f;
    for (size_t i = 0; i < cells; ++i) {
        float h = fields[0 * cells + i];
        float ddx = fields[1 * cells + i];
        float ddz = fields[2 * cells + i];
        float hx = fields[3 * cells + i];
        float hz = fields[4 * cells + i];
        float jxx = fields[5 * cells + i];
        float jzz = fields[6 * cells + i];
        float jxz = fields[7 * cells + i];
        float dxo = lambda * ddx;
        float dzo = lambda * ddz;
        float axx = 1.0f + lambda * jxx;
        float azz = 1.0f + lambda * jzz;
        float axz = lambda * jxz;
        float jac = axx * azz - axz * axz;
        float nx = -(hx * azz - axz * hz);
        float ny = jac;
        float nz = -(axx * hz - hx * axz);
        float len2 = nx * nx + ny * ny + nz * nz;
        float inv = (len2 > 0.0f) ? 1.0f / sqrtf(len2) : 0.0f;
        nx *= inv;
        ny *= inv;
        nz *= inv;
        float foam = (thr - jac) * inv_thr;
        if (foam < 0.0f) foam = 0.0f;
        if (foam > 1.0f) foam = 1.0f;
        disp[4 * i + 0] = dxo;
        disp[4 * i + 1] = h;
        disp[4 * i + 2] = dzo;
        disp[4 * i + 3] = foam;
        normal[4 * i + 0] = nx;
        normal[4 * i + 1] = ny;
        normal[4 * i + 2] = nz;
        normal[4 * i + 3] = jac;
        if (velocity && d->velocity) {
            velocity[4 * i + 0] = fields[8 * cells + i];
            velocity[4 * i + 1] = fields[9 * cells + i];
            velocity[4 * i + 2] = fields[10 * cells + i];
            velocity[4 * i + 3] = 0.0f;
        }
    }
}

void or_update(const or_desc* d, const float* tables, double t, float* fields, float* disp,
               float* normal, float* velocity)
{
    /* src/ocean.cpp:251-268: evolve, row FFTs, column FFTs, finalize. */
    const uint32_t n = d->n;
    const size_t cells = (size_t)n * n;
    const int nf = d->velocity ? 6 : 4;
    or_evolve(d, tables, t, fields);
    for (int f = 0; f < nf; ++f) {
        or_fft_2d(n, fields + (size_t)(2 * f) * cells, fields + (size_t)(2 * f + 1) * cells, +1);
    }
    or_finalize(d, fields, disp, normal, velocity);
}

/* ------------------------------------------------------------------------ */
/* Queries: src/ocean.cpp:322-452                                             */
/* ------------------------------------------------------------------------ */

typedef struct {
    size_t i00, i10, i01, i11;
    float w00, w10, w01, w11;
} tap_t;

static uint32_t wrap_index(int i, int n)
{
    i %= n;
    if (i < 0) i += n;
    return (uint32_t)i;
}

static tap_t make_tap(float u, float v, uint32_t n, float inv_cell)
{
    /* src/ocean.cpp:322-352 */
    tap_t t;
    float gu = u * inv_cell, gv = v * inv_cell;
    float fu = floorf(gu), fv = floorf(gv);
    int ni = (int)n;
    uint32_t x0 = wrap_index((int)fu, ni);
    uint32_t z0 = wrap_index((int)fv, ni);
    uint32_t x1 = (x0 + 1u) % n;
    uint32_t z1 = (z0 + 1u) % n;
    float tu = gu - fu, tv = gv - fv;
    t.i00 = ((size_t)z0 * n + x0) * 4;
    t.i10 = ((size_t)z0 * n + x1) * 4;
    t.i01 = ((size_t)z1 * n + x0) * 4;
    t.i11 = ((size_t)z1 * n + x1) * 4;
    t.w00 = (1.0f - tu) * (1.0f - tv);
    t.w10 = tu * (1.0f - tv);
    t.w01 = (1.0f - tu) * tv;
    t.w11 = tu * tv;
    return t;
}

static float fetch(const float* b, const tap_t* t, int c)
{
    /* src/ocean.cpp:354-358 */
    return b[t->i00 + c] * t->w00 + b[t->i10 + c] * t->w10 + b[t->i01 + c] * t->w01 +
           b[t->i11 + c] * t->w11;
}

void or_sample_at_iter(uint32_t n, float patch_length, const float* disp, const float* normal,
                       const float* velocity, float x, float z, int iters, float tol, float* out)
{
    /* src/ocean.cpp:375-452, with the fixed-point step count (the reference's
     * kInversionSteps = 4, src/ocean.cpp:366) as a parameter and an optional
     * stop once both parameter coordinates move by <= tol (tol = 0: never).
     * The step taken last is kept, as when the loop runs to its count. */
    const float inv_cell = (float)n / patch_length;
    float u = x, v = z;
    for (int it = 0; it < iters; ++it) {
        tap_t t = make_tap(u, v, n, inv_cell);
        const float un = x - fetch(disp, &t, 0);
        const float vn = z - fetch(disp, &t, 2);
        const int done = tol > 0.0f && fabsf(un - u) <= tol && fabsf(vn - v) <= tol;
        u = un;
        v = vn;
        if (done) break;
    }
    tap_t t = make_tap(u, v, n, inv_cell);
    out[1] = fetch(disp, &t, 0);
    out[0] = fetch(disp, &t, 1);
    out[2] = fetch(disp, &t, 2);
    out[6] = fetch(disp, &t, 3);
    float nx = fetch(normal, &t, 0);
    float ny = fetch(normal, &t, 1);
    float nz = fetch(normal, &t, 2);
    float len2 = nx * nx + ny * ny + nz * nz;
    if (len2 > 0.0f) {
        float inv = 1.0f / sqrtf(len2);
        nx *= inv;
        ny *= inv;
        nz *= inv;
    } else {
        nx = 0.0f;
        ny = 1.0f;
        nz = 0.0f;
    }
    out[3] = nx;
    out[4] = ny;
    out[5] = nz;
    if (velocity) {
        out[7] = fetch(velocity, &t, 0);
        out[8] = fetch(velocity, &t, 1);
        out[9] = fetch(velocity, &t, 2);
    } else {
        out[7] = out[8] = out[9] = 0.0f;
    }
}

void or_sample_at(uint32_t n, float patch_length, const float* disp, const float* normal,
                  const float* velocity, float x, float z, float* out)
{
    or_sample_at_iter(n, patch_length, disp, normal, velocity, x, z, 4, 0.0f, out);
}

void or_cascade_sample_many(uint32_t levels, const uint32_t* n, const float* patch_length,
                            const float* const* disp, const float* const* normal,
                            const float* const* velocity, const float* xz, uint64_t count, int iters,
                            float tol, float* out)
{
    /* src/cascade.cpp:80-153: levels visited in order, each with its own
     * inversion; height, offsets and velocity summed, normals summed then
     * renormalised, foam as 1 - prod(1 - foam_i). */
    float s[10];
    for (uint64_t i = 0; i < count; ++i) {
        const float x = xz[2 * i], z = xz[2 * i + 1];
        float height = 0.0f, offset_x = 0.0f, offset_z = 0.0f;
        float normal_x = 0.0f, normal_y = 0.0f, normal_z = 0.0f;
        float transparency = 1.0f;
        float vx = 0.0f, vy = 0.0f, vz = 0.0f;
        for (uint32_t l = 0; l < levels; ++l) {
            or_sample_at_iter(n[l], patch_length[l], disp[l], normal[l], velocity[l], x, z, iters, tol, s);
            height += s[0];
            offset_x += s[1];
            offset_z += s[2];
            normal_x += s[3];
            normal_y += s[4];
            normal_z += s[5];
            vx += s[7];
            vy += s[8];
            vz += s[9];
            transparency *= (1.0f - s[6]);
        }
        float* o = out + 10 * i;
        o[0] = height;
        o[1] = offset_x;
        o[2] = offset_z;
        o[6] = 1.0f - transparency;
        o[7] = vx;
        o[8] = vy;
        o[9] = vz;
        const float len2 = normal_x * normal_x + normal_y * normal_y + normal_z * normal_z;
        if (len2 > 0.0f) {
            const float inv = 1.0f / sqrtf(len2);
            o[3] = normal_x * inv;
            o[4] = normal_y * inv;
            o[5] = normal_z * inv;
        } else {
            o[3] = 0.0f;
            o[4] = 1.0f;
            o[5] = 0.0f;
        }
    }
}

void or_sample_many(uint32_t n, float patch_length, const float* disp, const float* normal,
                    const float* velocity, const float* xz, uint64_t count, float* out)
{
    for (uint64_t i = 0; i < count; ++i) {
        or_sample_at(n, patch_length, disp, normal, velocity, xz[2 * i], xz[2 * i + 1],
                     out + 10 * i);
    }
}

/* ------------------------------------------------------------------------ */
/* Persistent foam substep: src/foam.cpp:22-41 and :89-139                    */
/* ------------------------------------------------------------------------ */

static float sample_wrap(const float* f, float u, float v, int n)
{
    float fu = floorf(u), fv = floorf(v);
    float tu = u - fu, tv = v - fv;
    int x0 = (int)fu % n;
    if (x0 < 0) x0 += n;
    int z0 = (int)fv % n;
    if (z0 < 0) z0 += n;
    int x1 = (x0 + 1) % n;
    int z1 = (z0 + 1) % n;
    float a = f[(size_t)z0 * n + x0];
    float b = f[(size_t)z0 * n + x1];
    float c = f[(size_t)z1 * n + x0];
    float d = f[(size_t)z1 * n + x1];
    return a * (1.0f - tu) * (1.0f - tv) + b * tu * (1.0f - tv) + c * (1.0f - tu) * tv +
           d * tu * tv;
}

void or_foam_at_many(uint32_t n, float patch_length, const float* disp, const float* normal,
                     const float* foam, const float* xz, uint64_t count, float* out)
{
    /* src/foam.cpp:291-305: the ocean's inversion, then the wrapped fetch */
    const float cell = patch_length / (float)n;
    float s[10];
    for (uint64_t i = 0; i < count; ++i) {
        const float x = xz[2 * i], z = xz[2 * i + 1];
        or_sample_at(n, patch_length, disp, normal, NULL, x, z, s);
        const float u = (x - s[1]) / cell;
        const float v = (z - s[2]) / cell;
        out[i] = sample_wrap(foam, u, v, (int)n);
    }
}

void or_foam_step(uint32_t n, float cell, float dt, float decay, float gain, float scale,
                  float drift_x, float drift_z, const float* disp, const float* velocity,
                  const float* cur, float* next)
{
    const float inv_cell = 1.0f / cell;
    for (uint32_t z = 0; z < n; ++z) {
        for (uint32_t x = 0; x < n; ++x) {
            size_t i = (size_t)z * n + x;
            float vx = velocity[4 * i + 0] * scale + drift_x;
            float vz = velocity[4 * i + 2] * scale + drift_z;
            float su = (float)x - vx * dt * inv_cell;
            float sv = (float)z - vz * dt * inv_cell;
            float f = sample_wrap(cur, su, sv, (int)n);
            float src = disp[4 * i + 3];
            f = f * decay + src * gain;
            if (f > 1.0f) f = 1.0f;
            if (f < 0.0f) f = 0.0f;
            next[i] = f;
        }
    }
}

/* ------------------------------------------------------------------------ */
/* FP64 direct DFT (cf. tests/reference_dft.hpp:50-81): shares no structure  */
/* with the FFT; the phase index is reduced mod n before scaling.            */
/* ------------------------------------------------------------------------ */

static double* unit_circle(uint32_t n)
{
    double* cs = (double*)malloc(sizeof(double) * 2 * n);
    for (uint32_t j = 0; j < n; ++j) {
        double a = 6.283185307179586476925286766559 * (double)j / (double)n;
        cs[2 * j] = cos(a);
        cs[2 * j + 1] = sin(a);
    }
    return cs;
}

void or_dft2d_points(uint32_t n, const float* re, const float* im, uint32_t count,
                     const uint32_t* xs, const uint32_t* ys, double* out_re, double* out_im)
{
    double* cs = unit_circle(n);
    for (uint32_t p = 0; p < count; ++p) {
        const uint64_t x = xs[p], y = ys[p];
        double sr = 0.0, si = 0.0;
        for (uint32_t ky = 0; ky < n; ++ky) {
            const uint64_t base = (ky * y) % n;
            const float* rr = re + (size_t)ky * n;
            const float* ii = im + (size_t)ky * n;
            for (uint32_t kx = 0; kx < n; ++kx) {
                const uint64_t idx = (base + kx * x) % n;
                const double c = cs[2 * idx], s = cs[2 * idx + 1];
                const double xr = rr[kx], xi = ii[kx];
                sr += xr * c - xi * s;
                si += xr * s + xi * c;
            }
        }
        out_re[p] = sr;
        out_im[p] = si;
    }
    free(cs);
}

void or_dft2d_full(uint32_t n, const float* re, const float* im, double* out_re,
                   double* out_im)
{
    const size_t cells = (size_t)n * n;
    uint32_t* xs = (uint32_t*)malloc(sizeof(uint32_t) * cells);
    uint32_t* ys = (uint32_t*)malloc(sizeof(uint32_t) * cells);
    for (size_t i = 0; i < cells; ++i) {
        xs[i] = (uint32_t)(i % n);
        ys[i] = (uint32_t)(i / n);
    }
    or_dft2d_points(n, re, im, (uint32_t)cells, xs, ys, out_re, out_im);
    free(xs);
    free(ys);
}

/* ------------------------------------------------------------------------ */
/* iWave interaction field: src/core/iwave_step.cpp:7-124 and               */
/* src/interaction.cpp:212-391                                               */
/* ------------------------------------------------------------------------ */

void or_iwave_damping(uint32_t n, float damping, uint32_t absorb, float dt, float* c1, float* c2)
{
    /* src/interaction.cpp:212-241 */
    const float a0 = damping;
    const int w = (int)absorb;
    const float span = dt * (float)(w > 1 ? w : 1);
    const float a_edge = 4.0f / (span > 1e-6f ? span : 1e-6f);
    for (uint32_t z = 0; z < n; ++z) {
        for (uint32_t x = 0; x < n; ++x) {
            int dx = (int)x < (int)(n - 1 - x) ? (int)x : (int)(n - 1 - x);
            int dz = (int)z < (int)(n - 1 - z) ? (int)z : (int)(n - 1 - z);
            int d = dx < dz ? dx : dz;
            float alpha = a0;
            if (w > 0 && d < w) {
                float t = (float)(w - d) / (float)w;
                alpha += a_edge * t * t;
            }
            float ad = alpha * dt;
            size_t i = (size_t)z * n + x;
            c1[i] = 1.0f / (1.0f + ad);
            c2[i] = 1.0f - ad;
        }
    }
}

void or_iwave_step(uint32_t n, uint32_t p, size_t stride, const float* taps, const float* c1,
                   const float* c2, float gdt2, const float* cur, float* old)
{
    /* src/core/iwave_step.cpp:7-54: j outer, i inner, one float accumulator */
    const int pp = (int)p, w = 2 * pp + 1;
    for (uint32_t z = 0; z < n; ++z) {
        for (uint32_t x = 0; x < n; ++x) {
            const float* centre = cur + (size_t)z * stride + x;
            float acc = 0.0f;
            const float* tap = taps;
            for (int j = -pp; j <= pp; ++j) {
                const float* srow = centre + (ptrdiff_t)j * (ptrdiff_t)stride - pp;
                for (int i = 0; i < w; ++i) acc += tap[i] * srow[i];
                tap += w;
            }
            const size_t oi = (size_t)z * n + x;
            const float hc = *centre;
            const float hp = old[(size_t)z * stride + x];
            const float v = c1[oi] * (2.0f * hc - c2[oi] * hp - gdt2 * acc);
            old[(size_t)z * stride + x] = (v > -1.0e-30f && v < 1.0e-30f) ? 0.0f : v;
        }
    }
}

void or_iwave_finalize(uint32_t n, size_t stride, const float* cur, const float* old,
                       float inv_two_cell, float inv_dt, float* out)
{
    /* src/core/iwave_step.cpp:93-124 */
    for (uint32_t z = 0; z < n; ++z) {
        for (uint32_t x = 0; x < n; ++x) {
            const float* c = cur + (size_t)z * stride + x;
            float gx = (c[1] - c[-1]) * inv_two_cell;
            float gz = (c[stride] - c[-(ptrdiff_t)stride]) * inv_two_cell;
            float vy = (*c - old[(size_t)z * stride + x]) * inv_dt;
            float* d = out + ((size_t)z * n + x) * 4;
            d[0] = *c;
            d[1] = gx;
            d[2] = gz;
            d[3] = vy;
        }
    }
}

static float ricker(float r2, float inv2s2)
{
    float u = r2 * inv2s2;
    return (1.0f - u) * expf(-u);
}

/* One disturbance (world_x, world_z, radius, strength, velocity_y,
 * velocity_x, velocity_z) stamped into both levels (src/interaction.cpp:322-391). */
void or_iwave_inject(uint32_t n, size_t stride, float cell, int32_t origin_x, int32_t origin_z,
                     float dt, const float* d, float sub_time, float scale, float* cur, float* old)
{
    float sigma = d[2] > 0.25f * cell ? d[2] : 0.25f * cell;
    float inv2s2 = 1.0f / (2.0f * sigma * sigma);
    float wx = d[0] + d[5] * sub_time;
    float wz = d[1] + d[6] * sub_time;
    float gx = (wx - (float)origin_x * cell) / cell;
    float gz = (wz - (float)origin_z * cell) / cell;
    int rad = (int)ceilf(4.0f * sigma / cell);
    int fx = (int)floorf(gx), fz = (int)floorf(gz);
    int x0 = fx - rad < 0 ? 0 : fx - rad;
    int x1 = fx + rad > (int)n - 1 ? (int)n - 1 : fx + rad;
    int z0 = fz - rad < 0 ? 0 : fz - rad;
    int z1 = fz + rad > (int)n - 1 ? (int)n - 1 : fz + rad;
    if (x1 < x0 || z1 < z0) return;
    double sum = 0.0;
    for (int z = z0; z <= z1; ++z) {
        for (int x = x0; x <= x1; ++x) {
            float px = ((float)x + 0.5f) - gx;
            float pz = ((float)z + 0.5f) - gz;
            sum += ricker((px * px + pz * pz) * cell * cell, inv2s2);
        }
    }
    float mean = (float)(sum / ((double)(x1 - x0 + 1) * (double)(z1 - z0 + 1)));
    float disp = -d[3] * scale;
    float vel = d[4] * scale;
    for (int z = z0; z <= z1; ++z) {
        for (int x = x0; x <= x1; ++x) {
            float px = ((float)x + 0.5f) - gx;
            float pz = ((float)z + 0.5f) - gz;
            float r2 = (px * px + pz * pz) * cell * cell;
            float s = ricker(r2, inv2s2) - mean;
            float dd = disp * s;
            float dv = vel * s;
            size_t ci = (size_t)z * stride + (size_t)x;
            cur[ci] += dd;
            old[ci] += dd - dv * dt;
        }
    }
}

/* Nearest-fluid table by multi-source BFS (src/interaction.cpp:255-292);
 * returns the number of solid cells written to `solid`. */
uint32_t or_iwave_nearest(uint32_t n, const uint8_t* mask, uint32_t* nearest, uint32_t* solid)
{
    size_t cells = (size_t)n * n;
    uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * cells);
    size_t head = 0, tail = 0;
    uint32_t ns = 0;
    for (size_t i = 0; i < cells; ++i) {
        if (mask[i] == 0) {
            nearest[i] = (uint32_t)i;
            q[tail++] = (uint32_t)i;
        } else {
            nearest[i] = 0xFFFFFFFFu;
            solid[ns++] = (uint32_t)i;
        }
    }
    const int dx[4] = {1, -1, 0, 0}, dz[4] = {0, 0, 1, -1};
    while (head < tail) {
        uint32_t i = q[head++];
        int x = (int)(i % n), z = (int)(i / n);
        for (int e = 0; e < 4; ++e) {
            int nx = x + dx[e], nz = z + dz[e];
            if (nx < 0 || nz < 0 || nx >= (int)n || nz >= (int)n) continue;
            uint32_t j = (uint32_t)nz * n + (uint32_t)nx;
            if (nearest[j] == 0xFFFFFFFFu) {
                nearest[j] = nearest[i];
                q[tail++] = j;
            }
        }
    }
    free(q);
    return ns;
}

void or_iwave_obstruction(uint32_t n, size_t stride, const uint32_t* solid, uint32_t count,
                          const uint32_t* nearest, int dirichlet, float* cur)
{
    /* src/interaction.cpp:295-318 */
    for (uint32_t s = 0; s < count; ++s) {
        uint32_t i = solid[s];
        if (dirichlet) {
            cur[(i / n) * stride + (i % n)] = 0.0f;
        } else {
            uint32_t f = nearest[i];
            if (f == 0xFFFFFFFFu) continue;
            cur[(i / n) * stride + (i % n)] = cur[(f / n) * stride + (f % n)];
        }
    }
}
