// oceanlib-b200: iWave stencil fit (init-time, host, double precision).
//
// The stencil g is D4-symmetric: one unknown per orbit {(±a, ±b), (±b, ±a)}
// with 0 <= b <= a <= P. Its symbol is -sum_orbit g_ab * (phi_ab(k) - |orbit|)
// with phi_ab = sum over the orbit of cos(k . offset); the centre tap is fixed
// by requiring a zero symbol at k = 0. The remaining unknowns minimise a
// relative-error-weighted squared misfit to S(k) on a (fit_samples+1)^2 grid
// over the first quadrant of the resolved band (weight 1/S^2 in band,
// 0.02/S_edge^2 outside), solved by Cholesky on the normal equations with a
// tiny ridge. Then the realised symbol is scanned on a 193^2 grid for its
// extremes (the stability limit) and peak in-band error.
//
// Every double operation runs in the order of the reference's builder
// (src/core/iwave_kernel.cpp:177-437), so the float taps are the same bits and
// the device stencil step reproduces the reference field exactly.
#include "iwave_stencil.h"

#include <cmath>
#include <stdexcept>

namespace ocean_b200 {
namespace {

constexpr double kPi = 3.14159265358979323846;

double symbol(double k, double depth)
{
    if (k <= 0.0) return 0.0;
    if (depth <= 0.0) return k;
    return k * std::tanh(k * depth);
}

struct Orbit {
    int count = 0;
    int off[8][2];
};

// The members of orbit (a, b), in a fixed enumeration order (the order the
// cosines are summed in).
Orbit orbit(int a, int b)
{
    Orbit o;
    auto push = [&](int i, int j) {
        o.off[o.count][0] = i;
        o.off[o.count][1] = j;
        ++o.count;
    };
    if (a == 0) {
        push(0, 0);
        return o;
    }
    if (b == 0) {
        push(a, 0);
        push(-a, 0);
        push(0, a);
        push(0, -a);
        return o;
    }
    for (int sa : {a, -a})
        for (int sb : {b, -b}) push(sa, sb);
    if (a != b)
        for (int sa : {a, -a})
            for (int sb : {b, -b}) push(sb, sa);
    return o;
}

// In-place Cholesky factorisation and solve of the SPD system (n x n, row-major).
bool spd_solve(std::vector<double>& m, std::vector<double>& rhs, int n)
{
    auto at = [&](int i, int j) -> double& { return m[static_cast<size_t>(i) * n + j]; };
    for (int i = 0; i < n; ++i) {
        for (int j = 0; j <= i; ++j) {
            double s = at(i, j);
            for (int k = 0; k < j; ++k) s -= at(i, k) * at(j, k);
            if (i == j) {
                if (!(s > 0.0)) return false;
                at(i, i) = std::sqrt(s);
            } else {
                at(i, j) = s / at(j, j);
            }
        }
    }
    for (int i = 0; i < n; ++i) {
        double s = rhs[i];
        for (int k = 0; k < i; ++k) s -= at(i, k) * rhs[k];
        rhs[i] = s / at(i, i);
    }
    for (int i = n - 1; i >= 0; --i) {
        double s = rhs[i];
        for (int k = i + 1; k < n; ++k) s -= at(k, i) * rhs[k];
        rhs[i] = s / at(i, i);
    }
    return true;
}

}  // namespace

IWaveStencil build_iwave_stencil(uint32_t radius, double cell, double depth, uint32_t fit_samples,
                                 double band_low_frac)
{
    if (radius < 1 || radius > 12) throw std::invalid_argument("iwave kernel radius");
    if (!(cell > 0.0)) throw std::invalid_argument("iwave cell size");
    const int p = static_cast<int>(radius);
    const int width = 2 * p + 1;
    const double k_max = kPi / cell;

    IWaveStencil st;
    st.radius = radius;
    st.width = static_cast<uint32_t>(width);
    st.cell = static_cast<float>(cell);
    st.taps.assign(static_cast<size_t>(width) * width, 0.0f);

    // Orbit basis, a outer, b inner; basis 0 is the centre.
    std::vector<int> ba, bb;
    for (int a = 0; a <= p; ++a)
        for (int b = 0; b <= a; ++b) {
            ba.push_back(a);
            bb.push_back(b);
        }
    const int m = static_cast<int>(ba.size());
    const int u = m - 1;  // unknowns (centre eliminated)
    std::vector<Orbit> orbits(m);
    for (int t = 0; t < m; ++t) orbits[t] = orbit(ba[t], bb[t]);

    std::vector<double> ata(static_cast<size_t>(u) * u, 0.0), atb(u, 0.0), psi(u, 0.0);
    const double k_lo = band_low_frac * k_max;
    const int ns = static_cast<int>(fit_samples);
    for (int zi = 0; zi <= ns; ++zi) {
        for (int xi = 0; xi <= ns; ++xi) {
            const double kx = k_max * xi / ns;
            const double kz = k_max * zi / ns;
            const double kk = std::sqrt(kx * kx + kz * kz);
            const double s = symbol(kk, depth);
            const bool in_band = kk >= k_lo && kk <= k_max;
            const double ref = in_band ? s : symbol(kk < k_lo ? k_lo : k_max, depth);
            double w = 1.0 / (ref * ref);
            if (!in_band) w *= 0.02;
            for (int t = 1; t < m; ++t) {
                const Orbit& o = orbits[t];
                double phi = 0.0;
                for (int e = 0; e < o.count; ++e)
                    phi += std::cos(kx * o.off[e][0] * cell + kz * o.off[e][1] * cell);
                psi[t - 1] = phi - o.count;
            }
            for (int r = 0; r < u; ++r) {
                const double wr = w * psi[r];
                atb[r] += wr * s;
                for (int c = 0; c <= r; ++c) ata[static_cast<size_t>(r) * u + c] += wr * psi[c];
            }
        }
    }
    double trace = 0.0;
    for (int r = 0; r < u; ++r) trace += ata[static_cast<size_t>(r) * u + r];
    const double ridge = 1e-12 * trace / u;
    for (int r = 0; r < u; ++r) {
        ata[static_cast<size_t>(r) * u + r] += ridge;
        for (int c = r + 1; c < u; ++c)
            ata[static_cast<size_t>(r) * u + c] = ata[static_cast<size_t>(c) * u + r];
    }
    if (!spd_solve(ata, atb, u)) throw std::invalid_argument("iwave stencil fit is singular");

    std::vector<double> g(m, 0.0);
    double rest = 0.0;
    for (int t = 1; t < m; ++t) {
        g[t] = atb[t - 1];
        rest += orbits[t].count * g[t];
    }
    g[0] = -rest;
    for (int t = 0; t < m; ++t) {
        const float v = static_cast<float>(g[t]);
        for (int e = 0; e < orbits[t].count; ++e) {
            const int i = orbits[t].off[e][0], j = orbits[t].off[e][1];
            st.taps[static_cast<size_t>(j + p) * width + (i + p)] = v;
        }
    }

    // Realised symbol scan (reference: src/core/iwave_kernel.cpp:158-173, :410-437).
    const double dx = st.cell;
    constexpr int kScan = 192;
    double worst = 0.0, peak = 0.0, trough = 0.0;
    st.band_low = band_low_frac * k_max;
    for (int zi = 0; zi <= kScan; ++zi) {
        for (int xi = 0; xi <= kScan; ++xi) {
            const double kx = k_max * xi / kScan;
            const double kz = k_max * zi / kScan;
            const double kk = std::sqrt(kx * kx + kz * kz);
            double rs = 0.0;
            for (int j = -p; j <= p; ++j)
                for (int i = -p; i <= p; ++i)
                    rs += static_cast<double>(st.taps[static_cast<size_t>(j + p) * width + (i + p)]) *
                          std::cos(kx * i * dx + kz * j * dx);
            if (rs > peak) peak = rs;
            if (rs < trough) trough = rs;
            if (kk >= st.band_low && kk <= k_max) {
                const double tr = symbol(kk, depth);
                if (tr > 0.0) {
                    const double e = std::fabs(rs / tr - 1.0);
                    if (e > worst) worst = e;
                }
            }
        }
    }
    st.max_symbol = peak;
    st.min_symbol = trough;
    st.peak_relative_error = worst;
    return st;
}

}  // namespace ocean_b200
