// oceanlib-b200: device building blocks shared by the frame kernels.
//
// Everything here is compiled with -fmad=false (see build.py): no multiply is
// ever fused into an add, so each float/double operation rounds exactly where
// the reference's scalar kernels round. Where the "fast" FFT form wants fused
// multiply-adds it asks for them explicitly with __fmaf_rn.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace ocean_b200 {

// ---------------------------------------------------------------------------
// Constants shared with the reference's arithmetic. These are the values of
// src/core/trig.hpp:33-55 and src/core/spectrum.hpp:85-92 (the same IEEE
// numbers have to be used for the results to match bit for bit).
// ---------------------------------------------------------------------------
constexpr double kInvTwoPiD = 0.159154943091895335769;
constexpr double kTwoPiD = 6.28318530717958647692;

// ---------------------------------------------------------------------------
// Phase fold and sine/cosine (reference: src/core/trig.hpp:76-129).
// omega*t is folded into [0, 2pi) in double - the one place FP64 is used per
// frame - then a Cody-Waite quadrant reduction and two short minimax
// polynomials give sin and cos together in float.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float fold_phase(float omega, double t_over_2pi)
{
    const double d = static_cast<double>(omega) * t_over_2pi;
    return static_cast<float>((d - floor(d)) * kTwoPiD);
}

__device__ __forceinline__ void sincos_poly(float x, float& s_out, float& c_out)
{
    const float qf = floorf(x * 0.636619772367581343076f + 0.5f);
    const int q = static_cast<int>(qf);
    float y = x - qf * 1.5707963705062866f;
    y = y - qf * -4.3711388286737929e-8f;
    const float z = y * y;
    const float sy = y + ((-1.9515295891e-4f * z + 8.3321608736e-3f) * z + -1.6666654611e-1f) * z * y;
    const float cy = 1.0f - 0.5f * z +
                     ((2.443315711809948e-5f * z + -1.388731625493765e-3f) * z + 4.166664568298827e-2f) * z * z;
    const int quad = q & 3;
    const bool swap = (quad & 1) != 0;
    const float bs = swap ? cy : sy;
    const float bc = swap ? sy : cy;
    s_out = (quad & 2) ? -bs : bs;
    c_out = ((quad + 1) & 2) ? -bc : bc;
}

// ---------------------------------------------------------------------------
// Shared-memory layout of one N-point sequence: one float2 of padding after
// every 16 values. Every access pattern of the Stockham stage blocks below
// (lanes walking consecutive indices, or lanes writing 2^r-element runs) then
// touches 16 distinct 8-byte bank pairs per half-warp, and because the
// padding is additive the per-register offsets are compile-time constants
// (an XOR swizzle would cost integer work on every access).
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pad_idx(int i) { return i + (i >> 4); }

// float2 slots one padded sequence of n values occupies.
__host__ __device__ constexpr int padded_len(int n) { return n + n / 16; }

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }
__host__ __device__ constexpr int cmin(int a, int b) { return a < b ? a : b; }

template <int R>
__device__ __forceinline__ int bitrev(int s)
{
    int o = 0;
#pragma unroll
    for (int i = 0; i < R; ++i) o |= ((s >> i) & 1) << (R - 1 - i);
    return o;
}

// The transforms' arithmetic, a template argument AR of every stage block:
//   kArExact    the reference's operations in FP32, each multiply and add
//               rounded (bit-identical to src/core/fft_kernel_scalar.cpp);
//   kArFast     the same dataflow with fused multiply-adds;
//   kArPrecise  each stage block's butterflies in FP64 on the values held in
//               registers, rounded to FP32 once when the block stores them:
//               three roundings per point and dimension at N = 512 instead
//               of nine stages of them (within 1.5e-6 of FP64 on every
//               channel of a 512^2 frame, where the FP32 forms reach 3.5e-6).
constexpr int kArExact = 0;
constexpr int kArFast = 1;
constexpr int kArPrecise = 2;

// Butterfly of the radix-2 Stockham stage (reference:
// src/core/fft_kernel_scalar.cpp:19-33): a' = a + b, b' = (a - b) * w.
// kArExact keeps the reference's separate multiplies and adds; kArFast fuses.
template <int AR>
__device__ __forceinline__ void butterfly(float2& a, float2& b, float2 w)
{
    static_assert(AR != kArPrecise, "the precise form works on doubles (butterfly_f64)");
    const float ar = a.x, ai = a.y, br = b.x, bi = b.y;
    a.x = ar + br;
    a.y = ai + bi;
    const float dr = ar - br;
    const float di = ai - bi;
    if constexpr (AR == kArFast) {
        b.x = __fmaf_rn(dr, w.x, -(di * w.y));
        b.y = __fmaf_rn(dr, w.y, di * w.x);
    } else {
        b.x = dr * w.x - di * w.y;
        b.y = dr * w.y + di * w.x;
    }
}

// The same butterfly in FP64 (kArPrecise), the twiddle widened from FP32.
__device__ __forceinline__ void butterfly_f64(double& ar, double& ai, double& br, double& bi, float2 w)
{
    const double wx = w.x, wy = w.y;
    const double dr = ar - br, di = ai - bi;
    ar += br;
    ai += bi;
    br = fma(dr, wx, -(di * wy));
    bi = fma(dr, wy, di * wx);
}

// ---------------------------------------------------------------------------
// One block of r consecutive radix-2 Stockham stages, L0 .. L0+r-1, on a
// sequence of N = 2^LOG_N points held (swizzled) in shared memory and worked
// on by a group of G lanes. A group of one warp or less synchronises with
// __syncwarp; a sequence spanning several warps (G > 32) uses the CTA
// barrier, so every thread of the CTA must run the same transforms.
//
// Index algebra. At stage L0 an element index is [T : r bits][P : w bits]
// [q : L0 bits] with w = LOG_N - r - L0. The r stages pair the elements that
// differ only in T; a lane owns fixed (P, q) and keeps the 2^r values of T in
// registers. At block-local stage k the twiddle is W^(p << (L0+k)) with
// p = (R_k << w) | P, R_k being the T bits below the pairing bit; the table
// `tw` holds, for every stage l, the entries W^(p << l) contiguously from
// offset N - (N >> l). After the r stages the value in register slot S
// belongs at [P][bitrev_r(S)][q]. This performs exactly the butterflies of
// the reference's stage loop (src/core/fft.cpp:70-74) with the same operands
// and twiddles, so the EXACT form is bit-identical to it.
// ---------------------------------------------------------------------------
// Barrier for the lanes of one sequence group (see StageBlock).
template <int G>
__device__ __forceinline__ void group_sync()
{
    if constexpr (G > 32) {
        __syncthreads();
    } else {
        __syncwarp();
    }
}

template <int LOG_N, int G, int L0, int AR>
struct StageBlock {
    static constexpr int N = 1 << LOG_N;
    static constexpr int E = N / G;                  // values per lane
    static constexpr int RMAX = ilog2c(E);
    static constexpr int r = cmin(RMAX, LOG_N - L0);
    static constexpr int RR = 1 << r;
    static constexpr int C = (N >> r) / G;           // (P,q) combos per lane
    static constexpr int w = LOG_N - r - L0;

    __device__ __forceinline__ static void run(float2* seq, const float2* tw, int lane)
    {
        float2 v[C][RR];
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int c = lane + G * k;
#pragma unroll
            for (int t = 0; t < RR; ++t) v[k][t] = seq[pad_idx((t << (LOG_N - r)) | c)];
        }
        group_sync<G>();
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int c = lane + G * k;
            const int P = c >> L0;
            if constexpr (AR == kArPrecise) {
                double xr[RR], xi[RR];
#pragma unroll
                for (int t = 0; t < RR; ++t) {
                    xr[t] = v[k][t].x;
                    xi[t] = v[k][t].y;
                }
#pragma unroll
                for (int s = 0; s < r; ++s) {
                    const int half = RR >> (s + 1);
                    const float2* twl = tw + (N - (N >> (L0 + s)));
#pragma unroll
                    for (int S = 0; S < RR; ++S) {
                        if (S & half) continue;
                        butterfly_f64(xr[S], xi[S], xr[S + half], xi[S + half], twl[((S & (half - 1)) << w) | P]);
                    }
                }
#pragma unroll
                for (int t = 0; t < RR; ++t) v[k][t] = make_float2(__double2float_rn(xr[t]), __double2float_rn(xi[t]));
            } else {
#pragma unroll
                for (int s = 0; s < r; ++s) {
                    const int half = RR >> (s + 1);
                    const int l = L0 + s;
                    const float2* twl = tw + (N - (N >> l));
#pragma unroll
                    for (int S = 0; S < RR; ++S) {
                        if (S & half) continue;
                        const int Rk = S & (half - 1);
                        const float2 wv = twl[(Rk << w) | P];
                        butterfly<AR>(v[k][S], v[k][S + half], wv);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int c = lane + G * k;
            const int P = c >> L0;
            const int q = c & ((1 << L0) - 1);
#pragma unroll
            for (int S = 0; S < RR; ++S) {
                const int out = (P << (L0 + r)) | (bitrev<r>(S) << L0) | q;
                seq[pad_idx(out)] = v[k][S];
            }
        }
        group_sync<G>();
        if constexpr (L0 + r < LOG_N) StageBlock<LOG_N, G, L0 + r, AR>::run(seq, tw, lane);
    }
};

// The complete unnormalised inverse transform of one sequence.
template <int LOG_N, int G, int AR>
__device__ __forceinline__ void fft_sequence(float2* seq, const float2* tw, int lane)
{
    StageBlock<LOG_N, G, 0, AR>::run(seq, tw, lane);
}

// Lanes per sequence: each lane keeps 16 values (a 4-stage block) where the
// sequence is long enough, capped at one warp.
__host__ __device__ constexpr int lanes_for(int log_n)
{
    return (log_n - 4) >= 5 ? 32 : (1 << (log_n - 4 < 0 ? 0 : log_n - 4));
}

// ---------------------------------------------------------------------------
// Paired sequences: two sequences A and B of the same length transformed in
// lockstep, each register and shared-memory slot holding the same index of
// both. Shared memory holds a pair as float4 (A.re, B.re, A.im, B.im) per
// index, one float4 of padding after every 8; in registers (A.re, B.re) and
// (A.im, B.im) are each one 64-bit f32x2 operand. Blackwell's packed FP32
// instructions (add/sub/mul.rn.f32x2) do the two sequences' operations in one
// instruction, each lane rounded exactly as the scalar instruction rounds, so
// the results are bit-identical to transforming A and B one at a time.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int pad4(int i) { return i + (i >> 3); }
__host__ __device__ constexpr int padded_len4(int n) { return n + n / 8; }

// Lanes per sequence pair: twice the single-sequence count, so a pair of
// sequences takes as many threads as the two sequences alone, each lane
// keeping 8 indices (16 at N = 1024) of both.
__host__ __device__ constexpr int pair_lanes(int log_n) { return 2 * lanes_for(log_n); }

using f32x2 = unsigned long long;  // two floats, low word first

__device__ __forceinline__ f32x2 px_add(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 px_sub(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 px_mul(f32x2 a, f32x2 b)
{
    f32x2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f32x2 px_fma(f32x2 a, f32x2 b, f32x2 c)
{
    f32x2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ f32x2 px_pack(float lo, float hi)
{
    f32x2 d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ void px_unpack(f32x2 v, float& lo, float& hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}

// The radix-2 butterfly of `butterfly` on a pair: (ar, ai) and (br, bi) hold
// the real and imaginary parts of both sequences, (wx, wy) the twiddle's
// parts duplicated. EXACT: a' = a + b; b' = (dr wx - di wy, dr wy + di wx),
// every product rounded before the add. The assembler contracts a packed
// multiply into a packed add or subtract that consumes it (one fused
// multiply-add, rounded once) even with contraction disabled, so the four
// products are packed multiplies and the two sums that combine them are
// scalar adds of their halves. kArFast fuses as `butterfly<kArFast>` does.
template <int AR>
__device__ __forceinline__ void butterfly_pair(f32x2& ar, f32x2& ai, f32x2& br, f32x2& bi, f32x2 wx, f32x2 wy)
{
    const f32x2 dr = px_sub(ar, br);
    const f32x2 di = px_sub(ai, bi);
    ar = px_add(ar, br);
    ai = px_add(ai, bi);
    if constexpr (AR == kArFast) {
        const f32x2 nwy = wy ^ 0x8000000080000000ull;
        br = px_fma(dr, wx, px_mul(di, nwy));
        bi = px_fma(dr, wy, px_mul(di, wx));
    } else {
        float rx0, rx1, iy0, iy1, ry0, ry1, ix0, ix1;
        px_unpack(px_mul(dr, wx), rx0, rx1);
        px_unpack(px_mul(di, wy), iy0, iy1);
        px_unpack(px_mul(dr, wy), ry0, ry1);
        px_unpack(px_mul(di, wx), ix0, ix1);
        br = px_pack(__fsub_rn(rx0, iy0), __fsub_rn(rx1, iy1));
        bi = px_pack(__fadd_rn(ry0, ix0), __fadd_rn(ry1, ix1));
    }
}

// Barrier over the G2 lanes of one pair: the warp when the pair fits in one,
// else named barrier `id` (1 + the pair's index in the CTA) over its warps.
template <int G2>
__device__ __forceinline__ void pair_sync(int id)
{
    if constexpr (G2 <= 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(id), "n"(G2) : "memory");
    }
}

// StageBlock's r stages on a pair of sequences (same index algebra, lane
// ownership and twiddles; `tw` is the same float2 table as StageBlock's).
template <int LOG_N, int G2, int L0, int AR>
struct PairBlock {
    static constexpr int N = 1 << LOG_N;
    static constexpr int E = N / G2;
    static constexpr int RMAX = ilog2c(E);
    static constexpr int r = cmin(RMAX, LOG_N - L0);
    static constexpr int RR = 1 << r;
    static constexpr int C = (N >> r) / G2;
    static constexpr int w = LOG_N - r - L0;

    __device__ __forceinline__ static void run(ulonglong2* seq, const float2* tw, int lane, int bar_id)
    {
        f32x2 re[C][RR], im[C][RR];
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int c = lane + G2 * k;
#pragma unroll
            for (int t = 0; t < RR; ++t) {
                const ulonglong2 v = seq[pad4((t << (LOG_N - r)) | c)];
                re[k][t] = v.x;
                im[k][t] = v.y;
            }
        }
        pair_sync<G2>(bar_id);
        if constexpr (AR == kArPrecise) {
            // The pair's two sequences one after the other, each as doubles
            // (8 complex values: 32 registers), rounded back into its half
            // of the packed registers.
#pragma unroll
            for (int k = 0; k < C; ++k) {
                const int c = lane + G2 * k;
                const int P = c >> L0;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    double xr[RR], xi[RR];
#pragma unroll
                    for (int t = 0; t < RR; ++t) {
                        float r0, r1, i0, i1;
                        px_unpack(re[k][t], r0, r1);
                        px_unpack(im[k][t], i0, i1);
                        xr[t] = h ? r1 : r0;
                        xi[t] = h ? i1 : i0;
                    }
#pragma unroll
                    for (int s = 0; s < r; ++s) {
                        const int half = RR >> (s + 1);
                        const float2* twl = tw + (N - (N >> (L0 + s)));
#pragma unroll
                        for (int S = 0; S < RR; ++S) {
                            if (S & half) continue;
                            butterfly_f64(xr[S], xi[S], xr[S + half], xi[S + half], twl[((S & (half - 1)) << w) | P]);
                        }
                    }
#pragma unroll
                    for (int t = 0; t < RR; ++t) {
                        float r0, r1, i0, i1;
                        px_unpack(re[k][t], r0, r1);
                        px_unpack(im[k][t], i0, i1);
                        const float nr = __double2float_rn(xr[t]), ni = __double2float_rn(xi[t]);
                        re[k][t] = h ? px_pack(r0, nr) : px_pack(nr, r1);
                        im[k][t] = h ? px_pack(i0, ni) : px_pack(ni, i1);
                    }
                }
            }
        } else {
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int c = lane + G2 * k;
            const int P = c >> L0;
#pragma unroll
            for (int s = 0; s < r; ++s) {
                const int half = RR >> (s + 1);
                const int l = L0 + s;
                const float2* twl = tw + (N - (N >> l));
#pragma unroll
                for (int S = 0; S < RR; ++S) {
                    if (S & half) continue;
                    const int Rk = S & (half - 1);
                    // One 8-byte load, duplicated into both lanes of each
                    // f32x2 in registers (a 16-byte (wx, wx, wy, wy) table
                    // entry costs twice the shared-memory wavefronts).
                    const float2 wv = twl[(Rk << w) | P];
                    butterfly_pair<AR>(re[k][S], im[k][S], re[k][S + half], im[k][S + half], px_pack(wv.x, wv.x),
                                       px_pack(wv.y, wv.y));
                }
            }
        }
        }
#pragma unroll
        for (int k = 0; k < C; ++k) {
            const int c = lane + G2 * k;
            const int P = c >> L0;
            const int q = c & ((1 << L0) - 1);
#pragma unroll
            for (int S = 0; S < RR; ++S) {
                const int out = (P << (L0 + r)) | (bitrev<r>(S) << L0) | q;
                seq[pad4(out)] = make_ulonglong2(re[k][S], im[k][S]);
            }
        }
        pair_sync<G2>(bar_id);
        if constexpr (L0 + r < LOG_N) PairBlock<LOG_N, G2, L0 + r, AR>::run(seq, tw, lane, bar_id);
    }
};

// The unnormalised inverse transforms of the pair at `seq`.
template <int LOG_N, int G2, int AR>
__device__ __forceinline__ void fft_pair(ulonglong2* seq, const float2* tw, int lane, int bar_id)
{
    PairBlock<LOG_N, G2, 0, AR>::run(seq, tw, lane, bar_id);
}


}  // namespace ocean_b200
