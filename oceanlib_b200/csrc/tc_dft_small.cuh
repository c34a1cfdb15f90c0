// oceanlib-b200: the tensor-core DFT form at N = 64, 128 and 256 (sm_100a,
// tcgen05).
//
// The same four-step factorisation and exact digit-sliced GEMMs as the
// 512-point engine (tc_dft.cuh), with N = N1 x N2:
//
//   N = 256: 16 x 16     N = 128: 8 x 16     N = 64: 8 x 8
//
//   n = N2 n1 + n2,  k = k1 + N1 k2
//   Y[n2, k1] = sum_n1 W_N1^(n1 k1) x[N2 n1 + n2]         stage 1 (GEMM)
//   Z[n2, k1] = W_N^(n2 k1) Y[n2, k1]                     twiddle (FP64)
//   X[k1 + N1 k2] = sum_n2 W_N2^(n2 k2) Z[n2, k1]          stage 3 (GEMM)
//
// A frame task holds SEQS sequences with SEQS x N = 16 x threads (6144 with
// velocity, 4096 without, at every one of these sizes), so the operands are
// one size everywhere: stage 1 has SEQS x N2 rows of K = 2 N1, stage 3
// SEQS x N1 rows of K = 2 N2, each a whole number of M = 128 tiles, and each
// thread owns one or two rows of each stage. Row r of a stage sits in tensor
// memory lane r mod 128 of tile r / 128; a thread's rows are tid + i x
// threads with threads a multiple of 128, so warp w reads only lane quadrant
// w mod 4, as tcgen05.ld requires. Accumulators: tile t, level L at columns
// (4 t + L) NO, NO = 2 N1 (stage 1) or 2 N2 (stage 3): 384 columns with
// velocity (512 allocated, one CTA per SM), 256 without.
//
// The GEMMs are the 512-point engine's: rows scaled to [2^29, 2^30), four
// signed 8-bit digits in FP16, digit-pair levels 0..3 exact in FP32. The
// middle step is done in FP64 instead: the four levels of Y combine exactly
// (an integer below 2^47 times a power of two), the twiddles W_N^(n2 k1) are
// the exact ones (sincospi in double, not the FP32 table), and Z is rounded
// to FP32 once. With the FP32 middle step (three roundings of Y, the FP32
// twiddle, Kahan's difference of products) a 128^2 frame with velocity
// reached 2.14e-6 of FP64 on normal.x.
#pragma once

#include "tc_dft.cuh"

namespace ocean_b200 {
namespace tc {

template <int LOG_N, int SEQS>
struct SmallLayout {
    static constexpr int N = 1 << LOG_N;
    static_assert(LOG_N >= 6 && LOG_N <= 8, "the small engine covers N = 64, 128 and 256");
    static constexpr int N1 = LOG_N == 8 ? 16 : 8;
    static constexpr int N2 = N / N1;
    static constexpr int K1 = 2 * N1, NO1 = 2 * N1;  // stage 1: rows (s, n2), K = (p, n1)
    static constexpr int K3 = 2 * N2, NO3 = 2 * N2;  // stage 3: rows (s, k1), K = (p, n2)
    static constexpr int kThreads = SEQS * N / 16;
    static constexpr int kRows1 = SEQS * N2;
    static constexpr int kRows3 = SEQS * N1;
    static_assert(kRows1 % 128 == 0 && kRows3 % 128 == 0, "whole M = 128 tiles");
    static_assert(kThreads % 128 == 0, "a thread's rows share its lane quadrant");
    static constexpr int kTiles1 = kRows1 / 128;
    static constexpr int kTiles3 = kRows3 / 128;
    static constexpr int kRpt1 = kRows1 / kThreads;  // stage-1 rows per thread
    static constexpr int kRpt3 = kRows3 / kThreads;  // stage-3 rows per thread
    static_assert(kRpt1 * kThreads == kRows1 && kRpt3 * kThreads == kRows3 && kRpt1 >= 1 && kRpt3 >= 1,
                  "every thread owns whole rows");
    static constexpr int kCols1 = kTiles1 * kLevels * NO1;
    static constexpr int kCols3 = kTiles3 * kLevels * NO3;
    static constexpr int kColsUsed = kCols1 > kCols3 ? kCols1 : kCols3;
    static constexpr int kTmemCols = kColsUsed <= 32 ? 32 : (kColsUsed <= 64 ? 64 : (kColsUsed <= 128 ? 128 : (kColsUsed <= 256 ? 256 : 512)));
    static_assert(kColsUsed <= 512, "the accumulators fit in tensor memory");
    static constexpr int kAHalves = kRows1 * K1;  // halves per digit plane (== kRows3 * K3)
    static_assert(kRows1 * K1 == kRows3 * K3, "stage operands share one buffer");
    // Staged Z: row (s, k1) of 2 N2 floats (+2 against bank conflicts), inside
    // the sequences' own buffer.
    static constexpr int kZStride = 2 * N2 + 2;
    static constexpr int kOffA = 0;                                  // [digit][kAHalves]
    static constexpr int kOffB1 = kOffA + kDigits * kAHalves * 2;     // [digit][NO1 * K1]
    static constexpr int kOffB3 = kOffB1 + kDigits * NO1 * K1 * 2;    // [digit][NO3 * K3]
    static constexpr int kOffTw3 = kOffB3 + kDigits * NO3 * K3 * 2;   // double2[N1][N2]: W^(n2 k1)
    static constexpr int kOffBar = kOffTw3 + N1 * N2 * 16;            // uint64 mbarrier
    static constexpr int kOffTmem = kOffBar + 8;                      // uint32 tmem base
    static constexpr int kSmemBytes = kOffTmem + 8;
    static_assert(kOffB1 % 128 == 0 && kOffB3 % 128 == 0 && kOffTw3 % 128 == 0, "operands 128-byte aligned");
};

template <int LOG_N, int SEQS>
struct SmallEngine {
    using Lay = SmallLayout<LOG_N, SEQS>;
    static constexpr int N = Lay::N, N1 = Lay::N1, N2 = Lay::N2;
    unsigned char* smem;  // Lay::kSmemBytes, 128-byte aligned
    uint32_t tmem;        // tensor-memory base (lane 0, column 0)

    __device__ uint16_t* a(int digit) const
    {
        return reinterpret_cast<uint16_t*>(smem + Lay::kOffA) + digit * Lay::kAHalves;
    }
    __device__ uint32_t bar() const { return smem_u32(smem + Lay::kOffBar); }
    __device__ const double2* tw3() const { return reinterpret_cast<const double2*>(smem + Lay::kOffTw3); }

    // The digits of the real block form [[C, -S], [S, C]] of the M-point
    // inverse DFT at 2^30: row j = (q, k) output (q = 0 real, 1 imaginary),
    // column i = (p, n) input.
    __device__ static void dft_matrix(uint16_t* b, int m, int tid, int nthreads)
    {
        const int K = 2 * m, NO = 2 * m;
        const double scale = static_cast<double>(1ll << kBExp);
        for (int i = tid; i < NO * K; i += nthreads) {
            const int j = i / K, k = i % K;
            const int q = j / m, kk = j % m, p = k / m, n = k % m;
            double s, c;
            sincospi(2.0 * static_cast<double>((n * kk) % m) / m, &s, &c);
            const double v = (q == p) ? c : (q == 0 ? -s : s);
            uint16_t d[4];
            digits4(static_cast<int>(rint(v * scale)), d);
            for (int g = 0; g < kDigits; ++g) b[g * NO * K + kmajor(j, k, K)] = d[g];
        }
    }

    // Once per kernel, all threads: the DFT matrices' digits, the middle
    // step's twiddles [k1][n2] = W^(n2 k1) in double (W = e^(2 pi i / N)),
    // the mbarrier and (warp 0) the tensor-memory allocation. `tw` (the FP32
    // table) is not used: the middle step's twiddles are exact.
    __device__ void init(int tid, int nthreads, const float2* __restrict__ tw)
    {
        (void)tw;
        double2* t3 = reinterpret_cast<double2*>(smem + Lay::kOffTw3);
        for (int i = tid; i < N1 * N2; i += nthreads) {
            const int e = (i % N2) * (i / N2);  // n2 * k1 < N
            double sn, cs;
            sincospi(2.0 * static_cast<double>(e) / N, &sn, &cs);
            t3[i] = make_double2(cs, sn);
        }
        dft_matrix(reinterpret_cast<uint16_t*>(smem + Lay::kOffB1), N1, tid, nthreads);
        dft_matrix(reinterpret_cast<uint16_t*>(smem + Lay::kOffB3), N2, tid, nthreads);
        if (tid == 0) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar()) : "memory");
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        if (tid < 32) {
            const uint32_t slot = smem_u32(smem + Lay::kOffTmem);
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot),
                         "r"(Lay::kTmemCols)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        fence_proxy_async();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        tmem = *reinterpret_cast<volatile uint32_t*>(smem + Lay::kOffTmem);
    }

    // Once per kernel, all threads, after the last engine call.
    __device__ void release(int tid)
    {
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (tid < 32)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Lay::kTmemCols)
                         : "memory");
    }

    // One row's K values as digits into the four planes (K-major, 8 halves
    // a store), scaled by 2^e.
    template <int K>
    __device__ void put_row(int row, const float (&v)[K], int e)
    {
        const float sc = pow2f(e);
        uint16_t* a0p = a(0);
#pragma unroll
        for (int c = 0; c < K / 8; ++c) {
            float d[8][4];
#pragma unroll
            for (int q = 0; q < 8; ++q) digits4f(v[8 * c + q] * sc, d[q]);
            const int off = kmajor(row, 8 * c, K);
#pragma unroll
            for (int g = 0; g < kDigits; ++g)
                *reinterpret_cast<uint4*>(a0p + g * Lay::kAHalves + off) =
                    make_uint4(half2_bits(d[0][g], d[1][g]), half2_bits(d[2][g], d[3][g]),
                               half2_bits(d[4][g], d[5][g]), half2_bits(d[6][g], d[7][g]));
        }
    }

    // Tiles [0, tiles) of one stage, K / 16 steps x 10 digit pairs each,
    // committed to the mbarrier (thread 0 only).
    template <int K, int NO>
    __device__ void issue_stage(int tiles, uint32_t b_off) const
    {
        const uint32_t abase = smem_u32(a(0)), bbase = smem_u32(smem + b_off);
        constexpr uint32_t sbo = K * 16;
        constexpr uint32_t idesc = instr_desc(128, NO);
#pragma unroll 1
        for (int t = 0; t < tiles; ++t)
#pragma unroll 1
            for (int ks = 0; ks < K / 16; ++ks)
                Engine<8>::issue_levels(tmem + t * kLevels * NO, NO, abase, bbase, Lay::kAHalves * 2, NO * K * 2,
                                        ks * 256, t * 16 * sbo, sbo, sbo, idesc, ks == 0);
        mma_commit(bar());
    }

    // The four level accumulators of one row (NO columns each) from tensor
    // memory at `col`, combined exactly in FP64 for fixed-point exponent e:
    // level L weighs 2^(18 - 8 L - e), so the row value is 2^(-6 - e) times
    // the integer D0 2^24 + D1 2^16 + D2 2^8 + D3 (below 2^47).
    template <int NO>
    __device__ static void read_levels_exact(uint32_t col, int e, double (&y)[NO])
    {
        uint32_t r0[NO], r1[NO];
        if constexpr (NO == 32) {
            OCEAN_TMEM_LD32(col, r0);
            OCEAN_TMEM_LD32(col + NO, r1);
        } else {
            OCEAN_TMEM_LD16(col, r0);
            OCEAN_TMEM_LD16(col + NO, r1);
        }
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < NO; ++j)
            y[j] = fma(static_cast<double>(__uint_as_float(r0[j])), 0x1p24, static_cast<double>(__uint_as_float(r1[j])) * 0x1p16);
        if constexpr (NO == 32) {
            OCEAN_TMEM_LD32(col + 2 * NO, r0);
            OCEAN_TMEM_LD32(col + 3 * NO, r1);
        } else {
            OCEAN_TMEM_LD16(col + 2 * NO, r0);
            OCEAN_TMEM_LD16(col + 3 * NO, r1);
        }
        tmem_wait_ld();
        const double w = ldexp(1.0, -6 - e);
#pragma unroll
        for (int j = 0; j < NO; ++j)
            y[j] = fma(static_cast<double>(__uint_as_float(r0[j])), 0x1p8, y[j] + static_cast<double>(__uint_as_float(r1[j]))) * w;
    }

    // The same combined in FP32 (three roundings), for the outputs.
    template <int NO>
    __device__ static void read_levels(uint32_t col, int e, float (&y)[NO])
    {
        uint32_t r0[NO], r1[NO];
        if constexpr (NO == 32) {
            OCEAN_TMEM_LD32(col, r0);
            OCEAN_TMEM_LD32(col + NO, r1);
        } else {
            OCEAN_TMEM_LD16(col, r0);
            OCEAN_TMEM_LD16(col + NO, r1);
        }
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < NO; ++j) y[j] = level_sum(r0[j], r1[j], e);
        if constexpr (NO == 32) {
            OCEAN_TMEM_LD32(col + 2 * NO, r0);
            OCEAN_TMEM_LD32(col + 3 * NO, r1);
        } else {
            OCEAN_TMEM_LD16(col + 2 * NO, r0);
            OCEAN_TMEM_LD16(col + 3 * NO, r1);
        }
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < NO; ++j) y[j] = level_add(y[j], r0[j], r1[j], e);
    }

    // In-place inverse DFT of sequences s < count (<= SEQS) of length N at
    // data + s * seq_stride, element n at pad_idx(n). All threads of the CTA
    // call it (the first Lay::kThreads do the work); data must be complete on
    // entry, and is complete on return.
    __device__ void dft(float2* data, int seq_stride, int count, int tid, unsigned* error)
    {
        constexpr int T = Lay::kThreads;
        constexpr int K1 = Lay::K1, NO1 = Lay::NO1, K3 = Lay::K3, NO3 = Lay::NO3, ZS = Lay::kZStride;
        const bool worker = tid < T;
        const uint32_t quad = static_cast<uint32_t>(32 * ((tid >> 5) & 3)) << 16;
        const int tiles1 = (count * N2 + 127) / 128;
        const int tiles3 = (count * N1 + 127) / 128;

        // ---- stage 1 operand: row r = (s, n2), N1 complex x[N2 n1 + n2] ----
        int e1[Lay::kRpt1];
#pragma unroll
        for (int i = 0; i < Lay::kRpt1; ++i) {
            e1[i] = 0;
            const int r = tid + i * T;
            const int s = r / N2, n2 = r % N2;
            if (!worker || r >= tiles1 * 128) continue;
            float v[K1];
            float m = 0.0f;
            if (s < count) {
                const float2* seq = data + s * seq_stride;
#pragma unroll
                for (int n1 = 0; n1 < N1; ++n1) {
                    const float2 x = seq[pad_idx(N2 * n1 + n2)];
                    v[n1] = x.x;
                    v[N1 + n1] = x.y;
                    m = fmaxf(m, fmaxf(fabsf(x.x), fabsf(x.y)));
                }
            } else {
#pragma unroll
                for (int k = 0; k < K1; ++k) v[k] = 0.0f;
            }
            e1[i] = row_exp(m);
            put_row<K1>(r, v, e1[i]);
        }
        fence_proxy_async();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();

        if (tid == 0) issue_stage<K1, NO1>(tiles1, Lay::kOffB1);
        bar_wait(bar(), 0u, error);
        fence_after_sync();

        // ---- read Y, twiddle, stage Z as FP32 rows (s, k1) of 2 N2 floats ----
        // Every thread's inputs are in registers since stage 1, so Z may
        // overwrite the sequences: count * N1 * ZS floats fit inside them.
        float* zbuf = reinterpret_cast<float*>(data);
#pragma unroll
        for (int i = 0; i < Lay::kRpt1; ++i) {
            const int r = tid + i * T;
            if (!worker || r >= tiles1 * 128) continue;
            const int s = r / N2, n2 = r % N2;
            double y[NO1];
            read_levels_exact<NO1>(tmem + quad + (r >> 7) * kLevels * NO1, e1[i], y);
            if (s < count) {
#pragma unroll
                for (int k1 = 0; k1 < N1; ++k1) {
                    const double2 w = tw3()[k1 * N2 + n2];
                    float* zrow = zbuf + (s * N1 + k1) * ZS;
                    zrow[n2] = __double2float_rn(fma(y[k1], w.x, -(y[N1 + k1] * w.y)));
                    zrow[N2 + n2] = __double2float_rn(fma(y[k1], w.y, y[N1 + k1] * w.x));
                }
            }
        }
        __syncthreads();

        // ---- stage 3 operand: row r = (s, k1), K = (p, n2) ----
        int e3[Lay::kRpt3];
#pragma unroll
        for (int i = 0; i < Lay::kRpt3; ++i) {
            e3[i] = 0;
            const int r = tid + i * T;
            if (!worker || r >= tiles3 * 128) continue;
            const int s = r / N1;
            float v[K3];
            float m = 0.0f;
            if (s < count) {
                const float2* src = reinterpret_cast<const float2*>(zbuf + r * ZS);
#pragma unroll
                for (int q = 0; q < K3 / 2; ++q) {
                    const float2 f = src[q];
                    v[2 * q] = f.x;
                    v[2 * q + 1] = f.y;
                    m = fmaxf(m, fmaxf(fabsf(f.x), fabsf(f.y)));
                }
            } else {
#pragma unroll
                for (int k = 0; k < K3; ++k) v[k] = 0.0f;
            }
            e3[i] = row_exp(m);
            put_row<K3>(r, v, e3[i]);
        }
        fence_proxy_async();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();

        if (tid == 0) issue_stage<K3, NO3>(tiles3, Lay::kOffB3);
        bar_wait(bar(), 1u, error);
        fence_after_sync();

        // ---- read X: row (s, k1) holds X[k1 + N1 k2], real parts in its
        // first N2 columns, imaginary ones in the next N2 ----
#pragma unroll
        for (int i = 0; i < Lay::kRpt3; ++i) {
            const int r = tid + i * T;
            if (!worker || r >= tiles3 * 128) continue;
            const int s = r / N1, k1 = r % N1;
            float x[NO3];
            read_levels<NO3>(tmem + quad + (r >> 7) * kLevels * NO3, e3[i], x);
            if (s < count) {
                float2* seq = data + s * seq_stride;
#pragma unroll
                for (int k2 = 0; k2 < N2; ++k2) seq[pad_idx(k1 + N1 * k2)] = make_float2(x[k2], x[N2 + k2]);
            }
        }
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
    }
};

}  // namespace tc
}  // namespace ocean_b200
