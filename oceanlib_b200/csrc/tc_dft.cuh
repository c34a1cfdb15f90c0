// oceanlib-b200: the tensor-core DFT form (sm_100a, tcgen05).
//
// A 512-point inverse DFT (sign +, unnormalised, as src/core/fft.cpp) of 8
// sequences at a time, as the four-step factorisation 512 = 16 x 32:
//
//   n = 32 n1 + n2,  k = k1 + 16 k2
//   Y[n2, k1] = sum_n1 W16^(n1 k1) x[32 n1 + n2]          stage 1 (GEMM)
//   Z[n2, k1] = W512^(n2 k1) Y[n2, k1]                    twiddle (FP32)
//   X[k1 + 16 k2] = sum_n2 W32^(n2 k2) Z[n2, k1]           stage 3 (GEMM)
//
// Each stage is one real GEMM D = A B^T on the tensor cores
// (tcgen05.mma kind::f16: FP16 operands in shared memory, FP32 accumulators
// in tensor memory): the complex DFT matrix becomes the real block matrix
// [[C, -S], [S, C]] and a row of A holds one short sequence as (re..., im...).
// Stage 1 has 8 x 32 = 256 rows (two M = 128 tiles), K = 32, N = 32; stage 3
// has 8 x 16 = 128 rows, K = 64, N = 64.
//
// Precision: a plain FP16 split (hi + lo) still rounds every accumulation in
// FP32 against the dominant spectral terms of a row, which costs 2-3x the
// FP32 FFT's error. Here the GEMMs are made exact instead. Each row of A is
// scaled by a power of two so its largest magnitude lies in [2^29, 2^30),
// rounded to an integer (30 significant bits relative to the row maximum),
// and cut into four signed 8-bit digits a_i (weights 2^24, 2^16, 2^8, 1);
// the DFT matrices likewise at 2^30. FP16 holds the digits exactly, every
// product a_i b_j is an exact integer below 2^14, and a level
// D_L = sum over i + j = L of A_i B_j^T (at most 4 pairs x 64 terms) stays
// below 2^22 - so the FP32 accumulators hold every level EXACTLY, whatever
// order the tensor cores add in. Levels 0..3 (10 products per K step) are
// kept; the dropped ones weigh 2^-32 of the leading term. The four exact
// levels are then combined in FP32 (three roundings). The GEMMs are thus
// as good as FP64 ones; the remaining error is the FP32 twiddle step and the
// FP32 values between the stages - below the radix-2 FP32 FFT's own.
//
// One elected thread issues the MMAs and commits them to an mbarrier; every
// wait on it is bounded (the error word is set and the engine gives up
// rather than spin). Tensor memory: 256 columns per CTA, allocated once per
// kernel by warp 0 and released before exit.
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

#include "ocean_device.cuh"

namespace ocean_b200 {
namespace tc {

constexpr int kK1 = 32;          // stage 1 K (16 complex)
constexpr int kN1 = 32;          // stage 1 N (16 complex)
constexpr int kK3 = 64;          // stage 3 K (32 complex)
constexpr int kN3 = 64;          // stage 3 N (32 complex)
constexpr int kDigits = 4;       // signed 8-bit digits per value
constexpr int kLevels = 4;       // digit-pair levels kept (i + j < 4)
constexpr int kZStride = 68;     // floats per staged stage-3 row (64 + 4 against bank conflicts)
constexpr int kFixExp = 29;      // row max scaled into [2^29, 2^30)
constexpr int kBExp = 30;        // DFT matrices scaled by 2^30
constexpr unsigned long long kWaitNs = 1000000000ull;  // 1 s

// An engine call transforms SEQS sequences (8, or 12: a frame task's 2 rows
// x 6 fields) with SEQS x 32 threads. Stage 1 has SEQS x 32 rows (SEQS / 4
// tiles of M = 128); stage 3 has SEQS x 16 rows, one tile or two, the second
// holding rows 128..191 (its MMA also reads the 64 rows behind them, which
// lie inside the engine's shared memory and land in tensor-memory lanes that
// are never read). Accumulators (FP32 columns), one per level: stage 1 tile
// t, level L at 128 t + 32 L; stage 3 tile t, level L at 256 t + 64 L.
// Shared-memory layout in bytes, all offsets 128-byte aligned.
template <int SEQS>
struct Layout {
    static_assert(SEQS == 8 || SEQS == 12, "8 or 12 sequences per engine call");
    static constexpr int kRows1 = SEQS * 32;
    static constexpr int kTiles1 = kRows1 / 128;
    static constexpr int kRows3 = SEQS * 16;
    static constexpr int kTiles3 = (kRows3 + 127) / 128;
    static constexpr int kThreads = SEQS * 32;
    static constexpr int kTmemCols = kTiles3 > 1 ? 512 : 256;
    static constexpr int kAHalves = kRows1 * kK1;  // halves per digit plane (== kRows3 * kK3)
    static_assert(kRows1 * kK1 == kRows3 * kK3, "stage operands share one buffer");
    static constexpr int kOffA = 0;                                 // [digit][kAHalves]
    static constexpr int kOffB1 = kOffA + kDigits * kAHalves * 2;    // [digit][32*32]
    static constexpr int kOffB3 = kOffB1 + kDigits * kN1 * kK1 * 2;  // [digit][64*64]
    static constexpr int kOffE3 = kOffB3 + kDigits * kN3 * kK3 * 2;  // int[kRows3]
    static constexpr int kOffTw3 = kOffE3 + kRows3 * 4;              // float2[16][32]: W^(n2 k1)
    static constexpr int kOffBar = kOffTw3 + 16 * 32 * 8;            // uint64 mbarrier
    static constexpr int kOffTmem = kOffBar + 8;                     // uint32 tmem base
    static constexpr int kSmemBytes = kOffTmem + 8;
    // The second stage-3 tile's MMA reads rows 128..255 of each digit plane;
    // for the last plane those end inside B1.
    static_assert(kTiles3 == 1 || kOffA + (kDigits - 1) * kAHalves * 2 + 256 * kK3 * 2 <= kOffB3,
                  "stage-3 tile reads stay inside the engine's shared memory");
};

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Canonical K-major, no-swizzle layout of an R x K FP16 operand: 8-row x
// 16-byte core matrices; the K chunks of a row group lie 128 B apart (LBO),
// row groups K * 16 B apart (SBO). Offset in halves.
__device__ __forceinline__ int kmajor(int row, int k, int K)
{
    return (row >> 3) * (K * 8) + (k >> 3) * 64 + (row & 7) * 8 + (k & 7);
}

// Shared-memory matrix descriptor: start, LBO, SBO (all >> 4), version 1,
// base offset 0, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) |
           (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: FP16 A and B (K-major), FP32 accumulator, M x N.
__host__ __device__ constexpr uint32_t instr_desc(int m, int n)
{
    return (1u << 4) | (static_cast<uint32_t>(n >> 3) << 17) | (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
        :
        : "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait for mbarrier phase `parity`; false (and the error word set)
// when it does not complete within kWaitNs.
__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity, unsigned* error)
{
    uint32_t done = 0;
    unsigned long long t0 = 0;
    for (int spin = 0;; ++spin) {
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (spin == 0) t0 = now_ns();
        if ((spin & 63) == 63 && now_ns() - t0 > kWaitNs) {
            if (error) atomicCAS(error, 0u, 2u);
            return false;
        }
    }
}

#define OCEAN_TMEM_LD32(taddr, r)                                                                       \
    asm volatile(                                                                                       \
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "                                                       \
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"                                       \
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"                      \
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),          \
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),      \
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),   \
          "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),   \
          "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])                                           \
        : "r"(taddr)                                                                                    \
        : "memory")

#define OCEAN_TMEM_LD16(taddr, r)                                                                       \
    asm volatile(                                                                                       \
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "                                                       \
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"                               \
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),          \
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),      \
          "=r"(r[14]), "=r"(r[15])                                                                      \
        : "r"(taddr)                                                                                    \
        : "memory")

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// 2^e as a float, e clamped to the normal range.
__device__ __forceinline__ float pow2f(int e)
{
    e = e < -126 ? -126 : (e > 127 ? 127 : e);
    return __uint_as_float(static_cast<uint32_t>(e + 127) << 23);
}

// Exponent that scales `maxabs` into [2^29, 2^30) (0 for a zero row).
__device__ __forceinline__ int row_exp(float maxabs)
{
    if (!(maxabs > 0.0f)) return 0;
    int ex = static_cast<int>((__float_as_uint(maxabs) >> 23) & 0xFFu) - 127;
    if (ex < -126) ex = -126;  // subnormal maximum
    const int e = kFixExp - ex;
    return e > 120 ? 120 : (e < -120 ? -120 : e);
}

// A signed fixed-point value |v| < 2^30 as four signed 8-bit digits
// d0 2^24 + d1 2^16 + d2 2^8 + d3, as FP16 bit patterns (exact).
__device__ __forceinline__ void digits4(int v, uint16_t (&d)[4])
{
    const int d0 = (v + (1 << 23)) >> 24;
    int r = v - (d0 << 24);
    const int d1 = (r + (1 << 15)) >> 16;
    r -= d1 << 16;
    const int d2 = (r + (1 << 7)) >> 8;
    const int d3 = r - (d2 << 8);
    d[0] = __half_as_ushort(__int2half_rn(d0));
    d[1] = __half_as_ushort(__int2half_rn(d1));
    d[2] = __half_as_ushort(__int2half_rn(d2));
    d[3] = __half_as_ushort(__int2half_rn(d3));
}

// The operand form of digits4: signed digits of x, |x| < 2^30, as floats,
// x rounded to the nearest integer = t0 2^24 + t1 2^16 + t2 2^8 + t3 with
// |t_i| <= 128 (so every digit product is at most 2^14 and a level of 256
// terms at most 2^22, still exact in FP32). Each digit is the remaining value
// at its weight rounded to the nearest integer, halves up as digits4 rounds
// them (floor(y + 1/2): y + 1/2 by one rounding, then a round-down add onto
// the integer grid of 1.5 2^23), and each residual is exact: full-rate FP32
// operations only. Rounding halves to even instead measurably raised the
// worst-cell error of the frame's normals at late times.
__device__ __forceinline__ float nearest_half_up(float x, float scale)
{
    constexpr float M = 12582912.0f;  // 1.5 * 2^23
    return __fadd_rn(__fmaf_rd(__fmaf_rn(x, scale, 0.5f), 1.0f, M), -M);
}
__device__ __forceinline__ void digits4f(float x, float (&t)[4])
{
    t[0] = nearest_half_up(x, 0x1p-24f);
    const float x1 = __fmaf_rn(t[0], -0x1p24f, x);
    t[1] = nearest_half_up(x1, 0x1p-16f);
    const float x2 = __fmaf_rn(t[1], -0x1p16f, x1);
    t[2] = nearest_half_up(x2, 0x1p-8f);
    const float x3 = __fmaf_rn(t[2], -0x1p8f, x2);
    t[3] = nearest_half_up(x3, 1.0f);
}

// a b - c d with about one rounding (Kahan: the rounding error of c d is
// recovered exactly by a fused multiply-add and added back). The twiddle
// step Z = Y W uses it: rounding each product and the sum separately (three
// roundings) was the largest of the FP32 errors between the two exact GEMMs,
// and with it the frame's late-time normals stayed above 2e-6 of FP64.
__device__ __forceinline__ float diff_of_products(float a, float b, float c, float d)
{
    const float w = __fmul_rn(c, d);
    const float e = __fmaf_rn(-c, d, w);
    const float f = __fmaf_rn(a, b, -w);
    return __fadd_rn(f, e);
}

// Two digits as one FP16 pair (a in the low half), one conversion.
__device__ __forceinline__ uint32_t half2_bits(float a, float b)
{
    const __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&h);
}

// Read back, level D_L of a row with fixed-point exponent e weighs
// 2^(48 - 8 L - 30 - e) = 2^(18 - 8 L - e); the levels are added largest
// first. A level is an exact integer below 2^22 and its weight a power of
// two, so each weighted level is exact and a fused multiply-add rounds the
// running sum exactly as a multiply followed by an add would: the same
// bits in fewer instructions.
__device__ __forceinline__ float level_sum(uint32_t l0, uint32_t l1, int e)
{
    return __fmaf_rn(__uint_as_float(l1), pow2f(10 - e), __uint_as_float(l0) * pow2f(18 - e));
}
__device__ __forceinline__ float level_add(float acc, uint32_t l2, uint32_t l3, int e)
{
    return __fmaf_rn(__uint_as_float(l3), pow2f(-6 - e), __fmaf_rn(__uint_as_float(l2), pow2f(2 - e), acc));
}

template <int SEQS>
struct Engine {
    using Lay = Layout<SEQS>;
    unsigned char* smem;  // Lay::kSmemBytes, 128-byte aligned
    uint32_t tmem;        // tensor-memory base (lane 0, column 0)

    __device__ uint16_t* a(int digit) const
    {
        return reinterpret_cast<uint16_t*>(smem + Lay::kOffA) + digit * Lay::kAHalves;
    }
    __device__ int* e3() const { return reinterpret_cast<int*>(smem + Lay::kOffE3); }
    __device__ uint32_t bar() const { return smem_u32(smem + Lay::kOffBar); }

    __device__ const float2* tw3() const { return reinterpret_cast<const float2*>(smem + Lay::kOffTw3); }

    // Once per kernel, all threads: the DFT matrices' digits, the twiddles
    // of the middle step as [k1][n2] = W^(n2 k1) from the FP32 table `tw`
    // (W^p, p < 256, W = e^(2 pi i / 512); W^(p + 256) = -W^p), so a warp's
    // 32 lanes (n2) read 32 consecutive entries, the mbarrier, and (warp 0)
    // the tensor-memory allocation.
    __device__ void init(int tid, int nthreads, const float2* __restrict__ tw)
    {
        float2* t3 = reinterpret_cast<float2*>(smem + Lay::kOffTw3);
        for (int i = tid; i < 16 * 32; i += nthreads) {
            const int e = (i & 31) * (i >> 5);  // n2 * k1 < 512
            float2 w = tw[e & 255];
            if (e & 256) w = make_float2(-w.x, -w.y);
            t3[i] = w;
        }
        uint16_t* b1 = reinterpret_cast<uint16_t*>(smem + Lay::kOffB1);
        uint16_t* b3 = reinterpret_cast<uint16_t*>(smem + Lay::kOffB3);
        const double scale = static_cast<double>(1ll << kBExp);
        // B1[j][k]: j = (q, k1) output, k = (p, n1) input, angle 2 pi n1 k1 / 16
        for (int i = tid; i < kN1 * kK1; i += nthreads) {
            const int j = i / kK1, k = i % kK1;
            const int q = j >> 4, k1 = j & 15, p = k >> 4, n1 = k & 15;
            double s, c;
            sincospi(static_cast<double>((n1 * k1) & 15) / 8.0, &s, &c);
            const double v = (q == p) ? c : (q == 0 ? -s : s);
            uint16_t d[4];
            digits4(static_cast<int>(rint(v * scale)), d);
            for (int g = 0; g < kDigits; ++g) b1[g * kN1 * kK1 + kmajor(j, k, kK1)] = d[g];
        }
        // B3[j][k]: j = (q, k2), k = (p, n2), angle 2 pi n2 k2 / 32
        for (int i = tid; i < kN3 * kK3; i += nthreads) {
            const int j = i / kK3, k = i % kK3;
            const int q = j >> 5, k2 = j & 31, p = k >> 5, n2 = k & 31;
            double s, c;
            sincospi(static_cast<double>((n2 * k2) & 31) / 16.0, &s, &c);
            const double v = (q == p) ? c : (q == 0 ? -s : s);
            uint16_t d[4];
            digits4(static_cast<int>(rint(v * scale)), d);
            for (int g = 0; g < kDigits; ++g) b3[g * kN3 * kK3 + kmajor(j, k, kK3)] = d[g];
        }
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

    // The 10 digit-pair MMAs of one K step into the level accumulators at
    // `d` + 32 L (stage 1) or + 64 L (stage 3). `first` starts each level.
    __device__ static void issue_levels(uint32_t d, int level_stride, uint32_t a0, uint32_t b0, uint32_t a_digit,
                                        uint32_t b_digit, uint32_t kofs, uint32_t tile, uint32_t sbo_a,
                                        uint32_t sbo_b, uint32_t idesc, bool first)
    {
#pragma unroll
        for (int L = 0; L < kLevels; ++L) {
            bool started = !first;
#pragma unroll
            for (int i = 0; i <= L; ++i) {
                const int j = L - i;
                if (i >= kDigits || j >= kDigits) continue;
                const uint64_t da = smem_desc(a0 + i * a_digit + tile + kofs, 128, sbo_a);
                const uint64_t db = smem_desc(b0 + j * b_digit + kofs, 128, sbo_b);
                mma_f16(d + L * level_stride, da, db, idesc, started ? 1u : 0u);
                started = true;
            }
        }
    }

    // In-place inverse DFT of sequences s < count (<= SEQS) of length 512 at
    // data + s * seq_stride, element n at pad_idx(n). All threads of the CTA
    // call it (the first SEQS x 32 do the work); data must be complete on
    // entry, and is complete on return.
    __device__ void dft512(float2* data, int seq_stride, int count, int tid, unsigned* error)
    {
        const int warp = tid >> 5, lane = tid & 31;
        const bool worker = tid < Lay::kThreads;
        uint16_t* a0p = a(0);
        // Stage-1 tile t holds sequences 4t..4t+3, stage-3 tile t sequences
        // 8t..8t+7: tiles without sequences are skipped.
        const int tiles1 = (count + 3) / 4;
        const int tiles3 = (count + 7) / 8;

        // ---- stage 1 operand: row r = (s, n2), 16 complex x[32 n1 + n2] ----
        int e1 = 0;
        const int s_row = tid >> 5, n2 = tid & 31;
        if (worker && tid < tiles1 * 128) {
            float v[32];
            float m = 0.0f;
            if (s_row < count) {
                const float2* seq = data + s_row * seq_stride;
#pragma unroll
                for (int n1 = 0; n1 < 16; ++n1) {
                    const float2 x = seq[pad_idx(32 * n1 + n2)];
                    v[n1] = x.x;
                    v[16 + n1] = x.y;
                    m = fmaxf(m, fmaxf(fabsf(x.x), fabsf(x.y)));
                }
            } else {
#pragma unroll
                for (int k = 0; k < 32; ++k) v[k] = 0.0f;
            }
            e1 = row_exp(m);
            const float sc = pow2f(e1);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float d[8][4];
#pragma unroll
                for (int q = 0; q < 8; ++q) digits4f(v[8 * c + q] * sc, d[q]);
                const int off = kmajor(tid, 8 * c, kK1);
#pragma unroll
                for (int g = 0; g < kDigits; ++g)
                    *reinterpret_cast<uint4*>(a0p + g * Lay::kAHalves + off) =
                        make_uint4(half2_bits(d[0][g], d[1][g]), half2_bits(d[2][g], d[3][g]),
                                   half2_bits(d[4][g], d[5][g]), half2_bits(d[6][g], d[7][g]));
            }
        }
        fence_proxy_async();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();

        // ---- stage 1 MMAs: tiles1 tiles x 2 K steps x 10 digit pairs ----
        if (tid == 0) {
            const uint32_t abase = smem_u32(a0p), bbase = smem_u32(smem + Lay::kOffB1);
            constexpr uint32_t sbo = kK1 * 16;
            constexpr uint32_t idesc = instr_desc(128, kN1);
#pragma unroll 1
            for (int t = 0; t < tiles1; ++t)
#pragma unroll 1
                for (int ks = 0; ks < kK1 / 16; ++ks)
                    issue_levels(tmem + t * 128, kN1, abase, bbase, Lay::kAHalves * 2, kN1 * kK1 * 2, ks * 256,
                                 t * 16 * sbo, sbo, sbo, idesc, ks == 0);
            mma_commit(bar());
        }
        bar_wait(bar(), 0u, error);
        fence_after_sync();

        // ---- read Y, twiddle, stage 3 operand: row (s, k1), K = (p, n2) ----
        float* zbuf = reinterpret_cast<float*>(data);
        if (worker && (warp >> 2) < tiles1) {
            const int t = warp >> 2;
            const uint32_t col = tmem + (static_cast<uint32_t>(32 * (warp & 3)) << 16) + t * 128;
            float y[32];
            {
                uint32_t r0[32], r1[32];
                OCEAN_TMEM_LD32(col, r0);
                OCEAN_TMEM_LD32(col + 32, r1);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    y[j] = level_sum(r0[j], r1[j], e1);
            }
            {
                uint32_t r2[32], r3[32];
                OCEAN_TMEM_LD32(col + 64, r2);
                OCEAN_TMEM_LD32(col + 96, r3);
                tmem_wait_ld();
#pragma unroll
                for (int j = 0; j < 32; ++j)
                    y[j] = level_add(y[j], r2[j], r3[j], e1);
            }
            // Z staged as FP32, stage-3 row (s, k1) at zbuf + (s * 16 + k1) *
            // kZStride, K = (p, n2), in the sequences' own buffer: every
            // thread's inputs are in registers since stage 1, and the staging
            // (count * 4352 B) fits inside the count sequences' space.
            if (s_row < count) {
#pragma unroll
                for (int k1 = 0; k1 < 16; ++k1) {
                    const float2 w = tw3()[k1 * 32 + n2];
                    float* zrow = zbuf + (s_row * 16 + k1) * kZStride;
                    zrow[n2] = diff_of_products(y[k1], w.x, y[16 + k1], w.y);
                    zrow[32 + n2] = diff_of_products(y[k1], w.y, -y[16 + k1], w.x);
                }
            }
        }
        __syncthreads();
        // ---- stage 3 operand: two threads per row (s, k1), each 32 of its K ----
        // Warp w takes sequence w's 16 rows; a quarter warp takes 8 rows and
        // one half of K, so its float4 reads of the staged Z (row stride 68
        // floats) and its 16-byte digit stores (8 rows of one core matrix)
        // each touch 8 distinct bank groups. The row's other half sits 8
        // lanes away.
        if (worker) {
            const int row = warp * 16 + (lane & 7) + 8 * (lane >> 4), half_k = (lane >> 3) & 1;
            const int s = row >> 4;
            float v[32];
            float m = 0.0f;
            if (s < count) {
                const float4* src = reinterpret_cast<const float4*>(zbuf + row * kZStride + half_k * 32);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float4 f = src[q];
                    v[4 * q] = f.x;
                    v[4 * q + 1] = f.y;
                    v[4 * q + 2] = f.z;
                    v[4 * q + 3] = f.w;
                    m = fmaxf(m, fmaxf(fmaxf(fabsf(f.x), fabsf(f.y)), fmaxf(fabsf(f.z), fabsf(f.w))));
                }
            } else {
#pragma unroll
                for (int k = 0; k < 32; ++k) v[k] = 0.0f;
            }
            m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, 8));
            const int ex3 = row_exp(m);
            const float sc = pow2f(ex3);
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                float d[8][4];
#pragma unroll
                for (int q = 0; q < 8; ++q) digits4f(v[8 * c + q] * sc, d[q]);
                const int off = kmajor(row, half_k * 32 + 8 * c, kK3);
#pragma unroll
                for (int g = 0; g < kDigits; ++g)
                    *reinterpret_cast<uint4*>(a0p + g * Lay::kAHalves + off) =
                        make_uint4(half2_bits(d[0][g], d[1][g]), half2_bits(d[2][g], d[3][g]),
                                   half2_bits(d[4][g], d[5][g]), half2_bits(d[6][g], d[7][g]));
            }
            if (half_k == 0) e3()[row] = ex3;
        }
        fence_proxy_async();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();

        // ---- stage 3 MMAs: tiles3 tiles x 4 K steps x 10 digit pairs ----
        if (tid == 0) {
            const uint32_t abase = smem_u32(a0p), bbase = smem_u32(smem + Lay::kOffB3);
            constexpr uint32_t sbo = kK3 * 16;
            constexpr uint32_t idesc = instr_desc(128, kN3);
#pragma unroll 1
            for (int t = 0; t < tiles3; ++t)
#pragma unroll 1
                for (int ks = 0; ks < kK3 / 16; ++ks)
                    issue_levels(tmem + t * 256, kN3, abase, bbase, Lay::kAHalves * 2, kN3 * kK3 * 2, ks * 256,
                                 t * 16 * sbo, sbo, sbo, idesc, ks == 0);
            mma_commit(bar());
        }
        bar_wait(bar(), 1u, error);
        fence_after_sync();

        // ---- read X: row (s, k1) of stage-3 tile t in lane quadrant (row &
        // 127) / 32, where warp w may read quadrant w & 3. Tile 0: warps 0-3
        // take k2 < 16 and warps 4-7 k2 >= 16; tile 1 (rows 128..191, lanes
        // 0..63): warps 8 and 9, both halves. Each reads both parts (level
        // L's real parts in columns 256 t + 64 L + k2, imaginary ones 32
        // further), so every output is one float2 store and a half warp
        // writes 128 contiguous bytes ----
        if (worker) {
            const bool second = warp >= 8;
            const int t = second ? 1 : 0;
            if (!second || (t < tiles3 && warp < 10)) {
                const int row = 128 * t + 32 * (warp & 3) + lane;  // (s, k1)
                const int e = e3()[row];
                const int s = row >> 4, k1 = row & 15;
                float2* seq = data + s * seq_stride;
                const int h0 = second ? 0 : (warp >> 2), h1 = second ? 2 : h0 + 1;
#pragma unroll 1
                for (int half = h0; half < h1; ++half) {
                    const uint32_t col = tmem + (static_cast<uint32_t>(32 * (warp & 3)) << 16) + 256 * t + half * 16;
                    float xr[16], xi[16];
                    {
                        uint32_t r0[16], i0[16], r1[16], i1[16];
                        OCEAN_TMEM_LD16(col, r0);
                        OCEAN_TMEM_LD16(col + 32, i0);
                        OCEAN_TMEM_LD16(col + 64, r1);
                        OCEAN_TMEM_LD16(col + 96, i1);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            xr[j] = level_sum(r0[j], r1[j], e);
                            xi[j] = level_sum(i0[j], i1[j], e);
                        }
                    }
                    {
                        uint32_t r2[16], i2[16], r3[16], i3[16];
                        OCEAN_TMEM_LD16(col + 128, r2);
                        OCEAN_TMEM_LD16(col + 160, i2);
                        OCEAN_TMEM_LD16(col + 192, r3);
                        OCEAN_TMEM_LD16(col + 224, i3);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 16; ++j) {
                            xr[j] = level_add(xr[j], r2[j], r3[j], e);
                            xi[j] = level_add(xi[j], i2[j], i3[j], e);
                        }
                    }
                    if (s < count) {
#pragma unroll
                        for (int j = 0; j < 16; ++j)
                            seq[pad_idx(k1 + 16 * (half * 16 + j))] = make_float2(xr[j], xi[j]);
                    }
                }
            }
        }
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
    }
};

}  // namespace tc
}  // namespace ocean_b200
