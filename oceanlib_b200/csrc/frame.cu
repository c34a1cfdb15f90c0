// oceanlib-b200: the per-frame kernels.
//
// One frame of N x N oceans is two passes over HBM/L2:
//
//   row pass   (grid: row-pair groups x oceans)
//     h0 rows y and N-y -> shared memory; evolve every cell of both rows into
//     NF packed complex fields (src/core/evolve.cpp:28-184); 2*NF row FFTs in
//     shared memory, one lane group per sequence or per pair of sequences
//     (packed f32x2 arithmetic, at the sizes where pairs cost no extra pass);
//     write the rows to the intermediate, cell-major [y][x][field] so the
//     column pass reads whole 128-byte lines.
//
//   column pass (grid: W-column strips x oceans)
//     gather the strip's NF*W columns; column FFTs; finalize every cell
//     (src/core/evolve.cpp:238-327 and :186-203) straight into the RGBA32F
//     displacement / normal / velocity outputs; optionally the first
//     persistent-foam substep (src/foam.cpp:89-139) for the same cell, reading
//     only the previous foam state.
//
// Pairing rows y and N-y means h0(-k) - the conjugate-mirror table the
// reference stores separately (src/core/spectrum.cpp:329-338) - is read from
// the other row already in shared memory, so h0 is read from HBM once.
#include "frame_cells.cuh"
#include "ocean_device.cuh"
#include "query_device.cuh"
#include "spectrum.h"
#include "tc_dft.cuh"
#include "tc_dft_small.cuh"

#include <type_traits>

namespace ocean_b200 {
namespace {

constexpr int kPad = 4;   // float2 padding between sequences in shared memory
constexpr int kPad4 = 3;  // float4 padding between sequence pairs (stride = 3 mod 8 float4)

// Columns per CTA of the per-chunk column kernel: 4 at N = 512 (128-byte rows
// of the intermediate); 2 at N = 1024, where 32 values per lane leave room
// for fewer threads only.
template <int LOG_N>
struct Shape {
    static constexpr int N = 1 << LOG_N;
    static constexpr int G = lanes_for(LOG_N);
    static constexpr int W = LOG_N >= 10 ? 2 : cmin(N, (128 / G) > 4 ? 128 / G : 4);
};

// The plan of one size's tasks: how a sequence spreads over lanes, how the
// sequences sit in shared memory, and which rows a row task owns.
//
//   G lanes per sequence, each keeping N / G values (2^LANE_LOG): one stage
//   block of LANE_LOG radix-2 stages per pass through shared memory. The
//   default G (lanes_for) gives 16 values a lane (32 at N = 1024) within one
//   warp; a plan may take more lanes (N = 1024 over 64 lanes: 16 values, a
//   pass more, half the registers).
//
//   Paired: fields 2p and 2p+1 of a row or column as one pair (float4 per
//   index, stride SEQ4 float4 = 2 SEQ4 float2 per pair, so SEQ4 float2 per
//   sequence), transformed with packed f32x2 arithmetic over G2 = 2 G lanes.
//   Single: every sequence on its own (float2 per index, stride SEQ). A lane
//   keeps half as many indices of each sequence in a pair (it holds two), so
//   pairs are used where that adds no pass through shared memory (with the
//   default lanes: N = 32, 64, 512). The tensor-core form uses single
//   sequences. Both layouts read the same float2 twiddle table.
//
//   Row pairs (ROWS = 2 RP): RP row pairs (p, N-p), each row's h0(-k) read
//   from the other row of its pair, already staged (rows 0 and N/2 are their
//   own mirrors). Single rows (ROWS = RP): RP rows, each staged with a copy of
//   its mirror row (N - y) mod N beside it - twice the h0 reads (the second
//   from L2: the mirror row's task is the neighbouring ticket) for half the
//   threads. Column tasks of the persistent kernels cover PW = ROWS columns,
//   so both task kinds have the same thread count, ROWS * NF * G.
template <int LOG_N_, int G_, bool TC_, bool SINGLE_ROWS>
struct Plan {
    static constexpr int LOG_N = LOG_N_;
    static constexpr int N = 1 << LOG_N;
    static constexpr int G = G_;
    static constexpr bool TC = TC_;
    static constexpr int SEQ = padded_len(N) + kPad;                  // sequence stride (float2)
    static constexpr int SEQ4 = padded_len4(N) + kPad4;               // pair stride (float4)
    static constexpr int RP = cmin(N / 2, 32 / G > 1 ? 32 / G : 1);  // row pairs / task
    static constexpr int LANE_LOG = ilog2c(N / G);
    static_assert(LANE_LOG >= 2, "a lane keeps at least four values");
    static constexpr bool PAIRED =
        !TC && (LOG_N + LANE_LOG - 1) / LANE_LOG == (LOG_N + LANE_LOG - 2) / (LANE_LOG - 1);
    static constexpr int G2 = 2 * G;                                  // lanes per sequence pair
    static constexpr int SEQF2 = PAIRED ? SEQ4 : SEQ;                 // float2 per sequence
    static constexpr int TWF2 = N - 1;                                // float2 of the twiddle table
    static constexpr bool SINGLE = SINGLE_ROWS;
    static constexpr int ROWS = SINGLE ? RP : 2 * RP;                 // rows per row task
    static constexpr int H0ROWS = SINGLE ? 2 * ROWS : ROWS;           // h0 rows staged
    static constexpr int PW = ROWS;                                   // columns per column task
    static constexpr int RT = N / ROWS;                               // row tasks per ocean
    template <int NF>
    __host__ __device__ static constexpr int threads()
    {
        return ROWS * NF * G;
    }
};

// The persistent kernel's plan: default lanes, row pairs. Single rows were
// measured at N = 512 (64 oceans, velocity and persistent foam): 1.336 ms per
// frame against 1.117 ms with row pairs - the second h0 read and twice the
// tasks cost more than the smaller CTAs recover.
template <int LOG_N, bool TC>
using FramePlan = Plan<LOG_N, lanes_for(LOG_N), TC, false>;
// The per-chunk kernels' plan.
template <int LOG_N>
using ChunkPlan = Plan<LOG_N, lanes_for(LOG_N), false, false>;

// The persistent kernel's alternative plans, one per size that has them, for
// a batch's autotuner to time against the default (plan 0):
//   N = 256, 512  single rows (half the threads a task, twice the h0 reads);
//   N = 1024      64 lanes a sequence (16 values a lane: three passes
//                 instead of two, about half the registers, so two CTAs of
//                 single rows per SM instead of one of row pairs).
template <int LOG_N>
__host__ __device__ constexpr int frame_plan_count(bool tc)
{
    return (!tc && LOG_N >= 8 && LOG_N <= 10) ? 2 : 1;
}
template <int LOG_N, int V, bool TC>
struct PlanOfT {
    using type = FramePlan<LOG_N, TC>;
};
template <int LOG_N>
struct PlanOfT<LOG_N, 1, false> {
    using type = Plan<LOG_N, (LOG_N >= 10 ? 64 : lanes_for(LOG_N)), false, true>;
};
template <int LOG_N, int V, bool TC>
using PlanOf = typename PlanOfT<LOG_N, V, TC>::type;

// Column tasks over 2 columns shift their sequence pairs (pair s = field
// pair * W + column) by a few float4 so that the intermediate's stores (lanes
// walking field pair, column, row) and the finalize's reads (column, row)
// spread over the shared-memory banks: the shifts minimise the 16-byte
// wavefronts of both patterns together over a strip (a search over all
// shifts mod 8 with the padding of pad4 modelled).
template <int NF, int W>
__host__ __device__ constexpr int col_pair_shift(int s)
{
    return W != 2 ? 0 : (NF == 6 ? (s + 1) / 2 : s % 2);
}
// float2 the shifts add behind the last pair.
template <int NF, int W>
__host__ __device__ constexpr int col_shift_f2()
{
    return 2 * col_pair_shift<NF, W>(NF * W / 2 - 1);
}

// The shifts' float2 for a task of plan P (none for single sequences).
template <class P, int NF, int W>
__host__ __device__ constexpr int col_shift_f2_of()
{
    return P::PAIRED ? col_shift_f2<NF, W>() : 0;
}

// Foam window of a column task over W columns: columns x0 - 1 .. x0 + W of
// every row (WW floats per row), and its size in float2.
template <int W>
__host__ __device__ constexpr int foam_window()
{
    return W + 2;
}
template <int LOG_N, int W>
__host__ __device__ constexpr int foam_window_f2()
{
    return (1 << LOG_N) * foam_window<W>() / 2;
}

// The tensor-core engine of a task's sequences, one engine call per
// transform: at N = 512 the 2 NF sequences of a row pair or two columns (8
// without velocity, 12 with); at N = 64, 128 and 256 the ROWS x NF of the
// plan's rows or columns (16 x threads values in all). Sizes without a
// tensor-core form name the 512-point engine, which their kernels never use.
template <int LOG_N>
__host__ __device__ constexpr bool has_tc_form()
{
    return LOG_N >= 6 && LOG_N <= 9;
}
template <int LOG_N, int NF>
struct TcEngineOfT {
    using type = tc::Engine<2 * NF>;
};
template <int LOG_N, int NF>
    requires(LOG_N >= 6 && LOG_N <= 8)
struct TcEngineOfT<LOG_N, NF> {
    using type = tc::SmallEngine<LOG_N, FramePlan<LOG_N, true>::ROWS * NF>;
};
template <int LOG_N, int NF>
using TcEngineOf = typename TcEngineOfT<LOG_N, NF>::type;

// Copy the FP32 twiddle table into shared memory at `tws`.
template <class P>
__device__ __forceinline__ void load_twiddles(float2* tws, const float2* __restrict__ src, int tid, int nt)
{
    constexpr int N = P::N;
    for (int i = tid; i < N - 1; i += nt) tws[i] = src[i];
}

// The inverse DFT of the COUNT sequences of a task: the radix-2 Stockham FFT
// on single sequences (one lane group of G per sequence) or on sequence pairs
// (one lane group of G2 per pair, named barrier 1 + pair where a pair spans
// two warps), or with TC the tensor-core four-step DFT, 8 sequences per
// engine call (N = 512; its twiddles live in the engine).
template <class P, int AR, int COUNT, int COLW = 0, class Eng = tc::Engine<8>>
__device__ __forceinline__ void transform_all(float2* data, const float2* tws, int tid, Eng* eng,
                                              unsigned* error)
{
    if constexpr (P::TC && P::LOG_N == 9) {
        static_assert(P::SEQ * 2 >= 16 * tc::kZStride, "a sequence's space must hold its staged stage-3 rows");
        static_assert(COUNT == Eng::Lay::kThreads / 32, "one engine call holds the task's sequences");
        eng->dft512(data, P::SEQ, COUNT, tid, error);
    } else if constexpr (P::TC) {
        static_assert(has_tc_form<P::LOG_N>(), "the tensor-core form covers N = 64 to 512");
        static_assert(P::SEQ * 2 >= Eng::Lay::N1 * Eng::Lay::kZStride,
                      "a sequence's space must hold its staged stage-3 rows");
        static_assert(COUNT * P::N == 16 * Eng::Lay::kThreads, "one engine call holds the task's sequences");
        eng->dft(data, P::SEQ, COUNT, tid, error);
    } else if constexpr (!P::PAIRED) {
        fft_sequence<P::LOG_N, P::G, AR>(data + (tid / P::G) * P::SEQ, tws, tid % P::G);
    } else {
        constexpr int G2 = P::G2;
        static_assert(COUNT % 2 == 0, "sequences come in pairs");
        static_assert(G2 <= 32 || (COUNT / 2) < 16, "one named barrier per pair");
        const int pair = tid / G2;
        const int shift = COLW != 0 ? col_pair_shift<COUNT / (COLW != 0 ? COLW : 1), COLW>(pair) : 0;
        fft_pair<P::LOG_N, G2, AR>(reinterpret_cast<ulonglong2*>(data) + pair * P::SEQ4 + shift, tws, tid % G2,
                                     1 + pair);
    }
}

// ---------------------------------------------------------------------------
// Row task: RP row pairs of one ocean (evolve + row FFTs), written to the
// intermediate slot `inter_slot` (N*N*NF float2). `tws` already holds the
// twiddles in shared memory.
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// h0 rows by bulk asynchronous copy (TMA, untiled). A row task's h0 rows are
// contiguous in global memory and land unchanged in shared memory, so thread
// 0 copies each with one cp.async.bulk completing on an mbarrier and the CTA
// waits on it, instead of every thread moving 16-byte pieces through its
// registers (the shared-memory pipe is the frame's busiest unit). The other
// transfers of the frame change layout on the way (rows to cell-major, strips
// to padded sequences, transposes), which a TMA copy cannot do.
// ---------------------------------------------------------------------------
constexpr unsigned long long kH0WaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Once per CTA (thread 0), before the CTA's first barrier.
__device__ __forceinline__ void h0_bar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Thread 0: `rows` copies of row_f2 float2 each, src(r) -> dst + r * row_f2,
// all completing on `bar`. Addresses and sizes are multiples of 16 bytes.
template <typename RowSrc>
__device__ __forceinline__ void h0_rows_issue(uint64_t* bar, float2* dst, int rows, int row_f2, RowSrc src)
{
    const uint32_t b = smem_addr(bar);
    const unsigned bytes = static_cast<unsigned>(row_f2 * sizeof(float2));
    // The previous task accessed this memory through the generic proxy.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes * rows) : "memory");
    for (int r = 0; r < rows; ++r) {
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                         smem_addr(dst + r * row_f2)),
                     "l"(src(r)), "r"(bytes), "r"(b)
                     : "memory");
    }
}

// Every thread: wait for phase `parity` of `bar`, for at most limit_ns;
// then the error word is set (when there is one) and the task goes on.
__device__ __forceinline__ void h0_rows_wait(uint64_t* bar, uint32_t parity, unsigned* error,
                                             unsigned long long limit_ns = kH0WaitNs)
{
    const uint32_t b = smem_addr(bar);
    unsigned long long t0 = 0;
    for (int spin = 0;; ++spin) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred P;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P;\n\t}\n"
            : "=r"(done)
            : "r"(b), "r"(parity)
            : "memory");
        if (done) return;
        if (spin == 0) t0 = tc::now_ns();
        if ((spin & 63) == 63 && tc::now_ns() - t0 > limit_ns) {
            if (error != nullptr) atomicCAS(error, 0u, 1u);
            return;
        }
    }
}

// Release add at GPU scope: every write that happens before it (the CTA's,
// through the preceding barrier) is visible to an acquirer that sees the sum.
__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v)
{
    asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The persistent queues' counter adds that a task makes once its inputs are
// in shared memory (thread 0; pub = {previous task, this task}, either may be
// null). pub[0] is the CTA's previous task: its writes were all issued before
// the barrier this task began with, and the time the task spent loading lets
// them drain, so the release costs little here, where at the top of the loop
// it stalled the whole CTA. pub[1] is this task itself when it is a column
// task: it reads its intermediate slot only while staging, so the slot is
// free for the next ocean's row tasks from here on.
__device__ __forceinline__ void publish_staged(unsigned* const* pub, int tid)
{
    if (pub != nullptr && tid == 0) {
        if (pub[0] != nullptr) red_release_add(pub[0], 1u);
        if (pub[1] != nullptr) red_release_add(pub[1], 1u);
    }
}

template <class P, int NF, int AR>
__device__ __forceinline__ void row_task(const FrameArgs& a, int ocean, int group,
                                         float2* __restrict__ inter_slot, float2* smem,
                                         const float2* tws, int tid, uint64_t* h0_bar, uint32_t h0_parity,
                                         TcEngineOf<P::LOG_N, NF>* eng = nullptr, unsigned* error = nullptr,
                                         unsigned* const* pub = nullptr)
{
    using D = P;
    constexpr int LOG_N = P::LOG_N;
    constexpr int N = P::N, G = P::G, SEQ = P::SEQ, SEQ4 = P::SEQ4, ROWS = P::ROWS;
    constexpr int NT = ROWS * NF * G;
    constexpr int Q = NF / 2;
    constexpr bool PAIRED = P::PAIRED;

    float2* data = smem;                                   // sequences of rows jr, fields f
    float4* data4 = reinterpret_cast<float4*>(smem);       // the same as pairs (jr, f / 2)
    float2* h0s = data + ROWS * NF * P::SEQF2;             // [H0ROWS][N]

    OceanConsts cst;
    const float2* geom;
    const float* kvec;
    const float2* h0;
    if (a.table != nullptr) {
        const OceanSlot& s = a.table[ocean];
        cst = s.cst;
        geom = s.omega_kinv;
        kvec = s.kvec;
        h0 = s.h0;
    } else {
        cst = a.consts[ocean];
        geom = a.omega_kinv + static_cast<size_t>(cst.geom) * N * N;
        kvec = a.kvec + static_cast<size_t>(cst.geom) * N;
        h0 = a.h0 + static_cast<size_t>(ocean) * N * N;
    }
    const double top = a.t_over_2pi[ocean];

    // Row of slot jr: pair p = (jr's pair index) covers (p, N-p), or (0, N/2)
    // for p = 0. Paired tasks hold whole pairs (slot jr = 2 j + r); single-row
    // tasks take consecutive rows of that order, so a row and its mirror are
    // neighbouring tasks.
    auto row_of = [&](int jr) -> int {
        int p, r;
        if constexpr (D::SINGLE) {
            const int idx = group * ROWS + jr;
            p = idx >> 1;
            r = idx & 1;
        } else {
            p = group * P::RP + (jr >> 1);
            r = jr & 1;
        }
        if (p == 0) return r ? N / 2 : 0;
        return r ? N - p : p;
    };
    // Staged h0 row holding h0(-k) for slot jr's row: single rows keep a copy
    // of the mirror row in slot ROWS + jr; a pair's other row is the mirror
    // (rows 0 and N/2 mirror themselves).
    auto mirror_slot = [&](int jr) -> int {
        if constexpr (D::SINGLE) {
            return ROWS + jr;
        } else {
            const int p = group * P::RP + (jr >> 1);
            const int r = jr & 1;
            return (jr & ~1) + ((p == 0) ? r : 1 - r);
        }
    };

    // The h0 rows go first (bulk copies), then every thread loads the
    // geometry of its cells, so both latencies overlap ahead of the wait.
    static_assert((ROWS * NF * P::SEQF2 * sizeof(float2)) % 16 == 0 && (N * sizeof(float2)) % 16 == 0,
                  "the h0 rows start and end on 16-byte boundaries in shared memory");
    if (tid == 0) {
        h0_rows_issue(h0_bar, h0s, D::H0ROWS, N, [&](int k) {
            const int row = k < ROWS ? row_of(k) : ((N - row_of(k - ROWS)) & (N - 1));
            return h0 + static_cast<size_t>(row) * N;
        });
    }
    // HALVES: the paired FP32 plan with two rows, where row jr's Q field
    // pairs are worked by threads [jr * HT, (jr + 1) * HT): each row's warps
    // evolve, transform and store their own row and meet on a named barrier
    // (ids 8 and 9; the pair barriers take 1 + pair) instead of the CTA's, so
    // neither row waits on the other (the h0 rows both read are in place once
    // each thread's mbarrier wait returns). Same bits; 64 x 512^2 with velocity
    // and persistent foam 0.981 -> 0.977 ms a frame.
    constexpr bool HALVES = PAIRED && !P::TC && ROWS == 2;
    constexpr int HT = HALVES ? NT / 2 : NT;        // threads per barrier group
    constexpr int CELLS = HALVES ? N : ROWS * N;    // cells per group
    constexpr int ITER = (CELLS + HT - 1) / HT;
    const int hh = HALVES ? tid / HT : 0;
    const int lt = HALVES ? tid - hh * HT : tid;
    auto group_bar = [&]() {
        if constexpr (HALVES) {
            asm volatile("bar.sync %0, %1;" ::"r"(8 + hh), "r"(HT) : "memory");
        } else {
            __syncthreads();
        }
    };
    float2 wk_of[ITER];
    float kx_of[ITER], kz_of[ITER];
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int cell = hh * N + lt + it * HT;
        if (lt + it * HT < CELLS) {
            const int jr = cell >> LOG_N;
            const int x = cell & (N - 1);
            const int row = row_of(jr);
            wk_of[it] = __ldg(&geom[static_cast<size_t>(row) * N + x]);
            kx_of[it] = __ldg(&kvec[x]);
            kz_of[it] = __ldg(&kvec[row]);
        }
    }
    h0_rows_wait(h0_bar, h0_parity, error);
    group_bar();
    publish_staged(pub, tid);

    // Evolve (src/core/evolve.cpp:28-121 and :123-184), one cell at a time.
#pragma unroll
    for (int it = 0; it < ITER; ++it) {
        const int cell = hh * N + lt + it * HT;
        if (lt + it * HT >= CELLS) break;
        const int jr = cell >> LOG_N;
        const int x = cell & (N - 1);
        const float2 av = h0s[jr * N + x];
        const float2 bm = h0s[mirror_slot(jr) * N + ((N - x) & (N - 1))];
        float2 pv[NF];
        evolve_cell<NF>(av, bm, wk_of[it], kx_of[it], kz_of[it], top, pv);
        if constexpr (!PAIRED) {
            float2* base = data + (jr * NF) * SEQ + pad_idx(x);
#pragma unroll
            for (int f = 0; f < NF; ++f) base[f * SEQ] = pv[f];
        } else {
            float4* base = data4 + (jr * Q) * SEQ4 + pad4(x);
#pragma unroll
            for (int q = 0; q < Q; ++q)
                base[q * SEQ4] = make_float4(pv[2 * q].x, pv[2 * q + 1].x, pv[2 * q].y, pv[2 * q + 1].y);
        }
    }
    group_bar();

    transform_all<P, AR, ROWS * NF>(data, tws, tid, eng, error);
    group_bar();

    // Write the rows cell-major: inter[row][x][f], NF/2 float4 per cell.
    // HT is a multiple of Q, so each thread keeps one field pair fp and walks
    // cells with a constant stride (no division in the loop).
    constexpr int CSTEP = HT / Q;
    float4* inter = reinterpret_cast<float4*>(inter_slot);
    const int fp = lt % Q;
#pragma unroll 4
    for (int cell = hh * N + lt / Q; cell < (HALVES ? (hh + 1) * N : ROWS * N); cell += CSTEP) {
        const int jr = cell >> LOG_N;
        const int x = cell & (N - 1);
        const int row = row_of(jr);
        float4 o;
        if constexpr (!PAIRED) {
            const float2 v0 = data[(jr * NF + 2 * fp) * SEQ + pad_idx(x)];
            const float2 v1 = data[(jr * NF + 2 * fp + 1) * SEQ + pad_idx(x)];
            o = make_float4(v0.x, v0.y, v1.x, v1.y);
        } else {
            const float4 v = data4[(jr * Q + fp) * SEQ4 + pad4(x)];
            o = make_float4(v.x, v.z, v.y, v.w);
        }
        inter[(static_cast<size_t>(row) * N + x) * Q + fp] = o;
    }
}

// ---------------------------------------------------------------------------
// Column task: W columns of one ocean from intermediate slot `inter_slot`
// (column FFTs + finalize + optional foam substep). CG loads read the
// intermediate from L2: another CTA wrote it during this launch.
// ---------------------------------------------------------------------------
template <class P, int NF, int AR, bool FOAM, int W, bool CG>
__device__ __forceinline__ void col_task(const FrameArgs& a, int ocean, int strip,
                                         const float2* __restrict__ inter_slot, float2* smem,
                                         const float2* tws, int tid, TcEngineOf<P::LOG_N, NF>* eng = nullptr,
                                         unsigned* error = nullptr, unsigned* const* pub = nullptr)
{
    constexpr int N = P::N, G = P::G, SEQ = P::SEQ, SEQ4 = P::SEQ4;
    constexpr int NT = NF * W * G;
    constexpr int Q = NF / 2;
    constexpr bool PAIRED = P::PAIRED;
    float2* data = smem;                             // TC: sequence f*W + w
    float4* data4 = reinterpret_cast<float4*>(smem); // pairs: pair p*W + w holds fields 2p, 2p+1
    const int x0 = strip * W;
    constexpr bool FSTEP = NF == 6 && FOAM;
    constexpr int WW = foam_window<W>();

    const size_t base = static_cast<size_t>(ocean) * N * N;
    // With persistent foam: the previous foam state in columns x0 - 1 ..
    // x0 + W of every row, [y][WW] behind the sequences (foam_window_f2
    // float2 the caller reserves), loaded with the intermediate so the taps
    // of the foam step (within a cell of the strip for any velocity up to
    // cell / dt) come from shared memory.
    float* fwin = reinterpret_cast<float*>(smem + NF * W * P::SEQF2 + col_shift_f2_of<P, NF, W>());
    if constexpr (FSTEP) {
        // Asynchronous 4-byte copies straight into the window (no register
        // round trip, nothing to wait for until the finalize below).
        const float* cur = a.foam_cur + base;
        for (int k = tid; k < N * WW; k += NT) {
            const int xc = (x0 - 1 + k % WW) & (N - 1);
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(fwin + k)),
                         "l"(cur + static_cast<size_t>(k / WW) * N + xc)
                         : "memory");
        }
    }

    const float4* inter = reinterpret_cast<const float4*>(inter_slot);
    constexpr int CSTEP = NT / Q;  // NT is a multiple of Q
    const int fp = tid % Q;
    // Up to 8 loads per thread in flight before the first shared store.
    constexpr int LIT = (N * W + CSTEP - 1) / CSTEP;
    constexpr int LB = LIT < 8 ? LIT : 8;
#pragma unroll 1
    for (int b0 = 0; b0 < LIT; b0 += LB) {
        float4 buf[LB];
#pragma unroll
        for (int k = 0; k < LB; ++k) {
            const int cw = tid / Q + (b0 + k) * CSTEP;
            if (cw < N * W) {
                const float4* src = inter + (static_cast<size_t>(cw / W) * N + x0 + cw % W) * Q + fp;
                buf[k] = CG ? __ldcg(src) : *src;
            }
        }
#pragma unroll
        for (int k = 0; k < LB; ++k) {
            const int cw = tid / Q + (b0 + k) * CSTEP;
            if (cw < N * W) {
                const int y = cw / W;
                const int w = cw % W;
                const float4 v = buf[k];
                if constexpr (!PAIRED) {
                    data[((2 * fp) * W + w) * SEQ + pad_idx(y)] = make_float2(v.x, v.y);
                    data[((2 * fp + 1) * W + w) * SEQ + pad_idx(y)] = make_float2(v.z, v.w);
                } else {
                    data4[(fp * W + w) * SEQ4 + col_pair_shift<NF, W>(fp * W + w) + pad4(y)] =
                        make_float4(v.x, v.z, v.y, v.w);
                }
            }
        }
    }
    __syncthreads();
    publish_staged(pub, tid);

    transform_all<P, AR, NF * W, W>(data, tws, tid, eng, error);
    if constexpr (FSTEP) asm volatile("cp.async.wait_all;" ::: "memory");  // this thread's window copies
    __syncthreads();

    OceanConsts cst;
    float4* out_disp;
    float4* out_normal;
    float4* out_vel;
    if (a.table != nullptr) {
        const OceanSlot& s = a.table[ocean];
        cst = s.cst;
        out_disp = s.disp;
        out_normal = s.normal;
        out_vel = s.velocity;
    } else {
        cst = a.consts[ocean];
        out_disp = a.disp + base;
        out_normal = a.normal + base;
        out_vel = a.velocity + base;
    }
    const float lambda = cst.lambda;
    constexpr int FC = N * W;
    constexpr int FIT = (FC + NT - 1) / NT;
    const float* cur = a.foam_cur + base;
    // A tap in the window is read from shared memory, any other from global.
    auto foam_get = [&](int zz, int xx) {
        const int j = (xx - x0 + 1) & (N - 1);
        return j < WW ? fwin[zz * WW + j] : __ldg(&cur[static_cast<size_t>(zz) * N + xx]);
    };
#pragma unroll
    for (int it = 0; it < FIT; ++it) {
        const int i = tid + it * NT;
        if (i >= FC) break;
        const int y = i / W;
        const int w = i % W;
        const int x = x0 + w;
        float2 f0, f1, f2, f3, f4, f5;
        if constexpr (!PAIRED) {
            const int sy = pad_idx(y);
            f0 = data[(0 * W + w) * SEQ + sy];
            f1 = data[(1 * W + w) * SEQ + sy];
            f2 = data[(2 * W + w) * SEQ + sy];
            f3 = data[(3 * W + w) * SEQ + sy];
            if constexpr (NF == 6) {
                f4 = data[(4 * W + w) * SEQ + sy];
                f5 = data[(5 * W + w) * SEQ + sy];
            }
        } else {
            const int sy = pad4(y);
            const float4 q0 = data4[(0 * W + w) * SEQ4 + col_pair_shift<NF, W>(0 * W + w) + sy];
            const float4 q1 = data4[(1 * W + w) * SEQ4 + col_pair_shift<NF, W>(1 * W + w) + sy];
            f0 = make_float2(q0.x, q0.z);
            f1 = make_float2(q0.y, q0.w);
            f2 = make_float2(q1.x, q1.z);
            f3 = make_float2(q1.y, q1.w);
            if constexpr (NF == 6) {
                const float4 q2 = data4[(2 * W + w) * SEQ4 + col_pair_shift<NF, W>(2 * W + w) + sy];
                f4 = make_float2(q2.x, q2.z);
                f5 = make_float2(q2.y, q2.w);
            }
        }
        const CellOut c = finalize_cell(f0, f1, f2, f3, lambda, cst.foam_threshold, cst.inv_threshold);
        const size_t idx = static_cast<size_t>(y) * N + x;
        __stcs(&out_disp[idx], c.disp);
        __stcs(&out_normal[idx], c.normal);
        if constexpr (NF == 6) {
            __stcs(&out_vel[idx], make_float4(f4.x, f4.y, f5.x, 0.0f));
            if constexpr (FSTEP) {
                const FoamTaps t = foam_taps(N, x, y, f4.x, f5.x, a.foam_dt, a.foam_scale, a.foam_drift_x,
                                             a.foam_drift_z, a.foam_inv_cell, foam_get);
                __stcs(&a.foam_next[base + idx], foam_finish(t, c.disp.w, a.foam_decay, a.foam_gain));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Per-chunk kernels: grid (groups, oceans in the chunk); ocean o of the chunk
// uses intermediate slot o.
// ---------------------------------------------------------------------------
template <int LOG_N, int NF, int AR>
__global__ void __launch_bounds__(ChunkPlan<LOG_N>::template threads<NF>())
row_pass_kernel(FrameArgs a)
{
    using P = ChunkPlan<LOG_N>;
    constexpr int NT = P::template threads<NF>();
    extern __shared__ float4 smem4[];
    float2* smem = reinterpret_cast<float2*>(smem4);
    float2* tws = smem + P::ROWS * NF * P::SEQF2 + P::H0ROWS * P::N;
    __shared__ uint64_t h0_bar;
    if (threadIdx.x == 0) h0_bar_init(&h0_bar);
    load_twiddles<P>(tws, a.twiddles, threadIdx.x, NT);
    __syncthreads();  // the twiddles are complete before any transform reads them; the barrier is set up
    const int o = blockIdx.y;
    row_task<P, NF, AR>(a, a.ocean_base + o, blockIdx.x, a.inter + static_cast<size_t>(o) * P::N * P::N * NF,
                          smem, tws, threadIdx.x, &h0_bar, 0u, nullptr, a.error);
}

template <int LOG_N, int NF, int AR, bool FOAM>
__global__ void __launch_bounds__(NF * Shape<LOG_N>::W * Shape<LOG_N>::G)
col_pass_kernel(FrameArgs a)
{
    using S = Shape<LOG_N>;
    using P = ChunkPlan<LOG_N>;
    constexpr int NT = NF * S::W * S::G;
    extern __shared__ float4 smem4[];
    float2* smem = reinterpret_cast<float2*>(smem4);
    float2* tws = smem + NF * S::W * P::SEQF2 + col_shift_f2_of<P, NF, S::W>() + foam_window_f2<LOG_N, S::W>();
    load_twiddles<P>(tws, a.twiddles, threadIdx.x, NT);
    __syncthreads();  // the twiddles are complete before any transform reads them
    const int o = blockIdx.y;
    col_task<P, NF, AR, FOAM, S::W, false>(a, a.ocean_base + o, blockIdx.x,
                                             a.inter + static_cast<size_t>(o) * P::N * P::N * NF, smem, tws,
                                             threadIdx.x);
}

// ---------------------------------------------------------------------------
// Persistent frame kernel: one launch per frame for every ocean of the batch.
//
// CTAs take tickets from an ordered queue R(0) | R(1) C(0) | R(2) C(1) | ...
// | C(count-1), where R(b) are ocean b's row tasks and C(b) its column tasks.
// C(b) waits until all of R(b) finished; R(b) writes intermediate slot
// b % slots and first waits until C(b - slots) finished reading it. Every
// awaited task holds an earlier ticket, so it is already running on some CTA
// and never waits on a later one: the queue cannot deadlock, co-resident or
// not. Waits are bounded (QueueArgs::wait_ns); a CTA that gives up sets the error word
// and leaves, and the others give up in turn.
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Spin until *counter >= target or the error word is set or limit_ns passes.
// Returns false on timeout / abort.
__device__ bool wait_at_least(const unsigned* counter, unsigned target, unsigned* error,
                              unsigned long long limit_ns)
{
    if (ld_acquire(counter) >= target) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        __nanosleep(64);
        if (ld_acquire(counter) >= target) return true;
        if (ld_acquire(error) != 0u) return false;
        if (global_ns() - t0 > limit_ns) {
            atomicCAS(error, 0u, 1u);
            return false;
        }
    }
}

// Resident CTAs the persistent kernel is compiled for: 768 threads per SM
// (at N = 1024, whose 32 values per lane need the registers, two CTAs of
// single rows).
// (The tensor-core form needs about 150-170 KB of shared memory per CTA:
// one CTA per SM, which also bounds its tensor memory to 256 columns.)
template <class P, int NF>
constexpr int frame_min_blocks()
{
    constexpr int nt = P::template threads<NF>();
    if (P::TC) return 1;
    if (P::LANE_LOG >= 5) return 1;  // 32 values a lane: the registers allow one CTA
    return 768 / nt < 1 ? 1 : (768 / nt > 16 ? 16 : 768 / nt);
}

// Shared floats (float2 units) of a persistent task's data area (either
// kind), and the byte offset of the tensor-core engine's area behind the
// twiddles.
template <class P, int NF>
__host__ __device__ constexpr size_t frame_data_float2()
{
    constexpr size_t row = P::ROWS * NF * P::SEQF2 + P::H0ROWS * P::N;
    constexpr size_t col = NF * P::PW * P::SEQF2 + col_shift_f2_of<P, NF, P::PW>() + foam_window_f2<P::LOG_N, P::PW>();
    return row > col ? row : col;
}

template <int LOG_N, int NF>
__host__ __device__ constexpr size_t frame_engine_offset()
{
    return ((frame_data_float2<FramePlan<LOG_N, true>, NF>() + (size_t(1) << LOG_N)) * sizeof(float2) + 127) /
           128 * 128;
}

template <class P, int NF, int AR, bool FOAM>
__global__ void __launch_bounds__(P::template threads<NF>(), frame_min_blocks<P, NF>())
frame_kernel(FrameArgs a, QueueArgs q)
{
    constexpr int LOG_N = P::LOG_N;
    constexpr bool TC = P::TC;
    constexpr int N = P::N;
    constexpr int NT = P::template threads<NF>();
    constexpr int RT = P::RT;       // row tasks per ocean
    constexpr int CT = N / P::PW;   // column tasks per ocean
    constexpr size_t kDataFloat2 = frame_data_float2<P, NF>();
    static_assert(size_t(NF) * P::PW * P::SEQF2 + col_shift_f2_of<P, NF, P::PW>() +
                          foam_window_f2<LOG_N, P::PW>() <= kDataFloat2,
                  "the column task's foam window fits in the data area");
    extern __shared__ float4 smem4[];
    float2* smem = reinterpret_cast<float2*>(smem4);
    float2* tws = smem + kDataFloat2;
    __shared__ unsigned s_ticket;
    __shared__ int s_ok;
    // Thread 0's queue state between tasks, kept in shared memory so that it
    // takes no registers in the task code that every thread runs, except the
    // ticket drawn one task ahead: its atomic's result lands in a register
    // that thread 0 reads only at the next task, so the round trip to L2
    // overlaps the current task instead of holding thread 0 (and with it the
    // CTA's ticket barrier) until it returns. Same bits; 64 x 512^2 with
    // velocity and persistent foam 0.999 -> 0.981 ms a frame.
    __shared__ unsigned* s_publish;   // the current task's counter, added after it (row tasks)
    __shared__ unsigned* s_pub[2];    // publish_staged's pair for the current task
    unsigned r_next = 0;              // thread 0: the ticket drawn one task ahead
    int r_have_next = 0;
    __shared__ uint64_t h0_bar;   // the row tasks' h0 copies; phase k = k-th row task
    uint32_t h0_parity = 0;

    const int tid = threadIdx.x;
    if constexpr (!TC) load_twiddles<P>(tws, a.twiddles, tid, NT);
    TcEngineOf<LOG_N, NF> eng{reinterpret_cast<unsigned char*>(smem4) + frame_engine_offset<LOG_N, NF>(), 0};
    if constexpr (TC) {
        static_assert(NT == TcEngineOf<LOG_N, NF>::Lay::kThreads, "the engine works with the task's threads");
        eng.init(tid, NT, a.twiddles);
    }

    const unsigned count = static_cast<unsigned>(q.count);
    const unsigned total = count * (RT + CT);
    const size_t slot_f2 = static_cast<size_t>(N) * N * NF;
    // Ticket -> (row?, ocean, task index) for the queue order above.
    auto decode = [&](unsigned t, bool& row, unsigned& ocean, unsigned& idx) {
        if (t < RT) {
            row = true, ocean = 0, idx = t;
            return;
        }
        const unsigned u = t - RT, per = RT + CT, blk = u / per, off = u % per;
        if (blk + 1 < count) {
            row = off < RT;
            ocean = row ? blk + 1 : blk;
            idx = row ? off : off - RT;
        } else {
            row = false, ocean = count - 1, idx = off;
        }
    };

    // Thread 0 takes the next ticket and checks that task's inputs; one
    // barrier hands the ticket to the CTA. The previous task (a row task: a
    // column task publishes itself once staged) is published with a release
    // add (the barrier at the top of the loop orders every thread's writes
    // before it, the pattern grid-wide barriers use). With q.defer, and the
    // next task's inputs ready, the next task makes that add once it has
    // staged them (publish_staged); otherwise it comes here, before the wait,
    // since the next task may depend on the one just finished. So a CTA never
    // waits while it holds an unpublished task. Deferring pays with velocity
    // (64 x 512^2 with foam: 0.995 -> 0.984 ms a frame) and costs without it
    // (64 x 512^2: 0.608 -> 0.624 ms), where the column tasks wait on the
    // later adds; the batch defaults by field count and its autotuner times both.
    // Far from the end of the queue the following ticket is drawn one task
    // ahead; near the end tickets are drawn when a CTA is free, since a
    // ticket held by a CTA whose current task still waits would idle others
    // (in a short queue, e.g. 3 x 256^2 cascade levels on 296 CTAs, drawing
    // ahead cost 8 us per frame). A drawn ticket T runs right after the
    // CTA's current task (< T), which waits on nothing later, so the queue
    // stays deadlock-free.
    if (tid == 0) {
        h0_bar_init(&h0_bar);
        s_publish = nullptr;
        r_next = atomicAdd(q.ticket, 1u);
        r_have_next = 1;
    }
    while (true) {
        __syncthreads();  // previous task's writes issued; shared memory free
        if (tid == 0) {
            unsigned* prev = s_publish;
            const unsigned t = r_have_next ? r_next : atomicAdd(q.ticket, 1u);
            r_have_next = 0;
            int ok = 1;
            unsigned* publish = nullptr;
            unsigned* self = nullptr;
            const unsigned* dep = nullptr;
            unsigned need = 0;
            if (t < total) {
                if (t + 2u * gridDim.x < total) {
                    r_next = atomicAdd(q.ticket, 1u);
                    r_have_next = 1;
                }
                bool row;
                unsigned ocean, idx;
                decode(t, row, ocean, idx);
                if (row) {
                    if (ocean >= static_cast<unsigned>(q.slots)) dep = q.cols_done + (ocean - q.slots), need = CT;
                    publish = q.rows_done + ocean;
                } else {
                    dep = q.rows_done + ocean, need = RT;
                    self = q.cols_done + ocean;
                }
            }
            if (t >= total || !q.defer || (dep != nullptr && ld_acquire(dep) < need)) {
                if (prev != nullptr) red_release_add(prev, 1u);
                prev = nullptr;
                if (dep != nullptr) ok = wait_at_least(dep, need, q.error, q.wait_ns);
            }
            s_pub[0] = prev;
            s_pub[1] = self;
            s_publish = publish;
            s_ticket = t;
            s_ok = ok;
        }
        __syncthreads();
        const unsigned t = s_ticket;
        if (t >= total || !s_ok) break;
        bool row;
        unsigned ocean, idx;
        decode(t, row, ocean, idx);
        const unsigned slot = ocean % static_cast<unsigned>(q.slots);
        const int abs_ocean = a.ocean_base + static_cast<int>(ocean);
        if (row) {
            row_task<P, NF, AR>(a, abs_ocean, static_cast<int>(idx), a.inter + slot * slot_f2, smem, tws, tid,
                                  &h0_bar, h0_parity, &eng, q.error, s_pub);
            h0_parity ^= 1u;
        } else {
            col_task<P, NF, AR, FOAM, P::PW, true>(a, abs_ocean, static_cast<int>(idx),
                                                             a.inter + slot * slot_f2, smem, tws, tid,
                                                             &eng, q.error, s_pub);
        }
    }
    if constexpr (TC) eng.release(tid);
}

// ---------------------------------------------------------------------------
// Mixed-size frame kernel: the frames of several same-size groups of oceans in
// one persistent launch. Every size runs with 64 * NF threads (384 with
// velocity, 256 without): the default plans from N = 32 to 512 (row pairs,
// RP * G = 32), and N = 1024 over 64 lanes a sequence (16 values a lane, three
// passes, single rows) instead of the persistent kernel's 32 lanes x 32
// values, whose registers would cap every size at one CTA per SM. The queue
// holds group after group (each in the persistent kernel's order, with its
// own counters and intermediate ring), so a CTA picks up whichever size comes
// next, and the wave's tail is shared by all sizes. Each size's twiddle table
// sits in shared memory for the whole launch.
// ---------------------------------------------------------------------------
constexpr int kMixMinLog = 5;
constexpr int kMixMaxLog = 10;

template <int L>
using MixPlan = Plan<L, (L >= 10 ? 64 : lanes_for(L)), false, (L >= 10)>;

template <int NF, int L = kMixMinLog>
__host__ __device__ constexpr size_t mixed_data_float2()
{
    constexpr size_t here = frame_data_float2<MixPlan<L>, NF>();
    if constexpr (L >= kMixMaxLog) {
        return here;
    } else {
        constexpr size_t rest = mixed_data_float2<NF, L + 1>();
        return here > rest ? here : rest;
    }
}

// float2 of size log_n's twiddle table, rounded up to a 16-byte multiple.
__host__ __device__ constexpr int mix_twf2(int log_n)
{
    const int t = log_n == 5   ? MixPlan<5>::TWF2
                  : log_n == 6 ? MixPlan<6>::TWF2
                  : log_n == 7 ? MixPlan<7>::TWF2
                  : log_n == 8 ? MixPlan<8>::TWF2
                  : log_n == 9 ? MixPlan<9>::TWF2
                               : MixPlan<10>::TWF2;
    return (t + 1) & ~1;
}
// Offset of size log_n's table in the twiddle area (float2).
__host__ __device__ constexpr int mix_tw_offset(int log_n)
{
    int off = 0;
    for (int l = kMixMinLog; l < log_n; ++l) off += mix_twf2(l);
    return off;
}
__host__ __device__ constexpr size_t mixed_smem_bytes(int nf)
{
    return sizeof(float2) * ((nf == 4 ? mixed_data_float2<4>() : mixed_data_float2<6>()) +
                             mix_tw_offset(kMixMaxLog + 1));
}

template <int L>
__host__ __device__ constexpr int mix_rt()
{
    return MixPlan<L>::RT;
}
template <int L>
__host__ __device__ constexpr int mix_ct()
{
    return MixPlan<L>::N / MixPlan<L>::PW;
}
// (row tasks, column tasks) per ocean of size log_n.
__host__ __device__ inline void mix_tasks_per_ocean(int log_n, unsigned& rt, unsigned& ct)
{
    switch (log_n) {
        case 5: rt = mix_rt<5>(), ct = mix_ct<5>(); break;
        case 6: rt = mix_rt<6>(), ct = mix_ct<6>(); break;
        case 7: rt = mix_rt<7>(), ct = mix_ct<7>(); break;
        case 8: rt = mix_rt<8>(), ct = mix_ct<8>(); break;
        case 9: rt = mix_rt<9>(), ct = mix_ct<9>(); break;
        default: rt = mix_rt<10>(), ct = mix_ct<10>(); break;
    }
}

template <int L, int NF>
__device__ __forceinline__ void mix_load_twiddles(float2* area, const float2* __restrict__ src, int tid, int nt)
{
    load_twiddles<MixPlan<L>>(area + mix_tw_offset(L), src, tid, nt);
}

template <int L, int NF, int AR>
__device__ __noinline__ void mix_run(const MixedGroup& g, bool row, int ocean, int idx, float2* smem,
                                        const float2* tw_area, int tid, uint64_t* h0_bar, uint32_t h0_parity,
                                        unsigned* error, unsigned* const* pub)
{
    using P = MixPlan<L>;
    const unsigned slot = static_cast<unsigned>(ocean) % static_cast<unsigned>(g.slots);
    float2* inter = g.a.inter + static_cast<size_t>(slot) * P::N * P::N * NF;
    const float2* tws = tw_area + mix_tw_offset(L);
    if (row) {
        row_task<P, NF, AR>(g.a, ocean, idx, inter, smem, tws, tid, h0_bar, h0_parity, nullptr, error, pub);
    } else {
        col_task<P, NF, AR, false, P::PW, true>(g.a, ocean, idx, inter, smem, tws, tid, nullptr, error, pub);
    }
}

template <int NF, int AR>
__global__ void __launch_bounds__(64 * NF, 768 / (64 * NF)) mixed_frame_kernel(MixedArgs m)
{
    constexpr int NT = 64 * NF;
    static_assert(MixPlan<5>::template threads<NF>() == NT && MixPlan<6>::template threads<NF>() == NT &&
                      MixPlan<7>::template threads<NF>() == NT && MixPlan<8>::template threads<NF>() == NT &&
                      MixPlan<9>::template threads<NF>() == NT && MixPlan<10>::template threads<NF>() == NT,
                  "every size's tasks take the same threads");
    extern __shared__ float4 smem4[];
    float2* smem = reinterpret_cast<float2*>(smem4);
    float2* tw_area = smem + mixed_data_float2<NF>();
    __shared__ unsigned s_ticket;
    __shared__ int s_ok, s_group, s_row, s_ocean, s_idx;
    __shared__ unsigned* s_publish;
    __shared__ unsigned* s_pub[2];
    unsigned r_next = 0;              // thread 0: the ticket drawn one task ahead (as frame_kernel)
    int r_have_next = 0;
    __shared__ uint64_t h0_bar;
    // The group table in shared memory: tasks index it by a runtime group,
    // which on the kernel's parameters would take a copy per thread.
    __shared__ MixedGroup s_groups[kMaxMixedGroups];
    uint32_t h0_parity = 0;
    const int tid = threadIdx.x;
    {
        const int words = static_cast<int>(m.groups * sizeof(MixedGroup) / sizeof(unsigned));
        const unsigned* src = reinterpret_cast<const unsigned*>(m.g);
        unsigned* dst = reinterpret_cast<unsigned*>(s_groups);
        for (int i = tid; i < words; i += NT) dst[i] = src[i];
    }
    static_assert(sizeof(MixedGroup) % sizeof(unsigned) == 0, "the group table copies as words");

    for (int gi = 0; gi < m.groups; ++gi) {
        const float2* src = m.g[gi].a.twiddles;
        switch (m.g[gi].log_n) {
            case 5: mix_load_twiddles<5, NF>(tw_area, src, tid, NT); break;
            case 6: mix_load_twiddles<6, NF>(tw_area, src, tid, NT); break;
            case 7: mix_load_twiddles<7, NF>(tw_area, src, tid, NT); break;
            case 8: mix_load_twiddles<8, NF>(tw_area, src, tid, NT); break;
            case 9: mix_load_twiddles<9, NF>(tw_area, src, tid, NT); break;
            default: mix_load_twiddles<10, NF>(tw_area, src, tid, NT); break;
        }
    }
    if (tid == 0) {
        h0_bar_init(&h0_bar);
        s_publish = nullptr;
        r_next = atomicAdd(m.ticket, 1u);
        r_have_next = 1;
    }
    // The persistent kernel's protocol (frame_kernel), with a group lookup:
    // take a ticket (one ahead far from the end), check the task's inputs,
    // publish the previous task here only when they are not ready (before
    // waiting), else let the task publish it once staged; hand it to the CTA.
    while (true) {
        __syncthreads();
        if (tid == 0) {
            unsigned* prev = s_publish;
            const unsigned t = r_have_next ? r_next : atomicAdd(m.ticket, 1u);
            r_have_next = 0;
            int ok = 1;
            unsigned* publish = nullptr;
            unsigned* self = nullptr;
            const unsigned* dep = nullptr;
            unsigned need = 0;
            if (t < m.total) {
                if (t + 2u * gridDim.x < m.total) {
                    r_next = atomicAdd(m.ticket, 1u);
                    r_have_next = 1;
                }
                int gi = m.groups - 1;
                while (gi > 0 && t < m.g[gi].first) --gi;
                const MixedGroup& g = m.g[gi];
                unsigned rt, ct;
                mix_tasks_per_ocean(g.log_n, rt, ct);
                const unsigned count = static_cast<unsigned>(g.count);
                const unsigned lt = t - g.first;
                bool row;
                unsigned ocean, idx;
                if (lt < rt) {
                    row = true, ocean = 0, idx = lt;
                } else {
                    const unsigned u = lt - rt, per = rt + ct, blk = u / per, off = u % per;
                    if (blk + 1 < count) {
                        row = off < rt;
                        ocean = row ? blk + 1 : blk;
                        idx = row ? off : off - rt;
                    } else {
                        row = false, ocean = count - 1, idx = off;
                    }
                }
                if (row) {
                    if (ocean >= static_cast<unsigned>(g.slots)) dep = g.cols_done + (ocean - g.slots), need = ct;
                    publish = g.rows_done + ocean;
                } else {
                    dep = g.rows_done + ocean, need = rt;
                    self = g.cols_done + ocean;
                }
                s_group = gi;
                s_row = row ? 1 : 0;
                s_ocean = static_cast<int>(ocean);
                s_idx = static_cast<int>(idx);
            }
            if (t >= m.total || !m.defer || (dep != nullptr && ld_acquire(dep) < need)) {
                if (prev != nullptr) red_release_add(prev, 1u);
                prev = nullptr;
                if (dep != nullptr) ok = wait_at_least(dep, need, m.error, m.wait_ns);
            }
            s_pub[0] = prev;
            s_pub[1] = self;
            s_publish = publish;
            s_ticket = t;
            s_ok = ok;
        }
        __syncthreads();
        if (s_ticket >= m.total || !s_ok) break;
        const MixedGroup& g = s_groups[s_group];
        const bool row = s_row != 0;
        switch (g.log_n) {
            case 5: mix_run<5, NF, AR>(g, row, s_ocean, s_idx, smem, tw_area, tid, &h0_bar, h0_parity, m.error, s_pub); break;
            case 6: mix_run<6, NF, AR>(g, row, s_ocean, s_idx, smem, tw_area, tid, &h0_bar, h0_parity, m.error, s_pub); break;
            case 7: mix_run<7, NF, AR>(g, row, s_ocean, s_idx, smem, tw_area, tid, &h0_bar, h0_parity, m.error, s_pub); break;
            case 8: mix_run<8, NF, AR>(g, row, s_ocean, s_idx, smem, tw_area, tid, &h0_bar, h0_parity, m.error, s_pub); break;
            case 9: mix_run<9, NF, AR>(g, row, s_ocean, s_idx, smem, tw_area, tid, &h0_bar, h0_parity, m.error, s_pub); break;
            default: mix_run<10, NF, AR>(g, row, s_ocean, s_idx, smem, tw_area, tid, &h0_bar, h0_parity, m.error, s_pub); break;
        }
        if (row) h0_parity ^= 1u;
    }
}

template <int NF, int AR>
struct MixedLaunch {
    static constexpr int threads() { return 64 * NF; }
    static cudaError_t prepare()
    {
        return cudaFuncSetAttribute(mixed_frame_kernel<NF, AR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(mixed_smem_bytes(NF)));
    }
    static int blocks_per_sm()
    {
        if (prepare() != cudaSuccess) return 0;
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, mixed_frame_kernel<NF, AR>, threads(),
                                                          mixed_smem_bytes(NF)) != cudaSuccess)
            return 0;
        return n;
    }
    static cudaError_t launch(const MixedArgs& m, int grid, cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess) return e;
        mixed_frame_kernel<NF, AR><<<grid, threads(), mixed_smem_bytes(NF), st>>>(m);
        return cudaGetLastError();
    }
};

// Bounded waits that nothing completes, each of which must give up after
// limit_ns and set its error word: the queue's wait on a counter nothing
// increments (wait_at_least), and the h0 copy's wait on an mbarrier no
// thread arrives at and no copy targets (h0_rows_wait).
__global__ void wait_probe_kernel(const unsigned* counter, unsigned target, unsigned* error,
                                  unsigned* bar_error, unsigned long long limit_ns)
{
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) h0_bar_init(&bar);
    __syncthreads();
    if (threadIdx.x == 0) {
        wait_at_least(counter, target, error, limit_ns);
        h0_rows_wait(&bar, 0u, bar_error, limit_ns);
    }
}

__global__ void foam_step_kernel(int n, int count, const float4* __restrict__ disp,
                                 const float4* __restrict__ vel, const float* __restrict__ cur,
                                 float* __restrict__ next, float dt, float decay, float gain,
                                 float scale, float drift_x, float drift_z, float inv_cell)
{
    const uint64_t cells = static_cast<uint64_t>(n) * n;
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cells * count) return;
    const uint64_t o = i / cells;
    const uint64_t c = i % cells;
    const int z = static_cast<int>(c / n), x = static_cast<int>(c % n);
    const float4 v = vel[i];
    const float src = disp[i].w;
    next[i] = foam_cell(cur + o * cells, n, x, z, v.x, v.z, src, dt, decay, gain, scale, drift_x,
                        drift_z, inv_cell);
}

// ---------------------------------------------------------------------------
// World queries (src/ocean.cpp:322-452; sample_one in query_device.cuh)
// ---------------------------------------------------------------------------
using qdev::sample_one;

__global__ void sample_kernel(int n, float inv_cell, const float4* __restrict__ disp,
                              const float4* __restrict__ normal, const float4* __restrict__ vel,
                              const float2* __restrict__ xz, uint64_t count,
                              SurfaceEx* __restrict__ out)
{
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    out[i] = sample_one(n, inv_cell, disp, normal, vel, xz[i], 4, 0.0f);
}

// Summed surface of several cascade levels (src/cascade.cpp:82-153): height,
// offsets and velocity add exactly; normals add then renormalise; foam
// combines as 1 - prod(1 - foam_i). Levels are visited in order, so the float
// sums round as the reference's loop does.
__global__ void cascade_sample_kernel(CascadeLevels lv, const float2* __restrict__ xz,
                                      uint64_t count, SurfaceEx* __restrict__ out, int iters,
                                      float tol)
{
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float2 p = xz[i];
    float height = 0.0f, offset_x = 0.0f, offset_z = 0.0f;
    float normal_x = 0.0f, normal_y = 0.0f, normal_z = 0.0f;
    float transparency = 1.0f;
    float vx = 0.0f, vy = 0.0f, vz = 0.0f;
    for (int l = 0; l < lv.count; ++l) {
        const LevelView& L = lv.level[l];
        const SurfaceEx s = sample_one(L.n, L.inv_cell, L.disp, L.normal, L.velocity, p, iters, tol);
        height += s.height;
        offset_x += s.offset_x;
        offset_z += s.offset_z;
        normal_x += s.normal_x;
        normal_y += s.normal_y;
        normal_z += s.normal_z;
        vx += s.velocity_x;
        vy += s.velocity_y;
        vz += s.velocity_z;
        transparency *= (1.0f - s.foam);
    }
    SurfaceEx o;
    o.height = height;
    o.offset_x = offset_x;
    o.offset_z = offset_z;
    o.foam = 1.0f - transparency;
    o.velocity_x = vx;
    o.velocity_y = vy;
    o.velocity_z = vz;
    const float len2 = normal_x * normal_x + normal_y * normal_y + normal_z * normal_z;
    if (len2 > 0.0f) {
        const float inv = 1.0f / sqrtf(len2);
        o.normal_x = normal_x * inv;
        o.normal_y = normal_y * inv;
        o.normal_z = normal_z * inv;
    } else {
        o.normal_x = 0.0f;
        o.normal_y = 1.0f;
        o.normal_z = 0.0f;
    }
    out[i] = o;
}

// ---------------------------------------------------------------------------
// Launch helpers: compile-time dispatch over (log N, fields, form, foam).
// ---------------------------------------------------------------------------
template <int LOG_N, int NF>
constexpr size_t row_smem_bytes()
{
    using P = ChunkPlan<LOG_N>;
    return sizeof(float2) * (P::ROWS * NF * P::SEQF2 + P::H0ROWS * P::N + P::TWF2);
}
template <int LOG_N, int NF>
constexpr size_t col_smem_bytes()
{
    using S = Shape<LOG_N>;
    using P = ChunkPlan<LOG_N>;
    return sizeof(float2) *
           (NF * S::W * P::SEQF2 + col_shift_f2_of<P, NF, S::W>() + foam_window_f2<LOG_N, S::W>() + P::TWF2);
}

template <int LOG_N, int NF, int AR>
cudaError_t row_launch(const FrameArgs& a, cudaStream_t st)
{
    using P = ChunkPlan<LOG_N>;
    constexpr size_t smem = row_smem_bytes<LOG_N, NF>();
    auto k = row_pass_kernel<LOG_N, NF, AR>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    dim3 grid(P::RT, a.chunk);
    k<<<grid, P::template threads<NF>(), smem, st>>>(a);
    return cudaGetLastError();
}

template <int LOG_N, int NF, int AR, bool FOAM>
cudaError_t col_launch(const FrameArgs& a, cudaStream_t st)
{
    using S = Shape<LOG_N>;
    constexpr size_t smem = col_smem_bytes<LOG_N, NF>();
    auto k = col_pass_kernel<LOG_N, NF, AR, FOAM>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    dim3 grid(S::N / S::W, a.chunk);
    k<<<grid, NF * S::W * S::G, smem, st>>>(a);
    return cudaGetLastError();
}

template <class P, int NF>
constexpr size_t frame_smem_bytes()
{
    if (P::TC) return frame_engine_offset<P::LOG_N, NF>() + TcEngineOf<P::LOG_N, NF>::Lay::kSmemBytes;
    return sizeof(float2) * (frame_data_float2<P, NF>() + P::TWF2);
}

template <int LOG_N, int NF, int AR, bool FOAM, bool TC = false, int V = 0>
struct FrameLaunch {
    using P = PlanOf<LOG_N, V, TC>;
    using Eng = TcEngineOf<LOG_N, NF>;
    static constexpr int threads() { return P::template threads<NF>(); }
    static constexpr size_t smem() { return frame_smem_bytes<P, NF>(); }
    static_assert(frame_smem_bytes<P, NF>() <= 227 * 1024, "a task's shared memory fits one CTA");

    static cudaError_t prepare()
    {
        return cudaFuncSetAttribute(frame_kernel<P, NF, AR, FOAM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(smem()));
    }

    static int blocks_per_sm()
    {
        if (prepare() != cudaSuccess) return 0;
        int n = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, frame_kernel<P, NF, AR, FOAM>, threads(), smem()) !=
            cudaSuccess)
            return 0;
        // The tensor-core engine's tensor memory bounds its residency.
        if (TC && n * Eng::Lay::kTmemCols > 512) n = 512 / Eng::Lay::kTmemCols;
        return n;
    }

    static cudaError_t launch(const FrameArgs& a, const QueueArgs& q, int grid, cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess) return e;
        if (TC) {
            // Every resident CTA must obtain its tensor memory without waiting.
            int n = 0;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, frame_kernel<P, NF, AR, FOAM>, threads(), smem());
            if (e != cudaSuccess) return e;
            if (n * Eng::Lay::kTmemCols > 512) return cudaErrorInvalidConfiguration;
        }
        frame_kernel<P, NF, AR, FOAM><<<grid, threads(), smem(), st>>>(a, q);
        return cudaGetLastError();
    }
};

// The arithmetic `ar` (kArExact, kArFast, kArPrecise) as a compile-time
// constant for `fn`.
template <typename Fn>
auto with_arith(int ar, Fn&& fn)
{
    if (ar == kArFast) return fn(std::integral_constant<int, kArFast>{});
    if (ar == kArPrecise) return fn(std::integral_constant<int, kArPrecise>{});
    return fn(std::integral_constant<int, kArExact>{});
}

// form: an ocean_fft_form (exact, fast, tensor cores at N = 64 to 512, precise).
template <int LOG_N, int V, typename Fn>
auto frame_variant_plan(int nf, int ar, bool foam, Fn&& fn)
{
    return with_arith(ar, [&](auto A) {
        constexpr int AR = decltype(A)::value;
        if (nf == 4) return fn(FrameLaunch<LOG_N, 4, AR, false, false, V>{});
        if (foam) return fn(FrameLaunch<LOG_N, 6, AR, true, false, V>{});
        return fn(FrameLaunch<LOG_N, 6, AR, false, false, V>{});
    });
}

template <int LOG_N, typename Fn>
auto frame_variant(int nf, int form, bool foam, int plan, Fn&& fn)
{
    if constexpr (has_tc_form<LOG_N>()) {
        if (form == 2) {
            if (nf == 4) return fn(FrameLaunch<LOG_N, 4, kArExact, false, true>{});
            if (foam) return fn(FrameLaunch<LOG_N, 6, kArExact, true, true>{});
            return fn(FrameLaunch<LOG_N, 6, kArExact, false, true>{});
        }
    }
    const int ar = arith_of_form(form);
    if constexpr (frame_plan_count<LOG_N>(false) > 1) {
        if (plan == 1) return frame_variant_plan<LOG_N, 1>(nf, ar, foam, fn);
    }
    return frame_variant_plan<LOG_N, 0>(nf, ar, foam, fn);
}

template <typename Fn>
auto frame_dispatch(int log_n, int nf, int form, bool foam, int plan, Fn&& fn)
{
    switch (log_n) {
        case 4: return frame_variant<4>(nf, form, foam, plan, fn);
        case 5: return frame_variant<5>(nf, form, foam, plan, fn);
        case 6: return frame_variant<6>(nf, form, foam, plan, fn);
        case 7: return frame_variant<7>(nf, form, foam, plan, fn);
        case 8: return frame_variant<8>(nf, form, foam, plan, fn);
        case 9: return frame_variant<9>(nf, form, foam, plan, fn);
        default: return frame_variant<10>(nf, form, foam, plan, fn);
    }
}

template <int LOG_N>
cudaError_t row_dispatch_n(int nf, int ar, const FrameArgs& a, cudaStream_t st)
{
    return with_arith(ar, [&](auto A) {
        constexpr int AR = decltype(A)::value;
        return nf == 4 ? row_launch<LOG_N, 4, AR>(a, st) : row_launch<LOG_N, 6, AR>(a, st);
    });
}

template <int LOG_N>
cudaError_t col_dispatch_n(int nf, int ar, bool foam, const FrameArgs& a, cudaStream_t st)
{
    return with_arith(ar, [&](auto A) {
        constexpr int AR = decltype(A)::value;
        if (nf == 4) return col_launch<LOG_N, 4, AR, false>(a, st);
        return foam ? col_launch<LOG_N, 6, AR, true>(a, st) : col_launch<LOG_N, 6, AR, false>(a, st);
    });
}

}  // namespace

static_assert(frame_plan_count<8>(false) <= kMaxFramePlans && frame_plan_count<9>(false) <= kMaxFramePlans &&
                  frame_plan_count<10>(false) <= kMaxFramePlans,
              "the host sizes its per-plan tables by kMaxFramePlans");

int frame_plan_count(int log_n, int form)
{
    if (log_n < 4 || log_n > 10) return 0;
    return (form != 2 && log_n >= 8) ? 2 : 1;
}

int frame_blocks_per_sm(int log_n, int nf, int form, bool fuse_foam, int plan)
{
    if (log_n < 4 || log_n > 10) return 0;
    if (form == 2 && (log_n < 6 || log_n > 9)) return 0;
    if (plan < 0 || plan >= frame_plan_count(log_n, form)) return 0;
    return frame_dispatch(log_n, nf, form, fuse_foam, plan, [](auto L) { return decltype(L)::blocks_per_sm(); });
}

cudaError_t launch_frame(int log_n, int nf, int form, bool fuse_foam, const FrameArgs& a,
                         const QueueArgs& q, int grid, cudaStream_t st, int plan)
{
    if (log_n < 4 || log_n > 10) return cudaErrorInvalidValue;
    if (form == 2 && (log_n < 6 || log_n > 9)) return cudaErrorInvalidValue;
    if (plan < 0 || plan >= frame_plan_count(log_n, form)) return cudaErrorInvalidValue;
    return frame_dispatch(log_n, nf, form, fuse_foam, plan,
                          [&](auto L) { return decltype(L)::launch(a, q, grid, st); });
}


bool mixed_size_ok(int log_n) { return log_n >= kMixMinLog && log_n <= kMixMaxLog; }

uint32_t mixed_tasks(int log_n, int count)
{
    unsigned rt = 0, ct = 0;
    mix_tasks_per_ocean(log_n, rt, ct);
    return static_cast<uint32_t>(count) * (rt + ct);
}

int mixed_blocks_per_sm(int nf, int ar)
{
    return with_arith(ar, [&](auto A) {
        constexpr int AR = decltype(A)::value;
        return nf == 4 ? MixedLaunch<4, AR>::blocks_per_sm() : MixedLaunch<6, AR>::blocks_per_sm();
    });
}

cudaError_t launch_mixed_frame(int nf, int ar, const MixedArgs& m, int grid, cudaStream_t st)
{
    if (m.groups < 1 || m.groups > kMaxMixedGroups) return cudaErrorInvalidValue;
    for (int g = 0; g < m.groups; ++g)
        if (!mixed_size_ok(m.g[g].log_n) || m.g[g].count < 1 || m.g[g].slots < 1)
            return cudaErrorInvalidValue;
    return with_arith(ar, [&](auto A) {
        constexpr int AR = decltype(A)::value;
        return nf == 4 ? MixedLaunch<4, AR>::launch(m, grid, st) : MixedLaunch<6, AR>::launch(m, grid, st);
    });
}

cudaError_t launch_wait_probe(const unsigned* counter, unsigned target, unsigned* error, unsigned* bar_error,
                              unsigned long long limit_ns, cudaStream_t stream)
{
    wait_probe_kernel<<<1, 32, 0, stream>>>(counter, target, error, bar_error, limit_ns);
    return cudaGetLastError();
}

cudaError_t launch_row_pass(int log_n, int nf, int ar, const FrameArgs& a, cudaStream_t st)
{
    switch (log_n) {
        case 4: return row_dispatch_n<4>(nf, ar, a, st);
        case 5: return row_dispatch_n<5>(nf, ar, a, st);
        case 6: return row_dispatch_n<6>(nf, ar, a, st);
        case 7: return row_dispatch_n<7>(nf, ar, a, st);
        case 8: return row_dispatch_n<8>(nf, ar, a, st);
        case 9: return row_dispatch_n<9>(nf, ar, a, st);
        case 10: return row_dispatch_n<10>(nf, ar, a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_col_pass(int log_n, int nf, int ar, bool fuse_foam, const FrameArgs& a,
                            cudaStream_t st)
{
    switch (log_n) {
        case 4: return col_dispatch_n<4>(nf, ar, fuse_foam, a, st);
        case 5: return col_dispatch_n<5>(nf, ar, fuse_foam, a, st);
        case 6: return col_dispatch_n<6>(nf, ar, fuse_foam, a, st);
        case 7: return col_dispatch_n<7>(nf, ar, fuse_foam, a, st);
        case 8: return col_dispatch_n<8>(nf, ar, fuse_foam, a, st);
        case 9: return col_dispatch_n<9>(nf, ar, fuse_foam, a, st);
        case 10: return col_dispatch_n<10>(nf, ar, fuse_foam, a, st);
        default: return cudaErrorInvalidValue;
    }
}

size_t row_pass_smem(int log_n, int nf)
{
    switch (log_n) {
        case 4: return nf == 4 ? row_smem_bytes<4, 4>() : row_smem_bytes<4, 6>();
        case 5: return nf == 4 ? row_smem_bytes<5, 4>() : row_smem_bytes<5, 6>();
        case 6: return nf == 4 ? row_smem_bytes<6, 4>() : row_smem_bytes<6, 6>();
        case 7: return nf == 4 ? row_smem_bytes<7, 4>() : row_smem_bytes<7, 6>();
        case 8: return nf == 4 ? row_smem_bytes<8, 4>() : row_smem_bytes<8, 6>();
        case 9: return nf == 4 ? row_smem_bytes<9, 4>() : row_smem_bytes<9, 6>();
        case 10: return nf == 4 ? row_smem_bytes<10, 4>() : row_smem_bytes<10, 6>();
        default: return 0;
    }
}

size_t col_pass_smem(int log_n, int nf)
{
    switch (log_n) {
        case 4: return nf == 4 ? col_smem_bytes<4, 4>() : col_smem_bytes<4, 6>();
        case 5: return nf == 4 ? col_smem_bytes<5, 4>() : col_smem_bytes<5, 6>();
        case 6: return nf == 4 ? col_smem_bytes<6, 4>() : col_smem_bytes<6, 6>();
        case 7: return nf == 4 ? col_smem_bytes<7, 4>() : col_smem_bytes<7, 6>();
        case 8: return nf == 4 ? col_smem_bytes<8, 4>() : col_smem_bytes<8, 6>();
        case 9: return nf == 4 ? col_smem_bytes<9, 4>() : col_smem_bytes<9, 6>();
        case 10: return nf == 4 ? col_smem_bytes<10, 4>() : col_smem_bytes<10, 6>();
        default: return 0;
    }
}

cudaError_t launch_foam_step(int n, int count, const float4* disp, const float4* velocity,
                             const float* cur, float* next, float dt, float decay, float gain,
                             float scale, float drift_x, float drift_z, float inv_cell,
                             cudaStream_t stream)
{
    const uint64_t total = static_cast<uint64_t>(n) * n * count;
    const unsigned blocks = static_cast<unsigned>((total + 255) / 256);
    foam_step_kernel<<<blocks, 256, 0, stream>>>(n, count, disp, velocity, cur, next, dt, decay,
                                                 gain, scale, drift_x, drift_z, inv_cell);
    return cudaGetLastError();
}

cudaError_t launch_cascade_sample(const CascadeLevels& levels, const float2* xz, uint64_t count,
                                  SurfaceEx* out, int iters, float tol, cudaStream_t stream)
{
    if (count == 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
    cascade_sample_kernel<<<blocks, 256, 0, stream>>>(levels, xz, count, out, iters, tol);
    return cudaGetLastError();
}

cudaError_t launch_sample(int n, float inv_cell, const float4* disp, const float4* normal,
                          const float4* velocity, const float2* xz, uint64_t count,
                          SurfaceEx* out, cudaStream_t stream)
{
    if (count == 0) return cudaSuccess;
    const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
    sample_kernel<<<blocks, 256, 0, stream>>>(n, inv_cell, disp, normal, velocity, xz, count, out);
    return cudaGetLastError();
}

}  // namespace ocean_b200
