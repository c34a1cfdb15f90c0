// oceanlib-b200: the frame at N = 2048 and 4096.
//
// The persistent frame kernel (frame.cu) keeps every field of a row pair, or
// of a strip of columns, in one CTA's shared memory. Above N = 1024 that no
// longer fits: six 4096-point sequences alone are 209 KB. These sizes (the
// reference accepts N up to 4096, src/ocean.cpp:28-59) run three passes per
// chunk of oceans instead, through a field-major intermediate
// inter[ocean][field][y][x]:
//
//   rows      row y per task: evolve the row's cells once for all NF fields
//             (src/core/evolve.cpp:28-184; h0(-k) read from the mirrored row
//             in global memory, which the neighbouring task has just read),
//             field pair 0 into shared memory and the other pairs straight
//             into their rows of the intermediate; transform pair 0, then
//             each other pair from its row (just written, so read from L2)
//             back in place.
//   columns   four columns of one field per task, transformed in place.
//   finalize  one thread per cell: the NF fields to the RGBA32F outputs
//             (src/core/evolve.cpp:186-327) and, with persistent foam, the
//             first foam substep (src/foam.cpp:89-139).
//
// A sequence spans N/16 lanes holding 16 values each (4-stage blocks, three
// passes through shared memory at both sizes), i.e. several warps, which
// synchronise with the CTA barrier. Evolve, butterflies, twiddles, finalize
// and foam are the persistent kernel's own functions (frame_cells.cuh,
// ocean_device.cuh), so these sizes match the reference bit for bit too.
// A CTA runs several tasks so that each twiddle table load serves them all.
#include "frame_cells.cuh"
#include "ocean_device.cuh"
#include "spectrum.h"

#include <type_traits>

namespace ocean_b200 {
namespace {

template <int LOG_N>
struct Large {
    static constexpr int N = 1 << LOG_N;
    static constexpr int G = N / 16;               // lanes per sequence
    static constexpr int SEQ = padded_len(N) + 4;  // sequence stride (float2)
    static constexpr int W = 4;                    // columns per column task
    static constexpr int ROW_T = 2 * G;            // threads: two sequences
    static constexpr int COL_T = W * G;            // threads: W sequences
    static constexpr int ROW_TASKS = 2;            // rows per row CTA (a row and its mirror)
    // Resident row CTAs per SM the registers are capped for: two at N = 4096
    // (512 threads, 102 KB each; 7% faster than one), three at 2048 (256
    // threads, 51 KB each).
    static constexpr int ROW_BLOCKS = LOG_N >= 12 ? 2 : 3;
    static constexpr int COL_TASKS = 2;            // tasks per column CTA
    static constexpr size_t ROW_SMEM = sizeof(float2) * (2 * SEQ + N - 1);
    static constexpr size_t COL_SMEM = sizeof(float2) * (W * SEQ + N - 1);
    static_assert(COL_SMEM <= 227 * 1024, "a column CTA fits in shared memory");
};

template <int LOG_N, int NF, int AR>
__global__ void __launch_bounds__(Large<LOG_N>::ROW_T, Large<LOG_N>::ROW_BLOCKS)
large_row_kernel(FrameArgs a)
{
    using S = Large<LOG_N>;
    constexpr int N = S::N, NT = S::ROW_T, SEQ = S::SEQ, G = S::G;
    constexpr int NG = NF / 2;  // field pairs per row
    extern __shared__ float4 smem4[];
    float2* data = reinterpret_cast<float2*>(smem4);  // the task's two sequences
    float2* tws = data + 2 * SEQ;
    const int tid = threadIdx.x;
    const int o = blockIdx.y;
    const int ocean = a.ocean_base + o;
    const OceanConsts cst = a.consts[ocean];
    const size_t cells = static_cast<size_t>(N) * N;
    const float2* h0 = a.h0 + static_cast<size_t>(ocean) * cells;
    const float2* geom = a.omega_kinv + static_cast<size_t>(cst.geom) * cells;
    const float* kvec = a.kvec + static_cast<size_t>(cst.geom) * N;
    const double top = a.t_over_2pi[ocean];
    float2* inter = a.inter + static_cast<size_t>(o) * NF * cells;
    for (int i = tid; i < N - 1; i += NT) tws[i] = __ldg(&a.twiddles[i]);

#pragma unroll 1
    for (int k = 0; k < S::ROW_TASKS; ++k) {
        // Task t: row slot t, whose two members (p, N - p), or (0, N/2) for
        // p = 0, are each other's h0(-k) rows, so consecutive tasks reuse
        // what the L2 just fetched.
        const int j = blockIdx.x * S::ROW_TASKS + k;
        const int p = j >> 1, r = j & 1;
        const int y = p == 0 ? (r ? N / 2 : 0) : (r ? N - p : p);
        const int my = (N - y) & (N - 1);
        const float kz = __ldg(&kvec[y]);
        const size_t row = static_cast<size_t>(y) * N;
        __syncthreads();  // the twiddles are complete; the last task's reads are done
        // Evolve once: pair 0 to shared memory, pairs 1.. to their rows of
        // the intermediate (coalesced float2 stores, read back below).
        for (int x = tid; x < N; x += NT) {
            const float2 av = __ldg(&h0[row + x]);
            const float2 bm = __ldg(&h0[static_cast<size_t>(my) * N + ((N - x) & (N - 1))]);
            float2 pv[NF];
            evolve_cell<NF>(av, bm, __ldg(&geom[row + x]), __ldg(&kvec[x]), kz, top, pv);
            data[pad_idx(x)] = pv[0];
            data[SEQ + pad_idx(x)] = pv[1];
#pragma unroll
            for (int f = 2; f < NF; ++f) inter[static_cast<size_t>(f) * cells + row + x] = pv[f];
        }
#pragma unroll 1
        for (int g = 0; g < NG; ++g) {
            if (g > 0) {
                __syncthreads();  // the last pair's outputs are read out of shared memory
                // This CTA wrote the pair's row above; the barrier makes its
                // stores visible, and the loads go to L2.
                for (int i = tid; i < 2 * N; i += NT) {
                    const int s = i >> LOG_N, x = i & (N - 1);
                    data[s * SEQ + pad_idx(x)] = __ldcg(&inter[static_cast<size_t>(2 * g + s) * cells + row + x]);
                }
            }
            __syncthreads();
            fft_sequence<LOG_N, G, AR>(data + (tid / G) * SEQ, tws, tid % G);  // ends with a CTA barrier
            float2* out = inter + static_cast<size_t>(2 * g) * cells + row;
            for (int i = tid; i < 2 * N; i += NT) {
                const int s = i >> LOG_N, x = i & (N - 1);
                out[static_cast<size_t>(s) * cells + x] = data[s * SEQ + pad_idx(x)];
            }
        }
    }
}

template <int LOG_N, int AR>
__global__ void __launch_bounds__(Large<LOG_N>::COL_T) large_col_kernel(FrameArgs a, int nf)
{
    using S = Large<LOG_N>;
    constexpr int N = S::N, NT = S::COL_T, SEQ = S::SEQ, G = S::G, W = S::W;
    constexpr int H = W / 2;  // float4 (two columns) per row of a strip
    extern __shared__ float4 smem4[];
    float2* data = reinterpret_cast<float2*>(smem4);  // the task's W sequences
    float2* tws = data + W * SEQ;
    const int tid = threadIdx.x;
    const int o = blockIdx.y;
    const size_t cells = static_cast<size_t>(N) * N;
    for (int i = tid; i < N - 1; i += NT) tws[i] = __ldg(&a.twiddles[i]);

#pragma unroll 1
    for (int k = 0; k < S::COL_TASKS; ++k) {
        // Task t: strip t % (N / W) of field t / (N / W); neighbouring CTAs
        // take neighbouring strips, which share the rows' cache lines.
        const int t = blockIdx.x * S::COL_TASKS + k;
        const int f = t / (N / W);
        const int x0 = (t % (N / W)) * W;
        float2* plane = a.inter + (static_cast<size_t>(o) * nf + f) * cells;
        __syncthreads();  // the twiddles are complete; the last task's reads are done
        for (int i = tid; i < N * H; i += NT) {
            const int y = i / H, h = i % H;
            const float4 v = reinterpret_cast<const float4*>(plane + static_cast<size_t>(y) * N + x0)[h];
            data[(2 * h) * SEQ + pad_idx(y)] = make_float2(v.x, v.y);
            data[(2 * h + 1) * SEQ + pad_idx(y)] = make_float2(v.z, v.w);
        }
        __syncthreads();
        fft_sequence<LOG_N, G, AR>(data + (tid / G) * SEQ, tws, tid % G);  // ends with a CTA barrier
        for (int i = tid; i < N * H; i += NT) {
            const int y = i / H, h = i % H;
            const float2 u = data[(2 * h) * SEQ + pad_idx(y)];
            const float2 v = data[(2 * h + 1) * SEQ + pad_idx(y)];
            reinterpret_cast<float4*>(plane + static_cast<size_t>(y) * N + x0)[h] = make_float4(u.x, u.y, v.x, v.y);
        }
    }
}

template <int NF, bool FOAM>
__global__ void __launch_bounds__(256) large_finalize_kernel(FrameArgs a, int log_n)
{
    const int n = 1 << log_n;
    const size_t cells = static_cast<size_t>(n) * n;
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cells) return;
    const int o = blockIdx.y;
    const int ocean = a.ocean_base + o;
    const OceanConsts cst = a.consts[ocean];
    const float2* in = a.inter + static_cast<size_t>(o) * NF * cells + i;
    float2 f[NF];
#pragma unroll
    for (int k = 0; k < NF; ++k) f[k] = __ldcs(in + k * cells);
    const CellOut c = finalize_cell(f[0], f[1], f[2], f[3], cst.lambda, cst.foam_threshold, cst.inv_threshold);
    const size_t idx = static_cast<size_t>(ocean) * cells + i;
    __stcs(&a.disp[idx], c.disp);
    __stcs(&a.normal[idx], c.normal);
    if constexpr (NF == 6) {
        __stcs(&a.velocity[idx], make_float4(f[4].x, f[4].y, f[5].x, 0.0f));
        if constexpr (FOAM) {
            const int x = static_cast<int>(i & (n - 1));
            const int z = static_cast<int>(i >> log_n);
            __stcs(&a.foam_next[idx],
                   foam_cell(a.foam_cur + static_cast<size_t>(ocean) * cells, n, x, z, f[4].x, f[5].x, c.disp.w,
                             a.foam_dt, a.foam_decay, a.foam_gain, a.foam_scale, a.foam_drift_x, a.foam_drift_z,
                             a.foam_inv_cell));
        }
    }
}

template <int LOG_N, int NF, int AR>
cudaError_t rows_launch(const FrameArgs& a, cudaStream_t st)
{
    using S = Large<LOG_N>;
    auto k = large_row_kernel<LOG_N, NF, AR>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(S::ROW_SMEM));
    if (e != cudaSuccess) return e;
    static_assert(S::N % S::ROW_TASKS == 0, "row tasks divide evenly among CTAs");
    const dim3 grid(S::N / S::ROW_TASKS, a.chunk);
    k<<<grid, S::ROW_T, S::ROW_SMEM, st>>>(a);
    return cudaGetLastError();
}

template <int LOG_N, int AR>
cudaError_t cols_launch(int nf, const FrameArgs& a, cudaStream_t st)
{
    using S = Large<LOG_N>;
    auto k = large_col_kernel<LOG_N, AR>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(S::COL_SMEM));
    if (e != cudaSuccess) return e;
    static_assert((S::N / S::W) % S::COL_TASKS == 0, "column tasks divide evenly among CTAs");
    const dim3 grid((S::N / S::W) * nf / S::COL_TASKS, a.chunk);
    k<<<grid, S::COL_T, S::COL_SMEM, st>>>(a, nf);
    return cudaGetLastError();
}

// The arithmetic `ar` (kArExact, kArFast, kArPrecise) as a compile-time
// constant for `fn`.
template <typename Fn>
cudaError_t with_arith(int ar, Fn&& fn)
{
    if (ar == kArFast) return fn(std::integral_constant<int, kArFast>{});
    if (ar == kArPrecise) return fn(std::integral_constant<int, kArPrecise>{});
    return fn(std::integral_constant<int, kArExact>{});
}

template <int LOG_N>
cudaError_t rows_n(int nf, int ar, const FrameArgs& a, cudaStream_t st)
{
    return with_arith(ar, [&](auto A) {
        constexpr int AR = decltype(A)::value;
        return nf == 4 ? rows_launch<LOG_N, 4, AR>(a, st) : rows_launch<LOG_N, 6, AR>(a, st);
    });
}

}  // namespace

cudaError_t launch_large_rows(int log_n, int nf, int ar, const FrameArgs& a, cudaStream_t st)
{
    if (nf != 4 && nf != 6) return cudaErrorInvalidValue;
    switch (log_n) {
        case 11: return rows_n<11>(nf, ar, a, st);
        case 12: return rows_n<12>(nf, ar, a, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_large_cols(int log_n, int nf, int ar, const FrameArgs& a, cudaStream_t st)
{
    if (nf != 4 && nf != 6) return cudaErrorInvalidValue;
    return with_arith(ar, [&](auto A) {
        constexpr int AR = decltype(A)::value;
        switch (log_n) {
            case 11: return cols_launch<11, AR>(nf, a, st);
            case 12: return cols_launch<12, AR>(nf, a, st);
            default: return cudaErrorInvalidValue;
        }
    });
}

cudaError_t launch_large_finalize(int log_n, int nf, bool fuse_foam, const FrameArgs& a, cudaStream_t st)
{
    if (log_n != 11 && log_n != 12) return cudaErrorInvalidValue;
    if (fuse_foam && nf != 6) return cudaErrorInvalidValue;
    const size_t cells = size_t(1) << (2 * log_n);
    const dim3 grid(static_cast<unsigned>(cells / 256), a.chunk);
    if (nf == 4) {
        large_finalize_kernel<4, false><<<grid, 256, 0, st>>>(a, log_n);
    } else if (nf == 6) {
        if (fuse_foam) {
            large_finalize_kernel<6, true><<<grid, 256, 0, st>>>(a, log_n);
        } else {
            large_finalize_kernel<6, false><<<grid, 256, 0, st>>>(a, log_n);
        }
    } else {
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace ocean_b200
