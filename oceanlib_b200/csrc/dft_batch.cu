// oceanlib-b200: batched 1-D inverse DFTs of device sequences in each form
// (ocean_dft_batch): the radix-2 Stockham FFT (exact, bit-identical to
// src/core/fft.cpp), its fast and precise variants, and the tensor-core DFT (tc_dft.cuh at
// N = 512, tc_dft_small.cuh at N = 64, 128 and 256).
// The frame kernel runs the same code on its rows and columns; this entry
// point isolates the transform for accuracy checks against FP64.
#include "ocean_device.cuh"
#include "spectrum.h"
#include "tc_dft.cuh"
#include "tc_dft_small.cuh"

namespace ocean_b200 {
namespace {

constexpr int kSeqPad = 4;  // float2 between sequences in shared memory

// CTAs take chunks of 8 sequences in turn (several engine calls per CTA).
template <int LOG_N, int AR>
__global__ void __launch_bounds__(8 * lanes_for(LOG_N))
dft_fp32_kernel(const float2* __restrict__ in, float2* __restrict__ out, int count,
                const float2* __restrict__ tw)
{
    constexpr int N = 1 << LOG_N, G = lanes_for(LOG_N), NT = 8 * G;
    constexpr int SEQ = padded_len(N) + kSeqPad;
    extern __shared__ float4 smem4[];
    float2* data = reinterpret_cast<float2*>(smem4);
    float2* tws = data + 8 * SEQ;
    const int tid = threadIdx.x;
    for (int i = tid; i < N - 1; i += NT) tws[i] = tw[i];
    for (int base = blockIdx.x * 8; base < count; base += gridDim.x * 8) {
        const int k = min(8, count - base);
        __syncthreads();
        for (int i = tid; i < 8 * N; i += NT) {
            const int s = i >> LOG_N, n = i & (N - 1);
            data[s * SEQ + pad_idx(n)] = s < k ? in[static_cast<size_t>(base + s) * N + n] : make_float2(0.0f, 0.0f);
        }
        __syncthreads();
        fft_sequence<LOG_N, G, AR>(data + (tid / G) * SEQ, tws, tid % G);
        __syncthreads();
        for (int i = tid; i < k * N; i += NT) {
            const int s = i >> LOG_N, n = i & (N - 1);
            out[static_cast<size_t>(base + s) * N + n] = data[s * SEQ + pad_idx(n)];
        }
    }
}

using BatchEngine = tc::Engine<8>;  // 8 sequences per engine call

__global__ void __launch_bounds__(BatchEngine::Lay::kThreads)
dft_tc512_kernel(const float2* __restrict__ in, float2* __restrict__ out, int count,
                 const float2* __restrict__ tw, unsigned* error)
{
    constexpr int N = 512, NT = BatchEngine::Lay::kThreads;
    constexpr int SEQ = padded_len(N) + kSeqPad;
    static_assert(SEQ * 2 >= 16 * tc::kZStride, "a sequence's space must hold its staged stage-3 rows");
    extern __shared__ float4 smem4[];
    float2* data = reinterpret_cast<float2*>(smem4);
    float2* tws = data + 8 * SEQ;
    unsigned char* eng_smem = reinterpret_cast<unsigned char*>(smem4) +
                              ((8 * SEQ + N) * sizeof(float2) + 127) / 128 * 128;
    const int tid = threadIdx.x;
    for (int i = tid; i < N - 1; i += NT) tws[i] = tw[i];
    BatchEngine eng{eng_smem, 0};
    eng.init(tid, NT, tw);
    for (int base = blockIdx.x * 8; base < count; base += gridDim.x * 8) {
        const int k = min(8, count - base);
        __syncthreads();
        for (int i = tid; i < k * N; i += NT) {
            const int s = i >> 9, n = i & (N - 1);
            data[s * SEQ + pad_idx(n)] = in[static_cast<size_t>(base + s) * N + n];
        }
        __syncthreads();
        eng.dft512(data, SEQ, k, tid, error);
        for (int i = tid; i < k * N; i += NT) {
            const int s = i >> 9, n = i & (N - 1);
            out[static_cast<size_t>(base + s) * N + n] = data[s * SEQ + pad_idx(n)];
        }
    }
    eng.release(tid);
}

// N = 64, 128, 256: chunks of 6144 / N sequences (384 threads, one CTA per
// SM for its tensor memory).
template <int LOG_N>
using SmallBatchEngine = tc::SmallEngine<LOG_N, (6144 >> LOG_N)>;

template <int LOG_N>
__host__ __device__ constexpr size_t tc_small_data_bytes()
{
    return ((6144 >> LOG_N) * (padded_len(1 << LOG_N) + kSeqPad) * sizeof(float2) + 127) / 128 * 128;
}

template <int LOG_N>
__global__ void __launch_bounds__(SmallBatchEngine<LOG_N>::Lay::kThreads)
dft_tc_small_kernel(const float2* __restrict__ in, float2* __restrict__ out, int count,
                    const float2* __restrict__ tw, unsigned* error)
{
    using Eng = SmallBatchEngine<LOG_N>;
    constexpr int N = 1 << LOG_N, NT = Eng::Lay::kThreads, S = 6144 >> LOG_N;
    constexpr int SEQ = padded_len(N) + kSeqPad;
    static_assert(SEQ * 2 >= Eng::Lay::N1 * Eng::Lay::kZStride, "a sequence's space must hold its staged rows");
    extern __shared__ float4 smem4[];
    float2* data = reinterpret_cast<float2*>(smem4);
    const int tid = threadIdx.x;
    Eng eng{reinterpret_cast<unsigned char*>(smem4) + tc_small_data_bytes<LOG_N>(), 0};
    eng.init(tid, NT, tw);
    for (int base = blockIdx.x * S; base < count; base += gridDim.x * S) {
        const int k = min(S, count - base);
        __syncthreads();
        for (int i = tid; i < k * N; i += NT) {
            const int s = i >> LOG_N, n = i & (N - 1);
            data[s * SEQ + pad_idx(n)] = in[static_cast<size_t>(base + s) * N + n];
        }
        __syncthreads();
        eng.dft(data, SEQ, k, tid, error);
        for (int i = tid; i < k * N; i += NT) {
            const int s = i >> LOG_N, n = i & (N - 1);
            out[static_cast<size_t>(base + s) * N + n] = data[s * SEQ + pad_idx(n)];
        }
    }
    eng.release(tid);
}

template <int LOG_N>
cudaError_t tc_small_launch(const float2* in, float2* out, int count, const float2* tw, unsigned* error, int sms,
                            cudaStream_t st)
{
    using Eng = SmallBatchEngine<LOG_N>;
    constexpr int S = 6144 >> LOG_N;
    constexpr size_t smem = tc_small_data_bytes<LOG_N>() + Eng::Lay::kSmemBytes;
    static_assert(smem <= 227 * 1024, "one CTA's shared memory");
    cudaError_t e = cudaFuncSetAttribute(dft_tc_small_kernel<LOG_N>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    const int chunks = (count + S - 1) / S;
    dft_tc_small_kernel<LOG_N><<<chunks < sms ? chunks : sms, Eng::Lay::kThreads, smem, st>>>(in, out, count, tw,
                                                                                              error);
    return cudaGetLastError();
}

template <int LOG_N>
cudaError_t fp32_launch(int ar, const float2* in, float2* out, int count, const float2* tw, int grid,
                        cudaStream_t st)
{
    constexpr int N = 1 << LOG_N, G = lanes_for(LOG_N);
    const size_t smem = (8 * (padded_len(N) + kSeqPad) + N) * sizeof(float2);
    auto k = ar == kArFast ? dft_fp32_kernel<LOG_N, kArFast>
                           : (ar == kArPrecise ? dft_fp32_kernel<LOG_N, kArPrecise> : dft_fp32_kernel<LOG_N, kArExact>);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    k<<<grid, 8 * G, smem, st>>>(in, out, count, tw);
    return cudaGetLastError();
}

}  // namespace

size_t tc_dft_smem_bytes()
{
    constexpr int N = 512;
    return ((8 * (padded_len(N) + kSeqPad) + N) * sizeof(float2) + 127) / 128 * 128 + BatchEngine::Lay::kSmemBytes;
}

cudaError_t launch_dft_batch(int log_n, int form, const float2* in, float2* out, int count, const float2* tw,
                             unsigned* error, int grid, cudaStream_t st)
{
    if (count <= 0) return cudaSuccess;
    if (form == 2 && log_n >= 6 && log_n <= 8) {
        int dev = 0, sms = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess) return e;
        if (log_n == 6) return tc_small_launch<6>(in, out, count, tw, error, sms, st);
        if (log_n == 7) return tc_small_launch<7>(in, out, count, tw, error, sms, st);
        return tc_small_launch<8>(in, out, count, tw, error, sms, st);
    }
    if (form == 2) {
        if (log_n != 9) return cudaErrorInvalidValue;
        const size_t smem = tc_dft_smem_bytes();
        cudaError_t e = cudaFuncSetAttribute(dft_tc512_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             static_cast<int>(smem));
        if (e != cudaSuccess) return e;
        dft_tc512_kernel<<<grid, BatchEngine::Lay::kThreads, smem, st>>>(in, out, count, tw, error);
        return cudaGetLastError();
    }
    const int ar = arith_of_form(form);
    switch (log_n) {
        case 4: return fp32_launch<4>(ar, in, out, count, tw, grid, st);
        case 5: return fp32_launch<5>(ar, in, out, count, tw, grid, st);
        case 6: return fp32_launch<6>(ar, in, out, count, tw, grid, st);
        case 7: return fp32_launch<7>(ar, in, out, count, tw, grid, st);
        case 8: return fp32_launch<8>(ar, in, out, count, tw, grid, st);
        case 9: return fp32_launch<9>(ar, in, out, count, tw, grid, st);
        case 10: return fp32_launch<10>(ar, in, out, count, tw, grid, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace ocean_b200
