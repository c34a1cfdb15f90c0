// oceanlib-b200: one ocean frame that allocates nothing.
//
// Who needs this: code that must not call cudaMalloc while it runs - a game
// engine or renderer that owns every byte of GPU memory through its own
// allocator and budget and hands plug-ins only buffers it created, a
// real-time thread that cannot afford cudaMalloc's implicit device
// synchronisation and unbounded latency, or an embedded host that maps a
// fixed memory arena at start-up. Such a caller passes its own device
// buffers for the inputs (the spectrum tables) and the outputs; the frame's
// only other device memory, the row-pass intermediate, lives in the
// fixed-size array below instead of a cudaMalloc'd buffer.
//
// The array is a file-scope __device__ variable, so every GPU that loads
// this library holds it (kStaticScratchBytes, about 12 MiB) until the
// process exits. All calls on one device share it: two calls whose work
// overlaps on the GPU (for example on two different streams) race on it and
// corrupt each other's results. Nothing in it needs to start at zero: each
// call rewrites the whole header (its status word included, cleared to zero)
// and the row pass overwrites every intermediate value before the column
// pass reads it.
//
// The status word: the row pass's h0 copy completes on an mbarrier whose
// wait is bounded (1 s). A wait that gives up sets the word, and the frame's
// outputs are then not to be trusted. The call itself cannot see that (it
// returns when the work is queued), so ocean_frame_static_scratch_status
// waits for the stream and reads the word.
#include "../../include/ocean_b200.h"
#include "spectrum.h"

#include <cmath>
#include <cstddef>
#include <cstring>
#include <mutex>

namespace {

// Layout of the static array (bytes):
//   [0, 16)        OceanConsts of the frame
//   [16, 24)       t / (2 pi)
//   [24, 28)       status word: 0, or 1 once a bounded wait gave up
//   [28, 32)       zero (the self-test's counter that nothing increments)
//   [32, 36)       the self-test's scratch error word
//   [256, 8448)    per-stage twiddles, N - 1 float2 (N <= 1024 fits)
//   [8448, 12544)  signed wavenumbers, N floats
//   [12544, ...)   row-pass intermediate, N * N * fields float2
constexpr uint32_t kMaxStaticSize = 512;  // largest N this entry point accepts
constexpr size_t kTwiddleOffset = 256;
constexpr size_t kKvecOffset = kTwiddleOffset + 8192;
constexpr size_t kInterOffset = kKvecOffset + 4096;
constexpr size_t kInterBytes = size_t(kMaxStaticSize) * kMaxStaticSize * 6 * sizeof(float2);
constexpr size_t kStaticScratchBytes = kInterOffset + kInterBytes;  // 12,595,456 B

}  // namespace

// The scratch itself. In host code `g_frame_scratch` names a host-side
// stand-in, not device memory: only the address obtained from
// cudaGetSymbolAddress (below) may be handed to a kernel.
static __device__ __align__(256) unsigned char g_frame_scratch[kStaticScratchBytes];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Device address of g_frame_scratch on the current device, looked up once
// per device (with that device current) and cached.
cudaError_t scratch_address(unsigned char** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_ptr[dev] == nullptr) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_frame_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

int log2_exact(uint32_t v)
{
    int l = 0;
    while ((1u << l) < v) ++l;
    return l;
}

struct Header {
    ocean_b200::OceanConsts consts;
    double t_over_2pi;
    unsigned status;
    unsigned zero;
};
static_assert(offsetof(Header, status) == 24 && sizeof(Header) == 32, "header layout");
constexpr size_t kProbeErrorOffset = 32;

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// Waits for `stream` and reads the status word of the current device's array.
ocean_status read_status(cudaStream_t st)
{
    unsigned char* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return OCEAN_ERROR_DEVICE;
    unsigned word = 0;
    // A device-to-pageable copy returns once it has been made, after the
    // stream's earlier work; the synchronise also surfaces any launch error.
    if (cudaMemcpyAsync(&word, scratch + offsetof(Header, status), sizeof(word), cudaMemcpyDeviceToHost, st) !=
            cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return OCEAN_ERROR_DEVICE;
    return word != 0 ? OCEAN_ERROR_TIMEOUT : OCEAN_OK;
}

}  // namespace

extern "C" OCEAN_API ocean_status ocean_frame_static_scratch(
    uint32_t size, float patch_length, double time, float choppiness, float foam_threshold,
    const float* h0, const float* omega_kinv, float* displacement, float* normal,
    float* velocity, void* stream)
{
    const bool pow2 = size != 0 && (size & (size - 1)) == 0;
    if (!pow2 || size < 16 || size > kMaxStaticSize) return OCEAN_ERROR_INVALID_ARG;
    if (!(patch_length > 0.0f) || !(choppiness >= 0.0f)) return OCEAN_ERROR_INVALID_ARG;
    if (h0 == nullptr || omega_kinv == nullptr || displacement == nullptr || normal == nullptr)
        return OCEAN_ERROR_INVALID_ARG;
    // h0 rows arrive by bulk copies (16-byte aligned sources) and the outputs
    // are written as float4: a misaligned buffer is refused here, before any
    // work is queued, instead of faulting on the device.
    if (!aligned16(h0) || !aligned16(omega_kinv) || !aligned16(displacement) || !aligned16(normal) ||
        (velocity != nullptr && !aligned16(velocity)))
        return OCEAN_ERROR_INVALID_ARG;
    const int nf = velocity != nullptr ? 6 : 4;
    const size_t inter_bytes = size_t(size) * size * nf * sizeof(float2);
    if (inter_bytes > kInterBytes) return OCEAN_ERROR_INVALID_ARG;

    unsigned char* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return OCEAN_ERROR_DEVICE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    // Header, twiddles and wavenumbers are built on the host in fixed-size
    // automatic arrays (no heap) and copied into the static array. The
    // twiddles follow src/core/fft.cpp:24-33 (double cos/sin of 2 pi j / N,
    // narrowed), laid out per stage; the wavenumbers src/core/spectrum.hpp:85-92.
    Header hdr;
    hdr.consts.lambda = choppiness;
    hdr.consts.foam_threshold = foam_threshold;
    hdr.consts.inv_threshold = (foam_threshold > 1e-6f) ? (1.0f / foam_threshold) : 0.0f;
    hdr.consts.geom = 0;
    hdr.t_over_2pi = time * 0.159154943091895335769;
    hdr.status = 0;
    hdr.zero = 0;

    float2 base[kMaxStaticSize / 2];
    float2 tw[kMaxStaticSize];
    float kvec[kMaxStaticSize];
    constexpr double kTwoPi = 6.283185307179586476925286766559;
    for (uint32_t j = 0; j < size / 2; ++j) {
        const double angle = kTwoPi * static_cast<double>(j) / static_cast<double>(size);
        base[j] = make_float2(static_cast<float>(std::cos(angle)), static_cast<float>(std::sin(angle)));
    }
    const int log_n = log2_exact(size);
    for (int l = 0; l < log_n; ++l) {
        const uint32_t off = size - (size >> l);
        for (uint32_t p = 0; p < (size >> (l + 1)); ++p) tw[off + p] = base[size_t(p) << l];
    }
    for (uint32_t i = 0; i < size; ++i) {
        const int si = (i < size / 2) ? static_cast<int>(i) : static_cast<int>(i) - static_cast<int>(size);
        kvec[i] = 6.28318530717958647692f * static_cast<float>(si) / patch_length;
    }

    // Copies from pageable host memory return once the source has been
    // consumed, so the automatic arrays above may go out of scope.
    if (cudaMemcpyAsync(scratch, &hdr, sizeof(hdr), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(scratch + kTwiddleOffset, tw, (size - 1) * sizeof(float2),
                        cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(scratch + kKvecOffset, kvec, size * sizeof(float), cudaMemcpyHostToDevice,
                        st) != cudaSuccess)
        return OCEAN_ERROR_DEVICE;

    ocean_b200::FrameArgs a;
    std::memset(&a, 0, sizeof(a));
    a.h0 = reinterpret_cast<const float2*>(h0);
    a.omega_kinv = reinterpret_cast<const float2*>(omega_kinv);
    a.kvec = reinterpret_cast<const float*>(scratch + kKvecOffset);
    a.twiddles = reinterpret_cast<const float2*>(scratch + kTwiddleOffset);
    a.consts = reinterpret_cast<const ocean_b200::OceanConsts*>(scratch);
    a.t_over_2pi = reinterpret_cast<const double*>(scratch + offsetof(Header, t_over_2pi));
    a.inter = reinterpret_cast<float2*>(scratch + kInterOffset);
    a.disp = reinterpret_cast<float4*>(displacement);
    a.normal = reinterpret_cast<float4*>(normal);
    a.velocity = reinterpret_cast<float4*>(velocity);
    a.ocean_base = 0;
    a.chunk = 1;
    a.error = reinterpret_cast<unsigned*>(scratch + offsetof(Header, status));
    if (ocean_b200::launch_row_pass(log_n, nf, 0, a, st) != cudaSuccess) return OCEAN_ERROR_DEVICE;
    if (ocean_b200::launch_col_pass(log_n, nf, 0, false, a, st) != cudaSuccess)
        return OCEAN_ERROR_DEVICE;
    return OCEAN_OK;
}

extern "C" OCEAN_API ocean_status ocean_frame_static_scratch_status(void* stream)
{
    return read_status(static_cast<cudaStream_t>(stream));
}

extern "C" OCEAN_API ocean_status ocean_check_static_scratch_status(uint32_t timeout_ms)
{
    unsigned char* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return OCEAN_ERROR_DEVICE;
    // The probe's counter is the header's zero word (nothing increments it)
    // and its mbarrier wait reports into the status word.
    unsigned* status = reinterpret_cast<unsigned*>(scratch + offsetof(Header, status));
    if (cudaMemset(status, 0, sizeof(unsigned)) != cudaSuccess ||
        cudaMemset(scratch + kProbeErrorOffset, 0, sizeof(unsigned)) != cudaSuccess)
        return OCEAN_ERROR_DEVICE;
    if (ocean_b200::launch_wait_probe(reinterpret_cast<const unsigned*>(scratch + offsetof(Header, zero)), 1u,
                                      reinterpret_cast<unsigned*>(scratch + kProbeErrorOffset), status,
                                      uint64_t(timeout_ms) * 1000000ull, nullptr) != cudaSuccess)
        return OCEAN_ERROR_DEVICE;
    return read_status(nullptr);
}
