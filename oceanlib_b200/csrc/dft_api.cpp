// oceanlib-b200: ocean_dft_batch - the 1-D transform of every form on device
// sequences, for accuracy checks of the forms against an FP64 DFT.
#include "../../include/ocean_b200.h"
#include "host_util.h"
#include "ocean_host.h"
#include "spectrum.h"

#include <map>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

namespace ocean_b200 {

cudaError_t launch_dft_batch(int log_n, int form, const float2* in, float2* out, int count, const float2* tw,
                             unsigned* error, int grid, cudaStream_t st);

namespace {

struct DeviceTables {
    std::map<int, DevBuf<float2>> twiddles;  // by log2 N
    DevBuf<unsigned> error;
};

std::mutex g_dft_mutex;
std::map<int, std::unique_ptr<DeviceTables>> g_dft_tables;  // by device

}  // namespace
}  // namespace ocean_b200

extern "C" ocean_status ocean_dft_batch(uint32_t size, uint32_t count, int32_t form, const float* input,
                                        float* output, void* stream)
{
    using namespace ocean_b200;
    const bool pow2 = size != 0 && (size & (size - 1)) == 0;
    if (!pow2 || size < 16 || size > 1024 || input == nullptr || output == nullptr) return OCEAN_ERROR_INVALID_ARG;
    if (form != OCEAN_FFT_EXACT && form != OCEAN_FFT_FAST && form != OCEAN_FFT_TENSOR && form != OCEAN_FFT_PRECISE)
        return OCEAN_ERROR_INVALID_ARG;
    if (form == OCEAN_FFT_TENSOR && (size < 64 || size > 512)) return OCEAN_ERROR_INVALID_ARG;
    if (count == 0) return OCEAN_OK;
    return guarded([&] {
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        const int log_n = ilog2u(size);
        float2* tw = nullptr;
        unsigned* err = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_dft_mutex);
            auto& t = g_dft_tables[dev];
            if (!t) {
                t = std::make_unique<DeviceTables>();
                t->error = DevBuf<unsigned>(1);
                check(cudaMemset(t->error.p, 0, sizeof(unsigned)), "memset");
            }
            auto it = t->twiddles.find(log_n);
            if (it == t->twiddles.end()) {
                const std::vector<float2> host = stage_twiddles(size);
                DevBuf<float2> d(host.size());
                check(cudaMemcpy(d.p, host.data(), host.size() * sizeof(float2), cudaMemcpyHostToDevice), "twiddles");
                it = t->twiddles.emplace(log_n, std::move(d)).first;
            }
            tw = it->second.p;
            err = t->error.p;
        }
        int sms = 0;
        check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
        const int chunks = static_cast<int>((count + 7) / 8);
        const int grid = chunks < 2 * sms ? chunks : 2 * sms;
        check(launch_dft_batch(log_n, form, reinterpret_cast<const float2*>(input), reinterpret_cast<float2*>(output),
                               static_cast<int>(count), tw, err, grid, st), "dft kernel");
        unsigned e = 0;
        check(cudaMemcpyAsync(&e, err, sizeof(unsigned), cudaMemcpyDeviceToHost, st), "error word");
        check(cudaStreamSynchronize(st), "dft");
        if (e != 0) {
            check(cudaMemset(err, 0, sizeof(unsigned)), "memset");
            throw TimeoutError();
        }
    });
}
