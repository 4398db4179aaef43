// noalloc.cu -- fbp_residual_noalloc: residual subtraction with no device allocation.
//
// For callers that cannot call cudaMalloc (a plug-in inside a host that owns all
// device memory and forbids allocation while data stream).  The scratch that
// fbp_residual takes from the caller's workspace -- per-spike window ids and
// overlap flags, and the overlap counter -- lives here in one file-scope static
// device array of fixed size (FBP_NOALLOC_MAX_SPIKES spikes).  Host code must not
// pass the array's name to a kernel (that is a host-side stand-in, not a device
// address): the device address is looked up once per device with
// cudaGetSymbolAddress, with that device current, on the first call.
#include <mutex>

#include "fbp_internal.cuh"

namespace fbp {
namespace noalloc_detail {

constexpr size_t kMaxSpikes = FBP_NOALLOC_MAX_SPIKES;
constexpr size_t kWinOff = 0;                                          // u32 window id per spike
constexpr size_t kConfOff = kMaxSpikes * 4;                            // u8 overlap flag per spike
constexpr size_t kStatusOff = (kConfOff + kMaxSpikes + 255) / 256 * 256;  // DevStatus (counter)
constexpr size_t kBytes = kStatusOff + 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kBytes];

std::mutex g_mu;
void* g_dev_ptr[kMaxDevices] = {};

__global__ void window_of_kernel(const uint32_t* idx, uint32_t n, uint32_t W, uint32_t* win)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) win[i] = idx[i] / W;
}

}  // namespace noalloc_detail
}  // namespace fbp

using namespace fbp;

extern "C" int fbp_residual_noalloc(const fbp_dims* dims, float* voltage, const float* templates,
                                    const uint32_t* spike_idx, const uint32_t* spike_lab, uint32_t n,
                                    void* stream)
{
    namespace na = fbp::noalloc_detail;
    set_error("");
    Layout lay;
    if (!make_layout(dims, FBP_PLAIN_FP32, &lay)) return fail(FBP_E_ARG, "invalid dims");
    if (n == 0) return FBP_OK;
    if (n > na::kMaxSpikes)
        return fail(FBP_E_ARG, "fbp_residual_noalloc: n exceeds FBP_NOALLOC_MAX_SPIKES (65536)");
    if (!voltage || !templates || !spike_idx || !spike_lab) return fail(FBP_E_ARG, "null pointer argument");
    if (n > lay.nw) return fail(FBP_E_ARG, "more spikes than windows in the chunk");
    int dev = 0;
    FBP_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= na::kMaxDevices) return fail(FBP_E_ARG, "device ordinal out of range");
    void* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(na::g_mu);
        if (!na::g_dev_ptr[dev]) {
            void* p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, na::g_scratch);
            if (e != cudaSuccess || p == nullptr)
                return fail(FBP_E_CUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            na::g_dev_ptr[dev] = p;
        }
        base = na::g_dev_ptr[dev];
    }
    Layout sl = lay;
    sl.off_pwin = na::kWinOff;
    sl.off_pconf = na::kConfOff;
    sl.off_status = na::kStatusOff;
    Work w{&sl, static_cast<unsigned char*>(base)};
    const Dims d = dims_of(lay);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    na::window_of_kernel<<<(n + 255) / 256, 256, 0, st>>>(spike_idx, n, d.W, w.pwin());
    FBP_CUDA(cudaGetLastError());
    return launch_residual(d, w, voltage, templates, spike_idx, spike_lab, w.pwin(), n, st);
}
