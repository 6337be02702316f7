// First-collider search that allocates no device memory.
//
// Some callers cannot call cudaMalloc: frameworks that hand out all device
// memory from their own pool (a stray cudaMalloc bypasses the pool and fails
// once the pool holds nearly all of HBM), and long-running services that must
// not allocate after start-up.  bgwx_first_colliding_noalloc serves them: the
// caller passes every input and output in its own device memory, and the one
// work array the search needs -- the per-bubble candidate lists -- lives in
// the file-scope array below, sized for kNoAllocMaxBubbles radiating bubbles
// per call.  Every GPU that loads this library holds the array until the
// process exits.

#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "bgw_internal.h"
#include "device_common.cuh"
#include "masks.cuh"

namespace bgw {
namespace {

constexpr size_t kNoAllocMaxBubbles = 512;

// Candidate lists of up to kNoAllocMaxBubbles radiating bubbles followed by
// the fallback counter.  Shared by every call: the lists of the bubbles of a
// call are rewritten by that call, the counter is cleared by each call.
constexpr size_t kNoAllocBytes = kNoAllocMaxBubbles * sizeof(NbList) + 256;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
void* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  The first call
// on each device looks it up (host code cannot use the array's name as a
// device address); later calls reuse it.
void* scratch_address(int dev) {
    if (dev < 0 || dev >= kMaxDevices) throw Error{"device ordinal out of range for the no-allocation entry point"};
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            throw Error{std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                        cudaGetErrorString(e)};
        g_scratch_ptr[dev] = p;
    }
    return g_scratch_ptr[dev];
}

}  // namespace
}  // namespace bgw

extern "C" BgwStatus bgwx_first_colliding_noalloc(const double* d_bubbles, size_t n_interior, size_t n_total,
                                                   const uint32_t* d_selected, size_t n_selected,
                                                   const double* d_dirs, size_t n_dirs, int32_t* d_codes,
                                                   double* d_delta_tab, void* stream) {
    using namespace bgw;
    try {
        if (n_selected == 0 || n_dirs == 0) {
            clear_last_error();
            return BGW_STATUS_OK;
        }
        if (!d_bubbles || !d_selected || !d_dirs || !d_codes || !d_delta_tab)
            throw Error{"device pointers must not be null"};
        if (n_selected > kNoAllocMaxBubbles)
            throw Error{"n_selected=" + std::to_string(n_selected) + " exceeds the no-allocation limit of " +
                        std::to_string(kNoAllocMaxBubbles) + " radiating bubbles per call"};
        if (n_interior == 0 || n_interior > n_total) throw Error{"need 0 < n_interior <= n_total"};
        if (n_total > 0x7fffffffULL || n_dirs > 0x7fffffffULL) throw Error{"n_total or n_dirs too large"};
        int dev = 0;
        CUDA_OK(cudaGetDevice(&dev));
        unsigned char* base = static_cast<unsigned char*>(scratch_address(dev));
        NbList* lists = reinterpret_cast<NbList*>(base);
        unsigned long long* counter =
            reinterpret_cast<unsigned long long*>(base + kNoAllocMaxBubbles * sizeof(NbList));
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        CUDA_OK(cudaMemsetAsync(counter, 0, sizeof(unsigned long long), st));
        launch_masks_with_lists(st, reinterpret_cast<const D4*>(d_bubbles), n_interior, n_total, d_selected,
                                n_selected, reinterpret_cast<const D4*>(d_dirs), n_dirs, lists, d_delta_tab, d_codes,
                                counter);
        clear_last_error();
        return BGW_STATUS_OK;
    } catch (const Error& e) {
        set_last_error(e.msg);
        return BGW_STATUS_CALCULATION_ERROR;
    }
}
