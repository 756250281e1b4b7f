// Widest-path closure for callers that cannot allocate device memory.
//
// se_closure needs a caller-provided workspace. Some callers cannot produce one:
//   * a plugin inside a host application that owns the GPU's memory budget (a database, a
//     game engine, an inference server with its own pool) and forbids its guests from
//     calling cudaMalloc behind its back;
//   * latency-critical code that must not pay for cudaFree, which synchronises the whole
//     device, or for cudaMalloc, which can stall on the driver.
// For them, se_closure_noalloc runs the same closure with its scratch space in the
// file-scope device array below, a fixed 18 MiB that every GPU which loads this library
// holds until the process exits. That bounds the problem size: at most
// SE_NOALLOC_MAX_CANDIDATES (2048) candidates, in either lane mode.
//
// Host code must not hand the array's name to a kernel: on the host that name is a stand-in
// object, not a device address. The entry point looks up the array's device address with
// cudaGetSymbolAddress, once per device (on the first call made with that device current),
// and passes that address on as the workspace.
//
// The array is shared by every call and keeps the previous call's contents. The closure
// clears what must start at zero (its error word) and overwrites every cell of its working
// matrix before reading it. Calls that overlap on the GPU, e.g. on two streams, race on the
// array and must be serialised by the caller.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "common.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(18) << 20;

static __device__ __align__(256) unsigned char g_closure_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
constexpr int kMaxDevices = 256;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_closure_scratch on the current device, looked up on first use.
se_status_t scratch_address(void** out) {
    int dev = -1;
    SE_CUDA_TRY(cudaGetDevice(&dev));
    SE_REQUIRE(dev >= 0 && dev < kMaxDevices, SE_ERR_INVALID, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_closure_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            se::set_error("cudaGetSymbolAddress of the closure scratch array failed: %s", cudaGetErrorString(e));
            return SE_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SE_OK;
}

}  // namespace

extern "C" se_status_t se_closure_noalloc(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out,
                                          int64_t ld_out, int lane_bits, void* stream) {
    se::clear_error();
    SE_REQUIRE(C >= 1 && C <= SE_NOALLOC_MAX_CANDIDATES, SE_ERR_INVALID,
               "se_closure_noalloc handles 1 to %d candidates, got %d; pass a workspace to se_closure for "
               "larger elections",
               SE_NOALLOC_MAX_CANDIDATES, C);
    const int64_t need = se_closure_workspace_bytes(C, lane_bits, 0);
    SE_REQUIRE(need > 0 && size_t(need) <= kScratchBytes, SE_ERR_INVALID,
               "closure of %d candidates needs %lld bytes of scratch, more than the %zu-byte static array", C,
               (long long)need, kScratchBytes);
    void* scratch = nullptr;
    if (se_status_t st = scratch_address(&scratch)) return st;
    return se_closure(d_pref, ld_pref, C, d_out, ld_out, lane_bits, 0, scratch, int64_t(kScratchBytes), stream);
}
