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
// cudaGetSymbolAddress, once per device (on the first call made with that device current,
// and again if cudaDeviceReset has replaced the device's context since), and passes that
// address on as the workspace. It always runs the closure round by round, whatever
// se_closure_set_mode chose, since the dataflow form needs more scratch than the array.
//
// The array is shared by every call and keeps the previous call's contents. The closure
// clears what must start at zero (its error word) and overwrites every cell of its working
// matrix before reading it. Calls that overlap on the GPU, e.g. on two streams, race on the
// array and must be serialised by the caller.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "common.cuh"

namespace se {
namespace closure {
se_status_t closure_run(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out, int64_t ld_out,
                        int lane_bits, uint32_t value_offset, int tile, void* d_work, int64_t work_bytes,
                        void* stream, double* phase_ms, int mode_override, bool sync);
}
}  // namespace se

namespace {

constexpr size_t kScratchBytes = size_t(18) << 20;

static __device__ __align__(256) unsigned char g_closure_scratch[kScratchBytes];

std::mutex g_scratch_mutex;
constexpr int kMaxDevices = 256;
// Per device: the array's address and the id of the context it was looked up in. A context
// id is never reused within a process, so after cudaDeviceReset (a new primary context) the
// address is looked up again.
void* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};

using CtxGetId = CUresult (*)(CUcontext, unsigned long long*);
using CtxGetCurrent = CUresult (*)(CUcontext*);

// The current context's id (0 if the driver cannot say).
unsigned long long current_context_id() {
    static CtxGetId get_id = nullptr;
    static CtxGetCurrent get_current = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetId>(p);
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrent>(p);
        cudaGetLastError();
    });
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_id && get_current && get_current(&ctx) == CUDA_SUCCESS && ctx && get_id(ctx, &id) == CUDA_SUCCESS)
        return id;
    return 0;
}

// Device address of g_closure_scratch on the current device: looked up once per device (and
// again only if that device's context has been replaced), with the device current.
se_status_t scratch_address(void** out) {
    int dev = -1;
    SE_CUDA_TRY(cudaGetDevice(&dev));
    SE_REQUIRE(dev >= 0 && dev < kMaxDevices, SE_ERR_INVALID, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    // Before the first runtime call on a device no context may be current (id 0): look up.
    const unsigned long long ctx = current_context_id();
    if (g_scratch_addr[dev] == nullptr || ctx == 0 || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_closure_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            se::set_error("cudaGetSymbolAddress of the closure scratch array failed: %s", cudaGetErrorString(e));
            return SE_ERR_CUDA;
        }
        g_scratch_addr[dev] = p;
        g_scratch_ctx[dev] = current_context_id();  // the lookup made the device's context current
    }
    *out = g_scratch_addr[dev];
    return SE_OK;
}

}  // namespace

extern "C" se_status_t se_closure_noalloc(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out,
                                          int64_t ld_out, int lane_bits, void* stream) {
    return se::host_guard([&]() -> se_status_t {  // the mutex can throw std::system_error
        se::clear_error();
        SE_REQUIRE(C >= 1 && C <= SE_NOALLOC_MAX_CANDIDATES, SE_ERR_INVALID,
                   "se_closure_noalloc handles 1 to %d candidates, got %d; pass a workspace to se_closure for "
                   "larger elections",
                   SE_NOALLOC_MAX_CANDIDATES, C);
        SE_REQUIRE(lane_bits == 0 || lane_bits == 16 || lane_bits == 32, SE_ERR_INVALID,
                   "lane_bits must be 0, 16 or 32");
        const int64_t need = se_closure_workspace_bytes(C, lane_bits, 0);
        SE_REQUIRE(need > 0 && size_t(need) <= kScratchBytes, SE_ERR_INVALID,
                   "closure of %d candidates needs %lld bytes of scratch, more than the %zu-byte static array", C,
                   (long long)need, kScratchBytes);
        void* scratch = nullptr;
        if (se_status_t st = scratch_address(&scratch)) return st;
        // Always round by round: the dataflow form (se_closure_set_mode(2)) needs more scratch.
        return se::closure::closure_run(d_pref, ld_pref, C, d_out, ld_out, lane_bits, 0, 0, scratch,
                                        int64_t(kScratchBytes), stream, nullptr, 1, true);
    });
}
