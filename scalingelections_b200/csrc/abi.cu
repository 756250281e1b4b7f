// Error reporting, version and device information for the C ABI (include/se.h).
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <set>
#include <tuple>

#include "common.cuh"

namespace se {

namespace {
thread_local char g_last_error[1024] = {0};
}

void set_error(const char* fmt, ...) {
    va_list args;
    va_start(args, fmt);
    std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, args);
    va_end(args);
}

void clear_error() { g_last_error[0] = 0; }

se_status_t raise_smem_limit(const void* fn, int bytes, const char* what) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        set_error("cannot raise the shared-memory limit of %s: no current device", what);
        return SE_ERR_CUDA;
    }
    return host_guard([&]() -> se_status_t {  // the cache's insert can throw std::bad_alloc
        static std::mutex m;
        static std::set<std::tuple<const void*, int, int>> done;
        std::lock_guard<std::mutex> lock(m);
        if (done.count({fn, dev, bytes})) return SE_OK;
        const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            set_error("cannot raise the shared-memory limit of %s: %s", what, cudaGetErrorString(e));
            return SE_ERR_CUDA;
        }
        done.insert({fn, dev, bytes});
        return SE_OK;
    });
}

}  // namespace se

extern "C" const char* se_last_error(void) { return se::g_last_error; }

extern "C" int se_version(void) { return 1; }

// log_gpus (scaling_elections.cu:996-1016) raises "Failed to get device count" when the
// runtime cannot enumerate devices; the Python layer prints what this returns.
extern "C" se_status_t se_device_count(int* count) {
    se::clear_error();
    SE_REQUIRE(count != nullptr, SE_ERR_INVALID, "count must not be null");
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        se::set_error("Failed to get device count");
        return SE_ERR_CUDA;
    }
    return SE_OK;
}

extern "C" se_status_t se_device_info(int device, char* name, int name_capacity, int* sm_count,
                                      double* global_mem_gib, int* cc_major, int* cc_minor) {
    se::clear_error();
    cudaDeviceProp prop;
    cudaError_t e = cudaGetDeviceProperties(&prop, device);
    if (e != cudaSuccess) {
        cudaGetLastError();
        se::set_error("Failed to get device properties");
        return SE_ERR_CUDA;
    }
    if (name && name_capacity > 0) {
        std::strncpy(name, prop.name, static_cast<size_t>(name_capacity) - 1);
        name[name_capacity - 1] = 0;
    }
    if (sm_count) *sm_count = prop.multiProcessorCount;
    if (global_mem_gib) *global_mem_gib = static_cast<double>(prop.totalGlobalMem) / (1024.0 * 1024.0 * 1024.0);
    if (cc_major) *cc_major = prop.major;
    if (cc_minor) *cc_minor = prop.minor;
    return SE_OK;
}
