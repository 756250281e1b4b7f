// Shared helpers for the sm_100a Schulze kernels: status codes, the per-thread last-error
// string, the packed-lane (max, min) primitives and small PTX wrappers.
//
// Element types follow the reference (scaling_elections.cu:90-93): vote counts and
// strongest-path strengths are uint32. The closure can run them in two lane modes:
//   * u32  : one cell per 32-bit word;
//   * u16  : two cells per 32-bit word (`min.u16x2` / `max.u16x2`), legal when every count
//            fits in 16 bits (V < 65536 voters), which halves both the bytes moved and the
//            instructions issued per relaxation. Results are widened back to uint32.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <exception>

#include "../../include/se.h"

namespace se {

// ------------------------------------------------------------------------------------------
// Error handling: every C-ABI entry point returns an se_status_t and records a message that
// se_last_error() returns (thread-local, like errno).
// ------------------------------------------------------------------------------------------
void set_error(const char* fmt, ...);
void clear_error();

// Raises kernel fn's dynamic shared-memory limit to `bytes` on the current device. The setting
// is per device, so it is remembered per (kernel, device, bytes); thread-safe. On failure it
// records "cannot raise the shared-memory limit of <what>" and returns SE_ERR_CUDA.
se_status_t raise_smem_limit(const void* fn, int bytes, const char* what);

#define SE_CUDA_TRY(expr)                                                                     \
    do {                                                                                      \
        cudaError_t se_err_ = (expr);                                                         \
        if (se_err_ != cudaSuccess) {                                                         \
            ::se::set_error("%s failed: %s (%s:%d)", #expr, cudaGetErrorString(se_err_),      \
                            __FILE__, __LINE__);                                              \
            return SE_ERR_CUDA;                                                               \
        }                                                                                     \
    } while (0)

#define SE_CHECK_LAUNCH()                                                                     \
    do {                                                                                      \
        cudaError_t se_err_ = cudaGetLastError();                                             \
        if (se_err_ != cudaSuccess) {                                                         \
            ::se::set_error("kernel launch failed: %s (%s:%d)", cudaGetErrorString(se_err_),  \
                            __FILE__, __LINE__);                                              \
            return SE_ERR_CUDA;                                                               \
        }                                                                                     \
    } while (0)

#define SE_REQUIRE(cond, code, ...)                                                           \
    do {                                                                                      \
        if (!(cond)) {                                                                        \
            ::se::set_error(__VA_ARGS__);                                                     \
            return (code);                                                                    \
        }                                                                                     \
    } while (0)

// No C++ exception may leave an extern "C" entry point: its callers (C, ctypes, cgo) cannot
// catch one, and the process would end in std::terminate. The entry points that fill host
// containers (which can throw std::bad_alloc) run their body through this guard, which turns
// an exception into SE_ERR_HOST with its message.
template <class F>
se_status_t host_guard(F&& body) noexcept {
    try {
        return body();
    } catch (const std::exception& x) {
        set_error("host-side failure: %s", x.what());
    } catch (...) {
        set_error("host-side failure");
    }
    return SE_ERR_HOST;
}

inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// ------------------------------------------------------------------------------------------
// Lane primitives. A "word" is a 32-bit register holding one u32 cell or two u16 cells.
// Inline PTX keeps LLVM from folding max(max(c, x), x)-style chains, while ptxas still sees
// plain min/max instructions and is free to fuse a max-of-max into its 3-input form.
// ------------------------------------------------------------------------------------------
template <int LANE_BITS> struct lanes;

template <> struct lanes<32> {
    static constexpr int cells_per_word = 1;
    __device__ __forceinline__ static uint32_t vmin(uint32_t a, uint32_t b) {
        uint32_t r;
        asm("min.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
        return r;
    }
    __device__ __forceinline__ static uint32_t vmax(uint32_t a, uint32_t b) {
        uint32_t r;
        asm("max.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
        return r;
    }
    // max(a, b, c) as two PTX max instructions; ptxas may emit one 3-input min/max.
    __device__ __forceinline__ static uint32_t vmax3(uint32_t a, uint32_t b, uint32_t c) {
        uint32_t r;
        asm("{.reg .u32 t;\n\tmax.u32 t, %1, %2;\n\tmax.u32 %0, t, %3;}"
            : "=r"(r) : "r"(a), "r"(b), "r"(c));
        return r;
    }
    // Broadcast one cell of an A operand across a word (identity for u32).
    __device__ __forceinline__ static uint32_t splat(uint32_t cell) { return cell; }
};

template <> struct lanes<16> {
    static constexpr int cells_per_word = 2;
    __device__ __forceinline__ static uint32_t vmin(uint32_t a, uint32_t b) {
        uint32_t r;
        asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
        return r;
    }
    __device__ __forceinline__ static uint32_t vmax(uint32_t a, uint32_t b) {
        uint32_t r;
        asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
        return r;
    }
    __device__ __forceinline__ static uint32_t vmax3(uint32_t a, uint32_t b, uint32_t c) {
        uint32_t r;
        asm("{.reg .b32 t;\n\tmax.u16x2 t, %1, %2;\n\tmax.u16x2 %0, t, %3;}"
            : "=r"(r) : "r"(a), "r"(b), "r"(c));
        return r;
    }
    __device__ __forceinline__ static uint32_t splat(uint32_t cell) { return cell * 0x00010001u; }
};

// ------------------------------------------------------------------------------------------
// mbarrier + TMA (cp.async.bulk.tensor) wrappers. Loads only, never multicast: every tensor
// map here covers this GPU's own memory.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Programmatic dependent launch (a kernel launched with the programmatic stream serialization
// attribute): the previous kernel in the stream lets the next one start once each of its CTAs
// has called pdl_trigger (or exited); the next kernel's threads call pdl_wait before they read
// anything the previous kernel wrote, which returns once that kernel has completed and its
// memory is visible. Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Completes a phase that has no copy behind it (the barrier's single expected arrival).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait on an mbarrier phase. Returns false if the phase did not complete within
// `max_polls` polls or `max_ns` nanoseconds of wall time, whichever comes first (the caller
// records an error and skips the rest of its work), so a lost TMA completion can never hang
// the GPU.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t max_polls,
                                                  uint64_t max_ns = 2000000000ull) {
    uint32_t done = 0;
    uint64_t t0 = 0;
    for (uint32_t i = 0; i < max_polls; ++i) {
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(smem_u32(bar)), "r"(phase)
            : "memory");
        if (done) return true;
        if ((i & 255) == 0) {
            const uint64_t now = global_ns();
            if (i == 0) t0 = now;
            else if (now - t0 > max_ns) return false;
        }
    }
    return false;
}

__device__ __forceinline__ void tma_load_2d(void* smem_dst, const void* tmap, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4}], [%2];" ::"r"(smem_u32(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// Device-side error word shared by all kernels of one call: the first failure code wins.
__device__ __forceinline__ void raise_device_error(uint32_t* err, uint32_t code) {
    if (err) atomicCAS(err, 0u, code);
}

// Tile pair b of the upper triangle of an nt x nt tile grid, row by row: row I holds the pairs
// (I, I) .. (I, nt - 1), so pair b is (I, J) with I <= J.
__device__ __forceinline__ void upper_pair(int64_t b, int nt, int& I, int& J) {
    const double n2 = 2.0 * nt + 1.0;
    int64_t r = int64_t((n2 - sqrt(n2 * n2 - 8.0 * double(b))) * 0.5);
    auto start = [nt](int64_t x) { return x * nt - x * (x - 1) / 2; };
    while (r > 0 && start(r) > b) --r;
    while (r + 1 < nt && start(r + 1) <= b) ++r;
    I = int(r);
    J = int(r + (b - start(r)));
}

// A 64 x 64 tile of u32 cells staged in shared memory so that both its rows and its columns
// read conflict-free: element (r, c) sits at r * 64 + (c ^ 2 * ((r >> 2) & 15)). Row r's
// 4-groups stay 16-byte groups, and a warp reading column r of rows 4cx + q (cx = 0..15) for
// two neighbouring r hits 32 distinct banks.
__device__ __forceinline__ int swz64(int r, int c) { return r * 64 + (c ^ (2 * ((r >> 2) & 15))); }

// Stores cells (r, c0 .. c0+3), c0 a multiple of 4, of a swizzled tile with one 128-bit write.
__device__ __forceinline__ void swz64_store4(uint32_t* tile, int r, int c0, uint4 v) {
    const int s = 2 * ((r >> 2) & 15);
    if (s & 2) v = make_uint4(v.z, v.w, v.x, v.y);  // the two halves of the group swap
    *reinterpret_cast<uint4*>(tile + r * 64 + (c0 ^ (s & ~3))) = v;
}

// Cells (r, c0 .. c0+3), c0 a multiple of 4, of a swizzled tile with one 128-bit read.
__device__ __forceinline__ uint4 swz64_load4(const uint32_t* tile, int r, int c0) {
    const int s = 2 * ((r >> 2) & 15);
    const uint4 v = *reinterpret_cast<const uint4*>(tile + r * 64 + (c0 ^ (s & ~3)));
    return (s & 2) ? make_uint4(v.z, v.w, v.x, v.y) : v;
}

}  // namespace se
