// Integer min/max issue-rate microbenchmark: the denominator of the closure's roofline.
//
// The closure's inner loop is c = max(c, min(a, b)) over a register-blocked micro-tile whose
// operands come from shared memory. This kernel runs exactly that loop shape (8 x 8 words per
// thread, two 128-bit shared loads per operand per k-step) with no global traffic, for one of
// several instruction recipes, and reports relaxations per SM per clock. Which recipe is
// fastest on sm_100a, and whether int and float min/max pipes co-issue, is a measured fact
// that this file exists to establish; the closure kernels use the winner.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "common.cuh"

namespace se {
namespace {

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352dU;
    x ^= x >> 15;
    x *= 0x846ca68bU;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ uint32_t f16x2_min(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t f16x2_max(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.f16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t f32_min(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.f32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t f32_max(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.f32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t f32_max3(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm("max.f32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}

// Relaxation of one word over two k-steps: (a0, b0) then (a1, b1).
template <int RECIPE>
__device__ __forceinline__ uint32_t relax2(uint32_t c, uint32_t a0, uint32_t b0, uint32_t a1,
                                           uint32_t b1) {
    if constexpr (RECIPE == 0) {
        c = lanes<32>::vmax(c, lanes<32>::vmin(a0, b0));
        return lanes<32>::vmax(c, lanes<32>::vmin(a1, b1));
    } else if constexpr (RECIPE == 1) {
        return lanes<32>::vmax3(c, lanes<32>::vmin(a0, b0), lanes<32>::vmin(a1, b1));
    } else if constexpr (RECIPE == 2) {
        c = lanes<16>::vmax(c, lanes<16>::vmin(a0, b0));
        return lanes<16>::vmax(c, lanes<16>::vmin(a1, b1));
    } else if constexpr (RECIPE == 3) {
        return lanes<16>::vmax3(c, lanes<16>::vmin(a0, b0), lanes<16>::vmin(a1, b1));
    } else if constexpr (RECIPE == 4) {
        c = f16x2_max(c, f16x2_min(a0, b0));
        return f16x2_max(c, f16x2_min(a1, b1));
    } else if constexpr (RECIPE == 5) {
        c = f32_max(c, f32_min(a0, b0));
        return f32_max(c, f32_min(a1, b1));
    } else {  // RECIPE == 6
        return f32_max3(c, f32_min(a0, b0), f32_min(a1, b1));
    }
}

// Recipes 7 and 8 split the micro-tile rows between an integer and a float recipe.
template <int RECIPE, int ROW>
__device__ __forceinline__ uint32_t relax2_row(uint32_t c, uint32_t a0, uint32_t b0, uint32_t a1,
                                               uint32_t b1) {
    if constexpr (RECIPE == 7) {
        if constexpr (ROW < 4) return relax2<3>(c, a0, b0, a1, b1);
        else return relax2<4>(c, a0, b0, a1, b1);
    } else if constexpr (RECIPE == 8) {
        if constexpr (ROW < 4) return relax2<1>(c, a0, b0, a1, b1);
        else return relax2<6>(c, a0, b0, a1, b1);
    } else {
        return relax2<RECIPE>(c, a0, b0, a1, b1);
    }
}

template <int RECIPE> struct cells_of {
    static constexpr int value = (RECIPE == 2 || RECIPE == 3 || RECIPE == 4 || RECIPE == 7) ? 2 : 1;
};

constexpr int kPeakThreads = 256;
constexpr int kPeakK = 64;  // k-steps held in shared memory, reused cyclically

template <int RECIPE, int ROW>
__device__ __forceinline__ void relax_row(uint32_t (&c)[8][8], const uint32_t (&a0)[8],
                                          const uint32_t (&b0)[8], const uint32_t (&a1)[8],
                                          const uint32_t (&b1)[8]) {
#pragma unroll
    for (int j = 0; j < 8; ++j) c[ROW][j] = relax2_row<RECIPE, ROW>(c[ROW][j], a0[ROW], b0[j], a1[ROW], b1[j]);
}

template <int RECIPE>
__global__ void __launch_bounds__(kPeakThreads, 2)
    minmax_peak_kernel(uint32_t seed, int k_steps, uint32_t* __restrict__ sink,
                       unsigned long long* __restrict__ stamps) {
    __shared__ __align__(16) uint32_t As[kPeakK][64];
    __shared__ __align__(16) uint32_t Bs[kPeakK][64];
    // Every 16-bit lane <= 0x3FFF and every word <= 0x3FFF3FFF: valid non-negative finite
    // values whether read as u16x2, u32, f16x2 or f32.
    const uint32_t mask = 0x3FFF3FFFu;
    for (int i = threadIdx.x; i < kPeakK * 64; i += blockDim.x) {
        (&As[0][0])[i] = mix32(seed + 2 * i) & mask;
        (&Bs[0][0])[i] = mix32(seed + 2 * i + 1) & mask;
    }
    uint32_t c[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) c[i][j] = mix32(seed ^ (threadIdx.x * 64 + i * 8 + j)) & mask;
    __syncthreads();

    const int rg = threadIdx.x & 7;
    const int cg = (threadIdx.x >> 3) & 7;
    unsigned long long t0 = clock64(), g0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(g0));

#pragma unroll 1
    for (int k = 0; k < k_steps; k += 2) {
        const int kk = k & (kPeakK - 1);
        uint32_t a0[8], b0[8], a1[8], b1[8];
        *reinterpret_cast<uint4*>(&a0[0]) = *reinterpret_cast<const uint4*>(&As[kk][rg * 8]);
        *reinterpret_cast<uint4*>(&a0[4]) = *reinterpret_cast<const uint4*>(&As[kk][rg * 8 + 4]);
        *reinterpret_cast<uint4*>(&b0[0]) = *reinterpret_cast<const uint4*>(&Bs[kk][cg * 8]);
        *reinterpret_cast<uint4*>(&b0[4]) = *reinterpret_cast<const uint4*>(&Bs[kk][cg * 8 + 4]);
        *reinterpret_cast<uint4*>(&a1[0]) = *reinterpret_cast<const uint4*>(&As[kk + 1][rg * 8]);
        *reinterpret_cast<uint4*>(&a1[4]) = *reinterpret_cast<const uint4*>(&As[kk + 1][rg * 8 + 4]);
        *reinterpret_cast<uint4*>(&b1[0]) = *reinterpret_cast<const uint4*>(&Bs[kk + 1][cg * 8]);
        *reinterpret_cast<uint4*>(&b1[4]) = *reinterpret_cast<const uint4*>(&Bs[kk + 1][cg * 8 + 4]);
        relax_row<RECIPE, 0>(c, a0, b0, a1, b1);
        relax_row<RECIPE, 1>(c, a0, b0, a1, b1);
        relax_row<RECIPE, 2>(c, a0, b0, a1, b1);
        relax_row<RECIPE, 3>(c, a0, b0, a1, b1);
        relax_row<RECIPE, 4>(c, a0, b0, a1, b1);
        relax_row<RECIPE, 5>(c, a0, b0, a1, b1);
        relax_row<RECIPE, 6>(c, a0, b0, a1, b1);
        relax_row<RECIPE, 7>(c, a0, b0, a1, b1);
    }

    unsigned long long t1 = clock64(), g1;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(g1));
    uint32_t x = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) x ^= c[i][j];
    sink[blockIdx.x * blockDim.x + threadIdx.x] = x;
    if (threadIdx.x == 0) {
        stamps[blockIdx.x * 2 + 0] = t1 - t0;
        stamps[blockIdx.x * 2 + 1] = g1 - g0;
    }
}

using peak_kernel_t = void (*)(uint32_t, int, uint32_t*, unsigned long long*);

peak_kernel_t pick(int recipe, int* cells) {
    switch (recipe) {
    case 0: *cells = cells_of<0>::value; return minmax_peak_kernel<0>;
    case 1: *cells = cells_of<1>::value; return minmax_peak_kernel<1>;
    case 2: *cells = cells_of<2>::value; return minmax_peak_kernel<2>;
    case 3: *cells = cells_of<3>::value; return minmax_peak_kernel<3>;
    case 4: *cells = cells_of<4>::value; return minmax_peak_kernel<4>;
    case 5: *cells = cells_of<5>::value; return minmax_peak_kernel<5>;
    case 6: *cells = cells_of<6>::value; return minmax_peak_kernel<6>;
    case 7: *cells = cells_of<7>::value; return minmax_peak_kernel<7>;
    case 8: *cells = cells_of<8>::value; return minmax_peak_kernel<8>;
    default: return nullptr;
    }
}

}  // namespace
}  // namespace se

namespace se {
namespace {
se_status_t minmax_peak_impl(int recipe, int k_steps, double* relax_per_sm_clock, double* sm_mhz,
                             double* kernel_ms, double* relax_per_s) {
    clear_error();
    int cells = 1;
    peak_kernel_t kernel = pick(recipe, &cells);
    SE_REQUIRE(kernel != nullptr, SE_ERR_INVALID, "unknown min/max recipe %d", recipe);
    SE_REQUIRE(k_steps >= 2 && k_steps % 2 == 0, SE_ERR_INVALID, "k_steps must be even and >= 2");
    int device = 0, sms = 0;
    SE_CUDA_TRY(cudaGetDevice(&device));
    SE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    int per_sm = 0;
    SE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kPeakThreads, 0));
    SE_REQUIRE(per_sm >= 1, SE_ERR_CUDA, "min/max peak kernel cannot be resident");
    const int grid = sms * per_sm;

    // Host buffer for the per-block clock stamps, allocated before any device resource so
    // that a failed allocation (an exception, turned into a status by the caller) leaks none.
    std::vector<unsigned long long> host(static_cast<size_t>(grid) * 2);
    uint32_t* sink = nullptr;
    unsigned long long* stamps = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    se_status_t st = SE_OK;
    auto fail = [&](cudaError_t e, const char* what) {
        set_error("%s failed: %s", what, cudaGetErrorString(e));
        st = SE_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMalloc(&sink, sizeof(uint32_t) * grid * kPeakThreads)) != cudaSuccess) fail(e, "cudaMalloc");
    if (st == SE_OK && (e = cudaMalloc(&stamps, sizeof(unsigned long long) * grid * 2)) != cudaSuccess) fail(e, "cudaMalloc");
    if (st == SE_OK && (e = cudaEventCreate(&e0)) != cudaSuccess) fail(e, "cudaEventCreate");
    if (st == SE_OK && (e = cudaEventCreate(&e1)) != cudaSuccess) fail(e, "cudaEventCreate");
    float ms = 0.f;
    if (st == SE_OK) {
        kernel<<<grid, kPeakThreads>>>(12345u, 64, sink, stamps);  // warm-up
        cudaEventRecord(e0);
        kernel<<<grid, kPeakThreads>>>(777u, k_steps, sink, stamps);
        cudaEventRecord(e1);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) fail(e, "min/max peak kernel");
    }
    if (st == SE_OK && (e = cudaGetLastError()) != cudaSuccess) fail(e, "min/max peak launch");
    if (st == SE_OK) {
        cudaEventElapsedTime(&ms, e0, e1);
        if ((e = cudaMemcpy(host.data(), stamps, host.size() * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost)) != cudaSuccess)
            fail(e, "cudaMemcpy");
    }
    if (st == SE_OK) {
        double mhz_sum = 0;
        int n = 0;
        for (int b = 0; b < grid; ++b) {
            if (host[2 * b + 1] > 0) {
                mhz_sum += static_cast<double>(host[2 * b]) / static_cast<double>(host[2 * b + 1]) * 1e3;
                ++n;
            }
        }
        const double mhz = n ? mhz_sum / n : 0.0;
        const double total = static_cast<double>(grid) * kPeakThreads * k_steps * 64.0 * cells;
        const double rps = total / (ms * 1e-3);
        if (sm_mhz) *sm_mhz = mhz;
        if (kernel_ms) *kernel_ms = ms;
        if (relax_per_s) *relax_per_s = rps;
        if (relax_per_sm_clock) *relax_per_sm_clock = mhz > 0 ? rps / (sms * mhz * 1e6) : 0.0;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (sink) cudaFree(sink);
    if (stamps) cudaFree(stamps);
    return st;
}

}  // namespace
}  // namespace se

extern "C" se_status_t se_minmax_peak(int recipe, int k_steps, double* relax_per_sm_clock,
                                      double* sm_mhz, double* kernel_ms, double* relax_per_s) {
    return se::host_guard(
        [&] { return se::minmax_peak_impl(recipe, k_steps, relax_per_sm_clock, sm_mhz, kernel_ms, relax_per_s); });
}
