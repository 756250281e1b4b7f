// Seeded synthetic ballots on the device (no reference counterpart: the reference draws its
// ballots on the host with unseeded np.random.permutation, scaling_elections.py:477-481).
//
// Mallows(pi0, phi) by the repeated insertion model: item i of the reference order pi0 is
// inserted at slot j_i in {0..i} with P(j) ~ phi^(i - j); phi = 1 gives uniform permutations.
// Decoding runs backwards: item i takes the j_i-th still-free final place (later insertions
// only push it right). One thread per ballot walks a private Fenwick tree over the free
// places (node-major, ballot-minor in the workspace so the first levels coalesce), O(C log C).
// Randomness is a counter-based SplitMix64 of (seed, ballot, item): any ballot can be
// regenerated on its own, and the result does not depend on the launch shape.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"

namespace se {
namespace ballots {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// Uniform double in [0, 1) with 53 random bits.
__device__ __forceinline__ double uniform01(uint64_t seed, uint64_t v, uint64_t i) {
    const uint64_t h = splitmix64(seed ^ splitmix64(v * 0x100000001B3ull + i));
    return double(h >> 11) * (1.0 / 9007199254740992.0);
}

// Random preference matrix: the reference's benchmark input np.random.randint(0, C, (C, C))
// (scaling_elections.py:473-476) drawn on the device. Cell (i, j) is
// (hi32(splitmix64(seed ^ splitmix64(i * C + j))) * high) >> 32, a multiply-shift map of 32
// random bits onto [0, high) (bias at most high / 2^32). The diagonal is filled too, as in
// the reference; the closure ignores it.
__global__ void __launch_bounds__(256)
    random_matrix_kernel(int C, int64_t ld, uint32_t high, uint64_t seed, uint32_t* __restrict__ out) {
    const int64_t n = int64_t(C) * C;
    for (int64_t x = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; x < n; x += int64_t(gridDim.x) * blockDim.x) {
        const int64_t i = x / C, j = x - i * C;
        const uint64_t h = splitmix64(seed ^ splitmix64(uint64_t(x)));
        out[i * ld + j] = uint32_t(((h >> 32) * uint64_t(high)) >> 32);
    }
}

__global__ void __launch_bounds__(128)
    mallows_kernel(int64_t V, int C, int size, double phi, double log_phi, uint64_t seed,
                   const int32_t* __restrict__ pi0, int32_t* __restrict__ out, uint32_t* __restrict__ tree) {
    const int64_t v = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= V) return;
    // tree[k * V + v], k = 1..size: free places in (k - lowbit(k), k], clipped to C.
    for (int k = 1; k <= size; ++k) {
        const int low = k & -k;
        const int hi = k < C ? k : C;
        const int n = hi - (k - low);
        tree[int64_t(k) * V + v] = n > 0 ? uint32_t(n) : 0u;
    }
    int32_t* ballot = out + v * C;
    for (int i = C - 1; i >= 0; --i) {
        const double u = uniform01(seed, uint64_t(v), uint64_t(i));
        int j;
        if (phi >= 1.0) {
            j = int(u * double(i + 1));
        } else {
            // Truncated geometric displacement d = i - j in [0, i].
            const double tail = 1.0 - exp(double(i + 1) * log_phi);
            double d = floor(log1p(-u * tail) / log_phi);
            d = d < 0.0 ? 0.0 : (d > double(i) ? double(i) : d);
            j = i - int(d);
        }
        j = j < 0 ? 0 : (j > i ? i : j);
        // Fenwick descent: smallest place p with (#free places <= p) == j + 1.
        uint32_t want = uint32_t(j) + 1u;
        int idx = 0;
        for (int step = size; step; step >>= 1) {
            const int nxt = idx + step;
            if (nxt <= size) {
                const uint32_t t = tree[int64_t(nxt) * V + v];
                if (t < want) {
                    idx = nxt;
                    want -= t;
                }
            }
        }
        const int place = idx;  // 0-based; < C whenever j <= i, which the clamp above ensures
        if (place >= C) return;
        ballot[place] = pi0 ? pi0[i] : i;
        for (int k = place + 1; k <= size; k += k & -k) tree[int64_t(k) * V + v] -= 1u;
    }
}

int pow2_at_least(int C) {
    int s = 1;
    while (s < C) s <<= 1;
    return s;
}

}  // namespace ballots
}  // namespace se

using namespace se;

extern "C" int64_t se_mallows_workspace_bytes(int64_t V, int C) {
    if (V < 0 || C < 1) return -1;
    return (int64_t(ballots::pow2_at_least(C)) + 1) * std::max<int64_t>(V, 1) * 4;
}

extern "C" se_status_t se_mallows_ballots(int64_t V, int C, double phi, uint64_t seed, const int32_t* d_reference,
                                          int32_t* d_out, void* d_work, int64_t work_bytes, void* stream_) {
    clear_error();
    SE_REQUIRE(C >= 1 && C <= (1 << 24), SE_ERR_INVALID, "Number of candidates out of range (%d)", C);
    SE_REQUIRE(V >= 0, SE_ERR_INVALID, "Number of voters must be non-negative");
    SE_REQUIRE(phi > 0.0 && phi <= 1.0, SE_ERR_INVALID, "phi must be in (0, 1]");
    SE_REQUIRE(V == 0 || d_out, SE_ERR_INVALID, "null output");
    const int64_t need = se_mallows_workspace_bytes(V, C);
    SE_REQUIRE(d_work != nullptr && work_bytes >= need, SE_ERR_WORKSPACE,
               "workspace of %lld bytes is smaller than the %lld bytes required", (long long)work_bytes,
               (long long)need);
    if (V == 0) return SE_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    const int size = ballots::pow2_at_least(C);
    const double log_phi = phi < 1.0 ? log(phi) : 0.0;
    const int64_t blocks = (V + 127) / 128;
    SE_REQUIRE(blocks < (int64_t(1) << 31), SE_ERR_INVALID, "too many voters");
    ballots::mallows_kernel<<<unsigned(blocks), 128, 0, s>>>(V, C, size, phi, log_phi, seed, d_reference, d_out,
                                                             static_cast<uint32_t*>(d_work));
    SE_CHECK_LAUNCH();
    return SE_OK;
}

extern "C" se_status_t se_random_preferences(int C, uint32_t high, uint64_t seed, uint32_t* d_out, int64_t ld_out,
                                             void* stream_) {
    clear_error();
    SE_REQUIRE(C >= 0 && C <= (1 << 20), SE_ERR_INVALID, "Number of candidates out of range (%d)", C);
    SE_REQUIRE(C == 0 || (d_out && ld_out >= C), SE_ERR_INVALID, "bad output matrix");
    if (C == 0) return SE_OK;
    if (high == 0) high = uint32_t(C);
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    int sms = 0, dev = 0;
    SE_CUDA_TRY(cudaGetDevice(&dev));
    SE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t cells = int64_t(C) * C;
    const int64_t blocks = std::min<int64_t>((cells + 255) / 256, int64_t(sms) * 8);
    ballots::random_matrix_kernel<<<unsigned(blocks), 256, 0, s>>>(C, ld_out, high, seed, d_out);
    SE_CHECK_LAUNCH();
    return SE_OK;
}
