// Ranking on sm_100a: get_winner_and_ranking (scaling_elections.py:274-296) redesigned.
//
//   wins[i]    = #{j != i : S[i][j] > S[j][i]}                       (py:285-289)
//   ranking[r] = candidates by wins descending, ties by ascending index (py:291: Python's
//                stable sorted(..., key=wins, reverse=True) keeps ties in input order)
//
// wins_kernel reads each unordered pair of 32 x 32 tiles once, S[I][J] directly and S[J][I]
// through a shared-memory transpose, and credits both endpoints of every pair. place_kernel
// gives candidate i the place #{j : wins[j] > wins[i]} + #{j < i : wins[j] == wins[i]},
// which is exactly the stable order, by counting over 1024-candidate strips in shared
// memory; O(C^2) integer compares, a few microseconds at C = 32768.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace se {
namespace rank {

__global__ void __launch_bounds__(256)
    wins_kernel(const uint32_t* __restrict__ S, int64_t ld, int C, int32_t* __restrict__ wins) {
    const int bi = blockIdx.y, bj = blockIdx.x;
    if (bi > bj) return;
    __shared__ uint32_t tJI[32][33];  // tJI[x][y] = S[bj*32 + y][bi*32 + x]
    __shared__ int32_t wi[32], wj[32];
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    if (ty == 0) wi[tx] = 0, wj[tx] = 0;
    for (int y = ty; y < 32; y += 8) {
        const int r = bj * 32 + y, c = bi * 32 + tx;
        tJI[tx][y] = (r < C && c < C) ? S[int64_t(r) * ld + c] : 0u;
    }
    __syncthreads();
    for (int y = ty; y < 32; y += 8) {
        const int i = bi * 32 + y, j = bj * 32 + tx;
        if (i < C && j < C && (bi != bj || j > i)) {
            const uint32_t sij = S[int64_t(i) * ld + j];
            const uint32_t sji = tJI[y][tx];
            if (sij > sji) atomicAdd(&wi[y], 1);
            else if (sji > sij) atomicAdd(&wj[tx], 1);
        }
    }
    __syncthreads();
    if (ty == 0) {
        const int i = bi * 32 + tx, j = bj * 32 + tx;
        if (i < C && wi[tx]) atomicAdd(&wins[i], wi[tx]);
        if (j < C && wj[tx]) atomicAdd(&wins[j], wj[tx]);
    }
}

constexpr int kStrip = 1024;

__global__ void __launch_bounds__(256)
    place_kernel(const int32_t* __restrict__ wins, int C, int32_t* __restrict__ ranking) {
    __shared__ int32_t w[kStrip];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int wi = i < C ? wins[i] : 0;
    int place = 0;
    for (int j0 = 0; j0 < C; j0 += kStrip) {
        __syncthreads();
        for (int t = threadIdx.x; t < kStrip; t += blockDim.x) w[t] = j0 + t < C ? wins[j0 + t] : -1;
        __syncthreads();
        const int n = C - j0 < kStrip ? C - j0 : kStrip;
        for (int t = 0; t < n; ++t) {
            const int wj = w[t];
            place += (wj > wi) | ((wj == wi) & (j0 + t < i));
        }
    }
    if (i < C) ranking[place] = i;
}

}  // namespace rank
}  // namespace se

using namespace se;

extern "C" se_status_t se_rank(const uint32_t* d_S, int64_t ld, int C, int32_t* d_wins, int32_t* d_ranking,
                               void* stream_) {
    clear_error();
    SE_REQUIRE(C >= 1 && C <= (1 << 20), SE_ERR_INVALID, "Number of candidates out of range (%d)", C);
    SE_REQUIRE(d_S && d_wins && d_ranking, SE_ERR_INVALID, "null pointer");
    SE_REQUIRE(ld >= C, SE_ERR_INVALID, "row stride smaller than the number of candidates");
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    SE_CUDA_TRY(cudaMemsetAsync(d_wins, 0, sizeof(int32_t) * size_t(C), s));
    const int nb = (C + 31) / 32;
    rank::wins_kernel<<<dim3(nb, nb), dim3(32, 8), 0, s>>>(d_S, ld, C, d_wins);
    SE_CHECK_LAUNCH();
    rank::place_kernel<<<(C + 255) / 256, 256, 0, s>>>(d_wins, C, d_ranking);
    SE_CHECK_LAUNCH();
    return SE_OK;
}
