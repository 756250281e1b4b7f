// Ranking on sm_100a: get_winner_and_ranking (scaling_elections.py:274-296) redesigned.
//
//   wins[i]    = #{j != i : S[i][j] > S[j][i]}                       (py:285-289)
//   ranking[r] = candidates by wins descending, ties by ascending index (py:291: Python's
//                stable sorted(..., key=wins, reverse=True) keeps ties in input order)
//
// wins_kernel takes one pair of 64 x 64 tiles (I <= J, enumerated over the upper triangle so
// that no block idles): S[I][J] is read straight into registers and S[J][I] through a
// shared-memory transpose, every cell of S once, 128 coalesced bytes per warp load. Row wins
// are counted by warp ballots, column wins in registers; one global atomic per candidate per
// tile pair. place_kernel gives candidate i the place #{j : wins[j] > wins[i]} +
// #{j < i : wins[j] == wins[i]}, which is exactly the stable order, by counting over strips of
// the wins in shared memory (four per 128-bit load, eight slices of each strip counted side
// by side); a slice wholly before or after the block's candidates needs one compare per pair.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace se {
namespace rank {

constexpr int kRT = 64;  // tile edge of wins_kernel

// Tile pair b of the upper triangle, row by row: row I holds pairs (I, I) .. (I, nt - 1).
__device__ __forceinline__ void tile_pair(int64_t b, int nt, int& I, int& J) {
    const double n2 = 2.0 * nt + 1.0;
    int64_t r = int64_t((n2 - sqrt(n2 * n2 - 8.0 * double(b))) * 0.5);
    auto start = [nt](int64_t x) { return x * nt - x * (x - 1) / 2; };
    while (r > 0 && start(r) > b) --r;
    while (r + 1 < nt && start(r + 1) <= b) ++r;
    I = int(r);
    J = int(r + (b - start(r)));
}

__global__ void __launch_bounds__(256)
    wins_kernel(const uint32_t* __restrict__ S, int64_t ld, int C, int nt, int32_t* __restrict__ wins) {
    __shared__ uint32_t t[kRT][kRT + 1];  // t[x][y] = S[j0 + y][i0 + x]
    __shared__ int32_t wrow[2][kRT];      // row wins per half-row warp
    __shared__ int32_t wcol[4][kRT];      // column wins per row group
    int I, J;
    tile_pair(blockIdx.x, nt, I, J);
    const int i0 = I * kRT, j0 = J * kRT;
    const int tx = threadIdx.x & (kRT - 1), ty = threadIdx.x >> 6;  // 64 x 4
    const int j = j0 + tx, ci = i0 + tx;
    const bool full = i0 + kRT <= C && j0 + kRT <= C;
    uint32_t sij[kRT / 4];
    if (full) {  // interior tile pair: no bounds checks, addresses by one stride step
        const uint32_t* pd = S + int64_t(i0 + ty) * ld + j;
        const uint32_t* pt = S + int64_t(j0 + ty) * ld + ci;
        const int64_t step = 4 * ld;
#pragma unroll
        for (int s = 0; s < kRT / 4; ++s) {
            sij[s] = __ldg(pd + s * step);
            t[tx][ty + 4 * s] = __ldg(pt + s * step);
        }
    } else {
#pragma unroll
        for (int s = 0; s < kRT / 4; ++s) {
            const int y = ty + 4 * s;
            const int i = i0 + y, r = j0 + y;
            sij[s] = (i < C && j < C) ? __ldg(S + int64_t(i) * ld + j) : 0u;
            t[tx][y] = (r < C && ci < C) ? __ldg(S + int64_t(r) * ld + ci) : 0u;
        }
    }
    __syncthreads();
    int wj = 0;
#pragma unroll
    for (int s = 0; s < kRT / 4; ++s) {
        const int y = ty + 4 * s;
        const int i = i0 + y;
        const uint32_t sji = t[y][tx];
        const bool pair = i < C && j < C && (I != J || j > i);
        const bool win_i = pair && sij[s] > sji;
        wj += pair && sji > sij[s];
        const int n = __popc(__ballot_sync(0xFFFFFFFFu, win_i));
        if ((threadIdx.x & 31) == 0) wrow[tx >> 5][y] = n;
    }
    wcol[ty][tx] = wj;
    __syncthreads();
    if (threadIdx.x < kRT) {
        const int y = threadIdx.x;
        const int n = wrow[0][y] + wrow[1][y];
        if (n) atomicAdd(&wins[i0 + y], n);
    } else if (threadIdx.x < 2 * kRT) {
        const int x = threadIdx.x - kRT;
        const int n = wcol[0][x] + wcol[1][x] + wcol[2][x] + wcol[3][x];
        if (n) atomicAdd(&wins[j0 + x], n);
    }
}

// place_kernel: kPlaceCand candidates per CTA; each strip of kStrip wins in shared memory is
// split into kPlaceGroups slices, one per group of kPlaceCand threads, and the groups' partial
// counts are summed at the end.
constexpr int kPlaceCand = 64;
constexpr int kPlaceGroups = 8;
constexpr int kPlaceThreads = kPlaceCand * kPlaceGroups;  // 512
constexpr int kStrip = 2048;
constexpr int kSlice = kStrip / kPlaceGroups;             // 256

__global__ void __launch_bounds__(kPlaceThreads)
    place_kernel(const int32_t* __restrict__ wins, int C, int32_t* __restrict__ ranking) {
    __shared__ __align__(16) int32_t w[kStrip];
    __shared__ int32_t part[kPlaceGroups][kPlaceCand];
    const int c = threadIdx.x % kPlaceCand, grp = threadIdx.x / kPlaceCand;  // grp is warp-uniform
    const int i0 = blockIdx.x * kPlaceCand;
    const int i = i0 + c;
    const int wi = i < C ? wins[i] : 0;
    int p[4] = {0, 0, 0, 0};
    for (int j0 = 0; j0 < C; j0 += kStrip) {
        __syncthreads();
        for (int t = threadIdx.x; t < kStrip; t += kPlaceThreads) w[t] = j0 + t < C ? wins[j0 + t] : -1;
        __syncthreads();
        // This group's slice [js, js + kSlice). Entries past C hold -1, which never counts
        // (wins are >= 0).
        const int js = j0 + grp * kSlice;
        if (js >= C) continue;
        const int4* w4 = reinterpret_cast<const int4*>(w + grp * kSlice);
        if (js + kSlice <= i0) {  // every j precedes every i of the block: counts wins[j] >= wins[i]
#pragma unroll 8
            for (int t = 0; t < kSlice / 4; ++t) {
                const int4 v = w4[t];
                p[0] += v.x >= wi, p[1] += v.y >= wi, p[2] += v.z >= wi, p[3] += v.w >= wi;
            }
        } else if (js >= i0 + kPlaceCand) {  // every j follows: counts wins[j] > wins[i]
#pragma unroll 8
            for (int t = 0; t < kSlice / 4; ++t) {
                const int4 v = w4[t];
                p[0] += v.x > wi, p[1] += v.y > wi, p[2] += v.z > wi, p[3] += v.w > wi;
            }
        } else {
            const int* ws = w + grp * kSlice;
            for (int t = 0; t < kSlice; ++t) {
                const int wj = ws[t];
                p[t & 3] += (wj > wi) | ((wj == wi) & (js + t < i));
            }
        }
    }
    part[grp][c] = p[0] + p[1] + p[2] + p[3];
    __syncthreads();
    if (grp == 0 && i < C) {
        int place = 0;
#pragma unroll
        for (int g = 0; g < kPlaceGroups; ++g) place += part[g][c];
        ranking[place] = i;
    }
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
    const int nt = (C + rank::kRT - 1) / rank::kRT;
    const int64_t pairs = int64_t(nt) * (nt + 1) / 2;  // at most 2^27 at C = 2^20
    rank::wins_kernel<<<unsigned(pairs), 256, 0, s>>>(d_S, ld, C, nt, d_wins);
    SE_CHECK_LAUNCH();
    rank::place_kernel<<<(C + rank::kPlaceCand - 1) / rank::kPlaceCand, rank::kPlaceThreads, 0, s>>>(
        d_wins, C, d_ranking);
    SE_CHECK_LAUNCH();
    return SE_OK;
}
