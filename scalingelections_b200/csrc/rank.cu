// Ranking on sm_100a: get_winner_and_ranking (scaling_elections.py:274-296) redesigned.
//
//   wins[i]    = #{j != i : S[i][j] > S[j][i]}                       (py:285-289)
//   ranking[r] = candidates by wins descending, ties by ascending index (py:291: Python's
//                stable sorted(..., key=wins, reverse=True) keeps ties in input order)
//
// wins_kernel walks pairs of 64 x 64 tiles (I <= J, over the upper triangle in row order or, for
// a whole grid of 16 x 16 super-blocks, super-block by super-block), a few resident CTAs per SM
// each taking every gridDim.x-th pair: S[I][J] is read straight into
// registers and S[J][I] through a swizzled shared-memory tile, every cell of S once, in 128-bit
// loads, and the next pair's loads are issued before the current pair is counted. Both
// endpoints' wins accumulate in registers; one global atomic per candidate per tile pair. The
// transposed tile and the column partials are double-buffered: two barriers per pair.
//
// Candidate i's place is #{j : wins[j] > wins[i]} + #{j < i : wins[j] == wins[i]}, which is
// exactly the stable order. place_hist_kernel (C <= kHistMaxC) builds, per CTA, the histogram of
// all wins in shared memory (wins lie in [0, C)), reads the counts above each candidate's value
// from its suffix sums, and the ties before it from the histogram of the wins before the CTA's
// first candidate plus a scan of its own candidates: O(C) per CTA. place_kernel (larger C)
// counts over strips of the wins in shared memory (four per 128-bit load, eight slices of each
// strip counted side by side); a slice wholly before or after the block's candidates needs one
// compare per pair.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"

namespace se {
namespace rank {

constexpr int kRT = 64;  // tile edge of wins_kernel
constexpr int kWinsCtasPerSm = 4;

// Thread (ry, cx) of wins_kernel holds rows ry + 16p (p < 4) and columns 4cx .. 4cx+3 of the
// tile S[I][J] in registers (128-bit loads), and loads the same positions of S[J][I] into
// shared memory, where element (r, c) of that tile sits at r * 64 + (c ^ 2 * ((r >> 2) & 15)):
// rows stay 16-byte groups (stores are one 128-bit write, conflict free), and the column reads
// of the compare loop (row 4cx + q, column ry + 16p) fall on 32 distinct banks per warp.
// Pair (i, j) = (i0 + r, j0 + c) is then one shared load, two compares and two adds: row wins
// (S[i][j] > S[j][i]) and column wins (S[j][i] > S[i][j]) accumulate in registers. On a
// diagonal tile (I = J) every ordered pair is in the tile, so only row wins are counted.
__device__ __forceinline__ uint4 ldg4(const uint32_t* p) { return __ldg(reinterpret_cast<const uint4*>(p)); }

// Loads the thread's 4 x 4 cells of S[I][J] (a) and of S[J][I] at the same positions (b).
__device__ __forceinline__ void load_pair(const uint32_t* __restrict__ S, int64_t ld, int C, int vec, int i0, int j0,
                                          int ry, int cx, uint4 (&a)[4], uint4 (&b)[4]) {
    if (vec && i0 + kRT <= C && j0 + kRT <= C) {  // interior pair, 16-byte aligned rows
        const uint32_t* pa = S + int64_t(i0 + ry) * ld + j0 + 4 * cx;
        const uint32_t* pb = S + int64_t(j0 + ry) * ld + i0 + 4 * cx;
        const int64_t step = 16 * ld;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            a[p] = ldg4(pa + p * step);
            b[p] = ldg4(pb + p * step);
        }
    } else {
        auto at = [&](int r, int c) -> uint32_t { return (r < C && c < C) ? __ldg(S + int64_t(r) * ld + c) : 0u; };
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int ra = i0 + ry + 16 * p, ca = j0 + 4 * cx;
            const int rb = j0 + ry + 16 * p, cb = i0 + 4 * cx;
            a[p] = make_uint4(at(ra, ca), at(ra, ca + 1), at(ra, ca + 2), at(ra, ca + 3));
            b[p] = make_uint4(at(rb, cb), at(rb, cb + 1), at(rb, cb + 2), at(rb, cb + 3));
        }
    }
}

// Pair order. Row order: pair p is upper_pair(p, nt). Blocked order, for a tile grid that is a
// multiple of kSB tiles: super-blocks of kSB x kSB tile pairs in the upper-triangle order of
// the super-grid, the pairs of each super-block row by row; the pairs below the diagonal of a
// diagonal super-block are skipped. The CTAs in flight then read both tiles of their pairs as
// runs of kSB x 256 bytes per matrix row; in row order the transposed tiles come as 256-byte
// pieces of thousands of rows. Measured on a B200 (se_rank, warm): C = 8192 / 16384 / 32768
// 2-4 % faster blocked, C = 10000 1-2.5 % slower (a partial super-grid; row order there).
constexpr int kSB = 16;

template <bool BLOCKED>
__device__ __forceinline__ bool pair_at(int64_t p, int nt, int& I, int& J) {
    if constexpr (!BLOCKED) {
        upper_pair(p, nt, I, J);
        return true;
    } else {
        const int64_t q = p / (kSB * kSB);
        const int r = int(p - q * (kSB * kSB));
        int SI, SJ;
        upper_pair(q, nt / kSB, SI, SJ);
        I = SI * kSB + r / kSB;
        J = SJ * kSB + r % kSB;
        return I <= J;
    }
}

// Persistent over the tile pairs: block b takes pairs b, b + gridDim.x, ... and loads the next
// pair's cells into registers as soon as the current pair's transposed tile is in shared
// memory, so the loads are in flight while the current pair is compared and counted.
//
// Two barriers per pair. The transposed tile and the column partials are double-buffered:
// pair n uses bs[n & 1] and colpart[n & 1], and pair n + 2 rewrites them only after pair n + 1's
// first barrier, which every thread reaches after it has finished with pair n.
template <bool BLOCKED>
__global__ void __launch_bounds__(256, kWinsCtasPerSm)
    wins_kernel(const uint32_t* __restrict__ S, int64_t ld, int C, int nt, int vec, int32_t* __restrict__ wins) {
    __shared__ __align__(16) uint32_t tiles[2][kRT * kRT];
    __shared__ int32_t partials[2][16][kRT];  // column wins per row group ry
    const int64_t pairs = BLOCKED ? int64_t(nt / kSB) * (nt / kSB + 1) / 2 * (kSB * kSB)  // with the skipped ones
                                  : int64_t(nt) * (nt + 1) / 2;
    const int cx = threadIdx.x & 15, ry = threadIdx.x >> 4;
    // Row r = ry + 16p: the swizzle s = 2 * ((r >> 2) & 15) moves the thread's 4-group by s & ~3
    // and swaps its halves when bit 1 of s (bit 2 of r, which is bit 2 of ry) is set.
    const bool swap = (ry >> 2) & 1;
    uint4 a[4], b[4];  // a[p] = S[i0 + ry + 16p][j0 + 4cx ..], b[p] = S[j0 + ry + 16p][i0 + 4cx ..]
    int I, J;
    int64_t pb = blockIdx.x;
    while (pb < pairs && !pair_at<BLOCKED>(pb, nt, I, J)) pb += gridDim.x;
    if (pb < pairs) load_pair(S, ld, C, vec, I * kRT, J * kRT, ry, cx, a, b);
    for (int buf = 0; pb < pairs; buf ^= 1) {
        const int i0 = I * kRT, j0 = J * kRT;
        const bool diag = I == J;
        uint32_t* bs = tiles[buf];
        int32_t(*colpart)[kRT] = partials[buf];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int r = ry + 16 * p;
            const int g = (4 * cx) ^ (2 * ((r >> 2) & 15) & ~3);
            const uint4 v = swap ? make_uint4(b[p].z, b[p].w, b[p].x, b[p].y) : b[p];
            *reinterpret_cast<uint4*>(&bs[r * kRT + g]) = v;
        }
        const uint4 x0 = a[0], x1 = a[1], x2 = a[2], x3 = a[3];
        __syncthreads();
        int64_t nb = pb + gridDim.x;  // the next pair; its loads are in flight during this pair's counting
        while (nb < pairs && !pair_at<BLOCKED>(nb, nt, I, J)) nb += gridDim.x;
        if (nb < pairs) load_pair(S, ld, C, vec, I * kRT, J * kRT, ry, cx, a, b);
        uint32_t rw[4] = {0, 0, 0, 0}, cw[4] = {0, 0, 0, 0};
        const uint4 xs[4] = {x0, x1, x2, x3};
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const uint32_t x[4] = {xs[p].x, xs[p].y, xs[p].z, xs[p].w};
            const int col = (ry + 16 * p) ^ (2 * cx);  // column ry + 16p of rows 4cx + q, swizzled
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t y = bs[(4 * cx + q) * kRT + col];
                rw[p] += x[q] > y;
                cw[q] += y > x[q];
            }
        }
        // Row wins: the 16 threads of a half warp share the rows.
#pragma unroll
        for (int p = 0; p < 4; ++p) {
#pragma unroll
            for (int m = 8; m >= 1; m >>= 1) rw[p] += __shfl_xor_sync(0xFFFFFFFFu, rw[p], m);
        }
        if (cx < 4) {
            const int p = cx;  // lane cx of the half warp adds row ry + 16 * cx
            const uint32_t n = p == 0 ? rw[0] : p == 1 ? rw[1] : p == 2 ? rw[2] : rw[3];
            if (n) atomicAdd(&wins[i0 + ry + 16 * p], int(n));
        }
        if (!diag) {  // on a diagonal tile every ordered pair was counted as a row win
#pragma unroll
            for (int q = 0; q < 4; ++q) colpart[ry][4 * cx + q] = int(cw[q]);
        }
        __syncthreads();  // colpart is complete
        if (!diag && threadIdx.x < kRT) {
            int n = 0;
#pragma unroll
            for (int g = 0; g < 16; ++g) n += colpart[g][threadIdx.x];
            if (n) atomicAdd(&wins[j0 + threadIdx.x], n);
        }
        pb = nb;
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

// place_hist_kernel: kHistCand candidates per CTA, the histogram of all C wins in dynamic shared
// memory (C ints). Wins lie in [0, C); a value outside is skipped, which cannot happen for the
// wins that wins_kernel counts.
constexpr int kHistThreads = 512;
constexpr int kHistCand = 128;
constexpr int kHistMaxC = 49152;  // 192 KB of counts

__global__ void __launch_bounds__(kHistThreads)
    place_hist_kernel(const int32_t* __restrict__ wins, int C, int32_t* __restrict__ ranking) {
    extern __shared__ int32_t h[];                 // h[v] = #{j : wins[j] == v}, v < C
    __shared__ __align__(16) int32_t own[kHistCand];  // the CTA's candidates' wins
    __shared__ int32_t suffix[kHistThreads + 1];   // suffix[t] = counts of bins [t * L, C)
    const int tid = threadIdx.x;
    const int i0 = blockIdx.x * kHistCand;
    const int nb = min(kHistCand, C - i0);
    for (int v = tid; v < C; v += kHistThreads) h[v] = 0;
    if (tid < kHistCand) own[tid] = tid < nb ? wins[i0 + tid] : -1;
    // Adds wins[jb .. je) to the histogram; jb is 0 or i0, a multiple of 4, so 16-byte aligned
    // wins are read four at a time.
    const bool vec = (reinterpret_cast<uintptr_t>(wins) & 15) == 0;
    auto add = [&](int v) {
        if (unsigned(v) < unsigned(C)) atomicAdd(&h[v], 1);
    };
    auto add_range = [&](int jb, int je) {
        int j = jb;
        if (vec) {
            const int4* w4 = reinterpret_cast<const int4*>(wins + jb);
            const int n4 = (je - jb) >> 2;
#pragma unroll 2
            for (int q = tid; q < n4; q += kHistThreads) {
                const int4 v = w4[q];
                add(v.x), add(v.y), add(v.z), add(v.w);
            }
            j += 4 * n4;
        }
#pragma unroll 4
        for (j += tid; j < je; j += kHistThreads) add(wins[j]);
    };
    __syncthreads();
    add_range(0, i0);  // the wins before the CTA's first candidate
    __syncthreads();
    const int wi = tid < nb ? own[tid] : -1;
    const bool mine = unsigned(wi) < unsigned(C);
    int place = mine ? h[wi] : 0;  // ties before the CTA
    if (tid < kHistCand) {  // ties among the CTA's own candidates before this one (own[j] = -1 past nb)
        const int4* o4 = reinterpret_cast<const int4*>(own);
#pragma unroll 8
        for (int q = 0; q < kHistCand / 4; ++q) {
            const int4 v = o4[q];
            const int j = 4 * q;
            place += (v.x == wi && j < tid) + (v.y == wi && j + 1 < tid) + (v.z == wi && j + 2 < tid) +
                     (v.w == wi && j + 3 < tid);
        }
    }
    __syncthreads();  // every count above is read before the rest of the wins are added
    add_range(i0, C);
    __syncthreads();
    // Bins in chunks of L per thread; suffix[t] = sum of chunks t, t + 1, ... Thread t reads its
    // chunk starting at offset t % L and wrapping, so that the lanes of a warp read 32
    // consecutive bins at each step (distinct banks) instead of 32 bins L apart (one bank).
    const int L = (C + kHistThreads - 1) / kHistThreads;
    int sum = 0;
    {
        const int base = tid * L;
        int o = tid % L;
        for (int i = 0; i < L; ++i) {
            if (base + o < C) sum += h[base + o];
            if (++o == L) o = 0;
        }
    }
    // Inclusive suffix scan of the chunk sums: within the warp (from the higher lanes), then
    // over the warps' totals.
    const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int o = __shfl_down_sync(0xFFFFFFFFu, sum, d);
        if (lane + d < 32) sum += o;
    }
    __shared__ int32_t warp_total[kHistThreads / 32];
    if (lane == 0) warp_total[warp] = sum;  // lane 0 holds its warp's total
    __syncthreads();
    int later = 0;  // totals of the warps after this one
    for (int w = warp + 1; w < kHistThreads / 32; ++w) later += warp_total[w];
    suffix[tid] = sum + later;
    if (tid == 0) suffix[kHistThreads] = 0;
    __syncthreads();
    if (mine) {
        const int c = wi / L;  // #{j : wins[j] > wi}: later chunks, then this chunk's bins above wi
        place += suffix[c + 1];
        for (int v = wi + 1, e = min(C, (c + 1) * L); v < e; ++v) place += h[v];
        ranking[place] = i0 + tid;
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
    const int vec = (reinterpret_cast<uintptr_t>(d_S) % 16 == 0) && ld % 4 == 0;  // rows start 16-byte aligned
    // A few resident CTAs per SM, each walking the tile pairs with the next pair's loads in flight.
    int dev = 0, sms = 0;
    SE_CUDA_TRY(cudaGetDevice(&dev));
    SE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t grid = std::min<int64_t>(pairs, int64_t(sms) * rank::kWinsCtasPerSm);
    if (nt % rank::kSB == 0 && nt >= 8 * rank::kSB)  // a whole super-grid, at least 8 super-blocks across
        rank::wins_kernel<true><<<unsigned(grid), 256, 0, s>>>(d_S, ld, C, nt, vec, d_wins);
    else
        rank::wins_kernel<false><<<unsigned(grid), 256, 0, s>>>(d_S, ld, C, nt, vec, d_wins);
    SE_CHECK_LAUNCH();
    if (C <= rank::kHistMaxC) {
        const int bytes = int(sizeof(int32_t)) * rank::kHistMaxC;
        if (se_status_t st = raise_smem_limit(reinterpret_cast<const void*>(rank::place_hist_kernel), bytes,
                                              "the ranking's place kernel"))
            return st;
        rank::place_hist_kernel<<<(C + rank::kHistCand - 1) / rank::kHistCand, rank::kHistThreads,
                                  sizeof(int32_t) * size_t(C), s>>>(d_wins, C, d_ranking);
    } else {
        rank::place_kernel<<<(C + rank::kPlaceCand - 1) / rank::kPlaceCand, rank::kPlaceThreads, 0, s>>>(
            d_wins, C, d_ranking);
    }
    SE_CHECK_LAUNCH();
    return SE_OK;
}
