// Ballot tally on sm_100a: build_pairwise_preferences (scaling_elections.py:51-88) redesigned.
//
// The reference scatters d[r[a]][r[b]] += 1 for every ordered pair of every ballot (py:46-48),
// one voter at a time. Here the tally is a reduction over voters of a comparison:
//   d[i][j] = #{v : pos_v(i) < pos_v(j)}
// where pos_v is ballot v's rank position of each candidate after the reference's completion
// rule (missing ids appended in ascending order, py:75-83). Every completed ballot is a
// permutation, so for i != j exactly one of (i above j), (j above i) holds and
// d[j][i] = V - d[i][j]: only the upper-triangle tiles are computed.
//
// Kernel 1 (positions_kernel) writes pos as f32 [V][Cq] (exact integers), validating ids
// (range, repeats). Kernel 2 (pack_planes_kernel) packs each 32-voter chunk into bit planes.
//
// A ballot that names a candidate more than once is not a permutation, and the reference
// counts it pair by pair all the same (py:46-48; py:75 completes it only when its length
// differs from C). Such an "irregular" ballot gets place 0 for every candidate, so the
// bit-sliced count sees no pair for it in either direction, and it is left out of the
// complement V - d[i][j]. irregular_kernel then adds its pairs exactly as the reference does,
// diagonal included, with atomics.
// For C < 2048, places_planes_kernel does both in one pass and keeps the places in shared
// memory. Kernel 3 (count_bits_kernel, one CTA per upper tile) streams the planes of the two
// 128-candidate strips into shared memory with TMA and counts per 8 x 8 register micro-tile
// with a bit-serial borrow chain (one lop3 per plane) and a popc per 32 voters.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"
#include "positions.cuh"

namespace se {
namespace closure {
se_status_t make_map(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint64_t pitch_bytes,
                     uint32_t box_x, uint32_t box_y);
}

namespace tally {

constexpr int kTile = 128;     // candidates per tile edge
constexpr int kVC = 32;        // voters per TMA chunk
constexpr int kThreads = 512;  // 8 x 4 cells per thread
constexpr uint32_t kErrRange = 2;
constexpr uint32_t kErrTimeout = 1;
constexpr uint32_t kMaxPolls = 1u << 26;

int64_t padded(int C) { return round_up(C, kTile); }

// Irregular ballots (a repeated id) of one call, in the workspace after the error word:
// a count, the number per 32-voter chunk (the count kernel leaves them out of V - d[i][j]) and
// the list of their ballot indices (for irregular_kernel).
struct Irregular {
    uint32_t* n;         // irregular ballots recorded
    uint32_t* chunk;     // [ceil(V / 32)]: irregular ballots per 32-voter chunk
    uint32_t* list;      // [V]: their ballot indices, in no particular order
};

__device__ __forceinline__ void record_irregular(const Irregular& irr, int64_t v) {
    irr.list[atomicAdd(irr.n, 1u)] = uint32_t(v);
    atomicAdd(irr.chunk + v / 32, 1u);
}

// ------------------------------------------------------------------------------------------
// Positions (from C = 2048 on; below that places_planes_kernel keeps them on the SM):
// pos[v][c] = place of candidate c on completed ballot v, one CTA per ballot, the row built in
// shared memory up to C = 23552 (block_places_u16 in positions.cuh) and in global memory
// beyond (block_positions). Id is int32_t, or uint16_t / uint8_t for packed ballots.
// Ballot v is ids[offsets[v] - id_base, offsets[v + 1] - id_base), or ids[v * C, (v + 1) * C)
// when offsets is null (complete ballots).
// ------------------------------------------------------------------------------------------
constexpr int kPosThreads = 256;

// 16-bit place rows up to 46 KiB of dynamic shared memory: with the kernel's static shared
// memory that stays within the 48 KiB a block gets without raising its limit.
constexpr int kPosRowMaxCq = 23552;

// ROW: the place row is built in shared memory (block_places_u16, Cq halfwords of dynamic
// shared memory) and written out coalesced; else in global memory (block_positions).
template <typename Id, bool ROW>
__global__ void __launch_bounds__(kPosThreads)
    positions_kernel(const Id* __restrict__ ids, const int64_t* __restrict__ offsets, int64_t id_base, int64_t V,
                     int C, int64_t Cq, float* __restrict__ pos, Irregular irr, uint32_t* __restrict__ err) {
    extern __shared__ __align__(16) uint16_t row[];
    const int64_t v = blockIdx.x;
    const int64_t beg = offsets ? offsets[v] - id_base : v * C;
    const int64_t len = offsets ? offsets[v + 1] - offsets[v] : C;
    __shared__ int scratch[33];
    int code;
    if constexpr (ROW) code = block_places_u16(ids + beg, len, C, int(Cq), row, pos + v * Cq, scratch);
    else code = block_positions(ids + beg, len, C, Cq, pos + v * Cq, scratch);
    if (code == kPosRepeat) {  // every thread got the same code after the block-wide check
        for (int64_t c = threadIdx.x; c < Cq; c += blockDim.x) pos[v * Cq + c] = 0.0f;
        if (threadIdx.x == 0) record_irregular(irr, v);
    } else if (code != kPosOk && threadIdx.x == 0) {
        raise_device_error(err, uint32_t(code));
    }
}

template <typename Id>
void launch_positions(const Id* ids, const int64_t* offsets, int64_t id_base, int64_t V, int C, int64_t Cq,
                      float* pos, const Irregular& irr, uint32_t* err, cudaStream_t s) {
    if (Cq <= kPosRowMaxCq)
        positions_kernel<Id, true><<<unsigned(V), kPosThreads, size_t(Cq) * 2, s>>>(ids, offsets, id_base, V, C, Cq,
                                                                                 pos, irr, err);
    else
        positions_kernel<Id, false><<<unsigned(V), kPosThreads, 0, s>>>(ids, offsets, id_base, V, C, Cq, pos, irr,
                                                                        err);
}

// ------------------------------------------------------------------------------------------
// Bit-sliced counting. For a chunk of 32 voters, bit k of every voter's place of candidate c is
// gathered into one word: plane[ch][k][c] (bit v = bit k of pos_{32 ch + v}(c)). Then
// pos(i) < pos(j) for all 32 voters at once is the borrow out of the bit-serial subtraction
// pos(i) - pos(j): borrow' = MAJ(~a_k, b_k, borrow) over the planes from the least significant,
// one `lop3.b32` (LUT 0x8E) per plane, and one `popc` adds the 32 answers. With B = bits of
// C - 1 planes that is about (B + 2) / 32 ALU instructions per voter pair, against two FP32
// instructions in the direct form.
// ------------------------------------------------------------------------------------------
constexpr int kBitStages = 4;

// planes[(ch * B + k) * Cq + c] for the chunks of voters [0, V); voters past V count as place 0.
// B is a template parameter so that only B planes of bit work are done, in registers.
template <int B>
__global__ void __launch_bounds__(256)
    pack_planes_kernel(const float* __restrict__ pos, int64_t V, int64_t Cq, uint32_t* __restrict__ planes) {
    const int64_t c = int64_t(blockIdx.y) * blockDim.x + threadIdx.x;  // grid: (chunks, ceil(Cq / 256))
    const int64_t ch = blockIdx.x;
    if (c >= Cq) return;
    uint32_t p[32];
#pragma unroll
    for (int v = 0; v < 32; ++v) {
        const int64_t voter = ch * 32 + v;
        p[v] = voter < V ? uint32_t(pos[voter * Cq + c]) : 0u;
    }
#pragma unroll
    for (int k = 0; k < B; ++k) {
        uint32_t w = 0u;
#pragma unroll
        for (int v = 0; v < 32; ++v) w |= ((p[v] >> k) & 1u) << v;
        planes[(ch * B + k) * Cq + c] = w;
    }
}

// Places and planes in one pass, for C < 2048: one CTA of 32 warps per 32-ballot chunk. Warp
// w writes the places of ballot 32 ch + w as 16-bit values into row w of shared memory. Then
// each thread takes one candidate: it reads the candidate's 32 places down the column (lanes
// read neighbouring halfwords of one row, no bank conflicts) and builds each plane word in
// registers. The places never leave the SM.
constexpr int kFusedMaxCq = 2048;
inline size_t fused_smem(int64_t Cq) { return size_t(32) * size_t(Cq + 2) * 2; }

template <typename Id, int B>
__global__ void __launch_bounds__(1024)
    places_planes_kernel(const Id* __restrict__ ids, const int64_t* __restrict__ offsets, int64_t id_base,
                         int64_t V, int C, int Cq, uint32_t* __restrict__ planes, Irregular irr,
                         uint32_t* __restrict__ err) {
    extern __shared__ __align__(16) uint16_t rows[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pitch = Cq + 2;  // halfwords; rows start 4 bytes apart modulo 128
    const int64_t ch = blockIdx.x;
    const int64_t v = ch * 32 + warp;
    uint16_t* row = rows + warp * pitch;
    if (v < V) {
        const int64_t beg = offsets ? offsets[v] - id_base : v * C;
        const int64_t len = offsets ? offsets[v + 1] - offsets[v] : C;
        const int code = warp_places_u16(ids + beg, len, C, Cq, row);
        if (code == kPosRepeat) {  // an irregular ballot: place 0 everywhere, counted apart
            __syncwarp();
            for (int c = lane; c < Cq; c += 32) row[c] = 0;
            if (lane == 0) record_irregular(irr, v);
        } else if (code != kPosOk && lane == 0) {
            raise_device_error(err, uint32_t(code));
        }
    } else {
        for (int c = lane; c < Cq; c += 32) row[c] = 0;  // voters past V count as place 0
    }
    __syncthreads();
    for (int c = threadIdx.x; c < Cq; c += blockDim.x) {
        uint32_t p[32];
#pragma unroll
        for (int u = 0; u < 32; ++u) p[u] = rows[u * pitch + c];
#pragma unroll
        for (int k = 0; k < B; ++k) {
            uint32_t word = 0u;
#pragma unroll
            for (int u = 0; u < 32; ++u) word |= ((p[u] >> k) & 1u) << u;
            planes[(ch * B + k) * int64_t(Cq) + c] = word;
        }
    }
}

__device__ __forceinline__ uint32_t borrow_step(uint32_t a, uint32_t b, uint32_t br) {
    uint32_t r;
    asm("lop3.b32 %0, %1, %2, %3, 0x8E;" : "=r"(r) : "r"(a), "r"(b), "r"(br));
    return r;
}

inline size_t bits_smem(int B) { return size_t(kBitStages) * 2 * B * kTile * 4 + kBitStages * 8; }

// How the count's CTAs map to (upper tile, voter range). The first head_ctas CTAs take tiles
// 0 .. head_ctas / splits - 1, each cut into `splits` voter ranges; the rest take the remaining
// tiles (the launch's last, partial wave), each cut into tail_splits ranges, so that the tail
// does not hold a whole wave's time for a few tiles.
struct CountSplit {
    int64_t head_ctas;
    int splits;
    int tail_splits;
};

// Upper tile t (row by row: row I holds tiles (I, I) .. (I, R - 1)).
__device__ __forceinline__ void upper_tile(int64_t t, int R, int& I, int& J) {
    I = 0;
    while (t >= R - I) {
        t -= R - I;
        ++I;
    }
    J = I + int(t);
}

// Zeroes upper tile first + blockIdx.x and its mirror (J, I), row by row: the tiles whose counts
// arrive as atomic adds from several voter ranges.
__global__ void __launch_bounds__(256)
    zero_tiles_kernel(uint32_t* __restrict__ out, int64_t ld_out, int C, int R, int64_t first) {
    int I, J;
    upper_tile(first + blockIdx.x, R, I, J);
    for (int e = threadIdx.x; e < kTile * kTile; e += 256) {
        const int r = e / kTile, c = e % kTile;
        if (I * kTile + r < C && J * kTile + c < C) out[int64_t(I * kTile + r) * ld_out + J * kTile + c] = 0u;
        if (J * kTile + r < C && I * kTile + c < C) out[int64_t(J * kTile + r) * ld_out + I * kTile + c] = 0u;
    }
}

// Counting over one upper tile (I <= J): d[I][J] and, for I < J, d[J][I] = V - d[I][J]. One
// CTA per tile (and voter range): the two 128-candidate plane strips of each 32-voter chunk
// are staged by TMA (box {128, B}) through a 4-stage ring. With splits > 1 the voters are cut
// into `splits` ranges of whole chunks, one CTA per (tile, range), and each CTA adds its
// range's counts (and, below the diagonal, the range's voters minus them) to out with atomics:
// exact, since every count is an integer, and it keeps the grid full when there are few tiles
// and many voters.
// B (the planes per chunk) is a template parameter: the plane loop unrolls fully.
template <int B>
__global__ void __launch_bounds__(kThreads, 1)
    count_bits_kernel(const __grid_constant__ CUtensorMap mapPl, int64_t V, int C, int R, CountSplit sp,
                      uint32_t* __restrict__ out, int64_t ld_out, bool accumulate,
                      const uint32_t* __restrict__ irr_chunk, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint32_t* sI = reinterpret_cast<uint32_t*>(smem_raw);  // [kBitStages][B][kTile]
    uint32_t* sJ = sI + kBitStages * B * kTile;            // [kBitStages][B][kTile]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sJ + kBitStages * B * kTile);
    constexpr uint32_t stage_words = uint32_t(B) * kTile;
    constexpr uint32_t stage_bytes = 2u * stage_words * 4u;

    int64_t t;
    int split, splits;
    if (int64_t(blockIdx.x) < sp.head_ctas) {
        t = blockIdx.x / sp.splits, split = int(blockIdx.x % sp.splits), splits = sp.splits;
    } else {
        const int64_t b = int64_t(blockIdx.x) - sp.head_ctas;
        t = sp.head_ctas / sp.splits + b / sp.tail_splits, split = int(b % sp.tail_splits), splits = sp.tail_splits;
    }
    int I, J;
    upper_tile(t, R, I, J);
    const int total_ch = int((V + kVC - 1) / kVC);
    const int per = (total_ch + splits - 1) / splits;
    const int ch0 = split * per < total_ch ? split * per : total_ch;
    const int ch1 = ch0 + per < total_ch ? ch0 + per : total_ch;
    const int nch = ch1 - ch0;
    const int64_t vlo = int64_t(ch0) * kVC, vhi = int64_t(ch1) * kVC < V ? int64_t(ch1) * kVC : V;

    // done[s]: warps finished with stage s's current chunk. The last of them refills the stage
    // (see the end of the chunk loop), so no warp waits for another except on the data.
    __shared__ uint32_t done[kBitStages];
    __shared__ uint32_t irr_in_range;  // irregular ballots among this CTA's voters
    if (threadIdx.x < kBitStages) done[threadIdx.x] = 0u;
    if (threadIdx.x < 32) {
        uint32_t n = 0u;
        for (int c = ch0 + int(threadIdx.x); c < ch1; c += 32) n += irr_chunk[c];
#pragma unroll
        for (int o = 16; o; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
        if (threadIdx.x == 0) irr_in_range = n;
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kBitStages; ++s) mbar_init(&bars[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < kBitStages && s < nch; ++s) {
            mbar_arrive_expect_tx(&bars[s], stage_bytes);
            tma_load_2d(sI + s * stage_words, &mapPl, &bars[s], I * kTile, (ch0 + s) * B);
            tma_load_2d(sJ + s * stage_words, &mapPl, &bars[s], J * kTile, (ch0 + s) * B);
        }
    }
    // 16 warps: rows row0..row0+7 and columns col0..col0+3 of the tile per thread. A warp's 8
    // column groups read 128 contiguous bytes of a plane; its 4 row groups read 4 x 32 bytes.
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row0 = (warp & 3) * 32 + (lane >> 3) * 8;
    const int col0 = (warp >> 2) * 32 + (lane & 7) * 4;
    uint32_t acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = 0u;

    bool ok = true;
#pragma unroll 1
    for (int ch = 0; ch < nch; ++ch) {
        const int s = ch % kBitStages;
        if (ok && !mbar_wait_bounded(&bars[s], uint32_t(ch / kBitStages) & 1u, kMaxPolls)) ok = false;
        if (ok) {
            const uint32_t* pI = sI + s * stage_words;
            const uint32_t* pJ = sJ + s * stage_words;
            uint32_t br[8][4];
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int q = 0; q < 4; ++q) br[r][q] = 0u;
#pragma unroll
            for (int k = 0; k < B; ++k) {
                uint32_t a[8], b[4];
                const uint4 a0 = *reinterpret_cast<const uint4*>(pI + k * kTile + row0);
                const uint4 a1 = *reinterpret_cast<const uint4*>(pI + k * kTile + row0 + 4);
                const uint4 b0 = *reinterpret_cast<const uint4*>(pJ + k * kTile + col0);
                a[0] = a0.x, a[1] = a0.y, a[2] = a0.z, a[3] = a0.w, a[4] = a1.x, a[5] = a1.y, a[6] = a1.z, a[7] = a1.w;
                b[0] = b0.x, b[1] = b0.y, b[2] = b0.z, b[3] = b0.w;
#pragma unroll
                for (int r = 0; r < 8; ++r)
#pragma unroll
                    for (int q = 0; q < 4; ++q) br[r][q] = borrow_step(a[r], b[q], br[r][q]);
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int q = 0; q < 4; ++q) acc[r][q] += __popc(br[r][q]);
        }
        // This warp is done reading stage s. The last warp to get here refills it with chunk
        // ch + kBitStages: its lane 0 has seen every other warp's count (and, through the warp
        // barrier and the block fence, their reads of the stage come before the copy). Waiters
        // on bars[s] acquire the reset of done[s] with the stage's next phase.
        __syncwarp();
        if (lane == 0) {
            __threadfence_block();
            if (atomicAdd(&done[s], 1u) == uint32_t(kThreads / 32 - 1)) {
                done[s] = 0u;
                if (ok && ch + kBitStages < nch) {
                    fence_proxy_async();
                    mbar_arrive_expect_tx(&bars[s], stage_bytes);
                    tma_load_2d(sI + s * stage_words, &mapPl, &bars[s], I * kTile, (ch0 + ch + kBitStages) * B);
                    tma_load_2d(sJ + s * stage_words, &mapPl, &bars[s], J * kTile, (ch0 + ch + kBitStages) * B);
                }
            }
        }
    }
    if (!ok) {
        raise_device_error(err, kErrTimeout);
        return;
    }
    // Voters with a permutation ballot: each of them is counted in exactly one of d[i][j] and
    // d[j][i]. Irregular ballots (place 0 everywhere) are in neither and are added apart.
    const uint32_t Vu = uint32_t(vhi - vlo) - irr_in_range;
    if (nch == 0) return;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = I * kTile + row0 + r;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int j = J * kTile + col0 + q;
            const uint32_t n = acc[r][q];
            if (i < C && j < C) {
                uint32_t* ij = out + int64_t(i) * ld_out + j;
                uint32_t* ji = out + int64_t(j) * ld_out + i;
                if (splits > 1) {
                    if (I != J) {
                        atomicAdd(ij, n);
                        atomicAdd(ji, Vu - n);
                    } else if (i != j) {
                        atomicAdd(ij, n);
                    }
                } else if (accumulate) {
                    if (I != J) {
                        *ij += n;
                        *ji += Vu - n;
                    } else if (i != j) {
                        *ij += n;
                    }
                } else if (I == J) {
                    *ij = i == j ? 0u : n;
                } else {
                    *ij = n;
                    *ji = Vu - n;
                }
            }
        }
    }
}

// The pairs of the irregular ballots, as the reference counts them (py:46-48 over the ballot
// completed by py:75-83): with r the ballot as given (length len, ids in [0, C)) and M the ids
// absent from it in ascending order, appended only when len != C, the completed ballot is
// r ++ M and every position a before position b adds one to d[x_a][x_b]:
//   1. a < b within r;
//   2. every a of r with every m of M;
//   3. m1 < m2 within M.
// Every warp of the grid takes rows (a, or m1) of one ballot at a time, its lanes stride the
// partners, and each adds with an atomic. Each CTA keeps the ballot's presence bitmap
// (ceil(C / 32) words of dynamic shared memory) for 2 and 3. A call without irregular
// ballots returns at once.
constexpr int kIrrThreads = 512;
constexpr int kIrrMaxSmem = (1 << 20) / 8;  // the bitmap at the largest C (2^20 candidates)

template <typename Id>
__global__ void __launch_bounds__(kIrrThreads)
    irregular_kernel(const Id* __restrict__ ids, const int64_t* __restrict__ offsets, int64_t id_base, int C,
                     const uint32_t* __restrict__ irr_n, const uint32_t* __restrict__ irr_list,
                     uint32_t* __restrict__ out, int64_t ld_out) {
    extern __shared__ uint32_t present[];
    const uint32_t n = *irr_n;
    if (n == 0u) return;
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    const int64_t gw = int64_t(blockIdx.x) * warps + (threadIdx.x >> 5);
    const int64_t GW = int64_t(gridDim.x) * warps;
    const int words = (C + 31) >> 5;
    for (uint32_t q = 0; q < n; ++q) {
        const int64_t v = irr_list[q];
        const int64_t beg = offsets ? offsets[v] - id_base : v * C;
        const int64_t len = offsets ? offsets[v + 1] - offsets[v] : C;
        const Id* r = ids + beg;
        for (int64_t a = gw; a < len; a += GW) {
            uint32_t* row = out + int64_t(r[a]) * ld_out;
            for (int64_t b = a + 1 + lane; b < len; b += 32) atomicAdd(row + int64_t(r[b]), 1u);
        }
        if (len == int64_t(C)) continue;  // the same for every thread of the block
        __syncthreads();                  // the previous ballot's bitmap is no longer read
        for (int w = threadIdx.x; w < words; w += blockDim.x) present[w] = 0u;
        __syncthreads();
        for (int64_t a = threadIdx.x; a < len; a += blockDim.x) {
            const uint32_t id = uint32_t(r[a]);
            atomicOr(present + (id >> 5), 1u << (id & 31));
        }
        __syncthreads();
        auto absent = [&](int c) { return !((present[c >> 5] >> (c & 31)) & 1u); };
        for (int64_t a = gw; a < len; a += GW) {
            uint32_t* row = out + int64_t(r[a]) * ld_out;
            for (int m = lane; m < C; m += 32)
                if (absent(m)) atomicAdd(row + m, 1u);
        }
        for (int64_t m1 = gw; m1 < C; m1 += GW) {
            if (!absent(int(m1))) continue;
            uint32_t* row = out + m1 * ld_out;
            for (int64_t m2 = m1 + 1 + lane; m2 < C; m2 += 32)
                if (absent(int(m2))) atomicAdd(row + m2, 1u);
        }
    }
}

// The pack and count kernels for each plane count 1 .. kMaxPlanes.
template <typename Id>
using FusedKernel = void (*)(const Id*, const int64_t*, int64_t, int64_t, int, int, uint32_t*, Irregular, uint32_t*);

struct TallyKernels {
    void (*pack)(const float*, int64_t, int64_t, uint32_t*);
    void (*count)(CUtensorMap, int64_t, int, int, CountSplit, uint32_t*, int64_t, bool, const uint32_t*, uint32_t*);
    FusedKernel<uint8_t> fused8;  // places + planes for C < 2048 (B <= 11), else null
    FusedKernel<uint16_t> fused16;
    FusedKernel<int32_t> fused32;
};

template <int B> constexpr TallyKernels tally_entry() {
    if constexpr (B <= 11)
        return {pack_planes_kernel<B>, count_bits_kernel<B>, places_planes_kernel<uint8_t, B>,
                places_planes_kernel<uint16_t, B>, places_planes_kernel<int32_t, B>};
    else
        return {pack_planes_kernel<B>, count_bits_kernel<B>, nullptr, nullptr, nullptr};
}

template <int... Bs> struct TallyTable {
    static const TallyKernels* get() {
        static const TallyKernels t[] = {{nullptr, nullptr, nullptr, nullptr, nullptr}, tally_entry<Bs>()...};
        return t;
    }
};

const TallyKernels& tally_kernels(int B) {
    return TallyTable<1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15, 16, 17, 18, 19, 20>::get()[B];
}
static_assert(kMaxPlanes == 20, "the table instantiates planes 1 .. 20");

}  // namespace tally
}  // namespace se

using namespace se;
using namespace se::tally;

// Error word (256 B); the irregular-ballot record (16 B header holding the count, then one
// word per 32-voter chunk, then the ballot list, V words); the places f32 [V][Cq] (only from
// C = 2048 on: below that the places stay in shared memory); the bit planes u32
// [ceil(V/32) * B][Cq].
static int64_t chunks_of(int64_t V) { return (std::max<int64_t>(V, 1) + kVC - 1) / kVC; }
static int64_t irregular_header_bytes(int64_t V) { return 16 + 4 * chunks_of(V); }
static int64_t places_offset(int64_t V) {
    return 256 + round_up(irregular_header_bytes(V) + 4 * std::max<int64_t>(V, 1), 256);
}
static int64_t planes_offset(int64_t V, int C) {
    return C < kFusedMaxCq ? places_offset(V) : places_offset(V) + round_up(std::max<int64_t>(V, 1) * padded(C) * 4, 256);
}

extern "C" int64_t se_tally_workspace_bytes(int64_t V, int C) {
    if (V < 0 || C < 1) return -1;
    return planes_offset(V, C) + round_up(chunks_of(V) * planes_for(C) * padded(C) * 4, 256);
}

namespace {
se_status_t tally_impl(const void* d_ids, int id_bytes, const int64_t* d_offsets, int64_t id_base, int64_t V, int C,
                       unsigned flags, uint32_t* d_out, int64_t ld_out, void* d_work, int64_t work_bytes,
                       void* stream_) {
    clear_error();
    SE_REQUIRE(C >= 1 && C <= (1 << 20), SE_ERR_INVALID, "Number of candidates out of range (%d)", C);
    SE_REQUIRE(V >= 0 && V < (int64_t(1) << 24), SE_ERR_INVALID, "Number of voters out of range (%lld)",
               (long long)V);
    SE_REQUIRE(d_out != nullptr && ld_out >= C, SE_ERR_INVALID, "bad output matrix");
    SE_REQUIRE(id_bytes == 1 || id_bytes == 2 || id_bytes == 4, SE_ERR_INVALID, "id width must be 1, 2 or 4 bytes");
    SE_REQUIRE((flags & ~unsigned(SE_TALLY_ACCUMULATE | SE_TALLY_NO_SYNC | SE_TALLY_KEEP_ERROR)) == 0,
               SE_ERR_INVALID, "unknown tally flags %u", flags);
    SE_REQUIRE(V == 0 || d_ids, SE_ERR_INVALID, "null ballot pointer");
    SE_REQUIRE(d_offsets == nullptr || id_base >= 0, SE_ERR_INVALID, "negative id base");
    SE_REQUIRE((reinterpret_cast<uintptr_t>(d_ids) % unsigned(id_bytes)) == 0, SE_ERR_INVALID,
               "ballot ids are not aligned to their width");
    const bool accumulate = flags & SE_TALLY_ACCUMULATE;
    const bool check = !(flags & SE_TALLY_NO_SYNC);
    const int64_t need = se_tally_workspace_bytes(V, C);
    SE_REQUIRE(d_work != nullptr && work_bytes >= need, SE_ERR_WORKSPACE,
               "workspace of %lld bytes is smaller than the %lld bytes required", (long long)work_bytes,
               (long long)need);
    SE_REQUIRE((reinterpret_cast<uintptr_t>(d_work) & 255) == 0, SE_ERR_INVALID, "workspace must be 256-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    uint8_t* work = static_cast<uint8_t*>(d_work);
    uint32_t* err = reinterpret_cast<uint32_t*>(work);
    Irregular irr;
    irr.n = reinterpret_cast<uint32_t*>(work + 256);
    irr.chunk = irr.n + 4;
    irr.list = irr.chunk + chunks_of(V);
    float* pos = reinterpret_cast<float*>(work + places_offset(V));
    const int64_t Cq = padded(C);
    const int R = int(Cq / kTile);

    if (!(flags & SE_TALLY_KEEP_ERROR)) SE_CUDA_TRY(cudaMemsetAsync(work, 0, 256, s));
    if (V == 0) {
        if (!accumulate) SE_CUDA_TRY(cudaMemset2DAsync(d_out, size_t(ld_out) * 4, 0, size_t(C) * 4, size_t(C), s));
        return SE_OK;
    }
    SE_CUDA_TRY(cudaMemsetAsync(irr.n, 0, size_t(irregular_header_bytes(V)), s));
    const int B = planes_for(C);
    const TallyKernels& K = tally_kernels(B);
    if (se_status_t st = raise_smem_limit(reinterpret_cast<const void*>(K.count), int(bits_smem(B)), "the tally kernel"))
        return st;
    const int64_t nch_all = (V + kVC - 1) / kVC;
    uint32_t* planes = reinterpret_cast<uint32_t*>(work + planes_offset(V, C));
    if (C < kFusedMaxCq) {  // places and planes in one pass, places in shared memory
        const size_t smem = fused_smem(Cq);
        const int w = id_bytes == 1 ? 0 : id_bytes == 2 ? 1 : 2;
        const void* fn = w == 0 ? reinterpret_cast<const void*>(K.fused8)
                       : w == 1 ? reinterpret_cast<const void*>(K.fused16)
                                : reinterpret_cast<const void*>(K.fused32);
        if (se_status_t st = raise_smem_limit(fn, int(fused_smem(kFusedMaxCq)), "the places kernel")) return st;
        if (w == 0)
            K.fused8<<<unsigned(nch_all), 1024, smem, s>>>(static_cast<const uint8_t*>(d_ids), d_offsets, id_base, V, C,
                                                           int(Cq), planes, irr, err);
        else if (w == 1)
            K.fused16<<<unsigned(nch_all), 1024, smem, s>>>(static_cast<const uint16_t*>(d_ids), d_offsets, id_base, V,
                                                            C, int(Cq), planes, irr, err);
        else
            K.fused32<<<unsigned(nch_all), 1024, smem, s>>>(static_cast<const int32_t*>(d_ids), d_offsets, id_base, V,
                                                            C, int(Cq), planes, irr, err);
        SE_CHECK_LAUNCH();
    } else {
        if (id_bytes == 4)
            launch_positions(static_cast<const int32_t*>(d_ids), d_offsets, id_base, V, C, Cq, pos, irr, err, s);
        else if (id_bytes == 2)
            launch_positions(static_cast<const uint16_t*>(d_ids), d_offsets, id_base, V, C, Cq, pos, irr, err, s);
        else
            launch_positions(static_cast<const uint8_t*>(d_ids), d_offsets, id_base, V, C, Cq, pos, irr, err, s);
        SE_CHECK_LAUNCH();
        K.pack<<<dim3(unsigned(nch_all), unsigned((Cq + 255) / 256)), 256, 0, s>>>(pos, V, Cq, planes);
        SE_CHECK_LAUNCH();
    }
    CUtensorMap map;
    if (se_status_t st = se::closure::make_map(&map, planes, uint64_t(Cq), uint64_t(nch_all * B), uint64_t(Cq) * 4,
                                               kTile, uint32_t(B)))
        return st;
    const int64_t tiles = int64_t(R) * (R + 1) / 2;
    // Voter splits: each of the tiles x splits CTAs counts 1/splits of the voters, one CTA per
    // SM at a time, so a launch takes ceil(tiles x splits / SMs) waves of (the tile's counting
    // over all voters / splits + its output). Split outputs are atomic adds, dearer than the
    // plain stores of an unsplit launch. Costs in microseconds, measured on B200: counting
    // 0.15 per 32-voter chunk and plane-plus-two, output 12 (atomic) or 3 (stores) per tile.
    // Take the cheapest split count (the smallest within 1 %), keeping at least 32 chunks (1024
    // voters) per range. With few tiles and many voters this fills the SMs (C = 1024, 2^16
    // voters: 36 tiles x 37 splits = 9 full waves on 148 SMs); with many tiles it stays 1.
    // Then, unsplit, the last partial wave's tiles alone may be split the same way, when that
    // is cheaper than a whole wave for them (C = 4096, 4096 voters: 84 tiles in 3 ranges each;
    // C = 8192: 8 tiles in 4).
    int sms = 0, dev = 0;
    SE_CUDA_TRY(cudaGetDevice(&dev));
    SE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t chunks = (V + kVC - 1) / kVC;
    const int64_t max_splits = std::min<int64_t>(std::max<int64_t>(1, chunks / 32), 256);
    const double full_us = 0.15 * double(chunks) * double(B + 2);
    int splits = 1;
    double best = 0.0;
    for (int64_t sp = 1; sp <= max_splits; ++sp) {
        const double waves = double((tiles * sp + sms - 1) / sms);
        const double cost = waves * (full_us / double(sp) + (sp > 1 ? 12.0 : 3.0));
        if (sp == 1 || cost < best * 0.99) {
            best = cost;
            splits = int(sp);
        }
    }
    int64_t head = tiles;  // tiles in the head of the launch
    int tail_splits = 1;
    if (splits == 1 && tiles > sms && tiles % sms) {
        const int64_t rem = tiles % sms;
        double tail = full_us + 3.0;
        for (int64_t sp = 2; sp <= std::min<int64_t>(max_splits, 8); ++sp) {
            const double cost = double((rem * sp + sms - 1) / sms) * (full_us / double(sp) + 12.0);
            if (cost < tail * 0.99) {
                tail = cost;
                tail_splits = int(sp);
            }
        }
        if (tail_splits > 1) head = tiles - rem;
    }
    if (!accumulate) {
        if (splits > 1) {
            SE_CUDA_TRY(cudaMemset2DAsync(d_out, size_t(ld_out) * 4, 0, size_t(C) * 4, size_t(C), s));
        } else if (tail_splits > 1) {
            zero_tiles_kernel<<<unsigned(tiles - head), 256, 0, s>>>(d_out, ld_out, C, R, head);
            SE_CHECK_LAUNCH();
        }
    }
    const CountSplit layout{head * splits, splits, tail_splits};
    const int64_t grid = head * splits + (tiles - head) * tail_splits;
    K.count<<<unsigned(grid), kThreads, bits_smem(B), s>>>(map, V, C, R, layout, d_out, ld_out, accumulate, irr.chunk,
                                                           err);
    SE_CHECK_LAUNCH();
    // The irregular ballots' pairs, after the count's stores. Without any it returns at once.
    const size_t irr_smem = size_t((C + 31) / 32) * 4;
    const unsigned irr_grid = unsigned(2 * sms);
    if (id_bytes == 4) {
        auto fn = irregular_kernel<int32_t>;
        if (se_status_t st = raise_smem_limit(reinterpret_cast<const void*>(fn), kIrrMaxSmem, "the irregular-ballot kernel"))
            return st;
        fn<<<irr_grid, kIrrThreads, irr_smem, s>>>(static_cast<const int32_t*>(d_ids), d_offsets, id_base, C, irr.n,
                                                  irr.list, d_out, ld_out);
    } else if (id_bytes == 2) {
        auto fn = irregular_kernel<uint16_t>;
        if (se_status_t st = raise_smem_limit(reinterpret_cast<const void*>(fn), kIrrMaxSmem, "the irregular-ballot kernel"))
            return st;
        fn<<<irr_grid, kIrrThreads, irr_smem, s>>>(static_cast<const uint16_t*>(d_ids), d_offsets, id_base, C, irr.n,
                                                  irr.list, d_out, ld_out);
    } else {
        auto fn = irregular_kernel<uint8_t>;
        if (se_status_t st = raise_smem_limit(reinterpret_cast<const void*>(fn), kIrrMaxSmem, "the irregular-ballot kernel"))
            return st;
        fn<<<irr_grid, kIrrThreads, irr_smem, s>>>(static_cast<const uint8_t*>(d_ids), d_offsets, id_base, C, irr.n,
                                                  irr.list, d_out, ld_out);
    }
    SE_CHECK_LAUNCH();
    if (!check) return SE_OK;

    uint32_t code = 0;
    SE_CUDA_TRY(cudaMemcpyAsync(&code, err, 4, cudaMemcpyDeviceToHost, s));
    SE_CUDA_TRY(cudaStreamSynchronize(s));
    SE_REQUIRE(code != kErrRange, SE_ERR_DEVICE, "a ballot names a candidate outside [0, %d)", C);
    SE_REQUIRE(code == 0, SE_ERR_DEVICE, "tally kernel reported device error %u (TMA wait timed out)", code);
    return SE_OK;
}
}  // namespace

extern "C" se_status_t se_tally(const int32_t* d_ids, const int64_t* d_offsets, int64_t V, int C, uint32_t* d_out,
                                int64_t ld_out, void* d_work, int64_t work_bytes, void* stream) {
    clear_error();
    SE_REQUIRE(V == 0 || d_offsets != nullptr, SE_ERR_INVALID, "null ballot pointer");
    return tally_impl(d_ids, 4, d_offsets, 0, V, C, 0u, d_out, ld_out, d_work, work_bytes, stream);
}

extern "C" se_status_t se_tally_enqueue(const int32_t* d_ids, const int64_t* d_offsets, int64_t V, int C,
                                        uint32_t* d_out, int64_t ld_out, void* d_work, int64_t work_bytes,
                                        void* stream) {
    clear_error();
    SE_REQUIRE(V == 0 || d_offsets != nullptr, SE_ERR_INVALID, "null ballot pointer");
    return tally_impl(d_ids, 4, d_offsets, 0, V, C, SE_TALLY_NO_SYNC, d_out, ld_out, d_work, work_bytes, stream);
}

extern "C" se_status_t se_tally_ex(const void* d_ids, int id_bytes, const int64_t* d_offsets, int64_t id_base,
                                   int64_t V, int C, unsigned flags, uint32_t* d_out, int64_t ld_out, void* d_work,
                                   int64_t work_bytes, void* stream) {
    return tally_impl(d_ids, id_bytes, d_offsets, id_base, V, C, flags, d_out, ld_out, d_work, work_bytes, stream);
}
