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
// Kernel 1 (positions_kernel, one CTA per ballot) writes pos as f32 [V][Cq] (exact integers),
// validating ids (range, repeats). Kernel 2 (count_kernel, one CTA per upper tile) streams
// 32-voter chunks of the two 128-candidate position strips into shared memory with TMA and
// counts per 8 x 8 register micro-tile with `sub.sat.f32` (1.0 when pos_j > pos_i, the
// positions differ by at least 1) plus `add.f32`: both on the FP32 pipe, leaving the
// integer min/max pipe to the closure. Counts stay exact in f32 up to 2^24 voters.
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
constexpr int kStages = 3;     // chunk ring depth (3 x 32 KiB: fits beside a serving-engine CTA on one SM)
constexpr int kThreads = 256;  // 8 x 8 cells per thread
constexpr uint32_t kChunkBytes = kVC * kTile * 4;
constexpr size_t kSmem = size_t(kStages) * 2 * kVC * kTile * 4 + kStages * 8;
constexpr uint32_t kErrRange = 2;
constexpr uint32_t kErrRepeat = 3;
constexpr uint32_t kErrTimeout = 1;
constexpr uint32_t kMaxPolls = 1u << 26;

int64_t padded(int C) { return round_up(C, kTile); }

// ------------------------------------------------------------------------------------------
// Positions: pos[v][c] = place of candidate c on completed ballot v, one warp per ballot
// (positions.cuh), 8 ballots per CTA. Id is int32_t, or uint16_t / uint8_t for packed ballots.
// Ballot v is ids[offsets[v] - id_base, offsets[v + 1] - id_base), or ids[v * C, (v + 1) * C)
// when offsets is null (complete ballots).
// ------------------------------------------------------------------------------------------
constexpr int kPosWarps = 8;
constexpr int kPosBlockFromC = 2048;  // from this many candidates on, one CTA per ballot

// PER_WARP: one ballot per warp, kPosWarps ballots per CTA; else one ballot per CTA.
template <typename Id, bool PER_WARP>
__global__ void __launch_bounds__(32 * kPosWarps)
    positions_kernel(const Id* __restrict__ ids, const int64_t* __restrict__ offsets, int64_t id_base, int64_t V,
                     int C, int64_t Cq, float* __restrict__ pos, uint32_t* __restrict__ err) {
    const int64_t v = PER_WARP ? int64_t(blockIdx.x) * kPosWarps + (threadIdx.x >> 5) : int64_t(blockIdx.x);
    if (v >= V) return;  // warp-uniform (and CTA-uniform for one ballot per CTA)
    const int64_t beg = offsets ? offsets[v] - id_base : v * C;
    const int64_t len = offsets ? offsets[v + 1] - offsets[v] : C;
    int code;
    if constexpr (PER_WARP) {
        code = warp_positions(ids + beg, len, C, Cq, pos + v * Cq);
        if (code != kPosOk && (threadIdx.x & 31) == 0) raise_device_error(err, uint32_t(code));
    } else {
        __shared__ int scratch[33];
        code = block_positions(ids + beg, len, C, Cq, pos + v * Cq, scratch);
        if (code != kPosOk && threadIdx.x == 0) raise_device_error(err, uint32_t(code));
    }
}

template <typename Id>
void launch_positions(const Id* ids, const int64_t* offsets, int64_t id_base, int64_t V, int C, int64_t Cq,
                      float* pos, uint32_t* err, cudaStream_t s) {
    if (C >= kPosBlockFromC)
        positions_kernel<Id, false><<<unsigned(V), 32 * kPosWarps, 0, s>>>(ids, offsets, id_base, V, C, Cq, pos, err);
    else
        positions_kernel<Id, true><<<unsigned((V + kPosWarps - 1) / kPosWarps), 32 * kPosWarps, 0, s>>>(
            ids, offsets, id_base, V, C, Cq, pos, err);
}

__device__ __forceinline__ float sat_sub(float a, float b) {
    float r;
    asm("sub.sat.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

__device__ __forceinline__ void lds4f(float* dst, const float* src) {
    const float4 v = *reinterpret_cast<const float4*>(src);
    dst[0] = v.x, dst[1] = v.y, dst[2] = v.z, dst[3] = v.w;
}

// ------------------------------------------------------------------------------------------
// Counting over one upper tile (I <= J): d[I][J] and, for I < J, d[J][I] = V - d[I][J].
// With splits > 1 the voters are cut into `splits` ranges of whole 32-voter chunks, one CTA per
// (tile, range), and each CTA adds its range's counts (and, below the diagonal, the range's
// voters minus them) to out with atomics: exact, since every count is an integer, and it keeps
// the grid full when there are few tiles and many voters.
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kThreads, 1)
    count_kernel(const __grid_constant__ CUtensorMap mapPos, int64_t V, int C, int R, int splits,
                 uint32_t* __restrict__ out, int64_t ld_out, bool accumulate, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    float* sI = reinterpret_cast<float*>(smem_raw);           // [kStages][kVC][kTile]
    float* sJ = sI + kStages * kVC * kTile;                   // [kStages][kVC][kTile]
    uint64_t* bars = reinterpret_cast<uint64_t*>(sJ + kStages * kVC * kTile);

    // Upper-triangle tile index -> (I, J), row-major over I <= J.
    int64_t t = blockIdx.x / splits;
    const int split = int(blockIdx.x % splits);
    int I = 0;
    while (t >= R - I) {
        t -= R - I;
        ++I;
    }
    const int J = I + int(t);
    const int total_ch = int((V + kVC - 1) / kVC);
    const int per = (total_ch + splits - 1) / splits;
    const int ch0 = split * per < total_ch ? split * per : total_ch;
    const int ch1 = ch0 + per < total_ch ? ch0 + per : total_ch;
    const int nch = ch1 - ch0;
    const int64_t vlo = int64_t(ch0) * kVC, vhi = int64_t(ch1) * kVC < V ? int64_t(ch1) * kVC : V;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) mbar_init(&bars[s], 1);
        fence_barrier_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages && s < nch; ++s) {
            mbar_arrive_expect_tx(&bars[s], 2 * kChunkBytes);
            tma_load_2d(sI + s * kVC * kTile, &mapPos, &bars[s], I * kTile, (ch0 + s) * kVC);
            tma_load_2d(sJ + s * kVC * kTile, &mapPos, &bars[s], J * kTile, (ch0 + s) * kVC);
        }
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int row0 = (warp & 3) * 32 + (lane >> 3) * 8;
    const int col0 = (warp >> 2) * 64 + (lane & 7) * 4;  // cols col0..+3 and col0+32..+35
    float acc[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = 0.0f;

    bool ok = true;
#pragma unroll 1
    for (int ch = 0; ch < nch; ++ch) {
        const int s = ch % kStages;
        if (ok && !mbar_wait_bounded(&bars[s], uint32_t(ch / kStages) & 1u, kMaxPolls)) ok = false;
        if (ok) {
            const float* pI = sI + s * kVC * kTile;
            const float* pJ = sJ + s * kVC * kTile;
#pragma unroll 4
            for (int v = 0; v < kVC; ++v) {
                float a[8], b[8];
                lds4f(a, pI + v * kTile + row0);
                lds4f(a + 4, pI + v * kTile + row0 + 4);
                lds4f(b, pJ + v * kTile + col0);
                lds4f(b + 4, pJ + v * kTile + col0 + 32);
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[i][j] += sat_sub(b[j], a[i]);
            }
        }
        __syncthreads();  // every thread is done with stage s
        if (threadIdx.x == 0 && ok && ch + kStages < nch) {
            fence_proxy_async();  // order this stage's shared reads before the TMA rewrite
            mbar_arrive_expect_tx(&bars[s], 2 * kChunkBytes);
            tma_load_2d(sI + s * kVC * kTile, &mapPos, &bars[s], I * kTile, (ch0 + ch + kStages) * kVC);
            tma_load_2d(sJ + s * kVC * kTile, &mapPos, &bars[s], J * kTile, (ch0 + ch + kStages) * kVC);
        }
    }
    if (!ok) {
        raise_device_error(err, kErrTimeout);
        return;
    }
    const uint32_t Vu = uint32_t(vhi - vlo);
    if (nch == 0) return;  // an empty trailing range (more splits than chunks)
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = I * kTile + row0 + r;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int j = J * kTile + col0 + (q < 4 ? q : 28 + q);
            const uint32_t n = uint32_t(acc[r][q]);
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
                        *ij += n;  // the (j, i) cell of a diagonal tile is some thread's (i, j)
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

}  // namespace tally
}  // namespace se

using namespace se;
using namespace se::tally;

extern "C" int64_t se_tally_workspace_bytes(int64_t V, int C) {
    if (V < 0 || C < 1) return -1;
    return 256 + round_up(std::max<int64_t>(V, 1) * padded(C) * 4, 256);
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
    float* pos = reinterpret_cast<float*>(work + 256);
    const int64_t Cq = padded(C);
    const int R = int(Cq / kTile);

    if (!(flags & SE_TALLY_KEEP_ERROR)) SE_CUDA_TRY(cudaMemsetAsync(work, 0, 256, s));
    if (V == 0) {
        if (!accumulate) SE_CUDA_TRY(cudaMemset2DAsync(d_out, size_t(ld_out) * 4, 0, size_t(C) * 4, size_t(C), s));
        return SE_OK;
    }
    if (id_bytes == 4)
        launch_positions(static_cast<const int32_t*>(d_ids), d_offsets, id_base, V, C, Cq, pos, err, s);
    else if (id_bytes == 2)
        launch_positions(static_cast<const uint16_t*>(d_ids), d_offsets, id_base, V, C, Cq, pos, err, s);
    else
        launch_positions(static_cast<const uint8_t*>(d_ids), d_offsets, id_base, V, C, Cq, pos, err, s);
    SE_CHECK_LAUNCH();

    static bool smem_ok = cudaFuncSetAttribute(count_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(kSmem)) == cudaSuccess;
    SE_REQUIRE(smem_ok, SE_ERR_CUDA, "cannot raise the shared-memory limit of the tally kernel");
    CUtensorMap map;
    if (se_status_t st = se::closure::make_map(&map, pos, uint64_t(Cq), uint64_t(V), uint64_t(Cq) * 4, kTile, kVC))
        return st;
    const int64_t tiles = int64_t(R) * (R + 1) / 2;
    // Few tiles and many voters: split the voters so that the grid covers every SM about four
    // times, keeping at least 32 chunks (1024 voters) per range.
    int sms = 0, dev = 0;
    SE_CUDA_TRY(cudaGetDevice(&dev));
    SE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int64_t want = 4 * int64_t(sms);
    const int64_t chunks = (V + kVC - 1) / kVC;
    int splits = 1;
    if (tiles < want) splits = int(std::max<int64_t>(1, std::min<int64_t>((want + tiles - 1) / tiles, chunks / 32)));
    if (splits > 1 && !accumulate)
        SE_CUDA_TRY(cudaMemset2DAsync(d_out, size_t(ld_out) * 4, 0, size_t(C) * 4, size_t(C), s));
    count_kernel<<<unsigned(tiles * splits), kThreads, kSmem, s>>>(map, V, C, R, splits, d_out, ld_out, accumulate,
                                                                   err);
    SE_CHECK_LAUNCH();
    if (!check) return SE_OK;

    uint32_t code = 0;
    SE_CUDA_TRY(cudaMemcpyAsync(&code, err, 4, cudaMemcpyDeviceToHost, s));
    SE_CUDA_TRY(cudaStreamSynchronize(s));
    SE_REQUIRE(code != kErrRange, SE_ERR_DEVICE, "a ballot names a candidate outside [0, %d)", C);
    SE_REQUIRE(code != kErrRepeat, SE_ERR_DEVICE, "a ballot names the same candidate twice");
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
