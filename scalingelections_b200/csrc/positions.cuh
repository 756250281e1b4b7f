// Places of the candidates on one ballot, computed by one warp: the first step of the tally
// (build_pairwise_preferences, scaling_elections.py:51-88), shared by the tally kernels
// (tally.cu) and the serving engine's POS tasks (serve.cu).
//
// p[c] = place of candidate c on ballot r[0 .. len), as f32 (exact integers), for c < C; the
// padding p[C .. Cq) is 0. A ballot that omits candidates is completed by the reference's
// rule: the missing ids take places len, len + 1, ... in ascending id order (py:75-83). Every
// step is a warp-strided loop with warp barriers only, so a CTA works on several ballots at once
// (one per warp) and keeps many loads in flight. A complete ballot (len == C) needs no
// initialisation pass: its scatter writes every place once, and a repeated id (the only way a
// valid-looking complete ballot can miss a candidate) is caught by the check.
#pragma once

#include <stdint.h>

namespace se {

// Bit planes of places (the bit-sliced tally): places are below C, so B = bits of C - 1 planes
// (at least one) hold them; kMaxPlanes covers C <= 2^20.
constexpr int kMaxPlanes = 20;

__host__ __device__ inline int planes_for(int C) {
    int b = 0;
    for (uint32_t x = uint32_t(C > 1 ? C - 1 : 1); x; x >>= 1) ++b;
    return b;
}

constexpr int kPosOk = 0;
constexpr int kPosRange = 2;   // an id outside [0, C)
constexpr int kPosRepeat = 3;  // the same id twice

// COHERENT: read the ballot and the places through L2 (ld.global.cg). A persistent kernel needs
// this: its SM's L1 may still hold lines of an earlier request that used the same addresses.
template <bool COHERENT, typename T>
__device__ __forceinline__ T pos_load(const T* p) {
    if constexpr (COHERENT) return __ldcg(p);
    else return *p;
}

template <typename Id, bool COHERENT = false>
__device__ __forceinline__ int warp_positions(const Id* __restrict__ r, int64_t len, int C, int64_t Cq,
                                              float* __restrict__ p) {
    const int lane = threadIdx.x & 31;
    const bool complete = len >= C;
    for (int64_t c = complete ? C + lane : lane; c < Cq; c += 32) p[c] = c < C ? -1.0f : 0.0f;
    __syncwarp();
    int bad = 0;
#pragma unroll 4
    for (int64_t a = lane; a < len; a += 32) {
        const int64_t id = int64_t(pos_load<COHERENT>(r + a));
        if (id < 0 || id >= C) bad = 1;
        else p[id] = float(a);
    }
    if (__any_sync(0xffffffffu, bad)) return kPosRange;
    __syncwarp();  // the scatter's stores are visible to the whole warp
#pragma unroll 4
    for (int64_t a = lane; a < len; a += 32)
        if (pos_load<COHERENT>(p + int64_t(pos_load<COHERENT>(r + a))) != float(a))
            bad = 1;  // a repeated id left at most one of its places
    if (__any_sync(0xffffffffu, bad)) return kPosRepeat;
    if (complete) return kPosOk;
    // Missing ids (still -1) in ascending order: a ballot-and-popcount scan, 32 candidates a step.
    int64_t base = len;
    for (int64_t c0 = 0; c0 < C; c0 += 32) {
        const int64_t c = c0 + lane;
        const bool miss = c < C && pos_load<COHERENT>(p + c) < 0.0f;
        const uint32_t m = __ballot_sync(0xffffffffu, miss);
        if (miss) p[c] = float(base + __popc(m & ((1u << lane) - 1u)));
        base += __popc(m);
    }
    return kPosOk;
}

// The same places as 16-bit values in a row of shared memory (C < 65535, so every place fits),
// with 0xFFFF marking a missing id during the completion scan. Same checks and codes: with
// every id in range, a ballot longer than C must repeat one. COHERENT: read the ballot
// through L2, as warp_positions does.
template <typename Id, bool COHERENT = false>
__device__ __forceinline__ int warp_places_u16(const Id* __restrict__ r, int64_t len, int C, int Cq,
                                               uint16_t* __restrict__ p) {
    const int lane = threadIdx.x & 31;
    const bool complete = len >= C;
    for (int c = complete ? C + lane : lane; c < Cq; c += 32) p[c] = c < C ? uint16_t(0xFFFF) : uint16_t(0);
    __syncwarp();
    int bad = 0;
#pragma unroll 4
    for (int64_t a = lane; a < len; a += 32) {
        const int64_t id = int64_t(pos_load<COHERENT>(r + a));
        if (id < 0 || id >= C) bad = 1;
        else if (len <= C) p[id] = uint16_t(a);
    }
    if (__any_sync(0xffffffffu, bad)) return kPosRange;
    if (len > C) return kPosRepeat;
    __syncwarp();
#pragma unroll 4
    for (int64_t a = lane; a < len; a += 32)
        if (p[int64_t(pos_load<COHERENT>(r + a))] != uint16_t(a)) bad = 1;
    if (__any_sync(0xffffffffu, bad)) return kPosRepeat;
    if (complete) return kPosOk;
    int base = int(len);
    for (int c0 = 0; c0 < C; c0 += 32) {
        const int c = c0 + lane;
        const bool miss = c < C && p[c] == uint16_t(0xFFFF);
        const uint32_t m = __ballot_sync(0xffffffffu, miss);
        if (miss) p[c] = uint16_t(base + __popc(m & ((1u << lane) - 1u)));
        base += __popc(m);
    }
    return kPosOk;
}

// The same for one ballot per CTA (all blockDim.x threads, a multiple of 32, at most 1024):
// for long ballots, where one warp per ballot leaves too few warps in flight. Every thread of
// the block must call it with the same ballot. scratch: 32 + 1 ints of shared memory.
template <typename Id>
__device__ __forceinline__ int block_positions(const Id* __restrict__ r, int64_t len, int C, int64_t Cq,
                                               float* __restrict__ p, int* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool complete = len >= C;
    for (int64_t c = complete ? C + threadIdx.x : threadIdx.x; c < Cq; c += blockDim.x) p[c] = c < C ? -1.0f : 0.0f;
    __syncthreads();
    int bad = 0;
#pragma unroll 4
    for (int64_t a = threadIdx.x; a < len; a += blockDim.x) {
        const int64_t id = int64_t(r[a]);
        if (id < 0 || id >= C) bad = 1;
        else p[id] = float(a);
    }
    if (__syncthreads_or(bad)) return kPosRange;
#pragma unroll 4
    for (int64_t a = threadIdx.x; a < len; a += blockDim.x)
        if (p[int64_t(r[a])] != float(a)) bad = 1;
    if (__syncthreads_or(bad)) return kPosRepeat;
    if (complete) return kPosOk;
    // Missing ids in ascending order: a block-wide exclusive scan of the "missing" flags.
    int* warp_sums = scratch;
    int64_t base = len;
    for (int64_t c0 = 0; c0 < C; c0 += blockDim.x) {
        const int64_t c = c0 + threadIdx.x;
        const bool miss = c < C && p[c] < 0.0f;
        const uint32_t m = __ballot_sync(0xffffffffu, miss);
        if (lane == 0) warp_sums[warp] = __popc(m);
        __syncthreads();
        int before = __popc(m & ((1u << lane) - 1u)), total = 0;
        for (int w = 0; w < nw; ++w) {
            const int x = warp_sums[w];
            before += w < warp ? x : 0;
            total += x;
        }
        if (miss) p[c] = float(base + before);
        base += total;
        __syncthreads();
    }
    return kPosOk;
}

// block_positions with the place row in shared memory as 16-bit values (C < 65535; the
// caller provides Cq halfwords of p): the scatter and the repeat check stay on the SM, and the
// finished row goes out to `out` as f32 with coalesced stores. Same checks and codes.
template <typename Id>
__device__ __forceinline__ int block_places_u16(const Id* __restrict__ r, int64_t len, int C, int Cq,
                                                uint16_t* __restrict__ p, float* __restrict__ out, int* scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const bool complete = len >= C;
    for (int c = complete ? C + threadIdx.x : threadIdx.x; c < Cq; c += blockDim.x)
        p[c] = c < C ? uint16_t(0xFFFF) : uint16_t(0);
    __syncthreads();
    int bad = 0;
#pragma unroll 4
    for (int64_t a = threadIdx.x; a < len; a += blockDim.x) {
        const int64_t id = int64_t(r[a]);
        if (id < 0 || id >= C) bad = 1;
        else if (len <= C) p[id] = uint16_t(a);
    }
    if (__syncthreads_or(bad)) return kPosRange;
    if (len > C) return kPosRepeat;  // every id is in range, so one repeats
#pragma unroll 4
    for (int64_t a = threadIdx.x; a < len; a += blockDim.x)
        if (p[int64_t(r[a])] != uint16_t(a)) bad = 1;
    if (__syncthreads_or(bad)) return kPosRepeat;
    if (!complete) {  // missing ids in ascending order: a block-wide exclusive scan
        int* warp_sums = scratch;
        int base = int(len);
        for (int c0 = 0; c0 < C; c0 += blockDim.x) {
            const int c = c0 + threadIdx.x;
            const bool miss = c < C && p[c] == uint16_t(0xFFFF);
            const uint32_t m = __ballot_sync(0xffffffffu, miss);
            if (lane == 0) warp_sums[warp] = __popc(m);
            __syncthreads();
            int before = __popc(m & ((1u << lane) - 1u)), total = 0;
            for (int w = 0; w < nw; ++w) {
                const int x = warp_sums[w];
                before += w < warp ? x : 0;
                total += x;
            }
            if (miss) p[c] = uint16_t(base + before);
            base += total;
            __syncthreads();
        }
    }
    __syncthreads();
    for (int c = threadIdx.x; c < Cq; c += blockDim.x) out[c] = float(p[c]);
    return kPosOk;
}

}  // namespace se
