// Task routines of the persistent closure schedulers (batch.cu: a fixed batch; serve.cu: a
// queue fed while the kernel runs). Every task works on 128 x 128 tiles of one election:
//   SMALL      an election with C <= 128, whole in one CTA: defeat init from d, closure over
//              its C pivots in registers, u32 output, wins and ranking.
//   PIVOT k    close the pivot tile (k, k) in registers; emit dT.
//   ROW k, j   pivot-row panel tile (k, j)       = max(P, D (x) P)
//   COL k, i   pivot-column panel tile (i, k)    = max(P, P (x) D); emit AT (transposed).
//   REM k,i,j  remainder tile (i, j)             = max(S, AT (x) S[k][j])
// Tiles another CTA wrote are read through L2 (ld.global.cg) or TMA, never through L1.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "closure_core.cuh"

namespace se {
namespace batch {
using namespace se::closure;

enum : uint32_t { kSmall = 0, kPivot = 1, kRow = 2, kCol = 3, kRem = 4 };
constexpr uint64_t kNoTask = ~0ull;
constexpr uint32_t kErrTimeout = 1;
constexpr uint32_t kErrOverflow = 2;
constexpr uint32_t kErrDepTimeout = 3;
constexpr uint64_t kDepWaitNs = 5000000000ull;  // 5 s for one dependency

struct alignas(64) Elec {
    CUtensorMap mapS;   // working matrix, box {TW, 32}
    CUtensorMap mapAT;  // transposed column panel, box {128, 32}
    CUtensorMap mapDT;  // transposed pivot tile, box {128, 32}
    const uint32_t* d;
    int64_t ld;
    uint32_t* out;
    int64_t ld_out;
    int32_t* wins;
    int32_t* ranking;
    uint32_t* S;
    uint32_t* AT;
    uint32_t* dT;
    uint32_t* counters;  // [0, R): pivot done; [R, 2R): panels done; [2R, 3R): remainder done
    int32_t C, Cp, R, lanes;
    uint32_t base;  // u16 lanes store a kept value v as v - base (see init_kernel in closure.cu)
};

// Kept defeat value v -> stored u16 cell, or a flagged overflow outside [base+1, base+65535].
__device__ __forceinline__ uint32_t to_lane16(uint32_t v, uint32_t base, bool& over) {
    if (v == 0u) return 0u;
    if (v <= base || v - base > 0xFFFFu) {
        over = true;
        return 0xFFFFu;
    }
    return v - base;
}


__host__ __device__ inline uint64_t pack_task(uint32_t e, uint32_t type, uint32_t k, uint32_t i, uint32_t j) {
    return (uint64_t(e) << 39) | (uint64_t(type) << 36) | (uint64_t(k) << 24) | (uint64_t(i) << 12) | uint64_t(j);
}

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void fence_tensormap(const void* map) {
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

// Thread 0 only: wait until *ctr >= target or the abort flag rises or time runs out.
__device__ inline bool wait_counter(const uint32_t* ctr, uint32_t target, const uint32_t* abort_flag,
                                    uint64_t limit_ns = kDepWaitNs) {
    if (ld_acquire(ctr) >= target) return true;
    const uint64_t t0 = global_ns();
    for (uint32_t it = 0;; ++it) {
        if (ld_acquire(ctr) >= target) return true;
        if ((it & 63) == 0) {
            if (ld_acquire(abort_flag)) return false;
            if (global_ns() - t0 > limit_ns) return false;
        }
        __nanosleep(64);
    }
}

template <int LB> struct pcfg {
    using CF = cfg<LB>;
    static constexpr size_t A_REGION = size_t(kChunks) * CF::A_CHUNK * 4;  // 64 KiB
    static constexpr size_t B_REGION = size_t(kChunks) * CF::B_CHUNK * 4;  // 32 / 64 KiB
    static constexpr size_t SMALL_BYTES = size_t(kT) * (kT + 1) * 4;         // d tile, padded rows
    static constexpr size_t DATA = (A_REGION + B_REGION) > SMALL_BYTES ? (A_REGION + B_REGION) : SMALL_BYTES;
    static constexpr size_t SMEM = DATA + 8 * 8;                              // + 8 mbarriers
};

// ------------------------------------------------------------------------------------------
// SMALL: whole election in this CTA.
// ------------------------------------------------------------------------------------------
template <int LB>
__device__ void run_small(const Elec& E, uint8_t* smem, uint32_t (*rowbuf)[cfg<LB>::TW], uint32_t (*colbuf)[kT],
                          int32_t* s_wins, uint32_t* err) {
    constexpr int CPW = cfg<LB>::CPW;
    constexpr int P = kT + 1;  // padded row pitch: row and column walks are bank-conflict free
    uint32_t* dt = reinterpret_cast<uint32_t*>(smem);
    const int C = E.C;
    const geom g(threadIdx.x);
    for (int idx = threadIdx.x; idx < kT * kT; idx += blockDim.x) {
        const int r = idx / kT, c = idx % kT;
        dt[r * P + c] = (r < C && c < C) ? __ldcg(E.d + int64_t(r) * E.ld + c) : 0u;
    }
    __syncthreads();
    uint32_t c[8][8];
    bool over = false;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = g.row0 + r;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            uint32_t w = 0;
#pragma unroll
            for (int h = 0; h < CPW; ++h) {
                const int j = g.word(q) * CPW + h;
                const uint32_t dij = dt[i * P + j], dji = dt[j * P + i];
                uint32_t v = (i != j && dij > dji) ? dij : 0u;
                if constexpr (LB == 16) {
                    w |= to_lane16(v, E.base, over) << (16 * h);
                } else {
                    w = v;
                }
            }
            c[r][q] = w;
        }
    }
    if (over) raise_device_error(err, kErrOverflow);
    close_tile_in_registers<LB>(c, g, C, rowbuf, colbuf);
    // Output, and the u32 matrix again in shared memory for the ranking.
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = g.row0 + r;
#pragma unroll
        for (int q = 0; q < 8; ++q)
#pragma unroll
            for (int h = 0; h < CPW; ++h) {
                const int j = g.word(q) * CPW + h;
                uint32_t v = LB == 16 ? (c[r][q] >> (16 * h)) & 0xFFFFu : c[r][q];
                if (LB == 16 && v) v += E.base;
                if (i == j) v = 0u;
                dt[i * P + j] = v;
                if (i < C && j < C) E.out[int64_t(i) * E.ld_out + j] = v;
            }
    }
    if (E.wins == nullptr) return;
    __syncthreads();
    const int t = threadIdx.x;
    if (t < C) {
        int w = 0;
        for (int j = 0; j < C; ++j) w += dt[t * P + j] > dt[j * P + t];
        s_wins[t] = w;
        E.wins[t] = w;
    }
    __syncthreads();
    if (t < C) {
        const int wt = s_wins[t];
        int place = 0;
        for (int j = 0; j < C; ++j) {
            const int wj = s_wins[j];
            place += (wj > wt) | ((wj == wt) & (j < t));
        }
        E.ranking[place] = t;
    }
}

// ------------------------------------------------------------------------------------------
// Tile tasks of elections with R >= 2.
// ------------------------------------------------------------------------------------------
template <int LB, int NQ = 8>
__device__ void run_pivot(const Elec& E, int k, uint32_t (*rowbuf)[cfg<LB>::TW], uint32_t (*colbuf)[kT]) {
    using CF = cfg<LB>;
    const geomT<NQ> g(threadIdx.x);
    const int64_t ldw = E.Cp / CF::CPW;
    uint32_t* D = E.S + int64_t(k) * kT * ldw + int64_t(k) * CF::TW;
    uint32_t c[8][NQ];
    load_tile_regs<LB, true, NQ>(c, D, ldw, g);
    const int kmax = E.C - k * kT < kT ? E.C - k * kT : kT;  // pivots past C are zero padding
    close_tile_in_registers<LB, NQ>(c, g, kmax, rowbuf, colbuf);
    store_tile_regs<LB, NQ>(c, D, ldw, g);
    store_transposed_splat<LB, NQ>(c, E.dT, kT, g);
}

// Tile tasks of one pivot round K, all through one routine:
//   kTileRow  S[K][J] = max(S[K][J], D (x) S[K][J]):  A = dT, B = S[K][J] (TMA), C = S[K][J]
//   kTileCol  S[I][K] = max(S[I][K], S[I][K] (x) D):  A = the tile transposed in shared memory,
//             B = D = S[K][K] (TMA), C = S[I][K]; also emits the transposed panel AT[:, I]
//   kTileRem  S[I][J] = max(S[I][J], AT[:, I] (x) S[K][J]):  A = AT (TMA), B = S[K][J] (TMA)
// The (max, min) product, a fully unrolled loop of about 27 KB of code, has a single call site
// here, so every kind of tile task runs the same instructions: with a copy per kind, the rarely
// run panel copies missed in the instruction cache and took about 1.5x a remainder tile.
// E holds the election's scalars (it may be a shared-memory copy); G is the descriptor whose
// tensor maps the TMA unit reads. GLOBAL_MAPS: G lives in global memory and may have been
// rewritten since the last launch (batch and serving queues), so each use first acquires the
// tensor maps; false for a descriptor passed as a kernel parameter. bars[0, 4) use parity
// par_a, bars[4, 8) par_b; both are advanced here.
constexpr int kTileRow = 0;
constexpr int kTileCol = 1;
constexpr int kTileRem = 2;

// Split-K form of a tile task, for tasks on the critical path of a small closure: `parts` CTAs
// each run pivot chunks [q * kChunks / parts, (q + 1) * kChunks / parts) of the product from
// the tile's own cells and store that partial tile to scratch; the last of them to arrive
// folds every partial into its own with a lane-wise max and stores the tile as the unsplit
// task would. Exact: every partial is max(tile, part of the product), and max is associative
// and idempotent. The last part resets the counter for the next use and reports itself in
// `last` (a fused pivot that follows runs in that CTA only).
struct SplitK {
    int q, parts;
    uint32_t* scratch;  // this task's partial tiles, [parts][kT][TW] words
    uint32_t* counter;  // arrivals of this task's parts (0 before the first)
    bool last;
};

// The split-K epilogue of one part (SplitK): stores its partial tile, counts itself, and in the
// last part to arrive folds the other parts' partials into c. Returns whether this part is the
// last (which then stores the tile).
template <int LB, int NQ>
__device__ __forceinline__ bool fold_split(uint32_t (&c)[8][NQ], SplitK* split, const geomT<NQ>& g) {
    using L = lanes<LB>;
    constexpr int TW = cfg<LB>::TW;
    constexpr int64_t kTileWords = int64_t(kT) * TW;
    __shared__ uint32_t s_arrived;
    store_tile_regs<LB, NQ>(c, split->scratch + split->q * kTileWords, TW, g);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_arrived = atomicAdd(split->counter, 1u);
    __syncthreads();
    split->last = s_arrived == uint32_t(split->parts - 1);
    if (!split->last) return false;
    __threadfence();  // the other parts' partials, counted before our arrival, are visible
    for (int p = 0; p < split->parts; ++p) {
        if (p == split->q) continue;
        const uint32_t* src = split->scratch + p * kTileWords;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            uint32_t v[NQ];
            ld4_cg(v, src + int64_t(g.row0 + r) * TW + g.wbase);
            if constexpr (NQ == 8) ld4_cg(v + 4, src + int64_t(g.row0 + r) * TW + g.wbase + 32);
#pragma unroll
            for (int q = 0; q < NQ; ++q) c[r][q] = L::vmax(c[r][q], v[q]);
        }
    }
    if (threadIdx.x == 0) *split->counter = 0u;
    return true;
}

// mapB / kb: where the pivot rows S[K][*] (B of row and remainder tiles, D of column tiles)
// are read: by default G->mapS at row block K; a sharded closure passes the map of a
// received panel buffer (kb = 0) or of its own slab (kb = the local row block).
// kvalid / rvalid: pivots of round K and rows of the tile that lie inside the C candidates
// (by default from K and the tile's row block; a sharded closure, whose K and I are local,
// passes them). Padding holds zeros in both operands, and a cell's relaxation through a zero
// operand leaves it unchanged, so 32-pivot chunks and 32-row warps wholly past C skip the
// product (their copies too), with identical results. On the wide micro-tile, whose warps 4..7
// hold cells 64..127 of their rows, those warps skip it too when the tile's columns past 64 are
// all padding (a column tile's columns are round K's pivots: kvalid; otherwise block J's).
// NQ: words per thread, 8 (the default micro-tile) or 4 (the wide one, 256 threads, 16-bit
// lanes); the block must have tile_threads<LB, NQ>() threads.
// SPLIT / split: the split-K form above, compiled in only where a kernel may split (the whole
// product in this CTA when split is null); without it the routine has no split logic at all.
template <int LB, bool GLOBAL_MAPS = true, int NQ = 8, bool SPLIT = false>
__device__ bool run_tile(const Elec& E, const Elec* G, int kind, int K, int I, int J, uint8_t* smem, uint64_t* bars,
                         uint32_t& par_a, uint32_t& par_b, const CUtensorMap* mapB = nullptr, int kb = -1,
                         int kvalid = -1, int rvalid = -1, SplitK* split = nullptr) {
    using CF = cfg<LB>;
    constexpr int TW = CF::TW;
    uint32_t* As = reinterpret_cast<uint32_t*>(smem);
    uint32_t* Bs = reinterpret_cast<uint32_t*>(smem + pcfg<LB>::A_REGION);
    const geomT<NQ> g(threadIdx.x);
    const int64_t ldw = E.Cp / CF::CPW;
    uint32_t c[8][NQ];
    bool ok = true;
    uint64_t* wait_bars = bars;  // the product's chunk barriers and their parity
    uint32_t wait_par = par_a;
    uint32_t* Ct;
    if (mapB == nullptr) mapB = &G->mapS;
    if (kb < 0) kb = K;
    if (kvalid < 0) kvalid = E.C - K * kT;
    if (rvalid < 0) rvalid = E.C - (kind == kTileRow ? K : I) * kT;
    const int nch = kvalid >= kT ? kChunks : (kvalid + kKC - 1) / kKC;  // chunks holding pivots
    const int cvalid = kind == kTileCol ? kvalid : E.C - J * kT;         // the tile's columns inside C
    // This warp holds real rows and, on the wide micro-tile, real columns.
    const bool live = (g.row0 & ~31) < rvalid && (NQ == 8 || (g.wbase & ~31) * CF::CPW < cvalid);
    // This CTA's chunks [ch_lo, ch_end): all that hold pivots, or its part's share of them.
    int ch_lo = 0, ch_end = nch;
    if constexpr (SPLIT) {
        if (split) {
            ch_lo = split->q * (kChunks / split->parts);
            const int ch_hi = ch_lo + kChunks / split->parts;
            ch_end = nch < ch_hi ? nch : ch_hi;
        }
    }
    if (kind != kTileCol) {
        const bool rem = kind == kTileRem;
        const CUtensorMap* mapA = rem ? &G->mapAT : &G->mapDT;
        if (threadIdx.x == 0) {
            if constexpr (GLOBAL_MAPS) {
                fence_tensormap(mapA);
                fence_tensormap(mapB);
            }
            fence_proxy_async();  // this CTA's earlier shared reads before the TMA rewrites them
#pragma unroll
            for (int ch = 0; ch < kChunks; ++ch) {
                if (ch < ch_lo || ch >= ch_end) {
                    mbar_arrive(&bars[ch]);
                    continue;
                }
                mbar_arrive_expect_tx(&bars[ch], CF::A_BYTES + CF::B_BYTES);
                tma_load_2d(As + ch * CF::A_CHUNK, mapA, &bars[ch], rem ? I * kT : 0, ch * kKC);
                tma_load_2d(Bs + ch * CF::B_CHUNK, mapB, &bars[ch], J * TW, kb * kT + ch * kKC);
            }
        }
        Ct = E.S + int64_t(rem ? I : K) * kT * ldw + int64_t(J) * TW;
        load_tile_regs<LB, true, NQ>(c, Ct, ldw, g);
        par_a ^= 1u;
    } else {
        // The tile itself into Bs, transposed and duplicated into As; then D into Bs.
        if (threadIdx.x == 0) {
            if constexpr (GLOBAL_MAPS) fence_tensormap(&G->mapS);
            fence_proxy_async();
#pragma unroll
            for (int ch = 0; ch < kChunks; ++ch) {
                mbar_arrive_expect_tx(&bars[ch], CF::B_BYTES);
                tma_load_2d(Bs + ch * CF::B_CHUNK, &G->mapS, &bars[ch], K * TW, I * kT + ch * kKC);
            }
        }
#pragma unroll 1
        for (int ch = 0; ch < kChunks; ++ch) ok = ok && mbar_wait_bounded(&bars[ch], par_a, 1u << 26);
        if (ok) {
            constexpr int HALVES = tile_threads<LB, NQ>() / kT;
            constexpr int SPAN = TW / HALVES;
            const int i = threadIdx.x % kT;
            const int half = threadIdx.x / kT;
#pragma unroll 4
            for (int s = 0; s < SPAN; ++s) {
                const int w = half * SPAN + ((s + i) & (SPAN - 1));
                const uint32_t word = Bs[i * TW + w];
#pragma unroll
                for (int h = 0; h < CF::CPW; ++h) As[(w * CF::CPW + h) * kT + i] = cell_splat<LB>(word, h);
            }
            load_tile_regs<LB, false, NQ>(c, Bs, TW, g);
        }
        __syncthreads();  // the tile region is free again
        if (threadIdx.x == 0 && ok) {
            if constexpr (GLOBAL_MAPS) {
                if (mapB != &G->mapS) fence_tensormap(mapB);
            }
            fence_proxy_async();
#pragma unroll
            for (int ch = 0; ch < kChunks; ++ch) {
                if (ch < ch_lo || ch >= ch_end) {
                    mbar_arrive(&bars[kChunks + ch]);
                    continue;
                }
                mbar_arrive_expect_tx(&bars[kChunks + ch], CF::B_BYTES);
                tma_load_2d(Bs + ch * CF::B_CHUNK, mapB, &bars[kChunks + ch], K * TW, kb * kT + ch * kKC);
            }
        }
        Ct = E.S + int64_t(I) * kT * ldw + int64_t(K) * TW;
        wait_bars = bars + kChunks;
        wait_par = par_b;
        par_a ^= 1u;
        par_b ^= 1u;
    }
    if (ok) {
        // Chunks outside [ch_lo, ch_end): thread 0 completed their phases without a copy;
        // nobody waits.
#pragma unroll 1
        for (int ch = ch_lo; ch < ch_end; ++ch) {
            if (!mbar_wait_bounded(&wait_bars[ch], wait_par, 1u << 26)) {
                ok = false;
                break;
            }
            if (live) relax_chunk<LB, NQ>(c, As + ch * CF::A_CHUNK, Bs + ch * CF::B_CHUNK, g);
        }
    }
    if constexpr (SPLIT) {
        if (ok && split != nullptr) {
            if (!fold_split<LB, NQ>(c, split, g)) return ok;  // an earlier part: the last one stores
        }
    }
    if (ok) {
        store_tile_regs<LB, NQ>(c, Ct, ldw, g);
        if (kind == kTileCol) store_transposed_splat<LB, NQ>(c, E.AT + int64_t(I) * kT, E.Cp, g);
    }
    return ok;
}

}  // namespace batch
}  // namespace se
