// Device building blocks shared by the single-election closure (closure.cu) and the batched
// persistent closure (batch.cu): tile geometry, the register-blocked (max, min) product over
// TMA-staged shared operands, the in-register pivot-tile closure, and tile load/store.
#pragma once

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace se {
namespace closure {

constexpr int kT = 128;             // pivot block edge = tile edge, in cells
constexpr int kKC = 32;             // k-rows per TMA chunk
constexpr int kChunks = kT / kKC;   // chunks per tile
constexpr uint32_t kErrTmaTimeout = 1;

template <int LB> struct cfg {
    static constexpr int CPW = 32 / LB;               // cells per 32-bit word
    static constexpr int TW = kT / CPW;               // words per tile row: 64 (u16) / 128 (u32)
    static constexpr int WN = TW / 64;                // warps across a tile row
    static constexpr int THREADS = 32 * 4 * WN;       // 128 (u16) / 256 (u32)
    static constexpr int A_CHUNK = kKC * kT;          // words of one A chunk (k-major, 128 rows)
    static constexpr int B_CHUNK = kKC * TW;          // words of one B chunk
    static constexpr uint32_t A_BYTES = A_CHUNK * 4;
    static constexpr uint32_t B_BYTES = B_CHUNK * 4;
    // tile_kernel: all of K resident (no ring), one mbarrier per chunk.
    static constexpr size_t TILE_SMEM = size_t(kChunks) * (A_CHUNK + B_CHUNK) * 4 + kChunks * 8;
    // col_panel_kernel: the panel tile, its transposed-duplicated copy, and D.
    static constexpr size_t COL_SMEM = size_t(kT) * TW * 4 * 2 + size_t(kT) * kT * 4 + 2 * kChunks * 8;
};

// Thread geometry shared by every kernel of one lane mode: warp (wm, wn) of a 4 x WN grid,
// lane (tr, tc) of a 4 x 8 grid. With NQ = 8 words per thread (the default micro-tile) the
// thread owns rows row0 .. row0+7 and words wbase .. wbase+3 and wbase+32 .. wbase+35 of the
// tile, so the 8 threads of a row group read 128 contiguous bytes of B per shared load, and 4
// row groups read 4 disjoint bank groups of A. With NQ = 4 (16-bit lanes only: the wide
// micro-tile, 256 threads) warps 4..7 take words 32..63 and the thread owns words
// wbase .. wbase+3 of its rows: twice the warps on one tile, for tiles that run alone on an SM
// (pivot and panels), where four warps leave every scheduler with one warp and stall on
// instruction latency.
template <int NQ = 8> struct geomT {
    static_assert(NQ == 8 || NQ == 4, "8 or 4 words per thread");
    int row0, wbase;
    __device__ __forceinline__ explicit geomT(int tid) {
        const int warp = tid >> 5, lane = tid & 31;
        row0 = (warp & 3) * 32 + (lane >> 3) * 8;
        wbase = (warp >> 2) * (NQ == 8 ? 64 : 32) + (lane & 7) * 4;
    }
    __device__ __forceinline__ int word(int q) const { return wbase + (q < 4 ? q : 28 + q); }
};
using geom = geomT<8>;

// Threads of a CTA that holds one tile in lane mode LB with NQ words per thread.
template <int LB, int NQ> constexpr int tile_threads() {
    static_assert(NQ == 8 || LB == 16, "the wide micro-tile is for 16-bit lanes");
    return NQ == 8 ? cfg<LB>::THREADS : 256;
}

__device__ __forceinline__ void ld4(uint32_t* dst, const uint32_t* src) {
    const uint4 v = *reinterpret_cast<const uint4*>(src);
    dst[0] = v.x, dst[1] = v.y, dst[2] = v.z, dst[3] = v.w;
}
__device__ __forceinline__ void st4(uint32_t* dst, const uint32_t* src) {
    *reinterpret_cast<uint4*>(dst) = make_uint4(src[0], src[1], src[2], src[3]);
}

// Extract cell h (0 = low half) of a word and duplicate it across the word.
template <int LB> __device__ __forceinline__ uint32_t cell_splat(uint32_t w, int h);
template <> __device__ __forceinline__ uint32_t cell_splat<32>(uint32_t w, int) { return w; }
template <> __device__ __forceinline__ uint32_t cell_splat<16>(uint32_t w, int h) {
    return __byte_perm(w, 0, h ? 0x3232 : 0x1010);
}

// 128-bit global load that bypasses L1: for data another CTA of the same launch wrote.
__device__ __forceinline__ void ld4_cg(uint32_t* dst, const uint32_t* src) {
    const uint4 v = __ldcg(reinterpret_cast<const uint4*>(src));
    dst[0] = v.x, dst[1] = v.y, dst[2] = v.z, dst[3] = v.w;
}

template <int LB, bool COHERENT = false, int NQ = 8>
__device__ __forceinline__ void load_tile_regs(uint32_t (&c)[8][NQ], const uint32_t* base, int64_t ldw,
                                               const geomT<NQ>& g) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const uint32_t* p = base + int64_t(g.row0 + r) * ldw + g.wbase;
        if constexpr (COHERENT) {
            ld4_cg(&c[r][0], p);
            if constexpr (NQ == 8) ld4_cg(&c[r][4], p + 32);
        } else {
            ld4(&c[r][0], p);
            if constexpr (NQ == 8) ld4(&c[r][4], p + 32);
        }
    }
}

template <int LB, int NQ = 8>
__device__ __forceinline__ void store_tile_regs(const uint32_t (&c)[8][NQ], uint32_t* base, int64_t ldw,
                                                const geomT<NQ>& g) {
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        uint32_t* p = base + int64_t(g.row0 + r) * ldw + g.wbase;
        st4(p, &c[r][0]);
        if constexpr (NQ == 8) st4(p + 32, &c[r][4]);
    }
}

// One K-chunk of the semiring product: c = max(c, max_k min(A[k][row], B[k][word])).
// A is k-major [kKC][kT] (duplicated cells in u16 mode), B is [kKC][TW].
// The k loop is unrolled 4 pairs deep (about 6.6 KB of code instead of 27 KB fully unrolled):
// the loop overhead is negligible beside 416 instructions per iteration, and the smaller body
// stays in the instruction cache even in the persistent kernels, whose CTAs run several task
// routines side by side on one SM.
template <int LB, int NQ = 8>
__device__ __forceinline__ void relax_chunk(uint32_t (&c)[8][NQ], const uint32_t* __restrict__ As,
                                            const uint32_t* __restrict__ Bs, const geomT<NQ>& g) {
    using L = lanes<LB>;
    constexpr int TW = cfg<LB>::TW;
#pragma unroll 4
    for (int k = 0; k < kKC; k += 2) {
        uint32_t a0[8], a1[8], b0[NQ], b1[NQ];
        ld4(a0, As + k * kT + g.row0);
        ld4(a0 + 4, As + k * kT + g.row0 + 4);
        ld4(a1, As + (k + 1) * kT + g.row0);
        ld4(a1 + 4, As + (k + 1) * kT + g.row0 + 4);
        ld4(b0, Bs + k * TW + g.wbase);
        if constexpr (NQ == 8) ld4(b0 + 4, Bs + k * TW + g.wbase + 32);
        ld4(b1, Bs + (k + 1) * TW + g.wbase);
        if constexpr (NQ == 8) ld4(b1 + 4, Bs + (k + 1) * TW + g.wbase + 32);
#pragma unroll
        for (int r = 0; r < 8; ++r)
#pragma unroll
            for (int q = 0; q < NQ; ++q)
                c[r][q] = L::vmax3(c[r][q], L::vmin(a0[r], b0[q]), L::vmin(a1[r], b1[q]));
    }
}

// Writes the thread's cells transposed and duplicated: out[k][row] for every cell (row, k)
// it holds; out is k-major with row stride ld_out words.
template <int LB, int NQ = 8>
__device__ __forceinline__ void store_transposed_splat(const uint32_t (&c)[8][NQ], uint32_t* out,
                                                       int64_t ld_out, const geomT<NQ>& g) {
    constexpr int CPW = cfg<LB>::CPW;
#pragma unroll
    for (int q = 0; q < NQ; ++q)
#pragma unroll
        for (int h = 0; h < CPW; ++h) {
            const int k = g.word(q) * CPW + h;
            uint32_t v[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) v[r] = cell_splat<LB>(c[r][q], h);
            uint32_t* p = out + int64_t(k) * ld_out + g.row0;
            st4(p, v);
            st4(p + 4, v + 4);
        }
}

// Rows of the pivot-closure staging buffers (rowbuf[kPivotBufs][TW], colbuf[kPivotBufs][kT]):
// two phases, each holding the rows and columns of two pivots.
constexpr int kPivotBufs = 4;

// Publishes row k8 + J and column k8 + J of the tile into staging slot (row, col), for k8 a
// multiple of 8 and J < 8 known at compile time. Row k8 + J is register row J of the threads
// whose row0 is k8; column k8 + J is cell J % CPW of word (J / CPW) % 4 of a 4-word group,
// held by the threads whose wbase (or wbase + 32) starts that group. So one uniform test per
// row and per column group decides the stores, and the registers are indexed statically.
// Indices past the tile (k8 = 128) match no thread.
template <int LB, int NQ, int J>
__device__ __forceinline__ void publish_pivot8(const uint32_t (&c)[8][NQ], const geomT<NQ>& g, int k8, uint32_t* row,
                                               uint32_t* col) {
    constexpr int CPW = cfg<LB>::CPW;
    constexpr int QW = (J / CPW) & 3, H = J % CPW;
    if (g.row0 == k8) {
        st4(row + g.wbase, &c[J][0]);
        if constexpr (NQ == 8) st4(row + g.wbase + 32, &c[J][4]);
    }
    const int w4 = ((k8 + J) / CPW) & ~3;
    auto put_col = [&](int q) {
        uint32_t v[8];
#pragma unroll
        for (int r = 0; r < 8; ++r) v[r] = cell_splat<LB>(c[r][q], H);
        st4(col + g.row0, v);
        st4(col + g.row0 + 4, v + 4);
    };
    if (g.wbase == w4) put_col(QW);
    if constexpr (NQ == 8) {
        if (g.wbase + 32 == w4) put_col(4 + QW);
    }
}

// Pivots k = k8 + J and k + 1 (J even, known at compile time) from staging slots s, s + 1,
// then the publish of k + 2 and k + 3 into the other phase's slots and one barrier.
template <int LB, int NQ, int J>
__device__ __forceinline__ void pivot_pair(uint32_t (&c)[8][NQ], const geomT<NQ>& g, int k8,
                                           uint32_t (*rowbuf)[cfg<LB>::TW], uint32_t (*colbuf)[kT]) {
    using L = lanes<LB>;
    constexpr int CPW = cfg<LB>::CPW;
    constexpr int s = ((J >> 1) & 1) * 2, t = s ^ 2;
    uint32_t a0[8], b0[NQ], a1[8], b1[NQ];
    ld4(a0, &colbuf[s][g.row0]);
    ld4(a0 + 4, &colbuf[s][g.row0 + 4]);
    ld4(b0, &rowbuf[s][g.wbase]);
    if constexpr (NQ == 8) ld4(b0 + 4, &rowbuf[s][g.wbase + 32]);
    ld4(a1, &colbuf[s + 1][g.row0]);
    ld4(a1 + 4, &colbuf[s + 1][g.row0 + 4]);
    ld4(b1, &rowbuf[s + 1][g.wbase]);
    if constexpr (NQ == 8) ld4(b1 + 4, &rowbuf[s + 1][g.wbase + 32]);
    const uint32_t ckk1 = cell_splat<LB>(rowbuf[s][k8 / CPW + (J + 1) / CPW], (J + 1) % CPW);  // c[k][k+1]
    const uint32_t ck1k = colbuf[s][k8 + J + 1];                                             // c[k+1][k]
#pragma unroll
    for (int r = 0; r < 8; ++r) a1[r] = L::vmax(a1[r], L::vmin(a0[r], ckk1));
#pragma unroll
    for (int q = 0; q < NQ; ++q) b1[q] = L::vmax(b1[q], L::vmin(ck1k, b0[q]));
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int q = 0; q < NQ; ++q) c[r][q] = L::vmax3(c[r][q], L::vmin(a0[r], b0[q]), L::vmin(a1[r], b1[q]));
    if constexpr (J + 2 < 8) {
        publish_pivot8<LB, NQ, J + 2>(c, g, k8, rowbuf[t], colbuf[t]);
        publish_pivot8<LB, NQ, J + 3>(c, g, k8, rowbuf[t + 1], colbuf[t + 1]);
    } else {
        publish_pivot8<LB, NQ, 0>(c, g, k8 + 8, rowbuf[t], colbuf[t]);
        publish_pivot8<LB, NQ, 1>(c, g, k8 + 8, rowbuf[t + 1], colbuf[t + 1]);
    }
    __syncthreads();
}

// Closes the 128 x 128 tile held in registers (the thread's 8 x NQ words) in place over its
// first kmax pivots, two at a time. Rows and columns k and k+1 are published together (before
// this pair's steps) through double-buffered shared slots, one barrier per pair. Each thread
// applies step k to the row and column k+1 it reads:
//   c'[i][k+1] = max(c[i][k+1], min(c[i][k], c[k][k+1]))
//   c'[k+1][j] = max(c[k+1][j], min(c[k+1][k], c[k][j]))
// and then does both steps in one pass over its words:
//   c[i][j] = max(c[i][j], min(c[i][k], c[k][j]), min(c'[i][k+1], c'[k+1][j]))
// which is exactly two Floyd-Warshall steps. The pivot loop runs in groups of 8, so kmax is
// rounded up to a multiple of 8: the extra pivots' rows and columns are zero padding, and a
// step over a zero row and column changes nothing. Every thread of the block must call it.
template <int LB, int NQ = 8>
__device__ __forceinline__ void close_tile_in_registers(uint32_t (&c)[8][NQ], const geomT<NQ>& g, int kmax,
                                                        uint32_t (*rowbuf)[cfg<LB>::TW],
                                                        uint32_t (*colbuf)[kT]) {
    const int kend = kmax >= kT ? kT : (kmax + 7) & ~7;
    publish_pivot8<LB, NQ, 0>(c, g, 0, rowbuf[0], colbuf[0]);
    publish_pivot8<LB, NQ, 1>(c, g, 0, rowbuf[1], colbuf[1]);
    __syncthreads();
#pragma unroll 1
    for (int k8 = 0; k8 < kend; k8 += 8) {
        pivot_pair<LB, NQ, 0>(c, g, k8, rowbuf, colbuf);
        pivot_pair<LB, NQ, 2>(c, g, k8, rowbuf, colbuf);
        pivot_pair<LB, NQ, 4>(c, g, k8, rowbuf, colbuf);
        pivot_pair<LB, NQ, 6>(c, g, k8, rowbuf, colbuf);
    }
}

// 2-D u32 tensor map over this GPU's memory: dims {inner, outer} words, row pitch in bytes,
// box {box_x, box_y}. Defined in closure.cu.
se_status_t make_map(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint64_t pitch_bytes,
                     uint32_t box_x, uint32_t box_y);

// Defeat init of one election into a padded working matrix; defined in closure.cu.
se_status_t launch_defeat_init(const uint32_t* d, int64_t ld, int C, int Cp, void* S, int lane_bits, uint32_t base,
                               uint32_t* flags, cudaStream_t s);

}  // namespace closure
}  // namespace se
