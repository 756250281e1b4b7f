// One election's closure sharded across GPUs by row blocks (no reference counterpart: the
// reference closes one matrix on one GPU, scaling_elections.cu:490-578).
//
// A shard holds the row blocks [b0, b1) of the padded working matrix (its slab). Pivot round k
// has one exchange: the owner of row block k closes the pivot tile and updates its pivot-row
// panel S[k][*] (tiles (k, J) = max(S[k][J], D (x) S[k][J])); the caller then broadcasts that
// 128 x Cp panel (e.g. NCCL over NVLink) into every other shard's panel buffer. Each shard then
// updates only its own rows: the column-panel tiles (I, k) = max(S[I][k], S[I][k] (x) D), D read
// from the panel, and the remainder tiles (I, J) = max(S[I][J], S[I][k] (x) S[k][J]), S[k][*]
// read from the panel. These are the same three blocked Floyd-Warshall phases as the single-GPU
// closure, run through the same tile routine (batch_core.cuh). The remainder, nearly all of the
// work, splits evenly across shards, and the panel crosses the links once per round. The panel
// lands in local memory before any TMA load reads it: no load reads another GPU's memory.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <new>

#include "batch_core.cuh"

namespace se {
namespace shard {
using namespace se::closure;
using namespace se::batch;

// Defeat init of the slab rows [row0, row0 + nrows) from the full C x C matrix d (see
// init_kernel in closure.cu): S[i][j] = d[i][j] if d[i][j] > d[j][i], else 0; 16-bit lanes
// store v - base. Grid: (Cp / 32, nrows / 32) blocks of 32 x 8 threads.
template <int LB>
__global__ void __launch_bounds__(256)
    shard_init_kernel(const uint32_t* __restrict__ d, int64_t ld, int C, int Cp, int row0, void* __restrict__ Sv,
                      uint32_t base, uint32_t* __restrict__ err) {
    __shared__ uint32_t t[32][33];
    const int bx = blockIdx.x * 32, by = row0 + blockIdx.y * 32;  // S[by.., bx..], global rows
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = bx + y, cc = by + threadIdx.x;
        t[threadIdx.x][y] = (r < C && cc < C) ? d[int64_t(r) * ld + cc] : 0u;
    }
    __syncthreads();
    bool over = false;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int i = by + y, j = bx + threadIdx.x;
        uint32_t v = 0;
        if (i < C && j < C && i != j) {
            const uint32_t dij = d[int64_t(i) * ld + j];
            v = dij > t[y][threadIdx.x] ? dij : 0u;
        }
        const int64_t at = int64_t(i - row0) * Cp + j;
        if constexpr (LB == 16) static_cast<uint16_t*>(Sv)[at] = uint16_t(to_lane16(v, base, over));
        else static_cast<uint32_t*>(Sv)[at] = v;
    }
    if (over) raise_device_error(err, kErrOverflow);
}

// The owner's pivot tile S[k][k] (local row block kl): closed in place over its kmax real
// pivots, and emitted transposed and duplicated into dT for the row panel.
template <int LB>
__global__ void __launch_bounds__(cfg<LB>::THREADS, 1)
    shard_pivot_kernel(uint32_t* __restrict__ S, int64_t ldw, int kl, int k, int kmax, uint32_t* __restrict__ dT) {
    using CF = cfg<LB>;
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    const geom g(threadIdx.x);
    uint32_t c[8][8];
    uint32_t* D = S + int64_t(kl) * kT * ldw + int64_t(k) * CF::TW;
    load_tile_regs<LB>(c, D, ldw, g);
    close_tile_in_registers<LB>(c, g, kmax, rowbuf, colbuf);
    store_tile_regs<LB>(c, D, ldw, g);
    store_transposed_splat<LB>(c, dT, kT, g);
}

constexpr int kPhaseRowPanel = 0;
constexpr int kPhaseColPanel = 1;
constexpr int kPhaseRemainder = 2;

// The local row block of the b-th row the column-panel and remainder phases update: `only`
// >= 0 selects that row block alone; otherwise every local row block but kl (when own) and
// `skip` (when >= 0), in order.
__device__ __forceinline__ int selected_row(int b, int own, int kl, int only, int skip) {
    if (only >= 0) return only;
    int lo = own ? kl : -1, hi = skip;
    if (lo > hi) {
        const int t = lo;
        lo = hi;
        hi = t;
    }
    if (lo >= 0 && b >= lo) ++b;
    if (hi >= 0 && b >= hi) ++b;
    return b;
}

// One phase of round k on the slab. E describes the slab: S is its first row, mapS covers its
// rows, AT is indexed by local row block; b0 is the slab's first global row block. own: this
// shard holds row block k (local kl), so the
// pivot rows are read from its own slab; otherwise from the panel buffer (mapP, row block 0).
// only / skip: the rows the column-panel and remainder phases update (selected_row).
// fuse_next >= 0 (remainder phase only): this shard also holds row block k + 1, at local index
// fuse_next, and updates it in this launch. Block 0 then takes tile (k+1, k+1) and, after
// updating it, closes it as round k+1's pivot over kmax_next pivots and writes dT, while the
// other blocks go on: the next round's se_shard_pivot needs only its row panel. Nothing else
// in this launch reads that tile or dT.
template <int LB>
__global__ void __launch_bounds__(cfg<LB>::THREADS, 1)
    shard_tiles_kernel(const __grid_constant__ Elec E, const __grid_constant__ CUtensorMap mapP, int phase, int k,
                       int kl, int b0, int own, int only, int skip, int fuse_next, int kmax_next,
                       uint32_t* __restrict__ err) {
    using CF = cfg<LB>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + pcfg<LB>::DATA);
    if (threadIdx.x == 0) {
        for (int c = 0; c < 2 * kChunks; ++c) mbar_init(&bars[c], 1);
        fence_barrier_init();
    }
    __syncthreads();
    const CUtensorMap* mapB = own ? &E.mapS : &mapP;
    const int kb = own ? kl : 0;
    int b = blockIdx.x;
    const bool fuse = phase == kPhaseRemainder && fuse_next >= 0;
    if (fuse) {
        // Reduced coordinates of tile (k+1, k+1): its position among the selected rows (rows
        // without kl, or the one row `only`), columns without k.
        const int row = only >= 0 ? 0 : (own && fuse_next > kl ? fuse_next - 1 : fuse_next);
        const int p = row * (E.R - 1) + k;
        b = b == 0 ? p : (b == p ? 0 : b);
    }
    int kind, K = k, I = 0, J = 0;
    if (phase == kPhaseRowPanel) {  // owner only: tiles (k, J != k) of its row block kl
        kind = kTileRow;
        K = kl;
        J = b + (b >= k);
    } else if (phase == kPhaseColPanel) {  // the selected local row blocks (never k)
        kind = kTileCol;
        I = selected_row(b, own, kl, only, skip);
    } else {
        kind = kTileRem;
        const int R1 = E.R - 1;
        const int ii = b / R1, jj = b % R1;
        I = selected_row(ii, own, kl, only, skip);
        J = jj + (jj >= k);
    }
    uint32_t pa = 0, pb = 0;
    const int rblock = kind == kTileRow ? k : b0 + I;  // the tile's global row block
    const bool ok = run_tile<LB, false>(E, &E, kind, K, I, J, smem, bars, pa, pb, mapB, kb, E.C - k * kT,
                                        E.C - rblock * kT);
    if (!ok) {
        if (threadIdx.x == 0) raise_device_error(err, kErrTmaTimeout);
        return;
    }
    if (fuse && blockIdx.x == 0) {
        __syncthreads();  // the tile's stores are visible to the whole CTA
        const geom g(threadIdx.x);
        const int64_t ldw = E.Cp / CF::CPW;
        uint32_t* D = E.S + int64_t(fuse_next) * kT * ldw + int64_t(k + 1) * CF::TW;
        uint32_t c[8][8];
        load_tile_regs<LB, true>(c, D, ldw, g);
        close_tile_in_registers<LB>(c, g, kmax_next, rowbuf, colbuf);
        store_tile_regs<LB>(c, D, ldw, g);
        store_transposed_splat<LB>(c, E.dT, kT, g);
    }
}

// out rows [0, nrows) = global rows row0.. of the closure as u32, zero on the diagonal.
template <int LB>
__global__ void __launch_bounds__(256)
    shard_finalize_kernel(const void* __restrict__ Sv, int Cp, int C, int row0, int nrows, uint32_t* __restrict__ out,
                          int64_t ld_out, uint32_t base) {
    for (int il = blockIdx.y; il < nrows; il += gridDim.y)
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < C; j += gridDim.x * blockDim.x) {
            uint32_t v;
            if constexpr (LB == 16) {
                v = static_cast<const uint16_t*>(Sv)[int64_t(il) * Cp + j];
                v = v ? v + base : 0u;
            } else {
                v = static_cast<const uint32_t*>(Sv)[int64_t(il) * Cp + j];
            }
            out[int64_t(il) * ld_out + j] = (row0 + il == j) ? 0u : v;
        }
}

struct Layout {
    int64_t s_off, at_off, dt_off, p_off, total, panel_bytes;  // p_off: two panel buffers (round parity)
};

Layout layout(int C, int b0, int b1, int lanes) {
    const int64_t Cp = round_up(int64_t(C), kT);
    const int64_t cell = lanes == 16 ? 2 : 4;
    Layout L;
    L.s_off = 256;
    L.at_off = round_up(L.s_off + int64_t(b1 - b0) * kT * Cp * cell, 256);
    L.dt_off = round_up(L.at_off + int64_t(kT) * Cp * 4, 256);
    L.p_off = round_up(L.dt_off + int64_t(kT) * kT * 4, 256);
    L.panel_bytes = int64_t(kT) * Cp * cell;
    L.total = round_up(L.p_off + 2 * L.panel_bytes, 256);
    return L;
}

template <int LB> se_status_t set_smem() {
    return raise_smem_limit(reinterpret_cast<const void*>(shard_tiles_kernel<LB>), int(pcfg<LB>::SMEM),
                            "the sharded closure");
}

}  // namespace shard
}  // namespace se

using namespace se;
using namespace se::shard;

struct se_shard {
    Elec E;               // the slab: maps, pointers, C, Cp, R, lanes, base
    CUtensorMap mapP[2];  // the received pivot-row panels of even and odd rounds, 128 x Cp cells
    uint8_t* work;
    uint32_t* err;
    uint8_t* P;
    int64_t panel_bytes;
    int32_t b0, b1, nloc;
    int32_t pivot_ready;  // a round whose pivot tile the previous update already closed, or -1
};

extern "C" int64_t se_shard_workspace_bytes(int C, int b0, int b1, int lane_bits) {
    if (C < 1 || C > (1 << 20) || (lane_bits != 16 && lane_bits != 32)) return -1;
    const int R = int((C + kT - 1) / kT);
    if (b0 < 0 || b1 <= b0 || b1 > R) return -1;
    return layout(C, b0, b1, lane_bits).total;
}

extern "C" se_status_t se_shard_create(int C, int b0, int b1, int lane_bits, uint32_t value_offset, void* d_work,
                                       int64_t work_bytes, se_shard_t** out) {
    clear_error();
    SE_REQUIRE(out != nullptr, SE_ERR_INVALID, "null shard handle");
    SE_REQUIRE(C >= 1 && C <= (1 << 20), SE_ERR_INVALID, "Number of candidates out of range (%d)", C);
    SE_REQUIRE(lane_bits == 16 || lane_bits == 32, SE_ERR_INVALID, "lane_bits must be 16 or 32");
    SE_REQUIRE(lane_bits == 16 || value_offset == 0, SE_ERR_INVALID, "a value offset needs 16-bit lanes");
    const int R = int((C + kT - 1) / kT);
    SE_REQUIRE(b0 >= 0 && b1 > b0 && b1 <= R, SE_ERR_INVALID, "row blocks [%d, %d) outside [0, %d)", b0, b1, R);
    const Layout L = layout(C, b0, b1, lane_bits);
    SE_REQUIRE(d_work && work_bytes >= L.total, SE_ERR_WORKSPACE, "workspace of %lld bytes is below %lld",
               (long long)work_bytes, (long long)L.total);
    SE_REQUIRE((reinterpret_cast<uintptr_t>(d_work) & 255) == 0, SE_ERR_INVALID, "workspace must be 256-byte aligned");
    se_shard* h = new (std::nothrow) se_shard();
    SE_REQUIRE(h != nullptr, SE_ERR_INVALID, "out of host memory");
    uint8_t* w = static_cast<uint8_t*>(d_work);
    h->work = w;
    h->err = reinterpret_cast<uint32_t*>(w);
    h->P = w + L.p_off;
    h->panel_bytes = L.panel_bytes;
    h->b0 = b0;
    h->b1 = b1;
    h->nloc = b1 - b0;
    h->pivot_ready = -1;
    Elec& E = h->E;
    E.C = C;
    E.Cp = int(round_up(int64_t(C), kT));
    E.R = R;
    E.lanes = lane_bits;
    E.base = value_offset;
    E.S = reinterpret_cast<uint32_t*>(w + L.s_off);
    E.AT = reinterpret_cast<uint32_t*>(w + L.at_off);
    E.dT = reinterpret_cast<uint32_t*>(w + L.dt_off);
    const int cpw = 32 / lane_bits;
    const uint64_t ldw = uint64_t(E.Cp) / cpw, tw = uint64_t(kT) / cpw;
    se_status_t st = make_map(&E.mapS, E.S, ldw, uint64_t(h->nloc) * kT, ldw * 4, uint32_t(tw), kKC);
    if (!st) st = make_map(&E.mapAT, E.AT, uint64_t(E.Cp), kT, uint64_t(E.Cp) * 4, kT, kKC);
    if (!st) st = make_map(&E.mapDT, E.dT, kT, kT, kT * 4, kT, kKC);
    if (!st) st = make_map(&h->mapP[0], h->P, ldw, kT, ldw * 4, uint32_t(tw), kKC);
    if (!st) st = make_map(&h->mapP[1], h->P + h->panel_bytes, ldw, kT, ldw * 4, uint32_t(tw), kKC);
    if (st) {
        delete h;
        return st;
    }
    *out = h;
    return SE_OK;
}

extern "C" se_status_t se_shard_destroy(se_shard_t* sh) {
    delete sh;
    return SE_OK;
}

extern "C" se_status_t se_shard_init(se_shard_t* sh, const uint32_t* d_pref, int64_t ld, void* stream) {
    clear_error();
    SE_REQUIRE(sh && d_pref, SE_ERR_INVALID, "null argument");
    const Elec& E = sh->E;
    SE_REQUIRE(ld >= E.C, SE_ERR_INVALID, "bad preference matrix stride");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SE_CUDA_TRY(cudaMemsetAsync(sh->work, 0, 256, s));
    const dim3 grid(unsigned(E.Cp / 32), unsigned(sh->nloc * (kT / 32)));
    if (E.lanes == 16)
        shard_init_kernel<16><<<grid, dim3(32, 8), 0, s>>>(d_pref, ld, E.C, E.Cp, sh->b0 * kT, E.S, E.base, sh->err);
    else
        shard_init_kernel<32><<<grid, dim3(32, 8), 0, s>>>(d_pref, ld, E.C, E.Cp, sh->b0 * kT, E.S, 0u, sh->err);
    SE_CHECK_LAUNCH();
    return SE_OK;
}

namespace {
template <int LB> se_status_t pivot_impl(se_shard& h, int k, cudaStream_t s) {
    const Elec& E = h.E;
    if (se_status_t st = set_smem<LB>()) return st;
    const int kl = k - h.b0;
    if (h.pivot_ready != k) {  // not closed already by the previous round's remainder launch
        const int kmax = E.C - k * kT < kT ? E.C - k * kT : kT;  // pivots past C are zero padding
        shard_pivot_kernel<LB><<<1, cfg<LB>::THREADS, 0, s>>>(E.S, int64_t(E.Cp) / (32 / LB), kl, k, kmax, E.dT);
        SE_CHECK_LAUNCH();
    }
    h.pivot_ready = -1;
    if (E.R > 1) {
        shard_tiles_kernel<LB><<<unsigned(E.R - 1), cfg<LB>::THREADS, pcfg<LB>::SMEM, s>>>(
            E, h.mapP[k & 1], kPhaseRowPanel, k, kl, h.b0, 1, -1, -1, -1, 0, h.err);
        SE_CHECK_LAUNCH();
    }
    return SE_OK;
}

// part 0: every local row block but k; 1: row block k+1 alone (nothing unless this shard holds
// it); 2: every local row block but k and k+1. Row block k+1, when updated here, also closes
// round k+1's pivot tile inside the remainder launch.
template <int LB> se_status_t update_impl(se_shard& h, int k, int part, cudaStream_t s) {
    const Elec& E = h.E;
    if (se_status_t st = set_smem<LB>()) return st;
    const bool own = k >= h.b0 && k < h.b1;
    const int kl = own ? k - h.b0 : 0;
    const int next = k + 1;
    const int nl = next < E.R && next >= h.b0 && next < h.b1 ? next - h.b0 : -1;  // local index of k+1
    int only = -1, skip = -1, rows = own ? h.nloc - 1 : h.nloc;
    if (part == 1) {
        if (nl < 0) return SE_OK;
        only = nl;
        rows = 1;
    } else if (part == 2 && nl >= 0) {
        skip = nl;
        rows -= 1;
    }
    if (rows <= 0) return SE_OK;
    const CUtensorMap& mapP = h.mapP[k & 1];
    shard_tiles_kernel<LB><<<unsigned(rows), cfg<LB>::THREADS, pcfg<LB>::SMEM, s>>>(
        E, mapP, kPhaseColPanel, k, kl, h.b0, own ? 1 : 0, only, skip, -1, 0, h.err);
    SE_CHECK_LAUNCH();
    if (E.R > 1) {
        // Close round k+1's pivot inside this launch when it updates row block k+1.
        const int fuse = part != 2 ? nl : -1;
        const int kmax_next = fuse >= 0 ? (E.C - next * kT < kT ? E.C - next * kT : kT) : 0;
        shard_tiles_kernel<LB><<<unsigned(rows * (E.R - 1)), cfg<LB>::THREADS, pcfg<LB>::SMEM, s>>>(
            E, mapP, kPhaseRemainder, k, kl, h.b0, own ? 1 : 0, only, skip, fuse, kmax_next, h.err);
        SE_CHECK_LAUNCH();
        if (fuse >= 0) h.pivot_ready = next;
    }
    return SE_OK;
}
}  // namespace

extern "C" se_status_t se_shard_pivot(se_shard_t* sh, int k, void* stream) {
    clear_error();
    SE_REQUIRE(sh != nullptr, SE_ERR_INVALID, "null shard handle");
    SE_REQUIRE(k >= sh->b0 && k < sh->b1, SE_ERR_INVALID, "row block %d is not in this shard [%d, %d)", k, sh->b0,
               sh->b1);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return sh->E.lanes == 16 ? pivot_impl<16>(*sh, k, s) : pivot_impl<32>(*sh, k, s);
}

extern "C" int64_t se_shard_panel_offset(const se_shard_t* sh, int k) {
    if (!sh || k < 0 || k >= sh->E.R) return -1;
    if (k >= sh->b0 && k < sh->b1)  // the owner broadcasts straight from its slab rows
        return (reinterpret_cast<const uint8_t*>(sh->E.S) - sh->work) + int64_t(k - sh->b0) * sh->panel_bytes;
    return (sh->P - sh->work) + (k & 1) * sh->panel_bytes;  // a receiver's buffer of k's parity
}

extern "C" int64_t se_shard_panel_bytes(const se_shard_t* sh) { return sh ? sh->panel_bytes : -1; }

extern "C" se_status_t se_shard_update(se_shard_t* sh, int k, void* stream) {
    clear_error();
    SE_REQUIRE(sh != nullptr, SE_ERR_INVALID, "null shard handle");
    SE_REQUIRE(k >= 0 && k < sh->E.R, SE_ERR_INVALID, "round %d outside [0, %d)", k, sh->E.R);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return sh->E.lanes == 16 ? update_impl<16>(*sh, k, 0, s) : update_impl<32>(*sh, k, 0, s);
}

extern "C" se_status_t se_shard_update_part(se_shard_t* sh, int k, int part, void* stream) {
    clear_error();
    SE_REQUIRE(sh != nullptr, SE_ERR_INVALID, "null shard handle");
    SE_REQUIRE(k >= 0 && k < sh->E.R, SE_ERR_INVALID, "round %d outside [0, %d)", k, sh->E.R);
    SE_REQUIRE(part >= 0 && part <= 2, SE_ERR_INVALID, "part must be 0, 1 or 2 (got %d)", part);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    return sh->E.lanes == 16 ? update_impl<16>(*sh, k, part, s) : update_impl<32>(*sh, k, part, s);
}

extern "C" se_status_t se_shard_finalize(se_shard_t* sh, uint32_t* d_out, int64_t ld_out, void* stream) {
    clear_error();
    SE_REQUIRE(sh && d_out, SE_ERR_INVALID, "null argument");
    const Elec& E = sh->E;
    SE_REQUIRE(ld_out >= E.C, SE_ERR_INVALID, "bad output stride");
    const int row0 = sh->b0 * kT;
    const int nrows = std::min(sh->b1 * kT, E.C) - row0;
    if (nrows <= 0) return SE_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const dim3 grid(unsigned(std::min<int64_t>((E.C + 255) / 256, 64)), unsigned(std::min(nrows, 65535)));
    if (E.lanes == 16)
        shard_finalize_kernel<16><<<grid, 256, 0, s>>>(E.S, E.Cp, E.C, row0, nrows, d_out, ld_out, E.base);
    else
        shard_finalize_kernel<32><<<grid, 256, 0, s>>>(E.S, E.Cp, E.C, row0, nrows, d_out, ld_out, 0u);
    SE_CHECK_LAUNCH();
    return SE_OK;
}

extern "C" se_status_t se_shard_check(se_shard_t* sh, void* stream) {
    clear_error();
    SE_REQUIRE(sh != nullptr, SE_ERR_INVALID, "null shard handle");
    uint32_t code = 0;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    SE_CUDA_TRY(cudaMemcpyAsync(&code, sh->err, 4, cudaMemcpyDeviceToHost, s));
    SE_CUDA_TRY(cudaStreamSynchronize(s));
    SE_REQUIRE(code != kErrOverflow, SE_ERR_OVERFLOW, "a kept value does not fit the 16-bit lane window");
    SE_REQUIRE(code == 0, SE_ERR_DEVICE, "sharded closure reported device error %u (TMA wait timed out)", code);
    return SE_OK;
}
