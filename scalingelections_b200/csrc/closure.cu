// Widest-path closure over the (max, min) semiring on sm_100a: the blocked Floyd-Warshall
// that compute_strongest_paths_cuda (scaling_elections.cu:490-578) drives, redesigned.
//
// Layout in HBM (all inside the caller's workspace):
//   S   Cp x Cp cells, Cp = C rounded up to the 128-cell tile, u16 or u32 per cell. Padding
//       rows/columns are 0: a vertex with no edges, which no widest path can use.
//   AT  128 x Cp words: the closed pivot column panel of the current round, transposed
//       (k-major) and, in u16 mode, with every cell duplicated into both halves of its word
//       so it is a ready-made `min.u16x2` operand.
//   dT  128 x 128 words: the closed pivot tile, transposed and duplicated the same way.
//
// One round k (pivot block K = rows/cols [128k, 128k+128)):
//   pivot     close D = S[K][K] in place, k by k (the only sequential step); emit dT. Round
//             0 runs it as its own 1-CTA launch (diag_kernel); for round k+1 the first CTA of
//             round k's remainder launch does it right after updating that tile.
//   panels    one launch, 2(R-1) CTAs: S[K][J] = max(S[K][J], D (x) S[K][J]) and
//             S[I][K] = max(S[I][K], S[I][K] (x) D), the latter emitting AT.
//   remainder (R-1)^2 CTAs: S[I][J] = max(S[I][J], S[I][K] (x) S[K][J]).
// where (x) is the max-min product. Because D is closed, a panel needs no sequential k loop:
// a path k1 ->...-> k2 -> j inside block K is worth min(D*[k1][k2], S[k2][j]). So the
// panels and the remainder are the same register-blocked "semiring GEMM" (batch_core.cuh):
// operands staged into shared memory by TMA (this GPU's memory only, never multicast),
// 8 x 8 words per thread, c = max3(c, min(a0, b0), min(a1, b1)) per word and k-pair.
//
// The reference's masks (scaling_elections.py:118-121, cu:133-161) are dropped: the closure
// runs unmasked and the diagonal is zeroed at the end. That is exact: a relaxation through
// pivot i == j or i == k computes min(S[j][j], S[j][k]) <= S[j][k] or
// min(S[j][k], S[k][k]) <= S[j][k] and never changes an off-diagonal cell, and diagonal
// cells only feed such relaxations.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <atomic>
#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "batch_core.cuh"

namespace se {
namespace closure {

// Poll limit for one mbarrier phase: a TMA chunk lands in microseconds; ~2^26 polls is
// seconds. Hitting it means a lost completion, reported through the error word.
constexpr uint32_t kMaxPolls = 1u << 26;

// ------------------------------------------------------------------------------------------
// One round's panels in one launch: blocks [0, R-1) the pivot-row tiles S[K][J] =
// max(S[K][J], D (x) S[K][J]); blocks [R-1, 2(R-1)) the pivot-column tiles S[I][K] =
// max(S[I][K], S[I][K] (x) D), which also emit the transposed panel AT. 96 KiB of shared
// memory per CTA, so both sets are resident at once.
// ------------------------------------------------------------------------------------------
// With parts > 1 every panel tile runs split-K over `parts` consecutive blocks (batch::SplitK):
// split_ctr[b] and split_scr[b * parts ...] are tile b's counter and partial tiles.
template <int LB, int NQ = 8, bool SPLIT = false>
__global__ void __launch_bounds__(tile_threads<LB, NQ>(), 1)
    panels_kernel(const __grid_constant__ batch::Elec E, int K, int parts, uint32_t* __restrict__ split_ctr,
                  uint32_t* __restrict__ split_scr, uint32_t* __restrict__ err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + batch::pcfg<LB>::DATA);
    if (threadIdx.x == 0) {
        for (int c = 0; c < 2 * kChunks; ++c) mbar_init(&bars[c], 1);
        fence_barrier_init();
    }
    __syncthreads();
    pdl_trigger();  // the next launch may start filling SMs this grid has left
    pdl_wait();     // the previous launch's tiles are complete and visible
    const int R1 = E.R - 1;
    const int P = SPLIT ? parts : 1;
    const int b = blockIdx.x / P;
    bool ok;
    uint32_t par_a = 0, par_b = 0;
    const bool row = b < R1;
    const int x = row ? b : b - R1;
    batch::SplitK sp{int(blockIdx.x % P), P, SPLIT ? split_scr + int64_t(b) * P * kT * cfg<LB>::TW : nullptr,
                     SPLIT ? split_ctr + b : nullptr, false};
    ok = batch::run_tile<LB, false, NQ, SPLIT>(E, &E, row ? batch::kTileRow : batch::kTileCol, K, x + (x >= K),
                                               x + (x >= K), smem, bars, par_a, par_b, nullptr, -1, -1, -1,
                                               SPLIT ? &sp : nullptr);
    if (!ok && threadIdx.x == 0) raise_device_error(err, kErrTmaTimeout);
}

// ------------------------------------------------------------------------------------------
// One round's remainder tiles S[I][J] = max(S[I][J], AT (x) S[K][J]), I, J != K. With
// fuse_pivot, block 0 takes tile (K+1, K+1) and, after its update, closes it as the next
// round's pivot tile (and emits dT) while the other blocks continue: the next round needs no
// separate pivot launch. Nothing else in this launch reads that tile or dT.
// ------------------------------------------------------------------------------------------
// subset 0: all (R-1)^2 tiles of the round. subset 1: the tiles of row and column K+1 (2R - 3,
// tile (K+1, K+1) first); subset 2: every other tile ((R-2)^2). The two-stream schedule runs
// subset 1 and the next round's panels on the caller's stream while subset 2 runs on another.
// With fuse_pivot and parts > 1 (subset 0 only), blocks [0, parts) run tile (K+1, K+1) split-K
// (batch::SplitK, counter split_ctr, partials split_scr) and the last of them closes the
// pivot; the grid then has parts - 1 more blocks than tiles.
template <int LB, int NQ = 8, bool SPLIT = false>
__global__ void __launch_bounds__(tile_threads<LB, NQ>(), NQ == 4 ? 2 : 1)
    rem_kernel(const __grid_constant__ batch::Elec E, int K, int fuse_pivot, int subset, int parts,
               uint32_t* __restrict__ split_ctr, uint32_t* __restrict__ split_scr, uint32_t* __restrict__ err) {
    using CF = cfg<LB>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + batch::pcfg<LB>::DATA);
    if (threadIdx.x == 0) {
        for (int c = 0; c < kChunks; ++c) mbar_init(&bars[c], 1);
        fence_barrier_init();
    }
    __syncthreads();
    pdl_trigger();  // the next launch may start filling SMs this grid has left
    pdl_wait();     // the previous launch's tiles are complete and visible
    const int R1 = E.R - 1, R2 = E.R - 2;
    int t = blockIdx.x, I, J;
    const bool split = SPLIT && subset == 0 && fuse_pivot && parts > 1;
    const int q = split && t < parts ? t : -1;  // this block's part of tile (K+1, K+1)
    auto skip_k_k1 = [K](int n) { return n < K ? n : n + 2; };  // n-th block index other than K, K+1
    if (subset == 0) {
        if (fuse_pivot) {
            const int p = K * R1 + K;  // reduced coordinates of tile (K+1, K+1)
            if (split) t = q >= 0 ? 0 : t - parts + 1;
            t = t == 0 ? p : (t == p ? 0 : t);
        }
        const int ii = t / R1, jj = t % R1;
        I = ii + (ii >= K);
        J = jj + (jj >= K);
    } else if (subset == 1) {
        if (t == 0) {
            I = J = K + 1;
        } else if (t <= R2) {
            I = K + 1;
            J = skip_k_k1(t - 1);
        } else {
            I = skip_k_k1(t - 1 - R2);
            J = K + 1;
        }
    } else {
        I = skip_k_k1(t / R2);
        J = skip_k_k1(t % R2);
    }
    uint32_t par_a = 0, par_b = 0;
    batch::SplitK sp{q, parts, split_scr, split_ctr, false};
    const bool ok = batch::run_tile<LB, false, NQ, SPLIT>(E, &E, batch::kTileRem, K, I, J, smem, bars, par_a, par_b,
                                                          nullptr, -1, -1, -1, q >= 0 ? &sp : nullptr);
    if (!ok) {
        if (threadIdx.x == 0) raise_device_error(err, kErrTmaTimeout);
        return;
    }
    if (fuse_pivot && (q >= 0 ? sp.last : !split && blockIdx.x == 0)) {
        __syncthreads();  // the tile's stores are visible to the whole CTA
        batch::run_pivot<LB, NQ>(E, K + 1, rowbuf, colbuf);
    }
}

// ------------------------------------------------------------------------------------------
// Schedule 6: round K's remainder and round K+1's panels in one launch. Each CTA takes a
// ticket (an atomic counter, so every ticket below its own went to a CTA that is already
// running) and runs one task:
//   [0, 2R-3)              remainder tiles of row and column K+1; ticket 0 is tile (K+1, K+1),
//                          which it then closes as the next pivot (dT);
//   [2R-3, (R-1)^2)        the other remainder tiles of round K;
//   [(R-1)^2, +2(R-1))     the panel tiles of round K+1, which first wait (bounded) until all
//                          of the first group, the pivot included, are done.
// The panels then run in the remainder's last, partial wave instead of a launch of their own.
// They write AT[(K+1) % 2] while the remainder reads AT[K % 2] (descriptors E and En), and
// rows and columns K+1, which no remainder tile of the second group reads or writes; the tiles
// they read are exactly the first group's. state: this round's ticket and done counters.
// With parts > 1, tile (K+1, K+1) takes tickets [0, parts) and every panel tile `parts`
// consecutive tickets, split-K (batch::SplitK; counters and partials as in panels_kernel and
// rem_kernel): the last part of tile (K+1, K+1) closes the pivot and counts the tile done.
// ------------------------------------------------------------------------------------------
template <int LB, int NQ = 8, bool SPLIT = false>
__global__ void __launch_bounds__(tile_threads<LB, NQ>(), NQ == 4 ? 2 : 1)
    round_kernel(const __grid_constant__ batch::Elec E, const __grid_constant__ batch::Elec En, int K,
                 uint32_t* __restrict__ state, int parts, uint32_t* __restrict__ split_ctr,
                 uint32_t* __restrict__ split_scr, uint32_t* __restrict__ err) {
    using CF = cfg<LB>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    __shared__ uint32_t s_ticket;
    __shared__ int s_go;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + batch::pcfg<LB>::DATA);
    if (threadIdx.x == 0) {
        for (int c = 0; c < 2 * kChunks; ++c) mbar_init(&bars[c], 1);
        fence_barrier_init();
        s_ticket = atomicAdd(&state[0], 1u);
    }
    __syncthreads();
    pdl_trigger();  // the next round's launch may start filling SMs this grid has left
    pdl_wait();     // the previous launch's tiles are complete and visible
    const uint32_t t = s_ticket;
    const int R = E.R, R1 = R - 1, R2 = R - 2;
    const uint32_t P = SPLIT ? uint32_t(parts) : 1u;
    constexpr int64_t kTileWords = int64_t(kT) * CF::TW;
    // Remainder tickets: tile (K+1, K+1) in [0, P), the rest of the first group (row and column
    // K+1) up to P - 1 + first, the other tiles up to nrem.
    const uint32_t first = uint32_t(2 * R - 3), rem = uint32_t(R1) * uint32_t(R1), nrem = rem + P - 1;
    auto skip_k_k1 = [K](int n) { return n < K ? n : n + 2; };  // n-th block index other than K, K+1
    uint32_t par_a = 0, par_b = 0;
    if (t < nrem) {
        int I, J;
        const int q = P > 1 && t < P ? int(t) : -1;  // this ticket's part of tile (K+1, K+1)
        if (t < P) {
            I = J = K + 1;
        } else if (t < P - 1 + first) {
            const int x = int(t - P);
            I = x < R2 ? K + 1 : skip_k_k1(x - R2);
            J = x < R2 ? skip_k_k1(x) : K + 1;
        } else {
            const int x = int(t - (P - 1) - first);
            I = skip_k_k1(x / R2);
            J = skip_k_k1(x % R2);
        }
        batch::SplitK sp{q, int(P), SPLIT ? split_scr + int64_t(2 * R1) * P * kTileWords : nullptr,
                         SPLIT ? split_ctr + 2 * R1 : nullptr, false};
        const bool ok = batch::run_tile<LB, false, NQ, SPLIT>(E, &E, batch::kTileRem, K, I, J, smem, bars, par_a,
                                                              par_b, nullptr, -1, -1, -1, q >= 0 ? &sp : nullptr);
        if (!ok) {
            if (threadIdx.x == 0) raise_device_error(err, kErrTmaTimeout);
            return;
        }
        if (q >= 0 && !sp.last) return;  // an earlier part: the last one finishes the tile
        if (t < P) {
            __syncthreads();  // the tile's stores are visible to the whole CTA
            batch::run_pivot<LB, NQ>(E, K + 1, rowbuf, colbuf);
        }
        if (t < P - 1 + first) {  // publish: the tile (and the pivot) are done, for TMA reads too
            __threadfence();
            __syncthreads();
            if (threadIdx.x == 0) {
                batch::fence_proxy_async_global();
                atomicAdd(&state[1], 1u);
            }
        }
        return;
    }
    if (threadIdx.x == 0) {  // a panel of round K+1: wait for the tiles it reads and the pivot
        const bool ok = batch::wait_counter(&state[1], first, err, 2000000000ull);
        if (!ok) raise_device_error(err, kErrTmaTimeout);
        s_go = ok;
        batch::fence_proxy_async_global();
    }
    __syncthreads();
    if (!s_go) return;
    const int b = int((t - nrem) / P);  // the panel tile
    const bool row = b < R1;
    const int y = row ? b : b - R1;
    const int K1 = K + 1;
    batch::SplitK sp{int((t - nrem) % P), int(P), SPLIT ? split_scr + int64_t(b) * P * kTileWords : nullptr,
                     SPLIT ? split_ctr + b : nullptr, false};
    const bool ok = batch::run_tile<LB, false, NQ, SPLIT>(En, &En, row ? batch::kTileRow : batch::kTileCol, K1,
                                                          y + (y >= K1), y + (y >= K1), smem, bars, par_a, par_b,
                                                          nullptr, -1, -1, -1, SPLIT && P > 1 ? &sp : nullptr);
    if (!ok && threadIdx.x == 0) raise_device_error(err, kErrTmaTimeout);
}

// ------------------------------------------------------------------------------------------
// Dataflow closure: the same tasks as the round-by-round launches (pivot, panels, remainder),
// run by one persistent grid that walks a fixed task order with no barrier between rounds.
// Each task waits only for what it reads and for the readers of what it overwrites:
//   ver[i][j]   rounds applied to tile (i, j); a task of round k on a tile needs ver == k and
//               sets k + 1 (panels also need the pivot, the remainder needs both panels)
//   pdone[k]    panel tasks of round k done: the readers of the pivot tile (column panels read
//               it) and of dT[k % 2]
//   rdone[k]    remainder tasks of round k done: the readers of the row-panel tiles S[k][*]
//               and of AT[k % 2]
// so a round-k task that writes a tile of row k-1 also waits for pdone[k-1] and rdone[k-1],
// the column panels of round k wait for rdone[k-2] (AT is double-buffered), and the pivot of
// round k for pdone[k-2] (so is dT). The order (flow_decode) puts the next round's pivot and
// panels right after the tiles they need, ahead of the current round's bulk. Every task's
// prerequisites come earlier in the order and were taken by running CTAs, so the
// schedule cannot deadlock; waits are bounded and a timeout aborts the grid.
//
// A task's round picks the AT/dT buffer pair (k % 2). se_closure_flow_task exposes the order
// to the host; tests/test_flow_order.py checks it against these rules for every task, small R.
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void fence_proxy_async_global_flow() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ uint32_t flow_ld(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// n-th value of [0, count) without the excluded values a and b (either may be -1).
__host__ __device__ __forceinline__ int skip2(int n, int a, int b) {
    int lo = a < b ? a : b, hi = a < b ? b : a;
    if (lo < 0) {
        lo = hi;
        hi = -1;
    }
    if (lo >= 0 && n >= lo) ++n;
    if (hi >= 0 && n >= hi) ++n;
    return n;
}

struct FlowTask {
    int kind;  // 0 pivot, 1 row panel, 2 column panel, 3 remainder
    int k, i, j;
};

// Task t of the order. After [pivot 0][panels 0], round k's block is
//   A  remainder tiles of round k that round k+1 needs first: (k+1, k+1), row k+1, column k+1
//   B  pivot of round k+1
//   C  panels of round k+1 except the column tile (k, k+1)
//   D  the other remainder tiles of round k (rows other than k+1 and k-1)
//   E  remainder row k-1 (waits for round k-1 to finish)
//   F  column tile (k, k+1) of round k+1 (it overwrites a row-k tile: waits for round k)
// so the next round's pivot and panels run while round k's bulk is still in flight. Round
// R-1 has only D and E. Reduced coordinates of round k skip k; p = reduced k+1, q = reduced
// k-1.
__host__ __device__ FlowTask flow_decode(uint32_t t_in, int R) {
    const int R1 = R - 1;
    FlowTask T;
    const uint32_t head = uint32_t(1 + 2 * R1);
    if (t_in < head) {
        T.k = 0;
        if (t_in == 0) {
            T.kind = 0;
            T.i = T.j = 0;
        } else if (int(t_in) - 1 < R1) {
            T.kind = 1;
            T.i = 0;
            T.j = int(t_in);
        } else {
            T.kind = 2;
            T.i = int(t_in) - R1;
            T.j = 0;
        }
        return T;
    }
    const uint32_t t = t_in - head;
    const uint32_t B = uint32_t(R1 * R1) + head;
    int k = int(t / B);
    int r;
    if (k >= R - 1) {
        k = R - 1;
        r = int(t - uint32_t(R - 1) * B);
    } else {
        r = int(t % B);
    }
    const bool last = k + 1 >= R;
    const int p = last ? -1 : k;
    const int q = k >= 1 ? k - 1 : -1;
    auto full = [&](int red) { return red + (red >= k); };
    const int nA = last ? 0 : 1 + 2 * (R1 - 1);
    T.k = k;
    T.kind = 3;
    if (r < nA) {
        int ii, jj;
        if (r == 0) ii = jj = p;
        else if (r < R1) ii = p, jj = skip2(r - 1, p, -1);
        else ii = skip2(r - R1, p, -1), jj = p;
        T.i = full(ii);
        T.j = full(jj);
        return T;
    }
    r -= nA;
    if (!last) {
        const int k1 = k + 1;
        if (r == 0) {
            T.kind = 0;
            T.k = k1;
            T.i = T.j = k1;
            return T;
        }
        r -= 1;
        if (r < R1) {
            T.kind = 1;
            T.k = k1;
            T.i = k1;
            T.j = r + (r >= k1);
            return T;
        }
        r -= R1;
        if (r < R1 - 1) {
            T.kind = 2;
            T.k = k1;
            T.i = skip2(r, k, k1);
            T.j = k1;
            return T;
        }
        r -= R1 - 1;
    }
    const int ncols = R1 - (last ? 0 : 1);
    const int nmid = R1 - (last ? 0 : 1) - ((q >= 0 && q != p) ? 1 : 0);
    if (r < nmid * ncols) {
        T.i = full(skip2(r / ncols, p, q));
        T.j = full(skip2(r % ncols, p, -1));
        return T;
    }
    r -= nmid * ncols;
    if (q >= 0 && q != p && r < ncols) {
        T.i = full(q);
        T.j = full(skip2(r, p, -1));
        return T;
    }
    // F: column tile (k, k+1) of round k+1.
    T.kind = 2;
    T.k = k + 1;
    T.i = k;
    T.j = k + 1;
    return T;
}

template <int LB>
__global__ void __launch_bounds__(cfg<LB>::THREADS, 1)
    flow_kernel(const __grid_constant__ batch::Elec E0, const __grid_constant__ batch::Elec E1,
                uint32_t* __restrict__ state, uint32_t* __restrict__ err) {
    using CF = cfg<LB>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    __shared__ uint32_t s_t;
    __shared__ int s_go;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + batch::pcfg<LB>::DATA);
    if (threadIdx.x == 0) {
        for (int c = 0; c < 2 * kChunks; ++c) mbar_init(&bars[c], 1);
        fence_barrier_init();
    }
    __syncthreads();
    const int R = E0.R, R1 = R - 1;
    uint32_t* head = state;
    uint32_t* abort_flag = state + 1;
    uint32_t* ver = state + 4;
    uint32_t* pdone = ver + R * R;
    uint32_t* rdone = pdone + R;
    const uint32_t total = uint32_t(R) * uint32_t(R) * uint32_t(R);
    uint32_t par_a = 0, par_b = 0;
    for (;;) {
        if (threadIdx.x == 0) {
            uint32_t t = total;
            if (!flow_ld(abort_flag)) t = atomicAdd(head, 1u);
            s_t = t;
            s_go = 1;
            if (t < total) {
                const FlowTask T = flow_decode(t, R);
                const int k = T.k;
                const uint64_t t0 = global_ns();
                auto ready = [&]() -> bool {
                    const uint32_t kk = uint32_t(k);
                    if (T.kind == 0) {
                        if (flow_ld(&ver[k * R + k]) < kk) return false;
                        if (k >= 2 && flow_ld(&pdone[k - 2]) < uint32_t(2 * R1)) return false;
                        return true;
                    }
                    if (flow_ld(&ver[k * R + k]) < kk + 1) return false;  // the pivot of round k
                    if (flow_ld(&ver[T.i * R + T.j]) < kk) return false;
                    if (T.kind == 2 && k >= 2 && flow_ld(&rdone[k - 2]) < uint32_t(R1 * R1)) return false;
                    if (T.kind == 3) {
                        if (flow_ld(&ver[k * R + T.j]) < kk + 1) return false;
                        if (flow_ld(&ver[T.i * R + k]) < kk + 1) return false;
                    }
                    if (T.i == k - 1 && T.kind >= 2) {
                        if (flow_ld(&pdone[k - 1]) < uint32_t(2 * R1)) return false;
                        if (flow_ld(&rdone[k - 1]) < uint32_t(R1 * R1)) return false;
                    }
                    return true;
                };
                for (uint32_t it = 0; !ready(); ++it) {
                    if ((it & 31) == 0 && (flow_ld(abort_flag) || global_ns() - t0 > 2000000000ull)) {
                        atomicExch(abort_flag, 1u);
                        raise_device_error(err, kErrTmaTimeout + 2);
                        s_go = 0;
                        break;
                    }
                    __nanosleep(32);
                }
                fence_proxy_async_global_flow();
            }
        }
        __syncthreads();
        const uint32_t t = s_t;
        if (t >= total || !s_go) break;
        const FlowTask T = flow_decode(t, R);
        const batch::Elec& E = (T.k & 1) ? E1 : E0;
        bool ok = true;
        if (T.kind == 0) {
            batch::run_pivot<LB>(E, T.k, rowbuf, colbuf);
        } else {
            const int kind = T.kind == 1 ? batch::kTileRow : (T.kind == 2 ? batch::kTileCol : batch::kTileRem);
            ok = batch::run_tile<LB, false>(E, &E, kind, T.k, T.i, T.j, smem, bars, par_a, par_b);
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            if (!ok) {
                atomicExch(abort_flag, 1u);
                raise_device_error(err, kErrTmaTimeout);
            } else {
                fence_proxy_async_global_flow();
                atomicExch(&ver[T.i * R + T.j], uint32_t(T.k + 1));
                if (T.kind == 1 || T.kind == 2) atomicAdd(&pdone[T.k], 1u);
                if (T.kind == 3) atomicAdd(&rdone[T.k], 1u);
            }
        }
        if (!ok) break;
    }
}

// ------------------------------------------------------------------------------------------
// Pivot tile (phase 1): close D = S[K][K] in place, two pivots per barrier, then emit dT.
// ------------------------------------------------------------------------------------------
template <int LB, int NQ = 8>
__global__ void __launch_bounds__(tile_threads<LB, NQ>(), 1)
    diag_kernel(uint32_t* __restrict__ S, int64_t ldw, int K, uint32_t* __restrict__ dT) {
    using CF = cfg<LB>;
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    const geomT<NQ> g(threadIdx.x);
    uint32_t c[8][NQ];
    uint32_t* D = S + int64_t(K) * kT * ldw + int64_t(K) * CF::TW;
    pdl_trigger();
    pdl_wait();  // the tile's previous update is complete and visible
    load_tile_regs<LB, false, NQ>(c, D, ldw, g);
    close_tile_in_registers<LB, NQ>(c, g, kT, rowbuf, colbuf);
    store_tile_regs<LB, NQ>(c, D, ldw, g);
    store_transposed_splat<LB, NQ>(c, dT, kT, g);
}

// ------------------------------------------------------------------------------------------
// Defeat matrix into the padded working matrix (scaling_elections.py:105-112 /
// cu:495-503): S[i][j] = d[i][j] if d[i][j] > d[j][i] else 0, zero on the diagonal and in
// the padding. d[j][i] is read through a shared-memory transpose so both reads coalesce.
//
// In u16 mode every kept value v is stored as v - base. The widest-path closure only compares
// values: (max, min) commute with any strictly increasing map, and v -> v - base (0 -> 0) is
// one on {0} and [base + 1, inf). So the closure of the shifted matrix, shifted back, is the
// closure of the original, exactly, provided every kept value lies in [base + 1, base + 65535].
// Ballot counts from V voters always do for base = floor(V / 2): a kept d[i][j] > d[j][i]
// with d[i][j] + d[j][i] = V is in (V/2, V]. A value outside the window sets the overflow flag.
// ------------------------------------------------------------------------------------------
template <int LB>
__global__ void __launch_bounds__(256)
    init_kernel(const uint32_t* __restrict__ d, int64_t ld, int C, int Cp, void* __restrict__ Sv, uint32_t base,
                uint32_t* __restrict__ flags) {
    __shared__ uint32_t t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // this block writes S[by.., bx..]
    // Stage d[bx + y][by + x] (the transposed block) so t[x][y] = d[bx + y][by + x].
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
            const uint32_t dji = t[y][threadIdx.x];
            v = dij > dji ? dij : 0u;
        }
        if constexpr (LB == 16) {
            if (v != 0u) {
                if (v <= base || v - base > 0xFFFFu) {
                    over = true;
                    v = 0xFFFFu;
                } else {
                    v -= base;
                }
            }
            static_cast<uint16_t*>(Sv)[int64_t(i) * Cp + j] = static_cast<uint16_t>(v);
        } else {
            static_cast<uint32_t*>(Sv)[int64_t(i) * Cp + j] = v;
        }
    }
    if (over) atomicOr(&flags[1], 1u);
}

// Smallest and largest kept value of the defeat matrix (flags[2], flags[3]): decides whether
// 16-bit lanes, possibly shifted by a base, can hold the closure exactly.
__global__ void __launch_bounds__(256)
    kept_range_kernel(const uint32_t* __restrict__ d, int64_t ld, int C, uint32_t* __restrict__ flags) {
    __shared__ uint32_t t[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = bx + y, cc = by + threadIdx.x;
        t[threadIdx.x][y] = (r < C && cc < C) ? d[int64_t(r) * ld + cc] : 0u;
    }
    __syncthreads();
    uint32_t lo = 0xFFFFFFFFu, hi = 0u;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int i = by + y, j = bx + threadIdx.x;
        if (i < C && j < C && i != j) {
            const uint32_t dij = d[int64_t(i) * ld + j];
            if (dij > t[y][threadIdx.x]) {
                lo = dij < lo ? dij : lo;
                hi = dij > hi ? dij : hi;
            }
        }
    }
    for (int o = 16; o; o >>= 1) {
        lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
        hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (threadIdx.x == 0 && hi != 0u) {
        atomicMin(&flags[2], lo);
        atomicMax(&flags[3], hi);
    }
}

// out[i][j] = S[i][j] widened to u32 (and shifted back by base), 0 on the diagonal (the
// reference's masks).
template <int LB>
__global__ void __launch_bounds__(256)
    finalize_kernel(const void* __restrict__ Sv, int Cp, int C, uint32_t* __restrict__ out, int64_t ld_out,
                    uint32_t base) {
    pdl_wait();  // the closure's last launch is complete and visible
    for (int i = blockIdx.y; i < C; i += gridDim.y)
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < C; j += gridDim.x * blockDim.x) {
            uint32_t v;
            if constexpr (LB == 16) {
                v = static_cast<const uint16_t*>(Sv)[int64_t(i) * Cp + j];
                v = v ? v + base : 0u;
            } else {
                v = static_cast<const uint32_t*>(Sv)[int64_t(i) * Cp + j];
            }
            out[int64_t(i) * ld_out + j] = (i == j) ? 0u : v;
        }
}

// ------------------------------------------------------------------------------------------
// Host side.
// ------------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        else
            cudaGetLastError();
    });
    return fn;
}

// 2-D u32 tensor map: dims {inner, outer} words, row pitch in bytes, box {box_x, box_y}.
se_status_t make_map(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint64_t pitch_bytes,
                     uint32_t box_x, uint32_t box_y) {
    auto fn = encode_fn();
    SE_REQUIRE(fn != nullptr, SE_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable from the driver");
    cuuint64_t dims[2] = {inner, outer};
    cuuint64_t strides[1] = {pitch_bytes};
    cuuint32_t box[2] = {box_x, box_y};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<void*>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    SE_REQUIRE(r == CUDA_SUCCESS, SE_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", int(r));
    return SE_OK;
}

struct layout {
    int64_t C = 0;
    int64_t Cp = 0;
    int64_t flags_off = 0, s_off = 0, at_off = 0, dt_off = 0, total = 0;
    // Dataflow extras: second AT and dT buffers and the task state; then the split-K area of
    // the round-by-round schedules: 2R counters and the partial tiles of the 2(R-1) panel
    // tiles and the next pivot tile.
    int64_t at2_off = 0, dt2_off = 0, state_off = 0, split_ctr_off = 0, split_scr_off = 0, flow_total = 0;
};

// Parts of a split panel task for R row blocks: 4 up to R = 28 (C <= 3584), else 1. Measured on
// B200: 15-19 % off the whole closure at C = 512-2048 in the round-by-round schedules and up to
// 11 % in the one-launch-per-round ones; from R = 32 the remainder bulk, not the chain, bounds
// the rounds, and the split cost 7 % in the one-launch schedules at C = 4096-4608 (their unsplit
// panels already fill the remainder's last wave) and 1-2 % at R = 40-64 with 2 parts.
int split_parts(int R) { return R >= 2 && R <= 28 ? 4 : 1; }

layout plan(int C, int lane_bits) {
    layout L;
    L.C = C;
    L.Cp = round_up(C, kT);
    const int64_t cell = lane_bits == 16 ? 2 : 4;
    L.flags_off = 0;
    L.s_off = 256;
    L.at_off = L.s_off + round_up(L.Cp * L.Cp * cell, 256);
    L.dt_off = L.at_off + round_up(int64_t(kT) * L.Cp * 4, 256);
    L.total = L.dt_off + int64_t(kT) * kT * 4;
    const int64_t R = L.Cp / kT;
    L.at2_off = round_up(L.total, 256);
    L.dt2_off = L.at2_off + round_up(int64_t(kT) * L.Cp * 4, 256);
    L.state_off = L.dt2_off + round_up(int64_t(kT) * kT * 4, 256);
    L.split_ctr_off = round_up(L.state_off + (4 + R * R + 2 * R) * 4, 256);
    L.split_scr_off = L.split_ctr_off + round_up(2 * R * 4, 256);
    const int parts = split_parts(int(R));
    const int64_t split_tiles = parts > 1 ? (2 * (R - 1) + 1) * parts : 0;
    L.flow_total = L.split_scr_off + split_tiles * kT * kT * cell;
    return L;
}

// Closure schedules (se_closure_set_mode):
//   0  automatic: by C, from the variant table (se_closure_set_variant_table), else 1;
//   1  round by round, panels and pivots with the default micro-tile (8 x 8 words, 128
//      threads in 16-bit lanes), the next round's pivot fused into the remainder launch;
//   2  dataflow: one persistent grid (needs se_closure_workspace_bytes_flow() of workspace);
//   3  as 1 with the panels on the wide micro-tile (8 x 4 words, 256 threads; 16-bit lanes);
//   4  as 3 with every pivot tile closed by its own launch on the wide micro-tile, after the
//      whole remainder launch, instead of fused into its first CTA;
//   5  as 3 on two streams: round k's remainder tiles of row and column k+1 (with the fused
//      pivot) and round k+1's panels run on the caller's stream while the rest of round k's
//      remainder runs on a lower-priority second stream, so the next round's chain overlaps
//      the current round's bulk. AT is double-buffered (the dataflow layout's second buffer):
//      needs se_closure_workspace_bytes_flow() of workspace, and R >= 4;
//   6  round K's remainder and round K+1's panels in one launch (round_kernel): the panels
//      take the remainder's last, partial wave. AT is double-buffered as in 5;
//   7  as 3 with the remainder tiles on the wide micro-tile too, so the fused pivot closes on
//      eight warps;
//   8  as 6 with every tile on the wide micro-tile (16-bit lanes; 32-bit lanes run 6).
// 3 and 4 apply to 16-bit lanes; 32-bit lanes run 1 for them (5 without the wide panels). Round by round is the default:
// on B200 hardware block scheduling of one launch per phase beats the persistent grid's
// claim-and-poll overhead at every size measured.
std::atomic<int> g_closure_mode{0};

// The variant table of mode 0: modes[i] for C <= max_c[i] (the first entry that holds). The
// built-in table is autotune.tune_closure's result on one B200 with programmatic launches
// (16-bit lanes, ms per closure, 5 closures each; modes 3 / 6 / 7 / 8): C = 1024 0.441 / 0.473
// / 0.432 / 0.443, C = 2048 0.962 / 0.976 / 0.974 / 0.947, C = 3072 1.855 / 1.759 / 1.865 /
// 1.750, C = 4096 3.783 / 3.398 / 4.200 / 3.397, C = 5120 6.870 / 6.392 / 7.611 / 6.452, C =
// 6144 10.85 / 10.84 / 11.45 / 11.08. The table is within 2.2 % of the fastest mode at each.
constexpr int kMaxVariants = 8;
std::mutex g_variant_mutex;
int g_variant_n = 3;
int g_variant_max_c[kMaxVariants] = {1024, 4096, 1 << 20};
int g_variant_mode[kMaxVariants] = {7, 8, 6};

int automatic_mode(int C) {
    std::lock_guard<std::mutex> lock(g_variant_mutex);
    for (int i = 0; i < g_variant_n; ++i)
        if (C <= g_variant_max_c[i]) return g_variant_mode[i];
    return 1;
}

template <int LB> se_status_t set_smem_limits() {
    const int bytes = int(batch::pcfg<LB>::SMEM);
    auto raise = [bytes](const void* fn, const char* what) { return raise_smem_limit(fn, bytes, what); };
    auto both = [&](auto tag) -> se_status_t {  // every kernel of one micro-tile, whole and split
        constexpr int NQ = decltype(tag)::value;
        const void* fns[6] = {reinterpret_cast<const void*>(panels_kernel<LB, NQ, false>),
                              reinterpret_cast<const void*>(panels_kernel<LB, NQ, true>),
                              reinterpret_cast<const void*>(rem_kernel<LB, NQ, false>),
                              reinterpret_cast<const void*>(rem_kernel<LB, NQ, true>),
                              reinterpret_cast<const void*>(round_kernel<LB, NQ, false>),
                              reinterpret_cast<const void*>(round_kernel<LB, NQ, true>)};
        for (const void* fn : fns)
            if (se_status_t st = raise(fn, "the closure's tile kernels")) return st;
        return SE_OK;
    };
    if (se_status_t st = both(std::integral_constant<int, 8>{})) return st;
    if constexpr (LB == 16) {
        if (se_status_t st = both(std::integral_constant<int, 4>{})) return st;
    }
    return raise(reinterpret_cast<const void*>(flow_kernel<LB>), "the dataflow closure");
}

// Launches of the tile kernels. The split-K form (parts > 1) is a separate instantiation, so the
// whole-tile kernels that large closures run carry no split logic. Every launch is a
// programmatic dependent launch (pdl_trigger / pdl_wait): a round's grid may occupy the SM slots
// that the previous grid's last, partial wave leaves free and start its first tiles the moment
// that grid completes, without the launch gap.
template <typename... Params, typename... Args>
void launch_pdl(bool pdl, void (*kernel)(Params...), dim3 grid, int threads, size_t smem, cudaStream_t s,
                Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(unsigned(threads));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

template <int LB, int NQ>
void launch_panels(unsigned blocks, size_t smem, cudaStream_t s, const batch::Elec& E, int K, int parts,
                   uint32_t* ctr, uint32_t* scr, uint32_t* err, bool pdl = true) {
    constexpr int T = tile_threads<LB, NQ>();
    if (parts > 1) launch_pdl(pdl, panels_kernel<LB, NQ, true>, blocks, T, smem, s, E, K, parts, ctr, scr, err);
    else
        launch_pdl(pdl, panels_kernel<LB, NQ, false>, blocks, T, smem, s, E, K, 1, (uint32_t*)nullptr,
                   (uint32_t*)nullptr, err);
}

template <int LB, int NQ>
void launch_rem(unsigned blocks, size_t smem, cudaStream_t s, const batch::Elec& E, int K, int fuse, int subset,
                int parts, uint32_t* ctr, uint32_t* scr, uint32_t* err, bool pdl = true) {
    constexpr int T = tile_threads<LB, NQ>();
    if (parts > 1)
        launch_pdl(pdl, rem_kernel<LB, NQ, true>, blocks, T, smem, s, E, K, fuse, subset, parts, ctr, scr, err);
    else
        launch_pdl(pdl, rem_kernel<LB, NQ, false>, blocks, T, smem, s, E, K, fuse, subset, 1, (uint32_t*)nullptr,
                   (uint32_t*)nullptr, err);
}

template <int LB, int NQ>
void launch_round(unsigned blocks, size_t smem, cudaStream_t s, const batch::Elec& E, const batch::Elec& En, int K,
                  uint32_t* state, int parts, uint32_t* ctr, uint32_t* scr, uint32_t* err) {
    constexpr int T = tile_threads<LB, NQ>();
    if (parts > 1)
        launch_pdl(true, round_kernel<LB, NQ, true>, blocks, T, smem, s, E, En, K, state, parts, ctr, scr, err);
    else
        launch_pdl(true, round_kernel<LB, NQ, false>, blocks, T, smem, s, E, En, K, state, 1, (uint32_t*)nullptr,
                   (uint32_t*)nullptr, err);
}

// Rounds of the blocked closure on an initialised working matrix, in schedule `mode` (1, 3 or
// 4; see g_closure_mode). phase_ms (optional, 4 entries): accumulated device time of the pivot
// launches, the panel launches, (unused) and the remainder launches, from events recorded
// between launches.
// The second stream of the two-stream schedule, one per device, at the lowest priority so that
// the caller's stream (the per-round chain) gets SMs first.
se_status_t side_stream(cudaStream_t* out) {
    constexpr int kMaxDev = 64;
    static std::mutex m;
    static cudaStream_t streams[kMaxDev] = {};
    int dev = 0;
    SE_CUDA_TRY(cudaGetDevice(&dev));
    SE_REQUIRE(dev >= 0 && dev < kMaxDev, SE_ERR_INVALID, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lock(m);
    if (!streams[dev]) {
        int least = 0, greatest = 0;
        SE_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        SE_CUDA_TRY(cudaStreamCreateWithPriority(&streams[dev], cudaStreamNonBlocking, least));
    }
    *out = streams[dev];
    return SE_OK;
}

// Schedule 5 (see g_closure_mode). Per round k < R-1, with A the caller's stream and B the side
// stream, and E[k % 2] the descriptor whose AT buffer round k uses:
//   B: wait panels(k); remainder(k) off rows and columns k, k+1; record remB[k]
//   A: wait remB[k-1]; remainder(k) of row and column k+1, tile (k+1, k+1) first and closed as
//      the next pivot; panels(k+1) into the other AT buffer; record panels[k+1]
// then the last round's whole remainder on A after remB[R-2]. Reads and writes that could meet:
// panels(k+1) writes AT[(k+1) % 2] while remainder(k) reads AT[k % 2]; it writes rows and
// columns k+1, which no tile of B's remainder(k) reads or writes; remainder(k+1) of row and
// column k+2 waits for all of remainder(k) (it rewrites tiles of row k that remainder(k)
// reads); B's remainder(k+1) follows B's remainder(k) on B and waits for panels(k+1), which
// follows A's remainder(k) on A.
template <int LB>
se_status_t run_two_streams(const batch::Elec (&E)[2], int R, cudaStream_t A, uint32_t* S, int64_t ldw,
                            uint32_t* dT, uint32_t* err, double* phase_ms) {
    using CF = cfg<LB>;
    constexpr bool wide = LB == 16;
    const size_t smem = batch::pcfg<LB>::SMEM;
    cudaStream_t B = nullptr;
    if (se_status_t st = side_stream(&B)) return st;
    std::vector<cudaEvent_t> ev(size_t(2 * R + 2), nullptr);  // panels[0..R), remB[0..R), start, end
    struct Guard {
        std::vector<cudaEvent_t>& ev;
        ~Guard() {
            for (auto e : ev)
                if (e) cudaEventDestroy(e);
        }
    } guard{ev};
    for (size_t i = 0; i < ev.size(); ++i) {
        const unsigned flags = (phase_ms && i >= size_t(2 * R)) ? cudaEventDefault : cudaEventDisableTiming;
        SE_CUDA_TRY(cudaEventCreateWithFlags(&ev[i], flags));
    }
    cudaEvent_t* pan = ev.data();
    cudaEvent_t* remb = ev.data() + R;
    if (phase_ms) SE_CUDA_TRY(cudaEventRecord(ev[2 * R], A));
    auto panels = [&](int K) {
        if constexpr (wide)
            launch_panels<LB, 4>(unsigned(2 * (R - 1)), smem, A, E[K & 1], K, 1, nullptr, nullptr, err, false);
        else launch_panels<LB, 8>(unsigned(2 * (R - 1)), smem, A, E[K & 1], K, 1, nullptr, nullptr, err, false);
    };
    if constexpr (wide) diag_kernel<LB, 4><<<1, tile_threads<LB, 4>(), 0, A>>>(S, ldw, 0, dT);
    else diag_kernel<LB><<<1, CF::THREADS, 0, A>>>(S, ldw, 0, dT);
    panels(0);
    SE_CHECK_LAUNCH();
    SE_CUDA_TRY(cudaEventRecord(pan[0], A));
    const int R2 = R - 2;
    for (int K = 0; K + 1 < R; ++K) {
        SE_CUDA_TRY(cudaStreamWaitEvent(B, pan[K], 0));
        launch_rem<LB, 8>(unsigned(R2 * R2), smem, B, E[K & 1], K, 0, 2, 1, nullptr, nullptr, err, false);
        SE_CUDA_TRY(cudaEventRecord(remb[K], B));
        if (K > 0) SE_CUDA_TRY(cudaStreamWaitEvent(A, remb[K - 1], 0));
        launch_rem<LB, 8>(unsigned(2 * R - 3), smem, A, E[K & 1], K, 1, 1, 1, nullptr, nullptr, err, false);
        panels(K + 1);
        SE_CHECK_LAUNCH();
        SE_CUDA_TRY(cudaEventRecord(pan[K + 1], A));
    }
    SE_CUDA_TRY(cudaStreamWaitEvent(A, remb[R - 2], 0));
    launch_rem<LB, 8>(unsigned((R - 1) * (R - 1)), smem, A, E[(R - 1) & 1], R - 1, 0, 0, 1, nullptr, nullptr, err,
                      false);
    SE_CHECK_LAUNCH();
    if (phase_ms) {
        SE_CUDA_TRY(cudaEventRecord(ev[2 * R + 1], A));
        SE_CUDA_TRY(cudaEventSynchronize(ev[2 * R + 1]));
        float ms = 0.f;
        SE_CUDA_TRY(cudaEventElapsedTime(&ms, ev[2 * R], ev[2 * R + 1]));
        for (int q = 0; q < 4; ++q) phase_ms[q] = 0.0;
        phase_ms[3] = ms;  // the rounds overlap across the two streams: one figure for all
    }
    return SE_OK;
}

// split_room: the workspace holds the split-K area (layout split_ctr_off..flow_total).
template <int LB>
se_status_t run_rounds(uint8_t* work, const layout& P, cudaStream_t stream, double* phase_ms, int mode,
                       bool split_room) {
    using CF = cfg<LB>;
    if (se_status_t st = set_smem_limits<LB>(); st != SE_OK) return st;
    uint32_t* S = reinterpret_cast<uint32_t*>(work + P.s_off);
    uint32_t* AT = reinterpret_cast<uint32_t*>(work + P.at_off);
    uint32_t* dT = reinterpret_cast<uint32_t*>(work + P.dt_off);
    uint32_t* err = reinterpret_cast<uint32_t*>(work + P.flags_off);
    const int64_t ldw = P.Cp / CF::CPW;
    const int R = int(P.Cp / kT);
    const bool wide = LB == 16 && (mode == 3 || mode == 4 || mode == 7);
    const bool wide_rem = LB == 16 && mode == 7;
    const bool fused = !(LB == 16 && mode == 4);

    batch::Elec E;
    std::memset(&E, 0, sizeof(E));
    if (se_status_t st = make_map(&E.mapS, S, uint64_t(ldw), uint64_t(P.Cp), uint64_t(ldw) * 4, CF::TW, kKC); st)
        return st;
    if (se_status_t st = make_map(&E.mapAT, AT, uint64_t(P.Cp), kT, uint64_t(P.Cp) * 4, kT, kKC); st) return st;
    if (se_status_t st = make_map(&E.mapDT, dT, kT, kT, kT * 4, kT, kKC); st) return st;
    E.S = S;
    E.AT = AT;
    E.dT = dT;
    E.C = int(P.C);
    E.Cp = int(P.Cp);
    E.R = R;
    E.lanes = LB;
    const size_t smem = batch::pcfg<LB>::SMEM;
    // Split-K panels and next pivot tile (batch::SplitK) where the rounds are few enough for
    // the split tasks to fit one wave; the counters start at zero.
    const int parts = split_room && mode != 5 ? split_parts(R) : 1;
    uint32_t* split_ctr = parts > 1 ? reinterpret_cast<uint32_t*>(work + P.split_ctr_off) : nullptr;
    uint32_t* split_scr = parts > 1 ? reinterpret_cast<uint32_t*>(work + P.split_scr_off) : nullptr;
    if (parts > 1) SE_CUDA_TRY(cudaMemsetAsync(split_ctr, 0, size_t(2 * R) * 4, stream));
    if (mode == 5) {
        batch::Elec E2[2] = {E, E};
        uint32_t* AT2 = reinterpret_cast<uint32_t*>(work + P.at2_off);
        if (se_status_t st = make_map(&E2[1].mapAT, AT2, uint64_t(P.Cp), kT, uint64_t(P.Cp) * 4, kT, kKC); st)
            return st;
        E2[1].AT = AT2;
        return run_two_streams<LB>(E2, R, stream, S, ldw, dT, err, phase_ms);
    }
    if (mode == 6 || mode == 8) {
        const bool wide8 = LB == 16 && mode == 8;
        batch::Elec E2[2] = {E, E};
        uint32_t* AT2 = reinterpret_cast<uint32_t*>(work + P.at2_off);
        if (se_status_t st = make_map(&E2[1].mapAT, AT2, uint64_t(P.Cp), kT, uint64_t(P.Cp) * 4, kT, kKC); st)
            return st;
        E2[1].AT = AT2;
        uint32_t* state = reinterpret_cast<uint32_t*>(work + P.state_off);
        SE_CUDA_TRY(cudaMemsetAsync(state, 0, size_t(2 * R) * 4, stream));
        // Profiling: events after the round-0 pivot (phase 0), the round-0 panels (phase 1), and
        // every later launch (phase 3: each round's remainder with the next round's panels).
        std::vector<cudaEvent_t> ev;
        struct Guard {
            std::vector<cudaEvent_t>& ev;
            ~Guard() {
                for (auto e : ev) cudaEventDestroy(e);
            }
        } guard{ev};
        auto mark = [&]() -> se_status_t {
            if (!phase_ms) return SE_OK;
            cudaEvent_t e = nullptr;
            SE_CUDA_TRY(cudaEventCreate(&e));
            ev.push_back(e);
            SE_CUDA_TRY(cudaEventRecord(e, stream));
            return SE_OK;
        };
        if (se_status_t st = mark()) return st;
        if (wide8) {
            if constexpr (LB == 16) launch_pdl(true, diag_kernel<LB, 4>, 1u, tile_threads<LB, 4>(), 0, stream, S, ldw, 0, dT);
        } else {
            launch_pdl(true, diag_kernel<LB>, 1u, CF::THREADS, 0, stream, S, ldw, 0, dT);
        }
        if (se_status_t st = mark()) return st;
        const unsigned panel_blocks = unsigned(2 * (R - 1) * parts);
        if (wide8) {
            if constexpr (LB == 16)
                launch_panels<LB, 4>(panel_blocks, smem, stream, E2[0], 0, parts, split_ctr, split_scr, err);
        } else {
            launch_panels<LB, 8>(panel_blocks, smem, stream, E2[0], 0, parts, split_ctr, split_scr, err);
        }
        SE_CHECK_LAUNCH();
        if (se_status_t st = mark()) return st;
        const int tasks = (R - 1) * (R - 1) + (parts - 1) + 2 * (R - 1) * parts;
        for (int K = 0; K + 1 < R; ++K) {
            if (wide8) {
                if constexpr (LB == 16)
                    launch_round<LB, 4>(unsigned(tasks), smem, stream, E2[K & 1], E2[(K + 1) & 1], K, state + 2 * K,
                                        parts, split_ctr, split_scr, err);
            } else {
                launch_round<LB, 8>(unsigned(tasks), smem, stream, E2[K & 1], E2[(K + 1) & 1], K, state + 2 * K,
                                    parts, split_ctr, split_scr, err);
            }
            SE_CHECK_LAUNCH();
        }
        if (wide8) {
            if constexpr (LB == 16)
                launch_rem<LB, 4>(unsigned((R - 1) * (R - 1)), smem, stream, E2[(R - 1) & 1], R - 1, 0, 0, 1, nullptr,
                                  nullptr, err);
        } else {
            launch_rem<LB, 8>(unsigned((R - 1) * (R - 1)), smem, stream, E2[(R - 1) & 1], R - 1, 0, 0, 1, nullptr,
                              nullptr, err);
        }
        SE_CHECK_LAUNCH();
        if (se_status_t st = mark()) return st;
        if (phase_ms) {
            SE_CUDA_TRY(cudaEventSynchronize(ev.back()));
            float a = 0.f, b = 0.f, c = 0.f;
            SE_CUDA_TRY(cudaEventElapsedTime(&a, ev[0], ev[1]));
            SE_CUDA_TRY(cudaEventElapsedTime(&b, ev[1], ev[2]));
            SE_CUDA_TRY(cudaEventElapsedTime(&c, ev[2], ev[3]));
            phase_ms[0] = a;
            phase_ms[1] = b;
            phase_ms[2] = 0.0;
            phase_ms[3] = c;
        }
        return SE_OK;
    }

    // Events between launches when profiling: (phase, event recorded after the launch).
    std::vector<std::pair<int, cudaEvent_t>> ev;
    cudaEvent_t start = nullptr;
    se_status_t failed = SE_OK;
    auto mark = [&](int phase) {
        if (!phase_ms || failed) return;
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            failed = SE_ERR_CUDA;
            set_error("cannot create a profiling event");
            return;
        }
        cudaEventRecord(e, stream);
        ev.emplace_back(phase, e);
    };
    if (phase_ms) {
        if (cudaEventCreate(&start) != cudaSuccess) SE_CUDA_TRY(cudaGetLastError());
        cudaEventRecord(start, stream);
    }
    auto pivot = [&](int K) {
        if (wide) {
            if constexpr (LB == 16) launch_pdl(true, diag_kernel<LB, 4>, 1u, tile_threads<LB, 4>(), 0, stream, S, ldw, K, dT);
        } else {
            launch_pdl(true, diag_kernel<LB>, 1u, CF::THREADS, 0, stream, S, ldw, K, dT);
        }
        mark(0);
    };
    pivot(0);
    SE_CHECK_LAUNCH();
    for (int K = 0; K < R && R > 1; ++K) {
        if (K > 0 && !fused) pivot(K);
        const unsigned panel_blocks = unsigned(2 * (R - 1) * parts);
        if (wide) {
            if constexpr (LB == 16) launch_panels<LB, 4>(panel_blocks, smem, stream, E, K, parts, split_ctr, split_scr, err);
        } else {
            launch_panels<LB, 8>(panel_blocks, smem, stream, E, K, parts, split_ctr, split_scr, err);
        }
        mark(1);
        // Tile (K+1, K+1) and its pivot: counter and partials after the panel tiles'.
        const int fuse = fused && K + 1 < R ? 1 : 0;
        const unsigned rem_blocks = unsigned((R - 1) * (R - 1) + (fuse && parts > 1 ? parts - 1 : 0));
        uint32_t* pctr = split_ctr ? split_ctr + 2 * (R - 1) : nullptr;
        uint32_t* pscr = split_scr ? split_scr + int64_t(2 * (R - 1)) * parts * kT * CF::TW : nullptr;
        if (wide_rem) {
            if constexpr (LB == 16) launch_rem<LB, 4>(rem_blocks, smem, stream, E, K, fuse, 0, parts, pctr, pscr, err);
        } else {
            launch_rem<LB, 8>(rem_blocks, smem, stream, E, K, fuse, 0, parts, pctr, pscr, err);
        }
        mark(3);
        SE_CHECK_LAUNCH();
    }
    if (phase_ms) {
        for (int q = 0; q < 4; ++q) phase_ms[q] = 0.0;
        cudaError_t e = ev.empty() ? cudaSuccess : cudaEventSynchronize(ev.back().second);
        if (e == cudaSuccess) {
            cudaEvent_t prev = start;
            for (auto& x : ev) {
                float ms = 0.f;
                cudaEventElapsedTime(&ms, prev, x.second);
                phase_ms[x.first] += ms;
                prev = x.second;
            }
        }
        for (auto& x : ev) cudaEventDestroy(x.second);
        cudaEventDestroy(start);
        if (failed) return failed;
        SE_CUDA_TRY(e);
    }
    return SE_OK;
}

// The dataflow closure on an initialised working matrix (pivot of round 0 included).
template <int LB>
se_status_t run_flow(uint8_t* work, const layout& P, cudaStream_t stream, double* phase_ms) {
    using CF = cfg<LB>;
    if (se_status_t st = set_smem_limits<LB>(); st != SE_OK) return st;
    uint32_t* S = reinterpret_cast<uint32_t*>(work + P.s_off);
    uint32_t* err = reinterpret_cast<uint32_t*>(work + P.flags_off);
    const int64_t ldw = P.Cp / CF::CPW;
    const int R = int(P.Cp / kT);
    batch::Elec E[2];
    for (int b = 0; b < 2; ++b) {
        std::memset(&E[b], 0, sizeof(E[b]));
        uint32_t* AT = reinterpret_cast<uint32_t*>(work + (b ? P.at2_off : P.at_off));
        uint32_t* dT = reinterpret_cast<uint32_t*>(work + (b ? P.dt2_off : P.dt_off));
        if (se_status_t st = make_map(&E[b].mapS, S, uint64_t(ldw), uint64_t(P.Cp), uint64_t(ldw) * 4, CF::TW, kKC))
            return st;
        if (se_status_t st = make_map(&E[b].mapAT, AT, uint64_t(P.Cp), kT, uint64_t(P.Cp) * 4, kT, kKC)) return st;
        if (se_status_t st = make_map(&E[b].mapDT, dT, kT, kT, kT * 4, kT, kKC)) return st;
        E[b].S = S;
        E[b].AT = AT;
        E[b].dT = dT;
        E[b].C = int(P.C);
        E[b].Cp = int(P.Cp);
        E[b].R = R;
        E[b].lanes = LB;
    }
    uint32_t* state = reinterpret_cast<uint32_t*>(work + P.state_off);
    SE_CUDA_TRY(cudaMemsetAsync(state, 0, size_t(4 + R * R + 2 * R) * 4, stream));
    int device = 0, sms = 0, occ = 0;
    SE_CUDA_TRY(cudaGetDevice(&device));
    SE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    SE_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, flow_kernel<LB>, CF::THREADS,
                                                              batch::pcfg<LB>::SMEM));
    SE_REQUIRE(occ >= 1, SE_ERR_CUDA, "dataflow closure kernel cannot be resident");
    const int64_t total = int64_t(R) * R * R;
    const int grid = int(std::min<int64_t>(total, int64_t(sms) * occ));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (phase_ms) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
    }
    flow_kernel<LB><<<grid, CF::THREADS, batch::pcfg<LB>::SMEM, stream>>>(E[0], E[1], state, err);
    SE_CHECK_LAUNCH();
    if (phase_ms) {
        cudaEventRecord(e1, stream);
        cudaError_t e = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (e == cudaSuccess) cudaEventElapsedTime(&ms, e0, e1);
        for (int q = 0; q < 4; ++q) phase_ms[q] = 0.0;
        phase_ms[3] = ms;  // one launch: pivots, panels and remainders together
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        SE_CUDA_TRY(e);
    }
    return SE_OK;
}

template <int LB>
se_status_t launch_init(const uint32_t* d, int64_t ld, int C, const layout& P, uint8_t* work, uint32_t base,
                        cudaStream_t s) {
    const int nb = int(P.Cp / 32);
    init_kernel<LB><<<dim3(nb, nb), dim3(32, 8), 0, s>>>(d, ld, C, int(P.Cp), work + P.s_off, base,
                                                       reinterpret_cast<uint32_t*>(work + P.flags_off));
    SE_CHECK_LAUNCH();
    return SE_OK;
}

template <int LB>
se_status_t launch_finalize(const layout& P, uint8_t* work, int C, uint32_t* out, int64_t ld_out, uint32_t base,
                            cudaStream_t s) {
    const int gx = int((C + 255) / 256);
    const int gy = C < 65535 ? C : 65535;
    launch_pdl(true, finalize_kernel<LB>, dim3(unsigned(gx), unsigned(gy)), 256, 0, s,
               static_cast<const void*>(work + P.s_off), int(P.Cp), C, out, ld_out, base);
    SE_CHECK_LAUNCH();
    return SE_OK;
}

// Defeat init of one election into a padded working matrix (u16 lanes shifted by base, or
// u32), for callers outside this file (the serving engine).
se_status_t launch_defeat_init(const uint32_t* d, int64_t ld, int C, int Cp, void* S, int lane_bits, uint32_t base,
                               uint32_t* flags, cudaStream_t s) {
    const int nb = Cp / 32;
    if (lane_bits == 16)
        init_kernel<16><<<dim3(nb, nb), dim3(32, 8), 0, s>>>(d, ld, C, Cp, S, base, flags);
    else
        init_kernel<32><<<dim3(nb, nb), dim3(32, 8), 0, s>>>(d, ld, C, Cp, S, 0, flags);
    SE_CHECK_LAUNCH();
    return SE_OK;
}

}  // namespace closure
}  // namespace se

using namespace se;
using namespace se::closure;

extern "C" int64_t se_closure_workspace_bytes(int C, int lane_bits, int tile) {
    if (C < 1 || (tile != 0 && tile != kT)) return -1;
    return plan(C, lane_bits == 16 ? 16 : 32).total;
}

namespace se {
namespace closure {
se_status_t check_flags(const void* flags_dev, cudaStream_t s);

// The closure behind every entry point. mode: 0/1 round by round, 2 dataflow, -1 the
// process-wide choice (se_closure_set_mode). sync: read the flags back and report overflow or
// a device error (else the call is stream-ordered and se_closure_check reports them later).
// value_offset: the 16-bit lane shift when lane_bits is 16 (0 = none); the automatic mode
// (lane_bits 0) measures its own and needs sync.
se_status_t closure_run(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out, int64_t ld_out,
                        int lane_bits, uint32_t value_offset, int tile, void* d_work, int64_t work_bytes,
                        void* stream_, double* phase_ms, int mode_override, bool sync) {
    clear_error();
    SE_REQUIRE(C >= 1, SE_ERR_INVALID, "Number of candidates must be positive");
    SE_REQUIRE(C <= (1 << 20), SE_ERR_INVALID, "Number of candidates too large (%d)", C);
    SE_REQUIRE(d_pref && d_out, SE_ERR_INVALID, "null matrix pointer");
    SE_REQUIRE(ld_pref >= C && ld_out >= C, SE_ERR_INVALID, "row stride smaller than the number of candidates");
    SE_REQUIRE(lane_bits == 0 || lane_bits == 16 || lane_bits == 32, SE_ERR_INVALID, "lane_bits must be 0, 16 or 32");
    SE_REQUIRE(lane_bits != 0 || sync, SE_ERR_INVALID,
               "automatic lanes read the matrix's range back to the host; pass 16 or 32 to enqueue");
    SE_REQUIRE(value_offset == 0 || lane_bits == 16, SE_ERR_INVALID, "a value offset applies to 16-bit lanes only");
    SE_REQUIRE(tile == 0 || tile == kT, SE_ERR_UNSUPPORTED, "Unsupported tile size");
    const int64_t need = se_closure_workspace_bytes(C, lane_bits, tile);
    SE_REQUIRE(d_work != nullptr && work_bytes >= need, SE_ERR_WORKSPACE,
               "workspace of %lld bytes is smaller than the %lld bytes required", (long long)work_bytes,
               (long long)need);
    SE_REQUIRE((reinterpret_cast<uintptr_t>(d_work) & 255) == 0, SE_ERR_INVALID, "workspace must be 256-byte aligned");
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    uint8_t* work = static_cast<uint8_t*>(d_work);

    int lb = lane_bits == 0 ? 16 : lane_bits;
    uint32_t base = value_offset;
    SE_CUDA_TRY(cudaMemsetAsync(work, 0, 256, s));
    if (lane_bits == 0) {
        // Automatic lanes: 16-bit (shifted by a base if need be) whenever the kept values fit
        // a 65535-wide window, else 32-bit. One 8-byte read back.
        SE_CUDA_TRY(cudaMemsetAsync(work + 8, 0xFF, 4, s));
        const int nb = int(round_up(C, 32) / 32);
        kept_range_kernel<<<dim3(nb, nb), dim3(32, 8), 0, s>>>(d_pref, ld_pref, C,
                                                              reinterpret_cast<uint32_t*>(work));
        SE_CHECK_LAUNCH();
        uint32_t range[2] = {0, 0};
        SE_CUDA_TRY(cudaMemcpyAsync(range, work + 8, 8, cudaMemcpyDeviceToHost, s));
        SE_CUDA_TRY(cudaStreamSynchronize(s));
        const uint32_t lo = range[0], hi = range[1];
        if (hi <= 0xFFFFu) {
            lb = 16;
        } else if (hi - lo < 0xFFFFu) {
            lb = 16;
            base = lo - 1u;
        } else {
            lb = 32;
        }
    }
    const layout P = plan(C, lb);
    if (lb == 16) {
        if (se_status_t st = launch_init<16>(d_pref, ld_pref, C, P, work, base, s)) return st;
    } else {
        if (se_status_t st = launch_init<32>(d_pref, ld_pref, C, P, work, 0, s)) return st;
    }
    int mode = mode_override >= 0 ? mode_override : g_closure_mode.load();
    const bool automatic = mode == 0;
    if (automatic) mode = automatic_mode(C);
    if (mode == 5 && (P.Cp / kT < 4 || (automatic && work_bytes < P.flow_total))) mode = 3;
    if ((mode == 6 || mode == 8) && (P.Cp / kT < 2 || (automatic && work_bytes < P.flow_total))) mode = 1;
    const bool flow = mode == 2 && P.Cp > kT;
    SE_REQUIRE((mode != 2 && mode != 5 && mode != 6 && mode != 8) || work_bytes >= P.flow_total, SE_ERR_WORKSPACE,
               "the dataflow, two-stream and one-launch-per-round closures need a workspace of %lld bytes",
               (long long)P.flow_total);
    se_status_t st = flow ? (lb == 16 ? run_flow<16>(work, P, s, phase_ms) : run_flow<32>(work, P, s, phase_ms))
                          : (lb == 16 ? run_rounds<16>(work, P, s, phase_ms, mode, work_bytes >= P.flow_total)
                                      : run_rounds<32>(work, P, s, phase_ms, mode, work_bytes >= P.flow_total));
    if (st) return st;
    st = lb == 16 ? launch_finalize<16>(P, work, C, d_out, ld_out, base, s)
                  : launch_finalize<32>(P, work, C, d_out, ld_out, 0, s);
    if (st) return st;
    return sync ? check_flags(work + P.flags_off, s) : SE_OK;
}

// The flags word pair a closure leaves at the start of its workspace: [0] device error (a wait
// that timed out), [1] a kept value outside the 16-bit window. Synchronises s.
se_status_t check_flags(const void* flags_dev, cudaStream_t s) {
    uint32_t flags[2] = {0, 0};
    SE_CUDA_TRY(cudaMemcpyAsync(flags, flags_dev, 8, cudaMemcpyDeviceToHost, s));
    SE_CUDA_TRY(cudaStreamSynchronize(s));
    SE_REQUIRE(flags[1] == 0, SE_ERR_OVERFLOW,
               "a preference count exceeds 65535, which 16-bit lanes cannot hold; use 32-bit lanes");
    SE_REQUIRE(flags[0] == 0, SE_ERR_DEVICE, "closure kernel reported device error %u (TMA wait timed out)",
               flags[0]);
    return SE_OK;
}
}  // namespace closure
}  // namespace se

extern "C" se_status_t se_closure(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out, int64_t ld_out,
                                  int lane_bits, int tile, void* d_work, int64_t work_bytes, void* stream) {
    return host_guard([&] {
        return closure_run(d_pref, ld_pref, C, d_out, ld_out, lane_bits, 0, tile, d_work, work_bytes, stream, nullptr,
                           -1, true);
    });
}

extern "C" se_status_t se_closure_enqueue(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out,
                                          int64_t ld_out, int lane_bits, uint32_t value_offset, void* d_work,
                                          int64_t work_bytes, void* stream) {
    return host_guard([&] {
        return closure_run(d_pref, ld_pref, C, d_out, ld_out, lane_bits, value_offset, 0, d_work, work_bytes, stream,
                           nullptr, -1, false);
    });
}

extern "C" se_status_t se_closure_check(const void* d_work, void* stream) {
    return host_guard([&] {
        clear_error();
        SE_REQUIRE(d_work != nullptr, SE_ERR_INVALID, "null workspace");
        return check_flags(d_work, static_cast<cudaStream_t>(stream));
    });
}

extern "C" se_status_t se_closure_profiled(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out,
                                           int64_t ld_out, int lane_bits, int tile, void* d_work, int64_t work_bytes,
                                           void* stream, double* phase_ms, int* launches) {
    se_status_t st = host_guard([&] {  // the phase events' vector is filled before any event exists
        return closure_run(d_pref, ld_pref, C, d_out, ld_out, lane_bits, 0, tile, d_work, work_bytes, stream, phase_ms,
                           -1, true);
    });
    if (launches) *launches = se_closure_launch_count(C);
    return st;
}

extern "C" int64_t se_closure_workspace_bytes_flow(int C, int lane_bits, int tile) {
    if (C < 1 || (tile != 0 && tile != kT)) return -1;
    return plan(C, lane_bits == 16 ? 16 : 32).flow_total;
}

extern "C" se_status_t se_closure_flow_task(uint32_t t, int R, int* kind, int* k, int* i, int* j) {
    clear_error();
    SE_REQUIRE(R >= 2 && R <= 1024 && uint64_t(t) < uint64_t(R) * R * R, SE_ERR_INVALID, "task out of range");
    const FlowTask T = flow_decode(t, R);
    if (kind) *kind = T.kind;
    if (k) *k = T.k;
    if (i) *i = T.i;
    if (j) *j = T.j;
    return SE_OK;
}

extern "C" se_status_t se_closure_set_mode(int mode) {
    clear_error();
    SE_REQUIRE(mode >= 0 && mode <= 8, SE_ERR_INVALID, "closure mode must be 0 to 8");
    g_closure_mode.store(mode);
    return SE_OK;
}

extern "C" int se_closure_schedule(int C, int lane_bits, int64_t work_bytes) {
    if (C < 1) return -1;
    const layout P = plan(C, lane_bits == 32 ? 32 : 16);
    int mode = g_closure_mode.load();
    const bool automatic = mode == 0;
    if (automatic) mode = automatic_mode(C);
    if (mode == 5 && (P.Cp / kT < 4 || (automatic && work_bytes < P.flow_total))) mode = 3;
    if ((mode == 6 || mode == 8) && (P.Cp / kT < 2 || (automatic && work_bytes < P.flow_total))) mode = 1;
    if (lane_bits == 32 && (mode == 3 || mode == 4 || mode == 7)) mode = 1;
    if (lane_bits == 32 && mode == 8) mode = 6;
    return mode;
}

extern "C" se_status_t se_closure_set_variant_table(const int* max_c, const int* modes, int n) {
    return host_guard([&]() -> se_status_t {
        clear_error();
        SE_REQUIRE(n >= 0 && n <= kMaxVariants, SE_ERR_INVALID, "at most %d table entries", kMaxVariants);
        SE_REQUIRE(n == 0 || (max_c && modes), SE_ERR_INVALID, "null table");
        for (int i = 0; i < n; ++i)
            SE_REQUIRE(modes[i] == 1 || (modes[i] >= 3 && modes[i] <= 8), SE_ERR_INVALID,
                       "table modes must be 1 or 3 to 8 (got %d)", modes[i]);
        std::lock_guard<std::mutex> lock(g_variant_mutex);
        for (int i = 0; i < n; ++i) {
            g_variant_max_c[i] = max_c[i];
            g_variant_mode[i] = modes[i];
        }
        g_variant_n = n;
        return SE_OK;
    });
}

extern "C" int se_closure_launch_count(int C) {
    if (C < 1) return 0;
    const int R = int(round_up(C, kT) / kT);
    int mode = g_closure_mode.load();
    if (mode == 0) mode = automatic_mode(C);
    // init, pivot of round 0, R x (panels, remainder), finalize; mode 4 adds a pivot launch
    // per later round (in 16-bit lanes), mode 5 a second remainder launch per round but the last.
    if ((mode == 6 || mode == 8) && R >= 2) return 3 + R + 1;  // init, pivot, panels 0, R - 1 rounds, last, finalize
    return R == 1 ? 3 : 3 + 2 * R + (mode == 4 || (mode == 5 && R >= 4) ? R - 1 : 0);
}
