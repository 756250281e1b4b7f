// Batched persistent widest-path closure: many independent elections of uneven size in one
// launch per lane mode (no reference counterpart; the reference closes one matrix per call,
// scaling_elections.cu:863-989, one host-synchronised round at a time).
//
// Work is cut into tasks, all on 128 x 128 tiles:
//   SMALL      an election with C <= 128, whole in one CTA: defeat init from d, closure over
//              its C pivots in registers, u32 output, wins and ranking. Nothing in HBM but d
//              and the outputs.
//   PIVOT k    close the pivot tile (k, k) of a larger election in registers; emit dT.
//   ROW k, j   pivot-row panel tile (k, j)       = max(P, D (x) P)
//   COL k, i   pivot-column panel tile (i, k)    = max(P, P (x) D); emit AT (transposed).
//   REM k,i,j  remainder tile (i, j)             = max(S, AT (x) S[k][j])
// using the same device routines as the single-election kernels (closure_core.cuh).
//
// Scheduling: one persistent grid (every CTA resident) pulls tasks from a queue with an atomic
// counter. The queue is ordered so that every task comes after the tasks it depends on:
// round-major across elections (all pivots of round k, then all panels, then all remainders,
// largest elections first), then the SMALL tasks, which fill the tail. A task waits (thread 0,
// bounded by %globaltimer) on its election's per-round counters:
//   PIVOT k   needs REM k-1 complete ((R-1)^2 tiles)
//   ROW/COL k needs PIVOT k
//   REM k     needs all 2(R-1) panels of round k
// Because a task's prerequisites were dequeued earlier by CTAs that are running, and those only
// wait on even earlier tasks, the schedule cannot deadlock. A wait that times out sets the
// error word and an abort flag that makes every CTA drain the queue and exit.
//
// Memory ordering: a finished task's threads fence (gpu scope), the CTA barriers, and thread 0
// bumps the counter. A waiting task's thread 0 reads the counter with acquire semantics, then
// fences the async proxy before its TMA loads; generic loads of tiles another CTA wrote go
// through ld.global.cg (L2), never a possibly stale L1 line.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "batch_core.cuh"

namespace se {
namespace batch {
using namespace se::closure;

struct Header {
    uint32_t err;
    uint32_t abort;
    uint32_t head[3];  // queue heads of the persistent launches: u16, u32, u16 on the wide micro-tile
    uint32_t pad;
    // Profile: per task kind (SMALL, PIVOT, ROW, COL, REM) CTA-nanoseconds busy and tasks run;
    // CTA-nanoseconds waiting for dependencies.
    unsigned long long busy_ns[5];
    unsigned long long tasks[5];
    unsigned long long wait_ns;
};

// The counter a task of election E waits for and the value it must reach; false for a task
// with no dependency (SMALL, and PIVOT 0).
__device__ __forceinline__ bool task_dependency(const Elec& E, uint32_t type, uint32_t k, const uint32_t*& ctr,
                                                uint32_t& target) {
    const uint32_t R = uint32_t(E.R);
    if (type == kPivot && k > 0) {
        ctr = &E.counters[2 * R + k - 1];
        target = (R - 1) * (R - 1);
    } else if (type == kRow || type == kCol) {
        ctr = &E.counters[k];
        target = 1u;
    } else if (type == kRem) {
        ctr = &E.counters[R + k];
        target = 2u * (R - 1);
    } else {
        return false;
    }
    return true;
}

// One thread: claims the next task of the queue into s_next, and records whether its
// dependency is met already (counters only grow, so it stays met).
__device__ __forceinline__ void claim_task(const Elec* elecs, const uint64_t* tasks, uint32_t ntasks, Header* hdr,
                                           int queue, uint64_t& s_next, uint32_t& s_ready) {
    uint64_t t = kNoTask;
    uint32_t ready = 0;
    const uint32_t n = atomicAdd(&hdr->head[queue], 1u);
    if (n < ntasks && !ld_acquire(&hdr->abort)) {
        t = tasks[n];
        const uint32_t e = uint32_t(t >> 39), type = uint32_t(t >> 36) & 7u, k = uint32_t(t >> 24) & 0xFFFu;
        const uint32_t* ctr;
        uint32_t target;
        ready = !task_dependency(elecs[e], type, k, ctr, target) || ld_acquire(ctr) >= target;
    }
    s_next = t;
    s_ready = ready;
}

// NQ: the tile tasks' micro-tile, 8 (8 x 8 words, the default) or 4 (8 x 4 words, 256 threads,
// 16-bit lanes: elections with C > 128 whose size bucket the autotuner gave the wide one; small
// elections always run on the default, whose SMALL routine is written for it).
template <int LB, int NQ = 8>
__global__ void __launch_bounds__(tile_threads<LB, NQ>(), NQ == 4 ? 2 : 1)
    persistent_kernel(const Elec* __restrict__ elecs, const uint64_t* __restrict__ tasks, uint32_t ntasks,
                      Header* __restrict__ hdr, int queue, uint64_t dep_wait_ns) {
    using CF = cfg<LB>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    __shared__ int32_t s_wins[kT];
    __shared__ uint64_t s_task, s_next;
    __shared__ uint32_t s_go, s_ready;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + pcfg<LB>::DATA);
    if (threadIdx.x == 0) {
        for (int b = 0; b < 2 * kChunks; ++b) mbar_init(&bars[b], 1);
        fence_barrier_init();
    }
    if (threadIdx.x == 32) claim_task(elecs, tasks, ntasks, hdr, queue, s_next, s_ready);
    __syncthreads();
    uint32_t par_a = 0, par_b = 0;  // phase parity of barriers [0, 4) and [4, 8)

    // The next task is claimed by thread 32 (warp 1) while the current task's first copies are
    // in flight, so only its dependency wait, when not met at claim time, stays between tasks.
    // No task waits while it runs, and every dependency precedes its dependents in the queue,
    // so a task claimed ahead never blocks the tasks it depends on.
    for (;;) {
        if (threadIdx.x == 0) {
            const uint64_t t = s_next;
            s_task = t;
            s_go = 1;
            if (t != kNoTask) {
                if (!s_ready) {
                    const uint32_t e = uint32_t(t >> 39), type = uint32_t(t >> 36) & 7u,
                                   k = uint32_t(t >> 24) & 0xFFFu;
                    const uint32_t* ctr;
                    uint32_t target;
                    if (task_dependency(elecs[e], type, k, ctr, target)) {
                        const uint64_t w0 = global_ns();
                        const bool ok = wait_counter(ctr, target, &hdr->abort, dep_wait_ns);
                        atomicAdd(&hdr->wait_ns, (unsigned long long)(global_ns() - w0));
                        if (!ok) {
                            raise_device_error(&hdr->err, kErrDepTimeout);
                            atomicExch(&hdr->abort, 1u);
                            s_go = 0;
                        }
                    }
                }
                fence_proxy_async_global();
            }
        }
        __syncthreads();
        const uint64_t t = s_task;
        if (t == kNoTask || !s_go) break;
        if (threadIdx.x == 32) claim_task(elecs, tasks, ntasks, hdr, queue, s_next, s_ready);
        const uint32_t e = uint32_t(t >> 39), type = uint32_t(t >> 36) & 7u, k = uint32_t(t >> 24) & 0xFFFu;
        const uint32_t i = uint32_t(t >> 12) & 0xFFFu, j = uint32_t(t) & 0xFFFu;
        const Elec& E = elecs[e];
        bool ok = true;
        const uint64_t tb = threadIdx.x == 0 ? global_ns() : 0;
        if (type == kSmall) {
            if constexpr (NQ == 8) run_small<LB>(E, smem, rowbuf, colbuf, s_wins, &hdr->err);
            else ok = false;  // the host never queues one here
        } else if (type == kPivot) {
            run_pivot<LB, NQ>(E, int(k), rowbuf, colbuf);
        } else {
            const int kind = type == kRow ? kTileRow : (type == kCol ? kTileCol : kTileRem);
            ok = run_tile<LB, true, NQ>(E, &E, kind, int(k), int(i), int(j), smem, bars, par_a, par_b);
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            atomicAdd(&hdr->busy_ns[type], (unsigned long long)(global_ns() - tb));
            atomicAdd(&hdr->tasks[type], 1ull);
            if (!ok) {
                raise_device_error(&hdr->err, kErrTimeout);
                atomicExch(&hdr->abort, 1u);
            } else if (type != kSmall) {
                fence_proxy_async_global();
                const uint32_t R = uint32_t(E.R);
                const uint32_t slot = type == kPivot ? k : (type == kRem ? 2 * R + k : R + k);
                atomicAdd(&E.counters[slot], 1u);
            }
        }
        if (!ok) break;
    }
}

// ------------------------------------------------------------------------------------------
// Batched elementwise kernels over the elections with R >= 2: block b belongs to the big
// election m with prefix[m] <= b < prefix[m + 1].
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ int find_owner(const int64_t* prefix, int n, int64_t b) {
    int lo = 0, hi = n;  // prefix[lo] <= b < prefix[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (prefix[mid] <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

// The batched init and output kernels work on pairs of 64 x 64 tiles (I <= J over the
// election's Cp / 64 tiles per side, see upper_pair), 256 threads each. Thread (ry, cx) holds
// rows ry + 16p (p < 4) and columns 4cx .. 4cx+3 of both tiles, X[I][J] in a[] and X[J][I] in
// bt[], read once with 128-bit loads where the rows allow it. The tiles are also staged in
// shared memory (swz64), so every cell's transposed partner is one conflict-free read. (A form
// that moved the tiles through shared memory with lane-contiguous accesses instead, 128
// contiguous bytes per warp whatever the row stride, measured slower: output 7.5 against
// 4.2 ms per launch, init 3.3 against 3.0.)
constexpr int kPT = 64;

struct PairGeom {
    int I, J, i0, j0, cx, ry;
};

__device__ __forceinline__ PairGeom pair_geom(int64_t local, int Cp) {
    PairGeom g;
    upper_pair(local, Cp / kPT, g.I, g.J);
    g.i0 = g.I * kPT;
    g.j0 = g.J * kPT;
    g.cx = threadIdx.x & 15;
    g.ry = threadIdx.x >> 4;
    return g;
}

// X[row][c0 .. c0+3] of a C x C u32 matrix with row stride ld; cells past C read as 0.
__device__ __forceinline__ uint4 load4_u32(const uint32_t* X, int64_t ld, int C, int row, int c0, bool vec) {
    if (row >= C) return make_uint4(0u, 0u, 0u, 0u);
    const uint32_t* p = X + int64_t(row) * ld + c0;
    if (vec && c0 + 3 < C) return __ldg(reinterpret_cast<const uint4*>(p));
    return make_uint4(c0 < C ? __ldg(p) : 0u, c0 + 1 < C ? __ldg(p + 1) : 0u, c0 + 2 < C ? __ldg(p + 2) : 0u,
                      c0 + 3 < C ? __ldg(p + 3) : 0u);
}

// Resident CTAs per SM the init and output kernels are compiled for (registers): more CTAs keep
// more tile loads in flight.
constexpr int kPairCtasPerSm = 5;

// Block b of the init and output kernels works on pair `local` of election `e`.
struct PairOwner {
    int32_t e, local;
};

// Defeat matrix into the padded working matrix (see init_kernel in closure.cu): S[i][j] =
// d[i][j] if d[i][j] > d[j][i], else 0, for both tiles of the pair (on the diagonal d[i][i] >
// d[i][i] is false, and cells past C read 0, so the padding comes out 0). Also zeroes the
// election's wins.
__global__ void __launch_bounds__(256, kPairCtasPerSm)
    batch_init_kernel(const Elec* __restrict__ elecs, const PairOwner* __restrict__ owner, Header* __restrict__ hdr) {
    __shared__ __align__(16) uint32_t sa[kPT * kPT], sb[kPT * kPT];
    const PairOwner o = owner[blockIdx.x];
    const Elec& E = elecs[o.e];
    const int64_t local = o.local;
    const int C = E.C, Cp = E.Cp;
    const PairGeom g = pair_geom(local, Cp);
    if (local == 0 && E.wins)
        for (int x = threadIdx.x; x < C; x += 256) E.wins[x] = 0;
    const bool vec = E.ld % 4 == 0 && (reinterpret_cast<uintptr_t>(E.d) & 15) == 0;
    // Off the diagonal with both tiles inside the C candidates (CTA-uniform; i0 < j0), every
    // cell exists and the loads need no bounds.
    const bool interior = g.I != g.J && g.j0 + kPT <= C;
    // All eight 4-cell loads are issued before any is used (CTA-uniform branches around
    // straight-line code), so the CTA has both tiles in flight at once.
    uint4 a[4], bt[4];
    if (interior) {
        const uint32_t* pa = E.d + int64_t(g.i0 + g.ry) * E.ld + g.j0 + 4 * g.cx;
        const uint32_t* pb = E.d + int64_t(g.j0 + g.ry) * E.ld + g.i0 + 4 * g.cx;
        const int64_t step = 16 * E.ld;
        const bool half = E.ld % 2 == 0 && (reinterpret_cast<uintptr_t>(E.d) & 7) == 0;  // rows 8-byte aligned
        if (vec) {
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                a[p] = __ldg(reinterpret_cast<const uint4*>(pa + p * step));
                bt[p] = __ldg(reinterpret_cast<const uint4*>(pb + p * step));
            }
        } else if (half) {
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const uint2* x = reinterpret_cast<const uint2*>(pa + p * step);
                const uint2* y = reinterpret_cast<const uint2*>(pb + p * step);
                const uint2 x0 = __ldg(x), x1 = __ldg(x + 1), y0 = __ldg(y), y1 = __ldg(y + 1);
                a[p] = make_uint4(x0.x, x0.y, x1.x, x1.y);
                bt[p] = make_uint4(y0.x, y0.y, y1.x, y1.y);
            }
        } else {
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const uint32_t* x = pa + p * step;
                const uint32_t* y = pb + p * step;
                a[p] = make_uint4(__ldg(x), __ldg(x + 1), __ldg(x + 2), __ldg(x + 3));
                bt[p] = make_uint4(__ldg(y), __ldg(y + 1), __ldg(y + 2), __ldg(y + 3));
            }
        }
    } else if (vec) {
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int r = g.ry + 16 * p;
            a[p] = load4_u32(E.d, E.ld, C, g.i0 + r, g.j0 + 4 * g.cx, true);
            bt[p] = load4_u32(E.d, E.ld, C, g.j0 + r, g.i0 + 4 * g.cx, true);
        }
    } else {
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int r = g.ry + 16 * p;
            a[p] = load4_u32(E.d, E.ld, C, g.i0 + r, g.j0 + 4 * g.cx, false);
            bt[p] = load4_u32(E.d, E.ld, C, g.j0 + r, g.i0 + 4 * g.cx, false);
        }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int r = g.ry + 16 * p;
        swz64_store4(sa, r, 4 * g.cx, a[p]);
        swz64_store4(sb, r, 4 * g.cx, bt[p]);
    }
    __syncthreads();
    // Three CTA-uniform forms: u32 lanes; u16 lanes with base 0, where a kept value is its own
    // cell and one OR per cell finds any that would not fit (checked once at the end); and u16
    // lanes with a base, which checks each value against its window (to_lane16).
    const int form = E.lanes != 16 ? 0 : (E.base == 0 ? 1 : 2);
    const uint32_t base = E.base;
    bool over = false;
    uint32_t acc = 0;
    // One side: cells (x0 + r, y0 + 4cx + q), read back from their own tile's staging (so no
    // registers hold the tiles across the barrier), against their transposed partners in the
    // other tile's staging.
    auto emit = [&](auto form_tag, const uint32_t* own, const uint32_t* other, int x0, int y0) {
        constexpr int F = decltype(form_tag)::value;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int r = g.ry + 16 * p;
            const uint4 o4 = swz64_load4(own, r, 4 * g.cx);
            const uint32_t x[4] = {o4.x, o4.y, o4.z, o4.w};
            uint32_t v[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t y = other[swz64(4 * g.cx + q, r)];
                v[q] = x[q] > y ? x[q] : 0u;
            }
            const int64_t at = int64_t(x0 + r) * Cp + y0 + 4 * g.cx;
            if constexpr (F == 0) {
                *reinterpret_cast<uint4*>(E.S + at) = make_uint4(v[0], v[1], v[2], v[3]);
            } else {
                uint32_t h[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    if constexpr (F == 1) {
                        acc |= v[q];
                        h[q] = v[q];
                    } else {
                        h[q] = to_lane16(v[q], base, over);
                    }
                }
                *reinterpret_cast<uint2*>(reinterpret_cast<uint16_t*>(E.S) + at) =
                    make_uint2(__byte_perm(h[0], h[1], 0x5410), __byte_perm(h[2], h[3], 0x5410));
            }
        }
    };
    auto both = [&](auto form_tag) {
        emit(form_tag, sa, sb, g.i0, g.j0);
        if (g.I != g.J) emit(form_tag, sb, sa, g.j0, g.i0);
    };
    if (form == 0) both(std::integral_constant<int, 0>{});
    else if (form == 1) both(std::integral_constant<int, 1>{});
    else both(std::integral_constant<int, 2>{});
    if (over || acc > 0xFFFFu) raise_device_error(&hdr->err, kErrOverflow);
}

// Output (u32, zero diagonal) and wins, on the same tile pairs. Cells are widened from the
// working matrix (u16 lanes store v - base); wins compare the widened values, as the
// single-election ranking does. On a diagonal pair every ordered pair of the block is in the
// tile, so only row wins are counted there.
__global__ void __launch_bounds__(256, kPairCtasPerSm)
    batch_finalize_kernel(const Elec* __restrict__ elecs, const PairOwner* __restrict__ owner) {
    __shared__ __align__(16) uint32_t sb[kPT * kPT];  // X[J][I] staged: the transposed partners of a[]
    __shared__ int32_t colpart[16][kPT];
    const PairOwner o = owner[blockIdx.x];
    const Elec& E = elecs[o.e];
    const int C = E.C, Cp = E.Cp;
    const PairGeom g = pair_geom(o.local, Cp);
    const bool u16 = E.lanes == 16;
    // The working matrix covers Cp x Cp: no bounds. All eight loads are issued before any is
    // used (one CTA-uniform branch on the lane width around straight-line code); then the
    // 16-bit cells are widened (u16 lanes store v - base).
    uint4 a[4], bt[4];
    if (u16) {
        const uint16_t* S16 = reinterpret_cast<const uint16_t*>(E.S);
        uint2 wa[4], wb[4];
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int r = g.ry + 16 * p;
            wa[p] = __ldg(reinterpret_cast<const uint2*>(S16 + int64_t(g.i0 + r) * Cp + g.j0 + 4 * g.cx));
            wb[p] = __ldg(reinterpret_cast<const uint2*>(S16 + int64_t(g.j0 + r) * Cp + g.i0 + 4 * g.cx));
        }
        const uint32_t base = E.base;
        if (base == 0) {  // CTA-uniform: a cell is its value
            auto widen = [](uint2 w) { return make_uint4(w.x & 0xFFFFu, w.x >> 16, w.y & 0xFFFFu, w.y >> 16); };
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                a[p] = widen(wa[p]);
                bt[p] = widen(wb[p]);
            }
        } else {
            auto widen = [base](uint2 w) {
                const uint32_t h[4] = {w.x & 0xFFFFu, w.x >> 16, w.y & 0xFFFFu, w.y >> 16};
                return make_uint4(h[0] ? h[0] + base : 0u, h[1] ? h[1] + base : 0u, h[2] ? h[2] + base : 0u,
                                  h[3] ? h[3] + base : 0u);
            };
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                a[p] = widen(wa[p]);
                bt[p] = widen(wb[p]);
            }
        }
    } else {
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int r = g.ry + 16 * p;
            a[p] = __ldg(reinterpret_cast<const uint4*>(E.S + int64_t(g.i0 + r) * Cp + g.j0 + 4 * g.cx));
            bt[p] = __ldg(reinterpret_cast<const uint4*>(E.S + int64_t(g.j0 + r) * Cp + g.i0 + 4 * g.cx));
        }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p) swz64_store4(sb, g.ry + 16 * p, 4 * g.cx, bt[p]);
    // Off the diagonal, with both tiles inside the C candidates (CTA-uniform), the cells are
    // stored as they are: 128-bit stores where the output rows are 16-byte aligned.
    const bool interior = g.I != g.J && g.j0 + kPT <= C;  // i0 < j0, so i0 + kPT <= C too
    const bool vec_out = E.ld_out % 4 == 0 && (reinterpret_cast<uintptr_t>(E.out) & 15) == 0;
    const bool half_out = E.ld_out % 2 == 0 && (reinterpret_cast<uintptr_t>(E.out) & 7) == 0;
    auto store = [&](const uint4* own, int x0, int y0) {
        if (interior) {
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                uint32_t* at = E.out + int64_t(x0 + g.ry + 16 * p) * E.ld_out + y0 + 4 * g.cx;
                if (vec_out) {
                    *reinterpret_cast<uint4*>(at) = own[p];
                } else if (half_out) {
                    reinterpret_cast<uint2*>(at)[0] = make_uint2(own[p].x, own[p].y);
                    reinterpret_cast<uint2*>(at)[1] = make_uint2(own[p].z, own[p].w);
                } else {
                    at[0] = own[p].x, at[1] = own[p].y, at[2] = own[p].z, at[3] = own[p].w;
                }
            }
            return;
        }
#pragma unroll
        for (int p = 0; p < 4; ++p) {
            const int i = x0 + g.ry + 16 * p;
            if (i >= C) continue;
            const uint32_t x[4] = {own[p].x, own[p].y, own[p].z, own[p].w};
            uint32_t* row = E.out + int64_t(i) * E.ld_out;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const int j = y0 + 4 * g.cx + q;
                if (j < C) row[j] = i == j ? 0u : x[q];
            }
        }
    };
    store(a, g.i0, g.j0);
    if (g.I != g.J) store(bt, g.j0, g.i0);
    if (E.wins == nullptr) return;  // election-uniform
    __syncthreads();
    uint32_t rw[4] = {0, 0, 0, 0}, cw[4] = {0, 0, 0, 0};
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        const int r = g.ry + 16 * p;
        const uint32_t x[4] = {a[p].x, a[p].y, a[p].z, a[p].w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t y = sb[swz64(4 * g.cx + q, r)];  // S[j][i] for (i, j) = (i0 + r, j0 + 4cx + q)
            rw[p] += x[q] > y;
            cw[q] += y > x[q];
        }
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int msk = 8; msk >= 1; msk >>= 1) rw[p] += __shfl_xor_sync(0xFFFFFFFFu, rw[p], msk);
    if (g.cx < 4) {  // lane cx of the half warp adds row ry + 16 cx
        const uint32_t n = g.cx == 0 ? rw[0] : g.cx == 1 ? rw[1] : g.cx == 2 ? rw[2] : rw[3];
        const int i = g.i0 + g.ry + 16 * g.cx;
        if (n && i < C) atomicAdd(&E.wins[i], int(n));
    }
    if (g.I == g.J) return;  // CTA-uniform
#pragma unroll
    for (int q = 0; q < 4; ++q) colpart[g.ry][4 * g.cx + q] = int(cw[q]);
    __syncthreads();
    if (threadIdx.x < kPT) {
        int n = 0;
#pragma unroll
        for (int r = 0; r < 16; ++r) n += colpart[r][threadIdx.x];
        if (n && g.j0 + int(threadIdx.x) < C) atomicAdd(&E.wins[g.j0 + threadIdx.x], n);
    }
}

// Ranking of the elections with R >= 2 (see place_kernel in rank.cu).
__global__ void __launch_bounds__(256)
    batch_place_kernel(const Elec* __restrict__ elecs, const int32_t* __restrict__ big,
                       const int64_t* __restrict__ prefix, int nbig) {
    __shared__ int32_t w[1024];
    const int64_t b = blockIdx.x;
    const int m = find_owner(prefix, nbig, b);
    const Elec& E = elecs[big[m]];
    if (!E.wins) return;
    const int C = E.C;
    const int i = int(b - prefix[m]) * 256 + threadIdx.x;
    const int wi = i < C ? E.wins[i] : 0;
    int place = 0;
    for (int j0 = 0; j0 < C; j0 += 1024) {
        __syncthreads();
        for (int t = threadIdx.x; t < 1024; t += 256) w[t] = j0 + t < C ? E.wins[j0 + t] : -1;
        __syncthreads();
        const int n = C - j0 < 1024 ? C - j0 : 1024;
        for (int t = 0; t < n; ++t) {
            const int wj = w[t];
            place += (wj > wi) | ((wj == wi) & (j0 + t < i));
        }
    }
    if (i < C) E.ranking[place] = i;
}

// ------------------------------------------------------------------------------------------
// Host side: the plan lives in the caller's se_batch_plan_t; everything else in d_work.
// ------------------------------------------------------------------------------------------
struct Plan {
    uint8_t* work;
    int64_t work_bytes;
    int32_t n, nbig, nsmall;
    int64_t elec_off, big_off, init_prefix_off, fin_prefix_off, place_prefix_off, counters_off, counters_bytes;
    int64_t tasks_off[3];  // queues: u16, u32, u16 on the wide micro-tile
    uint32_t ntasks[3];
    int64_t init_blocks, fin_blocks, place_blocks;
    int32_t grid[3];
    cudaGraphExec_t graph;
    uint64_t dep_wait_ns;  // limit of one dependency wait of the persistent kernel
    int64_t pair_owner_off;  // PairOwner per block of the init and output kernels
};
static_assert(sizeof(Plan) <= sizeof(se_batch_plan_t), "se_batch_plan_t too small");

int64_t align256(int64_t x) { return round_up(x, 256); }

struct Sizes {
    int64_t total = 0, elec_off, big_off, init_prefix_off, fin_prefix_off, place_prefix_off, counters_off,
            counters_bytes, tasks_off[3], pair_owner_off, pairs = 0;
    std::vector<int64_t> s_off, at_off, dt_off, ctr_off;
    std::vector<int> lanes, R, Cp, queue;
    int nbig = 0, nsmall = 0;
    uint32_t ntasks[3] = {0, 0, 0};
};

// The persistent launch an election's tasks go to: 1 for 32-bit lanes; 2 for 16-bit lanes with
// C > 128 on the wide micro-tile; 0 otherwise.
int queue_of(int lanes, int R, int micro_tile) { return lanes != 16 ? 1 : (R > 1 && micro_tile == 4 ? 2 : 0); }

se_status_t size_batch(int n, const se_election_t* el, Sizes& z) {
    SE_REQUIRE(n >= 0, SE_ERR_INVALID, "negative election count");
    SE_REQUIRE(n < (1 << 24), SE_ERR_INVALID, "too many elections in one batch (%d)", n);
    z.s_off.assign(n, -1);
    z.at_off.assign(n, -1);
    z.dt_off.assign(n, -1);
    z.ctr_off.assign(n, -1);
    z.lanes.resize(n);
    z.R.resize(n);
    z.Cp.resize(n);
    z.queue.resize(n);
    int64_t off = 256;  // header
    z.elec_off = off;
    off = align256(off + int64_t(n) * int64_t(sizeof(Elec)));
    for (int e = 0; e < n; ++e) {
        SE_REQUIRE(el[e].C >= 1 && el[e].C <= (1 << 19), SE_ERR_INVALID, "election %d: bad candidate count %d", e,
                   el[e].C);
        SE_REQUIRE(el[e].lane_bits == 0 || el[e].lane_bits == 16 || el[e].lane_bits == 32, SE_ERR_INVALID,
                   "election %d: lane_bits must be 0, 16 or 32", e);
        z.lanes[e] = el[e].lane_bits == 16 ? 16 : 32;
        SE_REQUIRE(el[e].micro_tile == 0 || el[e].micro_tile == 8 || (el[e].micro_tile == 4 && z.lanes[e] == 16),
                   SE_ERR_INVALID, "election %d: micro_tile must be 0 or 8, or 4 with 16-bit lanes", e);
        z.Cp[e] = int(round_up(el[e].C, kT));
        z.R[e] = z.Cp[e] / kT;
        z.queue[e] = queue_of(z.lanes[e], z.R[e], el[e].micro_tile);
        SE_REQUIRE(z.R[e] <= 4095, SE_ERR_INVALID, "election %d too large for a batch", e);
        if (z.R[e] == 1) {
            ++z.nsmall;
            z.ntasks[z.queue[e]] += 1;
            continue;
        }
        ++z.nbig;
        const int64_t cell = z.lanes[e] == 16 ? 2 : 4;
        z.s_off[e] = off;
        off = align256(off + int64_t(z.Cp[e]) * z.Cp[e] * cell);
        z.at_off[e] = off;
        off = align256(off + int64_t(kT) * z.Cp[e] * 4);
        z.dt_off[e] = off;
        off = align256(off + int64_t(kT) * kT * 4);
        const uint64_t R = uint64_t(z.R[e]);
        z.ntasks[z.queue[e]] += uint32_t(R * R * R);
        const int64_t nt = z.Cp[e] / kPT;
        z.pairs += nt * (nt + 1) / 2;
    }
    z.counters_off = off;
    int64_t ctr = 0;
    for (int e = 0; e < n; ++e)
        if (z.R[e] > 1) {
            z.ctr_off[e] = z.counters_off + ctr;
            ctr += int64_t(3) * z.R[e] * 4;
        }
    z.counters_bytes = align256(ctr);
    off = z.counters_off + z.counters_bytes;
    z.big_off = off;
    off = align256(off + int64_t(z.nbig) * 4);
    z.init_prefix_off = off;
    off = align256(off + int64_t(z.nbig + 1) * 8);
    z.fin_prefix_off = off;
    off = align256(off + int64_t(z.nbig + 1) * 8);
    z.place_prefix_off = off;
    off = align256(off + int64_t(z.nbig + 1) * 8);
    z.pair_owner_off = off;
    off = align256(off + z.pairs * 8);
    for (int q = 0; q < 3; ++q) {
        z.tasks_off[q] = off;
        off = align256(off + int64_t(z.ntasks[q]) * 8);
    }
    z.total = off;
    return SE_OK;
}

template <int LB, int NQ = 8> int occupancy() {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_kernel<LB, NQ>, tile_threads<LB, NQ>(),
                                                  pcfg<LB>::SMEM);
    cudaGetLastError();
    return per_sm;
}

template <int LB, int NQ = 8> se_status_t set_persistent_smem() {
    return raise_smem_limit(reinterpret_cast<const void*>(persistent_kernel<LB, NQ>), int(pcfg<LB>::SMEM),
                            "the batched closure");
}

se_status_t enqueue(const Plan& P, cudaStream_t s) {
    Header* hdr = reinterpret_cast<Header*>(P.work);
    const Elec* elecs = reinterpret_cast<const Elec*>(P.work + P.elec_off);
    const int32_t* big = reinterpret_cast<const int32_t*>(P.work + P.big_off);
    SE_CUDA_TRY(cudaMemsetAsync(P.work, 0, 256, s));
    if (P.counters_bytes) SE_CUDA_TRY(cudaMemsetAsync(P.work + P.counters_off, 0, size_t(P.counters_bytes), s));
    if (P.nbig) {
        batch_init_kernel<<<unsigned(P.init_blocks), 256, 0, s>>>(
            elecs, reinterpret_cast<const PairOwner*>(P.work + P.pair_owner_off), hdr);
        SE_CHECK_LAUNCH();
    }
    if (P.ntasks[0]) {
        persistent_kernel<16><<<P.grid[0], cfg<16>::THREADS, pcfg<16>::SMEM, s>>>(
            elecs, reinterpret_cast<const uint64_t*>(P.work + P.tasks_off[0]), P.ntasks[0], hdr, 0, P.dep_wait_ns);
        SE_CHECK_LAUNCH();
    }
    if (P.ntasks[1]) {
        persistent_kernel<32><<<P.grid[1], cfg<32>::THREADS, pcfg<32>::SMEM, s>>>(
            elecs, reinterpret_cast<const uint64_t*>(P.work + P.tasks_off[1]), P.ntasks[1], hdr, 1, P.dep_wait_ns);
        SE_CHECK_LAUNCH();
    }
    if (P.ntasks[2]) {
        persistent_kernel<16, 4><<<P.grid[2], tile_threads<16, 4>(), pcfg<16>::SMEM, s>>>(
            elecs, reinterpret_cast<const uint64_t*>(P.work + P.tasks_off[2]), P.ntasks[2], hdr, 2, P.dep_wait_ns);
        SE_CHECK_LAUNCH();
    }
    if (P.nbig) {
        batch_finalize_kernel<<<unsigned(P.fin_blocks), 256, 0, s>>>(
            elecs, reinterpret_cast<const PairOwner*>(P.work + P.pair_owner_off));
        SE_CHECK_LAUNCH();
        batch_place_kernel<<<unsigned(P.place_blocks), 256, 0, s>>>(
            elecs, big, reinterpret_cast<const int64_t*>(P.work + P.place_prefix_off), P.nbig);
        SE_CHECK_LAUNCH();
    }
    return SE_OK;
}

}  // namespace batch
}  // namespace se

using namespace se;
using namespace se::batch;

extern "C" int64_t se_batch_workspace_bytes(int n, const se_election_t* elections) {
    clear_error();
    if (n > 0 && elections == nullptr) return -1;
    int64_t total = -1;
    host_guard([&] {  // size_batch fills host vectors
        Sizes z;
        const se_status_t st = size_batch(n, elections, z);
        if (st == SE_OK) total = z.total;
        return st;
    });
    return total;
}

// The batch's host-side planning: sizes, the task queues and their dependency prefixes, all in
// host vectors that are filled before anything is written to the device.
static se_status_t batch_prepare_impl(int n, const se_election_t* el, void* d_work, int64_t work_bytes, int order,
                                      int ctas_per_sm, se_batch_plan_t* plan_out) {
    clear_error();
    SE_REQUIRE(plan_out != nullptr, SE_ERR_INVALID, "null plan");
    SE_REQUIRE(n == 0 || el != nullptr, SE_ERR_INVALID, "null election array");
    Sizes z;
    if (se_status_t st = size_batch(n, el, z)) return st;
    SE_REQUIRE(d_work != nullptr && work_bytes >= z.total, SE_ERR_WORKSPACE,
               "workspace of %lld bytes is smaller than the %lld bytes required", (long long)work_bytes,
               (long long)z.total);
    SE_REQUIRE((reinterpret_cast<uintptr_t>(d_work) & 255) == 0, SE_ERR_INVALID, "workspace must be 256-byte aligned");
    for (int e = 0; e < n; ++e) {
        SE_REQUIRE(el[e].d_pref && el[e].d_out, SE_ERR_INVALID, "election %d: null matrix pointer", e);
        SE_REQUIRE(el[e].ld_pref >= el[e].C && el[e].ld_out >= el[e].C, SE_ERR_INVALID,
                   "election %d: row stride smaller than the number of candidates", e);
        SE_REQUIRE((el[e].d_wins == nullptr) == (el[e].d_ranking == nullptr), SE_ERR_INVALID,
                   "election %d: wins and ranking must both be given or both be null", e);
    }
    if (se_status_t st = set_persistent_smem<16>()) return st;
    if (se_status_t st = set_persistent_smem<32>()) return st;
    if (se_status_t st = set_persistent_smem<16, 4>()) return st;
    uint8_t* work = static_cast<uint8_t*>(d_work);

    std::vector<Elec> host(n);
    std::vector<int32_t> big;
    for (int e = 0; e < n; ++e) {
        Elec& E = host[e];
        std::memset(&E, 0, sizeof(Elec));
        E.d = el[e].d_pref;
        E.ld = el[e].ld_pref;
        E.out = el[e].d_out;
        E.ld_out = el[e].ld_out;
        E.wins = el[e].d_wins;
        E.ranking = el[e].d_ranking;
        E.C = el[e].C;
        E.Cp = z.Cp[e];
        E.R = z.R[e];
        E.lanes = z.lanes[e];
        E.base = E.lanes == 16 ? el[e].value_offset : 0u;
        if (E.R > 1) {
            big.push_back(e);
            const int cpw = E.lanes == 16 ? 2 : 1;
            const int64_t ldw = E.Cp / cpw;
            E.S = reinterpret_cast<uint32_t*>(work + z.s_off[e]);
            E.AT = reinterpret_cast<uint32_t*>(work + z.at_off[e]);
            E.dT = reinterpret_cast<uint32_t*>(work + z.dt_off[e]);
            E.counters = reinterpret_cast<uint32_t*>(work + z.ctr_off[e]);
            if (se_status_t st = make_map(&E.mapS, E.S, uint64_t(ldw), uint64_t(E.Cp), uint64_t(ldw) * 4,
                                          uint32_t(kT / cpw), kKC))
                return st;
            if (se_status_t st = make_map(&E.mapAT, E.AT, uint64_t(E.Cp), kT, uint64_t(E.Cp) * 4, kT, kKC)) return st;
            if (se_status_t st = make_map(&E.mapDT, E.dT, kT, kT, kT * 4, kT, kKC)) return st;
        }
    }
    // Task queues. Largest elections first inside every step.
    std::vector<int32_t> order_big(big);
    std::stable_sort(order_big.begin(), order_big.end(), [&](int a, int b) { return host[a].R > host[b].R; });
    int Rmax = 1;
    for (int e : big) Rmax = std::max(Rmax, host[e].R);
    std::vector<uint64_t> q[3];
    std::vector<uint64_t> small[2];
    for (int e = 0; e < n; ++e)
        if (host[e].R == 1) small[z.queue[e]].push_back(pack_task(e, kSmall, 0, 0, 0));
    if (order == 1)  // small elections first
        for (int l = 0; l < 2; ++l) q[l].insert(q[l].end(), small[l].begin(), small[l].end());
    for (int k = 0; k < Rmax; ++k) {
        for (int e : order_big)
            if (host[e].R > k) q[z.queue[e]].push_back(pack_task(e, kPivot, k, k, k));
        for (int e : order_big)
            if (host[e].R > k) {
                auto& Q = q[z.queue[e]];
                for (int x = 0; x < host[e].R; ++x)
                    if (x != k) {
                        Q.push_back(pack_task(e, kRow, k, k, x));
                        Q.push_back(pack_task(e, kCol, k, x, k));
                    }
            }
        for (int e : order_big)
            if (host[e].R > k) {
                auto& Q = q[z.queue[e]];
                for (int i = 0; i < host[e].R; ++i)
                    if (i != k)
                        for (int j = 0; j < host[e].R; ++j)
                            if (j != k) Q.push_back(pack_task(e, kRem, k, i, j));
            }
    }
    if (order != 1)
        for (int l = 0; l < 2; ++l) q[l].insert(q[l].end(), small[l].begin(), small[l].end());
    for (int l = 0; l < 3; ++l)
        SE_REQUIRE(q[l].size() == z.ntasks[l], SE_ERR_INVALID, "internal: task count mismatch");

    // Block prefixes of the batched elementwise kernels, and for init and finalize (one CTA per
    // pair of 64 x 64 tiles) each block's election and pair, so a CTA finds its work with one
    // load instead of a binary search over the prefixes.
    std::vector<int64_t> ip(big.size() + 1, 0), fp(big.size() + 1, 0), pp(big.size() + 1, 0);
    std::vector<PairOwner> owner;
    owner.reserve(size_t(z.pairs));
    for (size_t m = 0; m < big.size(); ++m) {
        const Elec& E = host[big[m]];
        const int64_t nt = E.Cp / kPT;
        ip[m + 1] = ip[m] + nt * (nt + 1) / 2;
        fp[m + 1] = fp[m] + nt * (nt + 1) / 2;
        pp[m + 1] = pp[m] + (E.C + 255) / 256;
        for (int64_t l = 0; l < nt * (nt + 1) / 2; ++l) owner.push_back(PairOwner{big[m], int32_t(l)});
    }
    SE_REQUIRE(int64_t(owner.size()) == z.pairs, SE_ERR_INVALID, "internal: pair count mismatch");
    // Upload (synchronous).
    SE_CUDA_TRY(cudaMemset(work, 0, 256));
    if (n) SE_CUDA_TRY(cudaMemcpy(work + z.elec_off, host.data(), sizeof(Elec) * size_t(n), cudaMemcpyHostToDevice));
    if (!big.empty()) {
        SE_CUDA_TRY(cudaMemcpy(work + z.big_off, big.data(), 4 * big.size(), cudaMemcpyHostToDevice));
        SE_CUDA_TRY(cudaMemcpy(work + z.init_prefix_off, ip.data(), 8 * ip.size(), cudaMemcpyHostToDevice));
        SE_CUDA_TRY(cudaMemcpy(work + z.fin_prefix_off, fp.data(), 8 * fp.size(), cudaMemcpyHostToDevice));
        SE_CUDA_TRY(cudaMemcpy(work + z.place_prefix_off, pp.data(), 8 * pp.size(), cudaMemcpyHostToDevice));
        SE_CUDA_TRY(cudaMemcpy(work + z.pair_owner_off, owner.data(), sizeof(PairOwner) * owner.size(),
                               cudaMemcpyHostToDevice));
    }
    for (int l = 0; l < 3; ++l)
        if (!q[l].empty())
            SE_CUDA_TRY(cudaMemcpy(work + z.tasks_off[l], q[l].data(), 8 * q[l].size(), cudaMemcpyHostToDevice));

    int device = 0, sms = 0;
    SE_CUDA_TRY(cudaGetDevice(&device));
    SE_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    Plan P;
    std::memset(&P, 0, sizeof(P));
    P.work = work;
    P.work_bytes = work_bytes;
    P.n = n;
    P.nbig = int32_t(big.size());
    P.nsmall = z.nsmall;
    P.elec_off = z.elec_off;
    P.big_off = z.big_off;
    P.init_prefix_off = z.init_prefix_off;
    P.fin_prefix_off = z.fin_prefix_off;
    P.place_prefix_off = z.place_prefix_off;
    P.pair_owner_off = z.pair_owner_off;
    P.counters_off = z.counters_off;
    P.counters_bytes = z.counters_bytes;
    for (int l = 0; l < 3; ++l) {
        P.tasks_off[l] = z.tasks_off[l];
        P.ntasks[l] = z.ntasks[l];
    }
    P.init_blocks = ip.back();
    P.fin_blocks = fp.back();
    P.place_blocks = pp.back();
    const int occ16 = occupancy<16>(), occ32 = occupancy<32>(), occ16w = occupancy<16, 4>();
    SE_REQUIRE(occ16 >= 1 && occ32 >= 1 && occ16w >= 1, SE_ERR_CUDA, "batched closure kernel cannot be resident");
    SE_REQUIRE(ctas_per_sm >= 0, SE_ERR_INVALID, "ctas_per_sm must be >= 0");
    const int per16 = ctas_per_sm > 0 ? std::min(occ16, ctas_per_sm) : occ16;
    const int per32 = ctas_per_sm > 0 ? std::min(occ32, ctas_per_sm) : occ32;
    const int per16w = ctas_per_sm > 0 ? std::min(occ16w, ctas_per_sm) : occ16w;
    P.grid[0] = int(std::min<int64_t>(P.ntasks[0], int64_t(sms) * per16));
    P.grid[1] = int(std::min<int64_t>(P.ntasks[1], int64_t(sms) * per32));
    P.grid[2] = int(std::min<int64_t>(P.ntasks[2], int64_t(sms) * per16w));
    P.graph = nullptr;
    P.dep_wait_ns = kDepWaitNs;
    std::memcpy(plan_out, &P, sizeof(P));
    return SE_OK;
}

extern "C" se_status_t se_batch_prepare(int n, const se_election_t* el, void* d_work, int64_t work_bytes, int order,
                                        int ctas_per_sm, se_batch_plan_t* plan_out) {
    return host_guard([&] { return batch_prepare_impl(n, el, d_work, work_bytes, order, ctas_per_sm, plan_out); });
}

extern "C" se_status_t se_batch_run(const se_batch_plan_t* plan, void* stream) {
    clear_error();
    SE_REQUIRE(plan != nullptr, SE_ERR_INVALID, "null plan");
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    return enqueue(P, static_cast<cudaStream_t>(stream));
}

extern "C" se_status_t se_batch_graph_build(se_batch_plan_t* plan) {
    clear_error();
    SE_REQUIRE(plan != nullptr, SE_ERR_INVALID, "null plan");
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    if (P.graph) {
        cudaGraphExecDestroy(P.graph);
        P.graph = nullptr;
    }
    cudaStream_t s;
    SE_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    se_status_t st = SE_OK;
    if (e == cudaSuccess) {
        st = enqueue(P, s);
        cudaError_t e2 = cudaStreamEndCapture(s, &g);
        if (st == SE_OK && e2 != cudaSuccess) e = e2;
    }
    if (st == SE_OK && e == cudaSuccess) e = cudaGraphInstantiate(&P.graph, g, 0);
    if (g) cudaGraphDestroy(g);
    cudaStreamDestroy(s);
    if (st != SE_OK) return st;
    SE_CUDA_TRY(e);
    std::memcpy(plan, &P, sizeof(P));
    return SE_OK;
}

extern "C" se_status_t se_batch_graph_launch(const se_batch_plan_t* plan, void* stream) {
    clear_error();
    SE_REQUIRE(plan != nullptr, SE_ERR_INVALID, "null plan");
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    SE_REQUIRE(P.graph != nullptr, SE_ERR_INVALID, "plan has no graph; call se_batch_graph_build first");
    SE_CUDA_TRY(cudaGraphLaunch(P.graph, static_cast<cudaStream_t>(stream)));
    return SE_OK;
}

extern "C" se_status_t se_batch_release(se_batch_plan_t* plan) {
    clear_error();
    if (!plan) return SE_OK;
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    if (P.graph) cudaGraphExecDestroy(P.graph);
    P.graph = nullptr;
    std::memcpy(plan, &P, sizeof(P));
    return SE_OK;
}

extern "C" se_status_t se_batch_set_wait_limit(se_batch_plan_t* plan, uint64_t limit_ns) {
    clear_error();
    SE_REQUIRE(plan != nullptr, SE_ERR_INVALID, "null plan");
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    P.dep_wait_ns = limit_ns;
    if (P.graph) cudaGraphExecDestroy(P.graph);  // it holds the old limit
    P.graph = nullptr;
    std::memcpy(plan, &P, sizeof(P));
    return SE_OK;
}

extern "C" se_status_t se_batch_check(const se_batch_plan_t* plan, void* stream) {
    clear_error();
    SE_REQUIRE(plan != nullptr, SE_ERR_INVALID, "null plan");
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    Header h;
    SE_CUDA_TRY(cudaMemcpyAsync(&h, P.work, sizeof(h), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
    SE_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    SE_REQUIRE(h.err != kErrOverflow, SE_ERR_OVERFLOW,
               "a kept preference count falls outside [value_offset + 1, value_offset + 65535] in an election "
               "run with 16-bit lanes");
    SE_REQUIRE(h.err == 0, SE_ERR_DEVICE, "batched closure reported device error %u (%s)", h.err,
               h.err == kErrDepTimeout ? "dependency wait timed out" : "TMA wait timed out");
    return SE_OK;
}

extern "C" se_status_t se_batch_profile(const se_batch_plan_t* plan, double* busy_ms, int64_t* tasks, double* wait_ms,
                                        void* stream) {
    clear_error();
    SE_REQUIRE(plan != nullptr, SE_ERR_INVALID, "null plan");
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    Header h;
    SE_CUDA_TRY(cudaMemcpyAsync(&h, P.work, sizeof(h), cudaMemcpyDeviceToHost, static_cast<cudaStream_t>(stream)));
    SE_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    for (int k = 0; k < 5; ++k) {
        if (busy_ms) busy_ms[k] = double(h.busy_ns[k]) * 1e-6;
        if (tasks) tasks[k] = int64_t(h.tasks[k]);
    }
    if (wait_ms) *wait_ms = double(h.wait_ns) * 1e-6;
    return SE_OK;
}

extern "C" int64_t se_batch_task_count(const se_batch_plan_t* plan, int queue) {
    if (!plan || queue < 0 || queue > 2) return -1;
    Plan P;
    std::memcpy(&P, plan, sizeof(P));
    return P.ntasks[queue];
}
