// Serving engine: continuous batching of elections on a persistent kernel that is fed while it
// runs (no reference counterpart).
//
// A request is a ballot set already in device memory. It occupies a slot and is a sequence of
// phases, each a set of independent tasks:
//   POS     ceil(V/64) tasks: place of every candidate on every (completed) ballot, built per
//           warp in a 16-bit row of shared memory when the rows fit and stored as exact
//           integers, then packed into bit planes (bit k of 32 ballots' places in one word)
//   TALLY   R(R+1) tasks: counts for one 128 x 64 half of an upper block pair (I <= J), by the
//           bit-sliced comparison (see tally.cu), written as the u32 preference matrix and,
//           shifted into 16 bits, as the closure's working matrix (d[j][i] = V - d[i][j]; no
//           separate defeat pass)
//   R == 1 (C <= 128): SMALL (closure, output, wins, ranking in one CTA)
//   R >= 2: PIVOT 0, then [PANELS k][REM k] for k < R, then FIN (output + wins per block pair)
//           and PLACE (ranking). REM k's task 0 is tile (k+1, k+1), which after its update
//           closes the next round's pivot (as the single-election closure's remainder launch
//           does), so no round but the first has a pivot phase of its own.
// The engine's CTAs (one or two per SM, resident while there is work) repeatedly scan the
// active slots, oldest first, and claim a task from the first request whose current phase is
// claimable: all tasks of the previous phase are done. Nothing waits on a dependency, so a
// request that arrives while others are mid-closure gets SMs as soon as the older ones have no
// claimable work: requests join and leave the running kernel at phase granularity, and the
// bit-sliced tally of one request (lop3 and popc on the integer ALU) shares the SMs with the
// closure of another (min/max).
//
// Slots are reused. Every claim counter carries the request's generation in its upper 32 bits
// and is advanced only by compare-and-swap against the expected generation, so a CTA that
// looked at a slot's previous occupant can never take a task of the new one. The request
// becomes visible only when the host's last write for it (active = 1) lands.
//
// Completion: the CTA finishing a request's last task writes (generation << 8 | status) to
// host-mapped memory; the host polls it without any CUDA call. All waits are bounded: after
// idle_ms with no active request the whole grid retires together (the host relaunches the
// engine when new work arrives); while requests are active a CTA waits at most 10 s for a
// claimable task; every mbarrier wait has a time limit; the host can raise a stop flag.
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <new>
#include <vector>

#include "batch_core.cuh"
#include "positions.cuh"

namespace se {
namespace serve {
using namespace se::batch;
using namespace se::closure;

constexpr int kMaxPhases = 3 * 256 + 4;  // R <= 256, i.e. C <= 32768 (2R + 5 phases are used)
constexpr size_t round_up_const(size_t x, size_t m) { return (x + m - 1) / m * m; }
constexpr uint32_t kStatusOverflow = 4;
constexpr uint32_t kStatusTally = 8;
constexpr int kPosChunk = 64;   // ballots per POS task
constexpr int kVC = 32;         // voters per TALLY chunk
constexpr int kTallyStages = 3;
constexpr size_t kEngineSmem = pcfg<16>::DATA + 16 * 8;                // data + 16 mbarrier slots

struct alignas(64) Req {
    Elec e;                      // e.d = the u32 preference matrix this request's TALLY writes
    CUtensorMap mapPl;           // bit planes u32 [ceil(V / 32) * B][Cq], box {64, B}
    const int32_t* ids;          // ballots: ids, most preferred first
    const int64_t* offsets;      // V + 1 CSR offsets, or null when every ballot has exactly C ids
    float* pos;                  // [V][Cq] places: f32, or u16 when the POS rows fit shared memory (POS)
    uint32_t* planes;            // word [ch * B + k][c]: bit k of the places of 32 ballots' candidate c
    int32_t B;                   // bit planes per 32-ballot chunk
    uint64_t* done_host;         // host-mapped completion word of this slot
    uint32_t* tally_host;        // host-mapped: the generation, once the TALLY phase is done
    uint32_t* flags;             // [0] ballot error (2 range, 3 repeat), [1] 16-bit lane overflow
    int64_t V;
    uint32_t gen;
    uint32_t active;
};

struct EngineHeader {
    uint32_t err;
    uint32_t stop;
    uint32_t slot_hi;
    uint32_t retire;  // raised by the first CTA to time out idle: the whole grid leaves together
    // Profile: per task kind, CTA-nanoseconds busy and tasks run; CTA-nanoseconds spent
    // looking for work. Kinds: POS, TALLY, SMALL, PIVOT, PANELS, REM, FIN, PLACE.
    unsigned long long busy_ns[8];
    unsigned long long tasks[8];
    unsigned long long search_ns;
};
constexpr int kKindCount = 8;

// Phases of a request with R row blocks: POS, TALLY, then SMALL (R = 1), or PIVOT 0,
// [PANELS k][REM k] for k < R, FIN, PLACE.
__host__ __device__ inline int phases_of(int R) { return R == 1 ? 3 : 2 * R + 5; }

__host__ __device__ inline uint32_t phase_size(int R, int64_t V, int f) {
    if (f == 0) return uint32_t((V + kPosChunk - 1) / kPosChunk);
    if (f == 1) return uint32_t(R * (R + 1));
    if (R == 1 || f == 2) return 1;
    const int g = f - 3;
    if (g < 2 * R) return g % 2 == 0 ? uint32_t(2 * (R - 1)) : uint32_t((R - 1) * (R - 1));
    return g == 2 * R ? uint32_t(R * (R + 1) / 2) : 1u;
}

__device__ __forceinline__ uint64_t ld_acquire64(const uint64_t* p) {
    uint64_t v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__host__ __device__ inline bool is_remainder_phase(int R, int f) { return R > 1 && f >= 3 && f - 3 < 2 * R && (f - 3) % 2 == 1; }

// Claims the next task of slot s (generation gen); returns the phase, the first index and how
// many consecutive tasks were taken (two remainder tiles at a time while two are left: the
// claim costs several L2 round trips, a remainder tile about 20 µs), or false.
// claims[0] = front (gen << 32 | phase), claims[1 + f] = gen << 32 | next index of phase f.
constexpr uint32_t kRemPerClaim = 2;

__device__ bool try_claim(uint64_t* claims, const uint32_t* dones, uint32_t gen, int R, int64_t V, int& f_out,
                          uint32_t& t_out, uint32_t& cnt_out) {
    const int nph = phases_of(R);
    for (int attempt = 0; attempt < 8; ++attempt) {
        const uint64_t fr = ld_acquire64(&claims[0]);
        if (uint32_t(fr >> 32) != gen) return false;
        const int f = int(uint32_t(fr));
        if (f >= nph) return false;
        if (f > 0 && ld_acquire(&dones[f - 1]) < phase_size(R, V, f - 1)) return false;  // not claimable yet
        const uint32_t size = phase_size(R, V, f);
        const uint64_t c = ld_acquire64(&claims[1 + f]);
        if (uint32_t(c >> 32) != gen) return false;
        const uint32_t n = uint32_t(c);
        if (n >= size) {
            // Everything in this phase is claimed: move the front on (harmless if another
            // CTA already did) and look again.
            atomicCAS(reinterpret_cast<unsigned long long*>(&claims[0]), (unsigned long long)fr,
                      (unsigned long long)(fr + 1));
            continue;
        }
        const uint32_t take = is_remainder_phase(R, f) && size - n >= kRemPerClaim ? kRemPerClaim : 1u;
        if (atomicCAS(reinterpret_cast<unsigned long long*>(&claims[1 + f]), (unsigned long long)c,
                      (unsigned long long)(c + take)) == (unsigned long long)c) {
            if (n + take == size)
                atomicCAS(reinterpret_cast<unsigned long long*>(&claims[0]), (unsigned long long)fr,
                          (unsigned long long)(fr + 1));
            f_out = f;
            t_out = n;
            cnt_out = take;
            return true;
        }
    }
    return false;
}

// Read-only look at slot state: true when the front phase of generation gen has an unclaimed
// task and its predecessor is complete. A front phase with nothing left to claim is moved on
// here (the same harmless CAS try_claim makes), so the next look sees the following phase.
__device__ bool claimable(uint64_t* claims, const uint32_t* dones, uint32_t gen, int R, int64_t V) {
    const uint64_t fr = ld_acquire64(&claims[0]);
    if (uint32_t(fr >> 32) != gen) return false;
    const int f = int(uint32_t(fr));
    if (f >= phases_of(R)) return false;
    if (f > 0 && ld_acquire(&dones[f - 1]) < phase_size(R, V, f - 1)) return false;
    const uint64_t c = ld_acquire64(&claims[1 + f]);
    if (uint32_t(c >> 32) != gen) return false;
    if (uint32_t(c) < phase_size(R, V, f)) return true;
    atomicCAS(reinterpret_cast<unsigned long long*>(&claims[0]), (unsigned long long)fr, (unsigned long long)(fr + 1));
    return false;
}

// Warp-wide search for a task: the 32 lanes look at 32 slots at once (lowest slot first), so a
// step costs a few L2 round trips however many requests are in flight; the candidates are then
// claimed one at a time in slot order. Returns the slot or kNoSlot; any_active reports whether
// any slot below hi holds a request.
constexpr uint32_t kNoSlot = 0xFFFFFFFFu;

__device__ uint32_t warp_find_task(Req* slots, uint64_t* claims, const uint32_t* dones, uint32_t hi, bool& any_active,
                                   int& f_out, uint32_t& t_out, uint32_t& cnt_out) {
    const int lane = threadIdx.x & 31;
    for (uint32_t s0 = 0; s0 < hi; s0 += 32) {
        const uint32_t s = s0 + lane;
        bool active = false, cand = false;
        uint32_t gen = 0;
        int R = 0;
        int64_t V = 0;
        if (s < hi && ld_acquire(&slots[s].active)) {
            active = true;
            gen = __ldcg(&slots[s].gen);
            R = __ldcg(&slots[s].e.R);
            V = __ldcg(&slots[s].V);
            cand = claimable(claims + size_t(s) * (kMaxPhases + 1), dones + size_t(s) * kMaxPhases, gen, R, V);
        }
        if (__any_sync(0xffffffffu, active)) any_active = true;
        uint32_t mask = __ballot_sync(0xffffffffu, cand);
        while (mask) {
            const int l = __ffs(mask) - 1;
            int f = 0;
            uint32_t t = 0, cnt = 0;
            int got = 0;
            if (lane == l)
                got = try_claim(claims + size_t(s) * (kMaxPhases + 1), dones + size_t(s) * kMaxPhases, gen, R, V, f, t,
                                cnt);
            got = __shfl_sync(0xffffffffu, got, l);
            if (got) {
                f_out = __shfl_sync(0xffffffffu, f, l);
                t_out = __shfl_sync(0xffffffffu, t, l);
                cnt_out = __shfl_sync(0xffffffffu, cnt, l);
                return s0 + l;
            }
            mask &= mask - 1;
        }
    }
    return kNoSlot;
}

// Output (u32, shifted back, zero diagonal) and wins for the 128-block pair (I, J), I <= J.
__device__ void run_fin(const Elec& E, int I, int J, uint8_t* smem) {
    uint16_t* tJI = reinterpret_cast<uint16_t*>(smem);  // [128][130]: S[J-block][I-block], padded
    int32_t* wsum = reinterpret_cast<int32_t*>(smem + 128 * 130 * 2);  // [256]: row wins, col wins
    const int C = E.C;
    const uint16_t* S = reinterpret_cast<const uint16_t*>(E.S);
    const int64_t Cp = E.Cp;
    for (int x = threadIdx.x; x < 256; x += blockDim.x) wsum[x] = 0;
    for (int idx = threadIdx.x; idx < 128 * 128; idx += blockDim.x) {
        const int r = idx / 128, c = idx % 128;  // S[J*128 + r][I*128 + c], coalesced in c
        tJI[r * 130 + c] = __ldcg(S + (int64_t(J) * 128 + r) * Cp + int64_t(I) * 128 + c);
    }
    __syncthreads();
    const uint32_t base = E.base;
    for (int idx = threadIdx.x; idx < 128 * 128; idx += blockDim.x) {
        const int r = idx / 128, c = idx % 128;  // cell (i, j) = (I*128 + r, J*128 + c)
        const int i = I * 128 + r, j = J * 128 + c;
        if (i >= C || j >= C) continue;
        uint32_t sij = __ldcg(S + int64_t(i) * Cp + j);
        uint32_t sji = tJI[c * 130 + r];
        sij = sij ? sij + base : 0u;
        sji = sji ? sji + base : 0u;
        E.out[int64_t(i) * E.ld_out + j] = i == j ? 0u : sij;
        if (I != J) E.out[int64_t(j) * E.ld_out + i] = sji;
        if (E.wins && (I != J || j > i)) {
            if (sij > sji) atomicAdd(&wsum[r], 1);
            else if (sji > sij) atomicAdd(&wsum[128 + c], 1);
        }
    }
    __syncthreads();
    if (E.wins)
        for (int x = threadIdx.x; x < 256; x += blockDim.x) {
            const int cand = x < 128 ? I * 128 + x : J * 128 + (x - 128);
            if (cand < C && wsum[x]) atomicAdd(&E.wins[cand], wsum[x]);
        }
}

// Ranking from the wins (stable by index), with the wins staged in shared memory.
__device__ void run_place(const Elec& E, uint8_t* smem) {
    int32_t* w = reinterpret_cast<int32_t*>(smem);
    constexpr int kChunk = 16384;  // 64 KiB of wins per pass
    const int C = E.C;
    for (int i0 = 0; i0 < C; i0 += blockDim.x * 8) {
        int wi[8], place[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * blockDim.x + threadIdx.x;
            wi[u] = i < C ? __ldcg(E.wins + i) : 0;
            place[u] = 0;
        }
        for (int j0 = 0; j0 < C; j0 += kChunk) {
            const int n = C - j0 < kChunk ? C - j0 : kChunk;
            __syncthreads();
            for (int t = threadIdx.x; t < n; t += blockDim.x) w[t] = __ldcg(E.wins + j0 + t);
            __syncthreads();
            for (int t = 0; t < n; ++t) {
                const int wj = w[t];
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const int i = i0 + u * blockDim.x + threadIdx.x;
                    place[u] += (wj > wi[u]) | ((wj == wi[u]) & (j0 + t < i));
                }
            }
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int i = i0 + u * blockDim.x + threadIdx.x;
            if (i < C) E.ranking[place[u]] = i;
        }
    }
}

// ------------------------------------------------------------------------------------------
// POS: ballots [v0, v1) -> places. Missing candidates go after the listed ones in ascending id
// order (the reference's completion rule, scaling_elections.py:75-83). Out-of-range or repeated
// ids set the request's ballot error word.
// ------------------------------------------------------------------------------------------
// smem: the task's free operand region (bytes). When a 16-bit row per warp fits there, each
// warp builds its ballot's places in its row (scatter, check and completion scan in shared
// memory) and then writes the row out with coalesced stores; otherwise it works in global
// memory through L2.
__device__ void run_positions(const Req& Q, int C, int Cq, int64_t v0, int64_t v1, uint8_t* smem, size_t smem_bytes) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const bool rows = size_t(nw) * size_t(Cq) * 2 <= smem_bytes && C < 0xFFFF;
    uint16_t* row = reinterpret_cast<uint16_t*>(smem) + size_t(warp) * Cq;
    for (int64_t v = v0 + warp; v < v1; v += nw) {  // one ballot per warp at a time
        const int64_t beg = Q.offsets ? __ldcg(Q.offsets + v) : v * C;
        const int64_t len = Q.offsets ? __ldcg(Q.offsets + v + 1) - beg : C;
        int code;
        if (rows) {
            // 16-bit places, copied out 8 at a time (Cq is a multiple of 128, so rows and
            // destinations are 16-byte aligned).
            code = warp_places_u16<int32_t, true>(Q.ids + beg, len, C, Cq, row);
            __syncwarp();
            if (code == kPosOk) {
                uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<uint16_t*>(Q.pos) + v * Cq);
                const uint4* src = reinterpret_cast<const uint4*>(row);
                for (int c = lane; c < Cq / 8; c += 32) dst[c] = src[c];
            }
            __syncwarp();  // the row is read before the next ballot rewrites it
        } else {
            code = warp_positions<int32_t, true>(Q.ids + beg, len, C, Cq, Q.pos + v * Cq);
        }
        if (code != kPosOk && lane == 0) atomicCAS(&Q.flags[0], 0u, uint32_t(code));
    }
    // Pack the task's 32-ballot chunks into bit planes (ballots past V count as place 0). The
    // places were written by this CTA's warps (u16 or f32, as above); read them back through L2.
    // Each thread turns one candidate's 32 places into the request's B plane words, one bit
    // extract and one bit insert per voter and plane (a loop over B, not over all 20 planes).
    __syncthreads();
    const int B = Q.B;
    const uint16_t* pos16 = reinterpret_cast<const uint16_t*>(Q.pos);
    for (int64_t ch = v0 / 32; ch * 32 < v1; ++ch)
        for (int64_t c = threadIdx.x; c < Cq; c += blockDim.x) {
            uint32_t p[32];
            if (rows) {  // CTA-uniform
#pragma unroll
                for (int v = 0; v < 32; ++v) {
                    const int64_t voter = ch * 32 + v;
                    p[v] = voter < Q.V ? uint32_t(__ldcg(pos16 + voter * Cq + c)) : 0u;
                }
            } else {
#pragma unroll
                for (int v = 0; v < 32; ++v) {
                    const int64_t voter = ch * 32 + v;
                    p[v] = voter < Q.V ? uint32_t(__ldcg(Q.pos + voter * Cq + c)) : 0u;
                }
            }
#pragma unroll 1
            for (int k = 0; k < B; ++k) {
                uint32_t word = 0u;
#pragma unroll
                for (int v = 0; v < 32; ++v) {
                    uint32_t bit;
                    asm("bfe.u32 %0, %1, %2, 1;" : "=r"(bit) : "r"(p[v]), "r"(k));
                    asm("bfi.b32 %0, %1, %2, %3, 1;" : "=r"(word) : "r"(bit), "r"(word), "r"(v));
                }
                Q.planes[(ch * B + k) * Cq + c] = word;
            }
        }
}

__device__ __forceinline__ uint32_t borrow_step(uint32_t a, uint32_t b, uint32_t br) {
    uint32_t r;
    asm("lop3.b32 %0, %1, %2, %3, 0x8E;" : "=r"(r) : "r"(a), "r"(b), "r"(br));  // MAJ(~a, b, br)
    return r;
}

// ------------------------------------------------------------------------------------------
// TALLY: counts n[i][j] = #{v : pos_v(i) < pos_v(j)} for rows I*128.. and the 64 columns
// J*128 + h*64.. (I <= J), streamed in 32-ballot chunks of bit planes through a 3-stage TMA
// ring. For each chunk the borrow of the bit-serial subtraction pos(i) - pos(j), one lop3 per
// plane, holds the 32 answers, and a popc adds them. Writes the u32 preferences d (both (i,j)
// and, for I < J, (j,i) = V - n) and, for R >= 2, the closure's working matrix: kept values
// (d > V - d) shifted by base into 16 bits, zero elsewhere, including the padding.
// ------------------------------------------------------------------------------------------
__device__ bool run_tally(const Req& Q, const Req* G, int I, int J, int h, uint8_t* smem, uint64_t* bars,
                          uint32_t& tpar) {
    const Elec& E = Q.e;
    const int B = Q.B;
    const int stage_words = 3 * B * 64;  // planes of rows I (two boxes of 64) and of the 64 columns
    uint32_t* sbuf = reinterpret_cast<uint32_t*>(smem);
    const int64_t V = Q.V;
    const int nch = int((V + kVC - 1) / kVC);
    const int xI = I * 128, xJ = J * 128 + h * 64;
    auto issue = [&](int ch, int st) {
        uint32_t* base = sbuf + st * stage_words;
        mbar_arrive_expect_tx(&bars[st], uint32_t(stage_words) * 4u);
        tma_load_2d(base, &G->mapPl, &bars[st], xI, ch * B);
        tma_load_2d(base + B * 64, &G->mapPl, &bars[st], xI + 64, ch * B);
        tma_load_2d(base + 2 * B * 64, &G->mapPl, &bars[st], xJ, ch * B);
    };
    if (threadIdx.x == 0) {
        fence_tensormap(&G->mapPl);
        fence_proxy_async();
        for (int st = 0; st < kTallyStages && st < nch; ++st) issue(st, st);
    }
    const geom g(threadIdx.x);
    uint32_t acc[8][8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[r][q] = 0u;
    bool ok = true;
    // Row r of the thread lives in box (row0 + r) / 64 at column (row0 + r) % 64.
    const int boxA = g.row0 / 64, colA = g.row0 % 64;
#pragma unroll 1
    for (int ch = 0; ch < nch; ++ch) {
        const int st = ch % kTallyStages;
        const uint32_t par = (tpar >> st) & 1u;
        if (ok && !mbar_wait_bounded(&bars[st], par, 1u << 26)) ok = false;
        tpar ^= 1u << st;
        if (ok) {
            const uint32_t* A = sbuf + st * stage_words + boxA * B * 64;
            const uint32_t* Bp = sbuf + st * stage_words + 2 * B * 64;
            uint32_t br[8][8];
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int q = 0; q < 8; ++q) br[r][q] = 0u;
#pragma unroll 2
            for (int k = 0; k < B; ++k) {
                uint32_t a[8], b[8];
                ld4(a, A + k * 64 + colA);
                ld4(a + 4, A + k * 64 + colA + 4);
                ld4(b, Bp + k * 64 + g.wbase);
                ld4(b + 4, Bp + k * 64 + g.wbase + 32);
#pragma unroll
                for (int r = 0; r < 8; ++r)
#pragma unroll
                    for (int q = 0; q < 8; ++q) br[r][q] = borrow_step(a[r], b[q], br[r][q]);
            }
#pragma unroll
            for (int r = 0; r < 8; ++r)
#pragma unroll
                for (int q = 0; q < 8; ++q) acc[r][q] += __popc(br[r][q]);
        }
        __syncthreads();  // everyone is done with stage st
        if (threadIdx.x == 0 && ok && ch + kTallyStages < nch) {
            fence_proxy_async();
            issue(ch + kTallyStages, st);
        }
    }
    if (!ok) return false;
    const int C = E.C, Cp = E.Cp;
    const uint32_t Vu = uint32_t(V);
    uint16_t* S16 = reinterpret_cast<uint16_t*>(E.S);
    const bool write_s = E.R > 1;
    bool over = false;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const int i = xI + g.row0 + r;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int j = xJ + g.wbase + (q < 4 ? q : 28 + q);
            const uint32_t n = acc[r][q], m = Vu - n;
            const bool live = i < C && j < C && i != j;
            if (i < C && j < C) {
                uint32_t* d = const_cast<uint32_t*>(E.d);
                d[int64_t(i) * C + j] = i == j ? 0u : n;
                if (I != J) d[int64_t(j) * C + i] = m;
            }
            if (write_s) {
                const uint32_t sij = (live && n > m) ? to_lane16(n, E.base, over) : 0u;
                S16[int64_t(i) * Cp + j] = uint16_t(sij);
                if (I != J) {
                    const uint32_t sji = (live && m > n) ? to_lane16(m, E.base, over) : 0u;
                    S16[int64_t(j) * Cp + i] = uint16_t(sji);
                }
            }
        }
    }
    if (over) atomicCAS(&Q.flags[1], 0u, 2u);
    return true;
}

constexpr uint64_t kStallNs = 10000000000ull;  // 10 s without a claim while requests are active

__global__ void __launch_bounds__(cfg<16>::THREADS, 1)
    engine_kernel(Req* __restrict__ slots, uint64_t* __restrict__ claims, uint32_t* __restrict__ dones,
                  EngineHeader* __restrict__ hdr, uint64_t idle_ns) {
    using CF = cfg<16>;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(16) uint32_t rowbuf[kPivotBufs][CF::TW];
    __shared__ __align__(16) uint32_t colbuf[kPivotBufs][kT];
    __shared__ int32_t s_wins[kT];
    __shared__ __align__(64) Req s_q;
    __shared__ uint32_t s_slot, s_t, s_cnt;
    __shared__ int s_f;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + pcfg<16>::DATA);  // [0,8) closure, [8,11) tally
    if (threadIdx.x == 0) {
        for (int b = 0; b < 2 * kChunks + kTallyStages; ++b) mbar_init(&bars[b], 1);
        fence_barrier_init();
    }
    __syncthreads();
    uint32_t par_a = 0, par_b = 0, tpar = 0;
    // The slot of the CTA's last task, whose descriptor is still in s_q: tried first, before
    // the ordered scan, because a request in a bulk phase (places, tally, remainder) usually
    // has more of it. Its claim counters carry the generation, so a slot reused by another
    // request fails this claim and the scan takes over.
    uint32_t last_slot = kNoSlot;

    for (;;) {
        uint64_t t_task = 0;
        if (threadIdx.x < 32) {
            uint32_t got = kNoSlot;
            bool fresh = true;  // the claimed slot's descriptor must be (re)loaded
            const uint64_t t0 = global_ns();
            if (last_slot != kNoSlot) {
                int ok_claim = 0, f = 0;
                uint32_t t = 0, cnt = 0;
                if (threadIdx.x == 0 && !ld_acquire(&hdr->stop) && !ld_acquire(&hdr->err))
                    ok_claim = try_claim(claims + size_t(last_slot) * (kMaxPhases + 1),
                                         dones + size_t(last_slot) * kMaxPhases, s_q.gen, s_q.e.R, s_q.V, f, t, cnt);
                if (__shfl_sync(0xffffffffu, ok_claim, 0)) {
                    got = last_slot;
                    fresh = false;
                    if (threadIdx.x == 0) {
                        s_f = f;
                        s_t = t;
                        s_cnt = cnt;
                    }
                }
            }
            while (got == kNoSlot) {
                int stop = 0;
                if (threadIdx.x == 0)
                    stop = ld_acquire(&hdr->stop) || ld_acquire(&hdr->err) || ld_acquire(&hdr->retire);
                if (__shfl_sync(0xffffffffu, stop, 0)) break;
                uint32_t hi = threadIdx.x == 0 ? ld_acquire(&hdr->slot_hi) : 0u;
                hi = __shfl_sync(0xffffffffu, hi, 0);
                bool any_active = false;
                int f = 0;
                uint32_t t = 0, cnt = 0;
                got = warp_find_task(slots, claims, dones, hi, any_active, f, t, cnt);
                if (got != kNoSlot && threadIdx.x == 0) {
                    s_f = f;
                    s_t = t;
                    s_cnt = cnt;
                }
                if (got == kNoSlot) {
                    // With no active request the CTA leaves after idle_ns (the host relaunches
                    // the engine for the next one). While requests are active but have nothing
                    // claimable (their current phase's last tasks are still running) it keeps
                    // looking, up to kStallNs without any claim, which no task comes close to.
                    // Lane 0 decides for the warp.
                    int leave = 0;
                    if (threadIdx.x == 0) {
                        const uint64_t waited = global_ns() - t0;
                        if (!any_active && waited > idle_ns) {
                            // Retire the whole grid, never part of it: a partial grid would
                            // keep serving the next request with a fraction of the SMs.
                            atomicExch(&hdr->retire, 1u);
                            leave = 1;
                        } else if (waited > kStallNs) {
                            atomicCAS(&hdr->err, 0u, 2u);
                            leave = 1;
                        }
                    }
                    if (__shfl_sync(0xffffffffu, leave, 0)) break;
                    __nanosleep(any_active ? 200 : 1000);
                }
            }
            if (threadIdx.x == 0) {
                s_slot = got;
                t_task = global_ns();
                atomicAdd(&hdr->search_ns, (unsigned long long)(t_task - t0));
            }
            last_slot = got;
            if (got != kNoSlot) {
                if (fresh) {
                    // The slot's descriptor may have been rewritten since this SM last read
                    // it: copy it through L2, one 16-byte piece per lane.
                    const uint4* src = reinterpret_cast<const uint4*>(&slots[got]);
                    uint4* dst = reinterpret_cast<uint4*>(&s_q);
                    for (int q = threadIdx.x; q < int(sizeof(Req) / 16); q += 32) dst[q] = __ldcg(src + q);
                }
                // Other CTAs' results that this task's TMA loads read were published with a
                // release after their own proxy fence; order the claim's acquire before them.
                fence_proxy_async_global();
            }
        }
        __syncthreads();
        const uint32_t s = s_slot;
        if (s == kNoSlot) break;
        const int f = s_f;
        const uint32_t t = s_t;
        const Req& Q = s_q;
        const Elec& E = Q.e;
        const Req* GQ = &slots[s];
        const Elec* G = &GQ->e;
        const int R = E.R;
        bool ok = true;
        bool last = false;
        if (f == 0) {
            const int64_t v0 = int64_t(t) * kPosChunk;
            const int64_t v1 = v0 + kPosChunk < Q.V ? v0 + kPosChunk : Q.V;
            run_positions(Q, E.C, E.Cp, v0, v1, smem, pcfg<16>::DATA);
        } else if (f == 1) {
            int q = int(t) >> 1, I = 0;
            while (q >= R - I) {
                q -= R - I;
                ++I;
            }
            ok = run_tally(Q, GQ, I, I + q, int(t) & 1, smem, bars + 2 * kChunks, tpar);
        } else if (R == 1) {
            run_small<16>(E, smem, rowbuf, colbuf, s_wins, Q.flags + 1);  // overflow -> this request
            last = true;
        } else if (f == 2) {
            run_pivot<16>(E, 0, rowbuf, colbuf);
        } else {
            const int g = f - 3;
            if (g < 2 * R) {
                const int k = g / 2, kind = 1 + g % 2;  // 1 panels, 2 remainder
                // Panels (row panels first, then column panels) or remainder tiles, one per
                // task; a remainder claim may hold two consecutive tiles. Remainder task 0 is
                // tile (k+1, k+1) (its index swapped with that tile's), closed afterwards as the
                // next round's pivot.
                const int R1 = R - 1;
                const int p_next = k * R1 + k;  // reduced coordinates of tile (k+1, k+1)
                const uint32_t cnt = s_cnt;
                for (uint32_t x = 0; x < cnt; ++x) {
                    // The previous tile's shared operands are read before the next TMA;
                    // the reduction keeps every thread's view of ok the same.
                    if (x > 0 && !__syncthreads_and(ok)) {
                        ok = false;
                        break;
                    }
                    int tt = int(t + x);
                    const bool pivot_next = kind == 2 && k + 1 < R && tt == 0;
                    int tk, ii, jj;
                    if (kind == 1) {
                        const bool row = tt < R1;
                        const int y = row ? tt : tt - R1;
                        tk = row ? kTileRow : kTileCol;
                        ii = jj = y + (y >= k);
                    } else {
                        if (k + 1 < R) tt = tt == 0 ? p_next : (tt == p_next ? 0 : tt);
                        tk = kTileRem;
                        ii = tt / R1;
                        jj = tt % R1;
                        ii += ii >= k;
                        jj += jj >= k;
                    }
                    ok = run_tile<16>(E, G, tk, k, ii, jj, smem, bars, par_a, par_b);
                    if (pivot_next && __syncthreads_and(ok)) {  // the tile's stores are visible
                        run_pivot<16>(E, k + 1, rowbuf, colbuf);
                    }
                }
            } else if (g == 2 * R) {
                int rem = int(t), I = 0;
                while (rem >= R - I) {
                    rem -= R - I;
                    ++I;
                }
                run_fin(E, I, I + rem, smem);
            } else {
                run_place(E, smem);
                last = true;
            }
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            const int kind = f == 0 ? 0 : f == 1 ? 1 : R == 1 ? 2 : f == 2 ? 3
                           : (f - 3 < 2 * R ? 4 + (f - 3) % 2 : (f - 3 == 2 * R ? 6 : 7));
            const uint32_t cnt = s_cnt;
            atomicAdd(&hdr->busy_ns[kind], (unsigned long long)(global_ns() - t_task));
            atomicAdd(&hdr->tasks[kind], (unsigned long long)cnt);
            if (!ok) {
                atomicCAS(&hdr->err, 0u, 1u);
            } else {
                fence_proxy_async_global();
                const uint32_t prev = atomicAdd(&dones[size_t(s) * kMaxPhases + f], cnt);
                if (f == 1 && prev + cnt == phase_size(R, Q.V, f)) {
                    // The ballot places are no longer needed: tell the host it may reuse them.
                    __threadfence_system();
                    asm volatile("st.release.sys.u32 [%0], %1;" ::"l"(Q.tally_host), "r"(Q.gen) : "memory");
                }
                if (last && prev + cnt == phase_size(R, Q.V, f)) {
                    uint32_t status = 0;
                    const uint32_t ballot_err = __ldcg(Q.flags);
                    if (__ldcg(Q.flags + 1)) status |= kStatusOverflow;
                    if (ballot_err) status |= kStatusTally | (ballot_err & 3u);
                    atomicExch(&slots[s].active, 0u);
                    __threadfence_system();
                    const unsigned long long word = (unsigned long long)Q.gen << 8 | status;
                    asm volatile("st.release.sys.u64 [%0], %1;" ::"l"(Q.done_host), "l"(word) : "memory");
                }
            }
        }
        if (!ok) break;
    }
}

// ------------------------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------------------------
struct Engine {
    std::mutex mu;
    uint8_t* work = nullptr;
    int max_slots = 0;
    EngineHeader* hdr = nullptr;
    Req* slots = nullptr;
    uint64_t* claims = nullptr;
    uint32_t* dones = nullptr;
    uint64_t* done_host = nullptr;  // host-mapped
    uint64_t* done_dev = nullptr;   // its device address
    uint32_t* tally_host = nullptr; // host-mapped: per slot, generation whose tally finished
    uint32_t* tally_dev = nullptr;
    std::vector<uint8_t> tally_reported;
    uint8_t* staging = nullptr;     // pinned, one region per slot: its H2D sources stay valid
                                    // until the slot is reused, i.e. long after the copies ran
    uint8_t* zeros = nullptr;       // pinned, kZeroBytes of zeros: the source of every clearing copy
    std::vector<uint32_t> gen;
    std::vector<uint8_t> busy;
    uint32_t slot_hi = 0;
    cudaStream_t stream = nullptr;   // the engine kernel's stream
    cudaEvent_t finished = nullptr;  // recorded after each engine launch
    bool launched = false;
    int64_t launches = 0;
    int grid = 0;
    uint64_t idle_ns = 0;
    int in_flight = 0;
};

constexpr size_t kStagingPerSlot = round_up_const(sizeof(Req) + 16 + (kMaxPhases + 1) * 8, 256);
// Submission clears a request's flags, wins and phase counters by copying from pinned zeros
// rather than with cudaMemsetAsync: a memset is a kernel, and while the engine is resident
// its CTAs hold every SM's registers, so a memset (and every copy queued behind it on the
// submitting stream) would wait for the whole grid to retire.
constexpr size_t kZeroBytes = std::max<size_t>(size_t(4) << 15, size_t(kMaxPhases) * 4);  // wins of C = 32768

int64_t offsets(int max_slots, int64_t* slots_off, int64_t* claims_off, int64_t* dones_off) {
    int64_t off = 256;
    *slots_off = off;
    off = round_up(off + int64_t(max_slots) * int64_t(sizeof(Req)), 256);
    *claims_off = off;
    off = round_up(off + int64_t(max_slots) * (kMaxPhases + 1) * 8, 256);
    *dones_off = off;
    off = round_up(off + int64_t(max_slots) * kMaxPhases * 4, 256);
    return off;
}

se_status_t launch_engine(Engine& E) {
    SE_CUDA_TRY(cudaMemsetAsync(&E.hdr->retire, 0, 4, E.stream));
    engine_kernel<<<E.grid, cfg<16>::THREADS, kEngineSmem, E.stream>>>(E.slots, E.claims, E.dones, E.hdr,
                                                                           E.idle_ns);
    SE_CHECK_LAUNCH();
    SE_CUDA_TRY(cudaEventRecord(E.finished, E.stream));
    E.launched = true;
    ++E.launches;
    return SE_OK;
}

// Relaunches the engine if it exited (idle) while requests are in flight.
se_status_t ensure_running(Engine& E) {
    if (E.in_flight == 0) return SE_OK;
    if (E.launched) {
        const cudaError_t q = cudaEventQuery(E.finished);
        if (q == cudaErrorNotReady) return SE_OK;
        SE_CUDA_TRY(q);
        EngineHeader h;
        SE_CUDA_TRY(cudaMemcpyAsync(&h, E.hdr, sizeof(h), cudaMemcpyDeviceToHost, E.stream));
        SE_CUDA_TRY(cudaStreamSynchronize(E.stream));
        SE_REQUIRE(h.err == 0, SE_ERR_DEVICE, "serving engine stopped on a device error (%u: %s)", h.err,
                   h.err == 2 ? "no task could be claimed for 10 s" : "lost TMA completion");
    }
    return launch_engine(E);
}

}  // namespace serve
}  // namespace se

using namespace se;
using namespace se::serve;

struct se_engine {
    Engine e;
};

extern "C" int64_t se_engine_workspace_bytes(int max_slots) {
    if (max_slots < 1 || max_slots > 65535) return -1;
    int64_t a, b, c;
    return offsets(max_slots, &a, &b, &c);
}

extern "C" se_status_t se_engine_create(void* d_work, int64_t work_bytes, int max_slots, int ctas_per_sm, int idle_ms,
                                        se_engine_t** out) {
    clear_error();
    SE_REQUIRE(out != nullptr, SE_ERR_INVALID, "null engine handle");
    SE_REQUIRE(max_slots >= 1 && max_slots <= 65535, SE_ERR_INVALID, "max_slots must be in [1, 65535]");
    SE_REQUIRE(ctas_per_sm >= 1 && ctas_per_sm <= 2, SE_ERR_INVALID, "ctas_per_sm must be 1 or 2");
    SE_REQUIRE(idle_ms >= 1 && idle_ms <= 10000, SE_ERR_INVALID, "idle_ms must be in [1, 10000]");
    int64_t so, co, dof;
    const int64_t need = offsets(max_slots, &so, &co, &dof);
    SE_REQUIRE(d_work && work_bytes >= need, SE_ERR_WORKSPACE, "engine workspace of %lld bytes is below %lld",
               (long long)work_bytes, (long long)need);
    SE_REQUIRE((reinterpret_cast<uintptr_t>(d_work) & 255) == 0, SE_ERR_INVALID, "workspace must be 256-byte aligned");
    if (se_status_t st = raise_smem_limit(reinterpret_cast<const void*>(engine_kernel), int(kEngineSmem),
                                          "the serving engine"))
        return st;
    auto* h = new (std::nothrow) se_engine();
    SE_REQUIRE(h != nullptr, SE_ERR_HOST, "cannot allocate the engine's host state");
    Engine& E = h->e;
    try {  // the host vectors first, while no CUDA resource is held yet
        E.gen.assign(max_slots, 0);
        E.busy.assign(max_slots, 0);
        E.tally_reported.assign(max_slots, 0);
    } catch (const std::exception& x) {
        delete h;
        set_error("cannot allocate the engine's host state: %s", x.what());
        return SE_ERR_HOST;
    }
    E.work = static_cast<uint8_t*>(d_work);
    E.max_slots = max_slots;
    E.hdr = reinterpret_cast<EngineHeader*>(E.work);
    E.slots = reinterpret_cast<Req*>(E.work + so);
    E.claims = reinterpret_cast<uint64_t*>(E.work + co);
    E.dones = reinterpret_cast<uint32_t*>(E.work + dof);
    E.idle_ns = uint64_t(idle_ms) * 1000000ull;
    auto fail = [&](cudaError_t err, const char* what) {
        set_error("%s failed: %s", what, cudaGetErrorString(err));
        if (E.done_host) cudaFreeHost(E.done_host);
        if (E.staging) cudaFreeHost(E.staging);
        if (E.zeros) cudaFreeHost(E.zeros);
        if (E.tally_host) cudaFreeHost(E.tally_host);
        if (E.stream) cudaStreamDestroy(E.stream);
        if (E.finished) cudaEventDestroy(E.finished);
        delete h;
        return se_status_t(SE_ERR_CUDA);
    };
    cudaError_t err;
    if ((err = cudaHostAlloc(&E.done_host, sizeof(uint64_t) * size_t(max_slots), cudaHostAllocMapped)) != cudaSuccess)
        return fail(err, "cudaHostAlloc");
    std::memset(E.done_host, 0, sizeof(uint64_t) * size_t(max_slots));
    if ((err = cudaHostAlloc(&E.staging, kStagingPerSlot * size_t(max_slots), cudaHostAllocDefault)) != cudaSuccess)
        return fail(err, "cudaHostAlloc");
    if ((err = cudaHostAlloc(&E.zeros, kZeroBytes, cudaHostAllocDefault)) != cudaSuccess)
        return fail(err, "cudaHostAlloc");
    std::memset(E.zeros, 0, kZeroBytes);
    if ((err = cudaHostAlloc(&E.tally_host, sizeof(uint32_t) * size_t(max_slots), cudaHostAllocMapped)) != cudaSuccess)
        return fail(err, "cudaHostAlloc");
    std::memset(E.tally_host, 0, sizeof(uint32_t) * size_t(max_slots));
    if ((err = cudaHostGetDevicePointer(reinterpret_cast<void**>(&E.tally_dev), E.tally_host, 0)) != cudaSuccess)
        return fail(err, "cudaHostGetDevicePointer");
    if ((err = cudaHostGetDevicePointer(reinterpret_cast<void**>(&E.done_dev), E.done_host, 0)) != cudaSuccess)
        return fail(err, "cudaHostGetDevicePointer");
    if ((err = cudaStreamCreateWithFlags(&E.stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(err, "cudaStreamCreate");
    if ((err = cudaEventCreateWithFlags(&E.finished, cudaEventDisableTiming)) != cudaSuccess)
        return fail(err, "cudaEventCreate");
    if ((err = cudaMemsetAsync(E.work, 0, size_t(need), E.stream)) != cudaSuccess) return fail(err, "cudaMemset");
    if ((err = cudaStreamSynchronize(E.stream)) != cudaSuccess) return fail(err, "cudaStreamSynchronize");
    int device = 0, sms = 0, occ = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, engine_kernel, cfg<16>::THREADS, kEngineSmem);
    if (occ < 1) return fail(cudaErrorInvalidConfiguration, "engine occupancy");
    E.grid = sms * std::min(occ, ctas_per_sm);
    *out = h;
    return SE_OK;
}

namespace {
struct ScratchLayout {
    int64_t Cq, flags, S, AT, dT, total;
};
ScratchLayout scratch_layout(int C) {
    ScratchLayout L;
    L.Cq = round_up(C, kT);
    L.flags = 0;
    L.S = 256;
    L.AT = round_up(L.S + L.Cq * L.Cq * 2, 256);
    L.dT = round_up(L.AT + int64_t(kT) * L.Cq * 4, 256);
    L.total = L.dT + int64_t(kT) * kT * 4;
    return L;
}
}  // namespace

extern "C" int64_t se_engine_request_scratch_bytes(int64_t V, int C) {
    if (V < 1 || C < 1) return -1;
    return scratch_layout(C).total;
}

// Places f32 [V][Cq], then the bit planes u32 [ceil(V / 32) * B][Cq].
static int64_t planes_offset(int64_t V, int C) { return round_up(V * round_up(C, kT) * 4, 256); }

extern "C" int64_t se_engine_request_positions_bytes(int64_t V, int C) {
    if (V < 1 || C < 1) return -1;
    return planes_offset(V, C) + (V + kVC - 1) / kVC * planes_for(C) * round_up(C, kT) * 4;
}

extern "C" se_status_t se_engine_submit(se_engine_t* h, const se_request_t* rq, void* stream_, int* slot_out,
                                        uint32_t* gen_out) {
    clear_error();
    SE_REQUIRE(h && rq && slot_out && gen_out, SE_ERR_INVALID, "null argument");
    Engine& E = h->e;
    std::lock_guard<std::mutex> lock(E.mu);
    const int C = rq->C;
    const int64_t V = rq->V;
    SE_REQUIRE(C >= 1 && C <= kT * 256, SE_ERR_INVALID, "the engine serves 1 to %d candidates, got %d", kT * 256, C);
    SE_REQUIRE(V >= 1 && V < (int64_t(1) << 24), SE_ERR_INVALID, "the engine serves 1 to 2^24 - 1 ballots");
    SE_REQUIRE(rq->d_ids && rq->d_prefs && rq->d_out && rq->d_wins && rq->d_ranking, SE_ERR_INVALID,
               "a request needs ballots, preference, output, wins and ranking buffers");
    const ScratchLayout L = scratch_layout(C);
    SE_REQUIRE(rq->d_scratch && rq->scratch_bytes >= L.total, SE_ERR_WORKSPACE,
               "request scratch of %lld bytes is below %lld", (long long)rq->scratch_bytes, (long long)L.total);
    const int64_t pos_need = V * L.Cq * 4;
    SE_REQUIRE(rq->d_positions && rq->positions_bytes >= pos_need, SE_ERR_WORKSPACE,
               "ballot-place buffer of %lld bytes is below %lld", (long long)rq->positions_bytes, (long long)pos_need);
    SE_REQUIRE((reinterpret_cast<uintptr_t>(rq->d_positions) & 255) == 0, SE_ERR_INVALID,
               "the ballot-place buffer must be 256-byte aligned");
    SE_REQUIRE((reinterpret_cast<uintptr_t>(rq->d_scratch) & 255) == 0, SE_ERR_INVALID,
               "scratch must be 256-byte aligned");
    int slot = -1;
    for (int s = 0; s < E.max_slots; ++s)
        if (!E.busy[s]) {
            slot = s;
            break;
        }
    SE_REQUIRE(slot >= 0, SE_ERR_UNSUPPORTED, "all %d engine slots are busy", E.max_slots);
    cudaStream_t s = static_cast<cudaStream_t>(stream_);
    uint8_t* sc = static_cast<uint8_t*>(rq->d_scratch);

    Req q;
    std::memset(&q, 0, sizeof(q));
    Elec& e = q.e;
    e.d = rq->d_prefs;
    e.ld = C;
    e.out = rq->d_out;
    e.ld_out = C;
    e.wins = rq->d_wins;
    e.ranking = rq->d_ranking;
    e.C = C;
    e.Cp = int(L.Cq);
    e.R = int(L.Cq / kT);
    e.lanes = 16;
    e.base = rq->value_offset;
    e.S = reinterpret_cast<uint32_t*>(sc + L.S);
    e.AT = reinterpret_cast<uint32_t*>(sc + L.AT);
    e.dT = reinterpret_cast<uint32_t*>(sc + L.dT);
    if (e.R > 1) {
        const int64_t ldw = L.Cq / 2;
        if (se_status_t st = make_map(&e.mapS, e.S, uint64_t(ldw), uint64_t(L.Cq), uint64_t(ldw) * 4, kT / 2, kKC))
            return st;
        if (se_status_t st = make_map(&e.mapAT, e.AT, uint64_t(L.Cq), kT, uint64_t(L.Cq) * 4, kT, kKC)) return st;
        if (se_status_t st = make_map(&e.mapDT, e.dT, kT, kT, kT * 4, kT, kKC)) return st;
    }
    q.pos = static_cast<float*>(rq->d_positions);
    q.B = planes_for(C);
    q.planes = reinterpret_cast<uint32_t*>(static_cast<uint8_t*>(rq->d_positions) + planes_offset(V, C));
    if (se_status_t st = make_map(&q.mapPl, q.planes, uint64_t(L.Cq), uint64_t((V + kVC - 1) / kVC * q.B),
                                  uint64_t(L.Cq) * 4, 64, uint32_t(q.B)))
        return st;
    q.ids = rq->d_ids;
    q.offsets = rq->d_offsets;
    q.flags = reinterpret_cast<uint32_t*>(sc + L.flags);
    q.V = V;
    const uint32_t gen = ++E.gen[slot];
    q.done_host = E.done_dev + slot;
    q.tally_host = E.tally_dev + slot;
    E.tally_reported[slot] = 0;
    q.gen = gen;
    q.active = 0;
    E.done_host[slot] = 0;

    // Host sources of this request's copies live in the slot's pinned staging region, so the
    // copies are truly asynchronous (a pageable source would synchronise the stream).
    const int nph = phases_of(e.R);
    uint8_t* stg = E.staging + kStagingPerSlot * size_t(slot);
    std::memcpy(stg, &q, sizeof(Req));
    uint32_t* stg_words = reinterpret_cast<uint32_t*>(stg + sizeof(Req));
    stg_words[0] = 1;  // active
    stg_words[1] = std::max(E.slot_hi, uint32_t(slot + 1));
    uint64_t* cl = reinterpret_cast<uint64_t*>(stg + sizeof(Req) + 16);
    for (int f = 0; f <= nph; ++f) cl[f] = uint64_t(gen) << 32;
    // Copies only (copy engines), no kernels: see kZeroBytes.
    SE_CUDA_TRY(cudaMemcpyAsync(sc, E.zeros, 256, cudaMemcpyHostToDevice, s));
    if (e.R > 1)
        SE_CUDA_TRY(cudaMemcpyAsync(rq->d_wins, E.zeros, sizeof(int32_t) * size_t(C), cudaMemcpyHostToDevice, s));
    SE_CUDA_TRY(cudaMemcpyAsync(E.claims + size_t(slot) * (kMaxPhases + 1), cl, size_t(nph + 1) * 8,
                                cudaMemcpyHostToDevice, s));
    SE_CUDA_TRY(cudaMemcpyAsync(E.dones + size_t(slot) * kMaxPhases, E.zeros, size_t(nph) * 4,
                                cudaMemcpyHostToDevice, s));
    SE_CUDA_TRY(cudaMemcpyAsync(&E.slots[slot], stg, sizeof(Req), cudaMemcpyHostToDevice, s));
    SE_CUDA_TRY(cudaMemcpyAsync(&E.slots[slot].active, &stg_words[0], 4, cudaMemcpyHostToDevice, s));
    if (uint32_t(slot + 1) > E.slot_hi) {
        E.slot_hi = uint32_t(slot + 1);
        SE_CUDA_TRY(cudaMemcpyAsync(&E.hdr->slot_hi, &stg_words[1], 4, cudaMemcpyHostToDevice, s));
    }
    E.busy[slot] = 1;
    ++E.in_flight;
    *slot_out = slot;
    *gen_out = gen;
    return ensure_running(E);
}

extern "C" se_status_t se_engine_poll(se_engine_t* h, int* slots_out, uint32_t* status_out, int max, int* n_out) {
    clear_error();
    SE_REQUIRE(h && n_out, SE_ERR_INVALID, "null argument");
    Engine& E = h->e;
    std::lock_guard<std::mutex> lock(E.mu);
    int n = 0;
    for (int s = 0; s < E.max_slots && n < max; ++s) {
        if (!E.busy[s]) continue;
        const uint64_t w = reinterpret_cast<volatile uint64_t*>(E.done_host)[s];
        if (uint32_t(w >> 8) == E.gen[s] && E.gen[s] != 0) {
            E.busy[s] = 0;
            --E.in_flight;
            if (slots_out) slots_out[n] = s;
            if (status_out) status_out[n] = uint32_t(w & 0xFF);
            ++n;
        }
    }
    *n_out = n;
    return ensure_running(E);
}

extern "C" se_status_t se_engine_poll_tallied(se_engine_t* h, int* slots_out, int max, int* n_out) {
    clear_error();
    SE_REQUIRE(h && n_out, SE_ERR_INVALID, "null argument");
    Engine& E = h->e;
    std::lock_guard<std::mutex> lock(E.mu);
    int n = 0;
    for (int s = 0; s < E.max_slots && n < max; ++s) {
        if (!E.busy[s] || E.tally_reported[s]) continue;
        if (reinterpret_cast<volatile uint32_t*>(E.tally_host)[s] == E.gen[s]) {
            E.tally_reported[s] = 1;
            if (slots_out) slots_out[n] = s;
            ++n;
        }
    }
    *n_out = n;
    return SE_OK;
}

extern "C" se_status_t se_engine_stats(se_engine_t* h, int64_t* launches, int* grid, int* in_flight,
                                       double* busy_ms, int64_t* tasks, double* search_ms) {
    clear_error();
    SE_REQUIRE(h != nullptr, SE_ERR_INVALID, "null engine");
    Engine& E = h->e;
    std::lock_guard<std::mutex> lock(E.mu);
    if (launches) *launches = E.launches;
    if (grid) *grid = E.grid;
    if (in_flight) *in_flight = E.in_flight;
    if (busy_ms || tasks || search_ms) {
        // The counters are read while the kernel may run: a snapshot, not a barrier.
        EngineHeader hd;
        cudaStream_t side;
        SE_CUDA_TRY(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
        cudaError_t e1 = cudaMemcpyAsync(&hd, E.hdr, sizeof(hd), cudaMemcpyDeviceToHost, side);
        cudaError_t e2 = cudaStreamSynchronize(side);
        cudaStreamDestroy(side);
        SE_CUDA_TRY(e1);
        SE_CUDA_TRY(e2);
        for (int k = 0; k < kKindCount; ++k) {
            if (busy_ms) busy_ms[k] = double(hd.busy_ns[k]) * 1e-6;
            if (tasks) tasks[k] = int64_t(hd.tasks[k]);
        }
        if (search_ms) *search_ms = double(hd.search_ns) * 1e-6;
    }
    return SE_OK;
}

extern "C" se_status_t se_engine_stop(se_engine_t* h) {
    clear_error();
    SE_REQUIRE(h != nullptr, SE_ERR_INVALID, "null engine");
    Engine& E = h->e;
    std::lock_guard<std::mutex> lock(E.mu);
    if (!E.launched) return SE_OK;
    const uint32_t one = 1;
    cudaStream_t side;
    SE_CUDA_TRY(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
    cudaError_t e1 = cudaMemcpyAsync(&E.hdr->stop, &one, 4, cudaMemcpyHostToDevice, side);
    cudaError_t e2 = cudaStreamSynchronize(side);
    cudaStreamDestroy(side);
    SE_CUDA_TRY(e1);
    SE_CUDA_TRY(e2);
    SE_CUDA_TRY(cudaEventSynchronize(E.finished));
    const uint32_t zero = 0;
    SE_CUDA_TRY(cudaMemcpy(&E.hdr->stop, &zero, 4, cudaMemcpyHostToDevice));
    E.launched = false;
    EngineHeader hd;
    SE_CUDA_TRY(cudaMemcpy(&hd, E.hdr, sizeof(hd), cudaMemcpyDeviceToHost));
    SE_REQUIRE(hd.err == 0, SE_ERR_DEVICE, "serving engine reported device error %u", hd.err);
    return SE_OK;
}

extern "C" se_status_t se_engine_destroy(se_engine_t* h) {
    clear_error();
    if (!h) return SE_OK;
    se_status_t st = se_engine_stop(h);
    Engine& E = h->e;
    if (E.done_host) cudaFreeHost(E.done_host);
    if (E.staging) cudaFreeHost(E.staging);
    if (E.zeros) cudaFreeHost(E.zeros);
    if (E.tally_host) cudaFreeHost(E.tally_host);
    if (E.stream) cudaStreamDestroy(E.stream);
    if (E.finished) cudaEventDestroy(E.finished);
    delete h;
    return st;
}
