/*
 * oracle.c - CPU restatement of the Schulze path of ashvardanian/ScalingElections.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker that tests, the smoke check and the
 * benchmark's CPU-baseline leg compare the CUDA path against. The product path
 * (scalingelections_b200, libse.so) never links, loads or calls it.
 *
 * Each function names the reference lines it restates (paths relative to the reference
 * project). The arithmetic is unsigned 32-bit integer, as in the reference
 * (scaling_elections.cu:90-93, scaling_elections.py:68 and :102).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define OR_API __attribute__((visibility("default")))

static inline uint32_t min_u32(uint32_t a, uint32_t b) { return a < b ? a : b; }

/*
 * Ballot tally, restating build_pairwise_preferences (scaling_elections.py:51-88) and
 * populate_preferences_from_ranking (scaling_elections.py:37-48):
 *   - C is fixed by the caller (the reference takes max(id) + 1, py:63-66);
 *   - a ballot shorter than C gets the ids it lacks appended in ascending order
 *     (py:75-83: np.nonzero over a presence mask);
 *   - then d[r[a]][r[b]] += 1 for every a < b (py:46-48).
 * Ballot v is ids[offsets[v] .. offsets[v+1]). Returns 0, or -1 for an id outside [0, C).
 * Ballots with repeated ids are counted exactly as the reference counts them.
 */
OR_API int or_tally_scatter(const int32_t* ids, const int64_t* offsets, int64_t V, int C,
                            uint32_t* d) {
    memset(d, 0, sizeof(uint32_t) * (size_t)C * (size_t)C);
    int64_t max_len = 0;
    for (int64_t v = 0; v < V; ++v) {
        int64_t len = offsets[v + 1] - offsets[v];
        if (len > max_len) max_len = len;
        for (int64_t a = offsets[v]; a < offsets[v + 1]; ++a)
            if (ids[a] < 0 || ids[a] >= C) return -1;
    }
    int32_t* buf = (int32_t*)malloc(sizeof(int32_t) * (size_t)(max_len + C + 1));
    unsigned char* present = (unsigned char*)malloc((size_t)C + 1);
    if (!buf || !present) {
        free(buf);
        free(present);
        return -2;
    }
    for (int64_t v = 0; v < V; ++v) {
        const int32_t* r = ids + offsets[v];
        int64_t len = offsets[v + 1] - offsets[v];
        int64_t n = 0;
        for (int64_t a = 0; a < len; ++a) buf[n++] = r[a];
        if (len != C) {
            /* py:75-83: append np.nonzero(~present), i.e. the absent ids ascending. */
            memset(present, 0, (size_t)C);
            for (int64_t a = 0; a < len; ++a) present[r[a]] = 1;
            for (int c = 0; c < C; ++c)
                if (!present[c]) buf[n++] = c;
        }
        for (int64_t a = 0; a < n; ++a) {
            uint32_t* row = d + (size_t)buf[a] * C;
            for (int64_t b = a + 1; b < n; ++b) row[buf[b]] += 1;
        }
    }
    free(buf);
    free(present);
    return 0;
}

/*
 * Same tally through rank positions, d[i][j] = #{v : pos_v(i) < pos_v(j)}, which equals the
 * scatter form above for ballots without repeated ids (every completed ballot is then a
 * permutation of 0..C-1). Parallel over rows i; used for sizes the scatter form is too slow
 * for, after a test shows both agree. pos must hold V * C int32 (scratch).
 */
OR_API int or_tally_positions(const int32_t* ids, const int64_t* offsets, int64_t V, int C,
                              uint32_t* d, int32_t* pos) {
    int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
    for (int64_t v = 0; v < V; ++v) {
        int32_t* p = pos + (size_t)v * C;
        for (int c = 0; c < C; ++c) p[c] = -1;
        const int32_t* r = ids + offsets[v];
        int64_t len = offsets[v + 1] - offsets[v];
        for (int64_t a = 0; a < len; ++a) {
            if (r[a] < 0 || r[a] >= C || p[r[a]] >= 0) {
                bad |= 1;
                break;
            }
            p[r[a]] = (int32_t)a;
        }
        int32_t next = (int32_t)len;
        for (int c = 0; c < C; ++c)
            if (p[c] < 0) p[c] = next++;
    }
    if (bad) return -1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int i = 0; i < C; ++i) {
        uint32_t* row = d + (size_t)i * C;
        memset(row, 0, sizeof(uint32_t) * (size_t)C);
        for (int64_t v = 0; v < V; ++v) {
            const int32_t* p = pos + (size_t)v * C;
            int32_t pi = p[i];
            for (int j = 0; j < C; ++j) row[j] += (uint32_t)(pi < p[j]);
        }
        row[i] = 0;
    }
    return 0;
}

/*
 * Defeat matrix, restating scaling_elections.py:105-112: S[i][j] = d[i][j] if
 * d[i][j] > d[j][i] else 0, diagonal 0. d has row stride ld.
 */
OR_API void or_defeats(const uint32_t* d, int64_t ld, int C, uint32_t* S) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C; ++i)
        for (int j = 0; j < C; ++j) {
            uint32_t dij = d[(size_t)i * ld + j], dji = d[(size_t)j * ld + i];
            S[(size_t)i * C + j] = (i != j && dij > dji) ? dij : 0;
        }
}

/*
 * Serial widest-path closure, restating compute_strongest_paths_numba_serial step 2
 * (scaling_elections.py:114-123): pivot i outermost, masks i != j, i != k, j != k.
 */
OR_API void or_closure_serial(uint32_t* S, int C) {
    for (int i = 0; i < C; ++i)
        for (int j = 0; j < C; ++j) {
            if (i == j) continue;
            uint32_t sji = S[(size_t)j * C + i];
            const uint32_t* row_i = S + (size_t)i * C;
            uint32_t* row_j = S + (size_t)j * C;
            for (int k = 0; k < C; ++k) {
                if (i == k || j == k) continue;
                uint32_t cand = min_u32(sji, row_i[k]);
                if (cand > row_j[k]) row_j[k] = cand;
            }
        }
}

/*
 * Masked tile relaxation, restating compute_strongest_paths_tile_numba
 * (scaling_elections.py:128-159), with the tile clipped at the matrix edge so any C works
 * (the reference requires C % tile == 0).
 */
static void tile_relax(uint32_t* S, int C, int c_row, int c_col, int a_row, int a_col,
                       int b_row, int b_col, int T) {
    int ti = T < C - c_row ? T : C - c_row;
    int tj = T < C - c_col ? T : C - c_col;
    int tk = T < C - a_col ? T : C - a_col;
    for (int k = 0; k < tk; ++k)
        for (int i = 0; i < ti; ++i)
            for (int j = 0; j < tj; ++j) {
                if (c_row + i == c_col + j || a_row + i == a_col + k || b_row + k == b_col + j)
                    continue;
                uint32_t rep = min_u32(S[(size_t)(a_row + i) * C + a_col + k],
                                       S[(size_t)(b_row + k) * C + b_col + j]);
                uint32_t* c = &S[(size_t)(c_row + i) * C + c_col + j];
                if (rep > *c) *c = rep;
            }
}

/*
 * Blocked closure, restating compute_strongest_paths_numba_parallel step 2
 * (scaling_elections.py:190-269): per pivot block k, the diagonal tile, then the column
 * tiles (i, k), the row tiles (k, j), then every independent tile (i, j), i, j != k.
 * The prange loops (py:211, 230, 249) become OpenMP loops. threads <= 0 keeps the default.
 */
OR_API void or_closure_blocked(uint32_t* S, int C, int T, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    int R = (C + T - 1) / T;
    for (int k = 0; k < R; ++k) {
        int ks = k * T;
        tile_relax(S, C, ks, ks, ks, ks, ks, ks, T);
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 0; i < R; ++i)
            if (i != k) tile_relax(S, C, i * T, ks, i * T, ks, ks, ks, T);
#pragma omp parallel for schedule(dynamic, 1)
        for (int j = 0; j < R; ++j)
            if (j != k) tile_relax(S, C, ks, j * T, ks, ks, ks, j * T, T);
#pragma omp parallel for schedule(dynamic, 1)
        for (int i = 0; i < R; ++i) {
            if (i == k) continue;
            for (int j = 0; j < R; ++j)
                if (j != k) tile_relax(S, C, i * T, j * T, i * T, ks, ks, j * T, T);
        }
    }
}

/*
 * Ranking, restating get_winner_and_ranking (scaling_elections.py:274-296):
 * wins[i] = #{j != i : S[i][j] > S[j][i]}; ranking = indices sorted by wins descending with
 * Python's stable sort (ties keep ascending index). Counting sort keeps that order.
 */
OR_API int or_rank(const uint32_t* S, int64_t ld, int C, int32_t* wins, int32_t* ranking) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < C; ++i) {
        int32_t w = 0;
        for (int j = 0; j < C; ++j)
            if (i != j && S[(size_t)i * ld + j] > S[(size_t)j * ld + i]) ++w;
        wins[i] = w;
    }
    int64_t* start = (int64_t*)calloc((size_t)C + 1, sizeof(int64_t));
    if (!start) return -2;
    for (int i = 0; i < C; ++i) start[wins[i]]++;
    int64_t acc = 0;
    for (int w = C - 1; w >= 0; --w) {
        int64_t n = start[w];
        start[w] = acc;
        acc += n;
    }
    for (int i = 0; i < C; ++i) ranking[start[wins[i]]++] = i;
    free(start);
    return 0;
}

/*
 * Widest paths from one source by a bottleneck Dijkstra over the defeat matrix S0 (as made by
 * or_defeats). Not a restatement of a reference routine: an independent O(C^2) check of one
 * row of the closure, straight from the definition the reference's closure computes
 * (scaling_elections.py:91-125): out[j] = max over paths src -> j of the weakest edge, and
 * out[src] = 0. Used to check rows of closures too large for a full C^3 oracle run.
 */
OR_API int or_widest_from(const uint32_t* S0, int64_t ld, int C, int src, uint32_t* out) {
    unsigned char* done = (unsigned char*)calloc((size_t)C, 1);
    if (!done) return -2;
    for (int j = 0; j < C; ++j) out[j] = 0;
    out[src] = 0xFFFFFFFFu;
    for (int it = 0; it < C; ++it) {
        int u = -1;
        uint32_t best = 0;
        for (int j = 0; j < C; ++j)
            if (!done[j] && (u < 0 || out[j] > best)) {
                u = j;
                best = out[j];
            }
        if (u < 0 || best == 0) break;
        done[u] = 1;
        const uint32_t* row = S0 + (size_t)u * ld;
        for (int v = 0; v < C; ++v) {
            if (done[v]) continue;
            uint32_t cand = min_u32(best, row[v]);
            if (cand > out[v]) out[v] = cand;
        }
    }
    out[src] = 0;
    free(done);
    return 0;
}

/*
 * Repeated-insertion decode for the Mallows sampler (test-input generation only, no
 * reference counterpart): slots[v][i] in [0, i] is where item i was inserted; pos[v][i]
 * receives item i's final place. Items are placed from last to first, each into the
 * slots[v][i]-th still-free place, found with a Fenwick tree over free places.
 */
OR_API int or_rim_decode(const int64_t* slots, int64_t V, int C, int64_t* pos) {
    int size = 1;
    while (size < C) size <<= 1;
    int bad = 0;
#pragma omp parallel reduction(| : bad)
    {
        int32_t* tree = (int32_t*)malloc(sizeof(int32_t) * ((size_t)size + 1));
        if (!tree) bad = 1;
#pragma omp for schedule(static)
        for (int64_t v = 0; v < V; ++v) {
            if (!tree) continue;
            for (int k = 1; k <= size; ++k) {
                int low = k & -k, hi = k < C ? k : C, n = hi - (k - low);
                tree[k] = n > 0 ? n : 0;
            }
            const int64_t* s = slots + (size_t)v * C;
            int64_t* p = pos + (size_t)v * C;
            for (int i = C - 1; i >= 0; --i) {
                int64_t want = s[i] + 1;
                int idx = 0;
                for (int step = size; step; step >>= 1) {
                    int nxt = idx + step;
                    if (nxt <= size && tree[nxt] < want) {
                        idx = nxt;
                        want -= tree[nxt];
                    }
                }
                if (idx >= C) {
                    bad = 1;
                    break;
                }
                p[i] = idx;
                for (int k = idx + 1; k <= size; k += k & -k) tree[k] -= 1;
            }
        }
        free(tree);
    }
    return bad ? -1 : 0;
}
