/*
 * se.h - C ABI of the sm_100a Schulze hot path (ballot tally, widest-path closure, ranking).
 *
 * Conventions (all entry points):
 *   - Pointers named d_* are DEVICE pointers owned by the caller. Nothing here allocates or
 *     frees memory on the compute paths; scratch space is passed in as `d_work`, sized by the
 *     matching *_workspace_bytes() query.
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream). Calls are
 *     stream-ordered and asynchronous unless the comment says otherwise.
 *   - The return value is an se_status_t; on failure se_last_error() returns a message
 *     (thread-local). Messages reuse the reference's wording where it has one.
 *   - Matrices are row-major uint32 with a row stride `ld` counted in elements.
 *
 * Reference interfaces replaced (paths relative to ashvardanian/ScalingElections):
 *   compute_strongest_paths      scaling_elections.cu:863-989, bound at :1034-1038
 *   compute_strongest_paths_cuda scaling_elections.cu:490-578
 *   log_gpus                     scaling_elections.cu:996-1016
 *   build_pairwise_preferences   scaling_elections.py:51-88 (+ populate_... :37-48)
 *   get_winner_and_ranking       scaling_elections.py:274-296
 */
#ifndef SE_H
#define SE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define SE_API __attribute__((visibility("default")))
#else
#define SE_API
#endif

typedef int se_status_t;

#define SE_OK 0
#define SE_ERR_INVALID 1     /* malformed argument (shape, range, null pointer) */
#define SE_ERR_CUDA 2        /* a CUDA runtime call or a kernel launch failed */
#define SE_ERR_UNSUPPORTED 3 /* e.g. a tile size this build does not provide */
#define SE_ERR_DEVICE 4      /* a kernel raised its device-side error word */
#define SE_ERR_OVERFLOW 5    /* a count does not fit the requested 16-bit lanes */
#define SE_ERR_WORKSPACE 6   /* d_work missing or smaller than the *_workspace_bytes() query */
#define SE_ERR_HOST 7        /* a host-side resource (memory, a lock) could not be obtained */

/* Lane modes for the closure: 16 = two u16 cells per 32-bit word (every count < 65536),
 * 32 = one u32 cell per word, 0 = choose on the device: 16-bit lanes whenever the kept
 * defeat values fit a window of 65535 (stored shifted by a base; the closure commutes with
 * that shift), which holds for any tally of up to 131070 ballots; else 32-bit. The automatic
 * choice costs one pass over d, an 8-byte device-to-host read and a stream synchronisation. */
#define SE_LANES_AUTO 0
#define SE_LANES_U16 16
#define SE_LANES_U32 32

/* Message of the last failed call on this thread ("" if none). */
SE_API const char* se_last_error(void);

/* ABI version, bumped on any signature change. */
SE_API int se_version(void);

/* ---------------------------------------------------------------------------------------
 * Device information. Replaces log_gpus (scaling_elections.cu:996-1016), which prints the
 * name, SM count, global memory and compute capability of every device.
 * ------------------------------------------------------------------------------------- */
SE_API se_status_t se_device_count(int* count);
SE_API se_status_t se_device_info(int device, char* name, int name_capacity, int* sm_count,
                           double* global_mem_gib, int* cc_major, int* cc_minor);

/* ---------------------------------------------------------------------------------------
 * Widest-path closure. Replaces compute_strongest_paths(preferences, allow_gpu=True, ...)
 * (scaling_elections.cu:863-989 -> compute_strongest_paths_cuda :490-578).
 *
 *   d_pref  C x C uint32 pairwise preference counts d[i][j], row stride ld_pref.
 *   d_out   C x C uint32 strongest-path strengths, row stride ld_out. Diagonal is 0.
 *           out[i][j] = widest path i->j in the graph with edge i->j of width d[i][j] when
 *           d[i][j] > d[j][i] (else no edge), exactly as scaling_elections.py:91-125.
 *   tile    pivot block edge; 0 picks the default. Unsupported values return
 *           SE_ERR_UNSUPPORTED ("Unsupported tile size", as scaling_elections.cu:900).
 *   d_work  scratch of at least se_closure_workspace_bytes(C, lane_bits, tile) bytes.
 * Any C >= 1 is accepted (the reference's GPU path needs C % tile == 0).
 * ------------------------------------------------------------------------------------- */
SE_API int64_t se_closure_workspace_bytes(int C, int lane_bits, int tile);
SE_API se_status_t se_closure(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out,
                       int64_t ld_out, int lane_bits, int tile, void* d_work,
                       int64_t work_bytes, void* stream);

/* se_closure without its closing synchronisation (same reference interface, cu:863-989):
 * every step is queued on `stream` and the call returns at once, so a caller can queue
 * several closures, or overlap their host<->device copies on another stream. lane_bits is
 * 16 or 32 (the automatic mode reads the matrix's range back and is not available here).
 * value_offset shifts 16-bit lanes as in se_batch (a kept count v is held as v - value_offset,
 * which must lie in [1, 65535]; 0 = no shift). Errors of the arguments return at once; errors
 * found on the device (a count outside the 16-bit window, a timed-out wait) are kept in the
 * first 8 bytes of d_work until se_closure_check reads them. d_work must not be reused by
 * another call before that check. A call may be captured into a CUDA graph once a first call
 * of the same lane width has run outside any capture (it sets the kernels' shared-memory
 * limits); each replay closes the captured matrices again. */
SE_API se_status_t se_closure_enqueue(const uint32_t* d_pref, int64_t ld_pref, int C,
                                      uint32_t* d_out, int64_t ld_out, int lane_bits,
                                      uint32_t value_offset, void* d_work, int64_t work_bytes,
                                      void* stream);

/* Synchronises `stream` and reports what the closure enqueued with d_work found on the
 * device: SE_OK, SE_ERR_OVERFLOW (a count outside the 16-bit window) or SE_ERR_DEVICE. */
SE_API se_status_t se_closure_check(const void* d_work, void* stream);

/* Same as se_closure, and also fills phase_ms[4] with the summed device time of the four
 * kernel kinds (pivot tile, pivot-row panel, pivot-column panel, remainder) from CUDA events
 * recorded between the launches, and *launches with the number of kernels launched.
 * Synchronous. For profiling: the events add a little time between launches. */
SE_API se_status_t se_closure_profiled(const uint32_t* d_pref, int64_t ld_pref, int C, uint32_t* d_out,
                                       int64_t ld_out, int lane_bits, int tile, void* d_work,
                                       int64_t work_bytes, void* stream, double* phase_ms, int* launches);

/* Workspace for every schedule of se_closure_set_mode at its fastest, a few MiB above
 * se_closure_workspace_bytes: the dataflow form (mode 2: one persistent launch whose task order
 * runs the next round's pivot and panels ahead of the current round's bulk; identical results,
 * slower on B200 than the round-by-round forms at every size measured), the second AT buffer
 * of modes 5, 6 and 8, and the split-K area of modes 1, 3, 4, 6, 7 and 8: with it, for R <= 28
 * row blocks (C <= 3584), each panel tile and the next pivot tile run as 4 CTAs over disjoint
 * pivot chunks whose partial tiles the last one folds with a lane-wise max (exact), which
 * shortens each round's chain at small C. */
SE_API int64_t se_closure_workspace_bytes_flow(int C, int lane_bits, int tile);

/* Task t (< R^3) of the dataflow closure's fixed order for R = ceil(C / 128) pivot blocks:
 * kind 0 pivot, 1 pivot-row panel, 2 pivot-column panel, 3 remainder; round k; tile (i, j).
 * Host-only (no GPU needed): lets tests check the order against the dependency rules. */
SE_API se_status_t se_closure_flow_task(uint32_t t, int R, int* kind, int* k, int* i, int* j);

/* Process-wide schedule of se_closure (results are identical in every one):
 *   0  automatic (default): by C, from the variant table below; 1 where it has no entry;
 *   1  round by round: pivot, panels and remainder launches per round, panels and pivots on
 *      the default micro-tile (8 x 8 words per thread), the next round's pivot closed by the
 *      first CTA of the remainder launch (with se_closure_workspace_bytes_flow() of workspace
 *      and C <= 3584, panel tiles and the next pivot tile split-K, as that function says);
 *   2  dataflow: one persistent launch (needs se_closure_workspace_bytes_flow() of workspace);
 *   3  as 1 with the panels on the wide micro-tile (8 x 4 words per thread, twice the warps);
 *   4  as 3 with every pivot tile closed by its own launch on the wide micro-tile;
 *   5  as 3 on two streams: each round's remainder tiles of the next pivot row and column, and
 *      the next round's panels, run on `stream` while the rest of the round's remainder runs
 *      on a second, lower-priority stream of the library's (joined before the call's last
 *      launch), so the next round's chain overlaps the current round's bulk. Needs
 *      se_closure_workspace_bytes_flow() of workspace and C > 384 (else it runs 3); the
 *      automatic schedule picks it only when the workspace is that large;
 *   6  one launch per round: round k's remainder tiles and round k+1's panel tiles, the
 *      panels taking the remainder's last, partial wave (they wait, bounded, for the tiles
 *      of row and column k+1 and the next pivot, which the launch runs first). Needs
 *      se_closure_workspace_bytes_flow() of workspace (else the automatic schedule runs 1);
 *   7  as 3 with the remainder tiles on the wide micro-tile too (the fused pivot then closes
 *      on eight warps);
 *   8  as 6 with every tile on the wide micro-tile.
 * 3, 4 and 7 differ from 1, and 8 from 6, in 16-bit lanes only. */
SE_API se_status_t se_closure_set_mode(int mode);

/* The variant table of the automatic schedule: for C <= max_c[i] (the first i that holds) use
 * modes[i] (1 or 3 to 8); C above every entry uses 1. n <= 8; n = 0 clears it. The built-in
 * table, measured on B200, is {C <= 1024: 7, C <= 4096: 8, larger: 6}. An autotuner
 * measures the variants per size bucket and installs the winners (scalingelections_b200
 * autotune.tune_closure). No reference counterpart: the reference's tile_size argument picks
 * among its kernels' tile templates (scaling_elections.cu:895-901). */
SE_API se_status_t se_closure_set_variant_table(const int* max_c, const int* modes, int n);

/* The schedule (1 to 8) an se_closure call would run now for C candidates with lane_bits 16
 * or 32 and work_bytes of workspace; -1 for C < 1. Host-only. */
SE_API int se_closure_schedule(int C, int lane_bits, int64_t work_bytes);

/* Number of kernels one se_closure call launches for C candidates in 16-bit lanes under the
 * current schedule (automatic lanes add at most one more). */
SE_API int se_closure_launch_count(int C);

/* Largest C that se_closure_noalloc accepts. */
#define SE_NOALLOC_MAX_CANDIDATES 2048

/* No counterpart in the reference. The same widest-path closure as se_closure for callers
 * that cannot allocate device memory: plugins whose host application owns the GPU memory
 * budget, and latency-critical code that cannot afford cudaMalloc/cudaFree (cudaFree
 * synchronises the device). The scratch space is a static 18 MiB device array inside this
 * library, held on every GPU that loads it until the process exits, so C is limited to
 * 1..SE_NOALLOC_MAX_CANDIDATES in any lane mode; larger C returns SE_ERR_INVALID with a
 * message. It always runs round by round (se_closure_set_mode does not apply). Nothing is
 * allocated or freed. The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress), and looks it up again after cudaDeviceReset: make that first call
 * before any stream capture. All calls share the array; calls that overlap on the GPU (e.g.
 * on different streams) race and must be serialised by the caller. Synchronises `stream`
 * once at the end, like se_closure. */
SE_API se_status_t se_closure_noalloc(const uint32_t* d_pref, int64_t ld_pref, int C,
                                      uint32_t* d_out, int64_t ld_out, int lane_bits,
                                      void* stream);

/* ---------------------------------------------------------------------------------------
 * Batched closure (no reference counterpart; the reference closes one matrix per call,
 * scaling_elections.cu:863-989): many independent elections of uneven size, all tasks in
 * one persistent launch per lane mode, optionally replayed as a CUDA graph.
 *
 * Each election gives its preference matrix, output matrix and (optionally, both or
 * neither) wins/ranking arrays, with the same meaning as se_closure and se_rank. Elections
 * with C <= 128 run whole inside one CTA; larger ones are cut into 128 x 128 tile tasks
 * scheduled by per-election round counters. lane_bits per election: 16 or 32 (0 means 32).
 * 16-bit lanes hold every kept value v (d[i][j] > d[j][i]) as v - value_offset, which must
 * lie in [1, 65535]; the closure commutes with that shift, so results stay exact. For counts
 * from V ballots, value_offset = V / 2 (rounded down) works for every V <= 131070, and 0 for
 * V < 65536. A value outside the window makes se_batch_check report SE_ERR_OVERFLOW.
 *
 *   se_batch_workspace_bytes   device bytes for the batch (host-only computation).
 *   se_batch_prepare           builds the task queues and tensor maps and uploads them into
 *                              d_work (synchronous copies); fills the caller's plan.
 *                              order: 0 = small elections after the tiled ones, 1 = before.
 *                              ctas_per_sm: persistent CTAs per SM (0 = as many as fit).
 *   se_batch_run               enqueues one whole batch on `stream` (asynchronous, no host
 *                              synchronisation, capturable).
 *   se_batch_graph_build       captures se_batch_run into a CUDA graph held by the plan;
 *   se_batch_graph_launch      replays it on `stream`; se_batch_release frees the graph.
 *   se_batch_check             reads the batch's device error word (synchronises `stream`).
 * The plan refers to d_work and to the elections' buffers: keep them alive while it is used.
 * ------------------------------------------------------------------------------------- */
typedef struct se_election {
    const uint32_t* d_pref;
    int64_t ld_pref;
    uint32_t* d_out;
    int64_t ld_out;
    int32_t* d_wins;    /* C entries, or NULL */
    int32_t* d_ranking; /* C entries, or NULL */
    int32_t C;
    int32_t lane_bits;
    uint32_t value_offset; /* 16-bit lanes only */
    /* Micro-tile of the tile tasks: 0 or 8 the default (8 x 8 words per thread), 4 the wide
     * one (8 x 4 words, 256-thread CTAs; 16-bit lanes, used for C > 128). The batch runs each
     * kind in its own persistent launch; the autotuner picks one per size bucket. */
    int32_t micro_tile;
} se_election_t;

typedef struct se_batch_plan {
    int64_t opaque[40];
} se_batch_plan_t;

SE_API int64_t se_batch_workspace_bytes(int n, const se_election_t* elections);
SE_API se_status_t se_batch_prepare(int n, const se_election_t* elections, void* d_work,
                                    int64_t work_bytes, int order, int ctas_per_sm,
                                    se_batch_plan_t* plan);
SE_API se_status_t se_batch_run(const se_batch_plan_t* plan, void* stream);
SE_API se_status_t se_batch_graph_build(se_batch_plan_t* plan);
SE_API se_status_t se_batch_graph_launch(const se_batch_plan_t* plan, void* stream);
SE_API se_status_t se_batch_release(se_batch_plan_t* plan);
SE_API se_status_t se_batch_check(const se_batch_plan_t* plan, void* stream);
/* Limit of one dependency wait of the batch's persistent kernel (default 5 s): a task whose
 * prerequisite is not complete within it sets the batch's error word, every CTA drains the
 * queue and exits, and se_batch_check returns SE_ERR_DEVICE; the GPU stays usable. Applies
 * to runs enqueued after the call; a graph built before it is released (build it again). */
SE_API se_status_t se_batch_set_wait_limit(se_batch_plan_t* plan, uint64_t limit_ns);
/* Profile of the last run (synchronises `stream`): per task kind (small election, pivot,
 * row panel, column panel, remainder) CTA-milliseconds busy and tasks run, and the
 * CTA-milliseconds spent waiting for dependencies. Any pointer may be NULL. */
SE_API se_status_t se_batch_profile(const se_batch_plan_t* plan, double* busy_ms, int64_t* tasks,
                                    double* wait_ms, void* stream);
/* Number of tasks in queue 0 (16-bit lanes), 1 (32-bit lanes) or 2 (16-bit lanes on the wide
 * micro-tile) of a prepared plan. */
SE_API int64_t se_batch_task_count(const se_batch_plan_t* plan, int queue);

/* ---------------------------------------------------------------------------------------
 * Serving engine (no reference counterpart): continuous batching of whole elections (tally,
 * closure, ranking) on one persistent kernel that keeps running while requests are added.
 * Each request's work is split into phases of independent tasks; the kernel's CTAs take
 * claimable tasks from the oldest requests first, so new requests join the running kernel.
 *
 *   se_engine_workspace_bytes        device bytes for an engine with max_slots request slots.
 *   se_engine_create                 ctas_per_sm in {1, 2}; idle_ms: the kernel exits after
 *                                    that long without work, and the next submit or poll
 *                                    relaunches it.
 *   se_engine_request_scratch_bytes  per-request scratch (working matrix, panels) for C
 *                                    candidates; se_engine_request_positions_bytes the ballot
 *                                    places, which are released early (se_engine_poll_tallied).
 *   se_engine_submit                 publishes a request on `stream` (a few small copies and
 *                                    memsets; asynchronous). Returns its slot and generation.
 *   se_engine_poll                   requests finished since the last poll: slot and status
 *                                    (0 ok, 4 = a kept count outside the 16-bit window,
 *                                    8|2 = ballot id out of range, 8|3 = repeated id).
 *   se_engine_stop / destroy         stop the kernel (waits for it) / also free host state.
 * Every buffer of a request must stay alive until poll reports it.
 * ------------------------------------------------------------------------------------- */
typedef struct se_request {
    const int32_t* d_ids;      /* ballots, most preferred first (see se_tally) */
    const int64_t* d_offsets;  /* V + 1 CSR offsets, or NULL: every ballot lists exactly C ids */
    int64_t V;
    int32_t C;
    uint32_t value_offset;     /* 16-bit lane shift, as in se_election_t (V / 2 above 65535) */
    uint32_t* d_prefs;         /* out: C x C preference counts, row stride C */
    uint32_t* d_out;           /* out: C x C strongest paths, row stride C */
    int32_t* d_wins;           /* out: C */
    int32_t* d_ranking;        /* out: C */
    void* d_scratch;           /* se_engine_request_scratch_bytes(V, C), 256-byte aligned */
    int64_t scratch_bytes;
    void* d_positions;         /* ballot places: se_engine_request_positions_bytes(V, C), 256-byte
                                  aligned; free for reuse once se_engine_poll_tallied reports it */
    int64_t positions_bytes;
} se_request_t;

typedef struct se_engine se_engine_t;
SE_API int64_t se_engine_workspace_bytes(int max_slots);
SE_API se_status_t se_engine_create(void* d_work, int64_t work_bytes, int max_slots, int ctas_per_sm,
                                    int idle_ms, se_engine_t** engine);
SE_API int64_t se_engine_request_scratch_bytes(int64_t V, int C);
SE_API int64_t se_engine_request_positions_bytes(int64_t V, int C);
SE_API se_status_t se_engine_submit(se_engine_t* engine, const se_request_t* request, void* stream,
                                    int* slot, uint32_t* generation);
SE_API se_status_t se_engine_poll(se_engine_t* engine, int* slots, uint32_t* statuses, int max,
                                  int* n_finished);
/* Requests whose tally finished since the last call: their ballot-place buffer (usually the
 * largest part of a request's memory) may be reused from now on. */
SE_API se_status_t se_engine_poll_tallied(se_engine_t* engine, int* slots, int max, int* n);
/* Kernel launches so far, the engine's grid size, requests in flight and, when the arrays
 * are given, a profile snapshot: busy_ms[8] / tasks[8] per task kind (positions, tally,
 * small election, round 0's pivot, panels, remainder (which closes the later pivots: the task
 * that updates a round's next pivot tile closes it), output + wins, ranking), summed over
 * CTAs, and the CTA-milliseconds spent looking for work (any pointer may be NULL). */
SE_API se_status_t se_engine_stats(se_engine_t* engine, int64_t* launches, int* grid, int* in_flight,
                                   double* busy_ms, int64_t* tasks, double* search_ms);
SE_API se_status_t se_engine_stop(se_engine_t* engine);
SE_API se_status_t se_engine_destroy(se_engine_t* engine);

/* ---------------------------------------------------------------------------------------
 * One election's closure sharded across GPUs by row blocks (no reference counterpart: the
 * reference closes one matrix on one GPU, scaling_elections.cu:490-578).
 *
 * With R = ceil(C / 128) row blocks of 128 candidates, each GPU (rank) holds a shard: the row
 * blocks [b0, b1) of the working matrix. For every pivot round k = 0 .. R-1, in order:
 *   1. the shard that holds block k calls se_shard_pivot(k): it closes the pivot tile and
 *      updates its pivot-row panel;
 *   2. the caller broadcasts that panel, se_shard_panel_bytes() bytes at byte offset
 *      se_shard_panel_offset(k) of the owner's workspace, into the same offset of every other
 *      shard's workspace (e.g. one NCCL broadcast; the offsets differ between owner and
 *      receivers, so each rank asks its own shard; receivers have one buffer per round
 *      parity, so panel k+1 may arrive while round k still reads panel k);
 *   3. every shard calls se_shard_update(k): column panels and remainder tiles of its rows.
 * Look-ahead order, which lets panel k+1 cross the links during round k's remainder: in round
 * k the shard holding row block k+1 first calls se_shard_update_part(k, 1) (that row block
 * alone, closing the next pivot tile) and se_shard_pivot(k+1); the broadcast of panel k+1
 * then starts (asynchronously) on every rank, and every shard calls se_shard_update_part(k, 2)
 * (all its other rows) while it is in flight. Both orders give identical results.
 * Before round 0 each shard calls se_shard_init with the whole C x C preference matrix on its
 * GPU; after round R-1, se_shard_finalize writes its rows [128 b0, min(128 b1, C)) of the
 * strongest-path matrix (u32, zero diagonal). Results equal se_closure's bit for bit.
 * lane_bits 16 (value_offset as in se_election_t) or 32. All calls are stream-ordered;
 * se_shard_check synchronises and reports device errors.
 * ------------------------------------------------------------------------------------- */
typedef struct se_shard se_shard_t;
SE_API int64_t se_shard_workspace_bytes(int C, int b0, int b1, int lane_bits);
SE_API se_status_t se_shard_create(int C, int b0, int b1, int lane_bits, uint32_t value_offset,
                                   void* d_work, int64_t work_bytes, se_shard_t** shard);
SE_API se_status_t se_shard_destroy(se_shard_t* shard);
SE_API se_status_t se_shard_init(se_shard_t* shard, const uint32_t* d_pref, int64_t ld_pref, void* stream);
SE_API se_status_t se_shard_pivot(se_shard_t* shard, int k, void* stream);
SE_API int64_t se_shard_panel_offset(const se_shard_t* shard, int k);
SE_API int64_t se_shard_panel_bytes(const se_shard_t* shard);
SE_API se_status_t se_shard_update(se_shard_t* shard, int k, void* stream);
/* se_shard_update in parts: part 0 all of it; 1 row block k+1 alone (no launch unless this
 * shard holds it), its tile (k+1, k+1) then closed as the next pivot; 2 every row but k+1.
 * Parts 1 then 2 of one round do what part 0 does. */
SE_API se_status_t se_shard_update_part(se_shard_t* shard, int k, int part, void* stream);
SE_API se_status_t se_shard_finalize(se_shard_t* shard, uint32_t* d_out, int64_t ld_out, void* stream);
SE_API se_status_t se_shard_check(se_shard_t* shard, void* stream);

/* ---------------------------------------------------------------------------------------
 * Ballot tally. Replaces build_pairwise_preferences (scaling_elections.py:51-88).
 *
 *   Ballots are given in CSR form: ballot v is d_ids[d_offsets[v] .. d_offsets[v+1]), the
 *   candidate ids from most to least preferred. A ballot whose length differs from C is
 *   completed by appending the ids it lacks in ascending order (scaling_elections.py:75-83).
 *   C must be at least max(id) + 1 (the reference uses exactly max(id) + 1, :63-66).
 *   d_out receives d[i][j] = the number of (ballot, position of i, later position of j)
 *   triples (uint32, row stride ld_out), the reference's pair-by-pair count (py:46-48): for
 *   ballots that name each id once, the number of ballots ranking i above j, with diagonal 0.
 *   A ballot that repeats an id is counted the same way, so its pairs can reach the diagonal
 *   and push counts above V. Ids outside [0, C) return SE_ERR_DEVICE with a message (the
 *   reference takes C = max(id) + 1, so it never meets one).
 * ------------------------------------------------------------------------------------- */
SE_API int64_t se_tally_workspace_bytes(int64_t V, int C);
SE_API se_status_t se_tally(const int32_t* d_ids, const int64_t* d_offsets, int64_t V, int C,
                     uint32_t* d_out, int64_t ld_out, void* d_work, int64_t work_bytes,
                     void* stream);

/* se_tally without the final synchronisation: fully stream-ordered. Malformed ballots are
 * reported in the first 4 bytes of d_work (0 = fine, 2 = id out of range, 1 = lost TMA
 * completion), which the caller reads after the stream reaches that point. */
SE_API se_status_t se_tally_enqueue(const int32_t* d_ids, const int64_t* d_offsets, int64_t V, int C,
                                    uint32_t* d_out, int64_t ld_out, void* d_work,
                                    int64_t work_bytes, void* stream);

/* Tally of streamed or packed ballots, e.g. a ballot file read in chunks (no reference
 * counterpart: the reference only tallies in-memory ballots, scaling_elections.py:51-88).
 *   id_bytes   1, 2 or 4: ids are uint8, uint16 or int32 (d_ids aligned to that width).
 *   d_offsets  V + 1 offsets: ballot v is d_ids[d_offsets[v] - id_base .. d_offsets[v+1] - id_base),
 *              so a slice of a larger CSR index works with id_base = its first offset; or NULL:
 *              every ballot lists exactly C ids (ballot v starts at v * C).
 *   flags      SE_TALLY_ACCUMULATE adds this call's counts to d_out (the diagonal is left
 *              as it is), so a tally over chunks equals the tally of all ballots at once;
 *              SE_TALLY_NO_SYNC returns without synchronising, leaving the error code in the
 *              first 4 bytes of d_work as se_tally_enqueue does; SE_TALLY_KEEP_ERROR does not
 *              reset that code first, so a sequence of calls reports the first error of any.
 * Workspace: se_tally_workspace_bytes(V, C). */
#define SE_TALLY_ACCUMULATE 1u
#define SE_TALLY_NO_SYNC 2u
#define SE_TALLY_KEEP_ERROR 4u
SE_API se_status_t se_tally_ex(const void* d_ids, int id_bytes, const int64_t* d_offsets, int64_t id_base,
                               int64_t V, int C, unsigned flags, uint32_t* d_out, int64_t ld_out,
                               void* d_work, int64_t work_bytes, void* stream);

/* ---------------------------------------------------------------------------------------
 * Ranking. Replaces get_winner_and_ranking (scaling_elections.py:274-296).
 *
 *   d_wins[i]    = #{j != i : S[i][j] > S[j][i]}
 *   d_ranking[r] = candidate at place r: candidates sorted by wins, descending, ties in
 *                  ascending index order (Python's stable `sorted(..., reverse=True)`).
 *   The winner is d_ranking[0]. S is C x C uint32 with row stride ld.
 * ------------------------------------------------------------------------------------- */
SE_API se_status_t se_rank(const uint32_t* d_S, int64_t ld, int C, int32_t* d_wins,
                    int32_t* d_ranking, void* stream);

/* ---------------------------------------------------------------------------------------
 * Seeded synthetic ballots on the device (no reference counterpart; the reference draws
 * unseeded np.random.permutation ballots on the host, scaling_elections.py:477-481).
 *   d_out[v*C .. v*C+C) = ballot v, a permutation of 0..C-1 drawn from the Mallows model
 *   around d_reference (C ids; NULL = identity) with dispersion phi in (0, 1]; phi = 1 is
 *   uniform. Deterministic in (seed, v). d_work: se_mallows_workspace_bytes(V, C) bytes.
 * ------------------------------------------------------------------------------------- */
SE_API int64_t se_mallows_workspace_bytes(int64_t V, int C);
SE_API se_status_t se_mallows_ballots(int64_t V, int C, double phi, uint64_t seed,
                                      const int32_t* d_reference, int32_t* d_out, void* d_work,
                                      int64_t work_bytes, void* stream);

/* Random preference matrix on the device: the reference's benchmark input
 * np.random.randint(0, C, (C, C)) (scaling_elections.py:473-476) as a seeded, counter-based
 * draw. Cell (i, j) = (hi32(splitmix64(seed ^ splitmix64(i*C + j))) * high) >> 32, uniform in
 * [0, high) up to a bias of high / 2^32; high = 0 means C. Deterministic in (seed, i, j). */
SE_API se_status_t se_random_preferences(int C, uint32_t high, uint64_t seed, uint32_t* d_out,
                                         int64_t ld_out, void* stream);

/* ---------------------------------------------------------------------------------------
 * Integer min/max issue-rate microbenchmark (no reference counterpart): measures the
 * relaxations c = max(c, min(a, b)) per SM per clock that one instruction recipe reaches on
 * this GPU, with operands read from shared memory by a register-blocked 8 x 8 micro-kernel.
 * This is the denominator of the closure's roofline. Synchronous; allocates its own small
 * buffers (diagnostic only).
 *   recipe: 0 u32 min+max, 1 u32 min+min+max3, 2 u16x2 min+max, 3 u16x2 min+min+max3,
 *           4 f16x2 min+max, 5 f32 min+max, 6 f32 min+min+max3,
 *           7 half rows recipe 3 / half rows recipe 4, 8 half rows recipe 1 / half recipe 6
 * ------------------------------------------------------------------------------------- */
SE_API se_status_t se_minmax_peak(int recipe, int k_steps, double* relax_per_sm_clock,
                           double* sm_mhz, double* kernel_ms, double* relax_per_s);

#ifdef __cplusplus
}
#endif

#endif /* SE_H */
