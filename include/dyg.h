/*
 * dyg.h -- C ABI of the B200 dyGRASS update path.
 *
 * The reference has no library API: its boundary is two executables and a
 * file contract.  Each entry point below replaces one piece of what those
 * executables do between reading the .mtx files and writing the result:
 *
 *   dyg_graph_create_from_edges  <- read_graph + gpu_graph ctor + copyToDevice
 *   dyg_graph_create_from_csr       (and CSRGraph ctor + GPU_Dual_Graph ctor,
 *                                    dynamic_update/functions.cpp:308-587,
 *                                    dynamic_update/gpu_graph.cuh:283-333)
 *                                   (random_walk_incremental/functions.cpp:58-239,
 *                                    random_walk_incremental/gpu_graph.cuh:123-162, 205-275;
 *                                    random_walk_decremental/functions.cpp:69-281,
 *                                    random_walk_decremental/gpu_graph.cuh:179-268, 479-489)
 *   dyg_incremental_batch        <- one iteration of the batch loop:
 *                                   random_walk<<<>>> + get_result + updateGraphFromResult
 *                                   (random_walk_incremental/main.cu:301-328,
 *                                    random_walk_incremental/gpu_graph.cuh:292-336, 551-554)
 *   dyg_incremental_stream       <- the whole loop with the reference batching
 *                                   (random_walk_incremental/main.cu:297-340,
 *                                    random_walk_incremental/gpu_graph.cuh:135, 395-413)
 *   dyg_decremental_batch        <- removeAndUpdateDelEdges + random_walk_decremental<<<>>>
 *                                   + incrementalUpdateSparse + random_walk_small<<<>>>
 *                                   + heuristicRecovery
 *                                   (random_walk_decremental/gpu_graph.cuh:328-615,
 *                                    random_walk_decremental/main.cu:77-290, 392-408)
 *   dyg_decremental_stream       <- the decremental batch loop (random_walk_decremental/main.cu:388-444)
 *   dyg_stream_file              <- one stream_*.mtx file of the mixed updater:
 *                                   preprocessStreamEdges + the chunked
 *                                   NBRW_incremental / NBRW_decremental loop +
 *                                   updateSparsiferFromResult
 *                                   (dynamic_update/main.cu:96-126,
 *                                    dynamic_update/gpu_graph.cuh:361-465, 620-723)
 *   dyg_graph_export             <- saveCurrentMtx / save_added_edges data source
 *                                   (random_walk_incremental/gpu_graph.cuh:427-454,
 *                                    random_walk_decremental/gpu_graph.cuh:633-646)
 *   dyg_last_error_string        <- HandleError / HRR printing (random_walk_incremental/gpu_graph.cuh:38-50,
 *                                   random_walk_incremental/herror.h:1-11); errors are
 *                                   returned, never exit().
 *
 * Conventions: the caller owns every host buffer; the library owns device
 * graph state.  Array arguments may be host or device pointers (detected per
 * call); device pointers must be memory of the graph's own GPU (or managed
 * memory), else DYG_EINVAL.  Inputs are checked before anything changes:
 * an endpoint >= |V| or a weight that is not finite and > 0, in host or
 * device memory, makes the call return DYG_EINVAL with G and H unchanged.
 * With host outputs the call returns after the results are on the
 * host.  A handle is not thread-safe; distinct handles are.  Calls are
 * ordered on the given CUDA stream (NULL = legacy default stream).
 * No torch types cross this boundary.
 */
#ifndef DYG_H
#define DYG_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define DYG_ABI_VERSION 1

typedef enum dyg_status {
    DYG_OK = 0,
    DYG_EINVAL = 1,    /* bad argument (walkers not a multiple of 32, vertex id out of range, ...) */
    DYG_ENOMEM = 2,    /* device or host allocation failed                                         */
    DYG_ECUDA = 3,     /* a CUDA runtime call failed; see dyg_last_error_string()                  */
    DYG_ERANGE = 4,    /* a result did not fit the caller's buffer                                 */
    DYG_ESTATE = 5,    /* handle in an unusable state (previous device error)                      */
    DYG_ENOTSUP = 6,   /* feature not supported on this device                                     */
    DYG_EIO = 7        /* file I/O error (MTX reader/writer)                                       */
} dyg_status;

typedef struct dyg_graph dyg_graph;
/* Same object as cudaStream_t. */
typedef struct CUstream_st *dyg_stream_t;

/* Transition rules for the walk. */
#define DYG_TRANSITION_UNIFORM 0u   /* the reference's non-backtracking uniform choice */
#define DYG_TRANSITION_WEIGHTED 1u  /* opt-in: weight-proportional, not reference parity */

/* dyg_walk_params.flags bits.  By default a walker stops as soon as its 1/R
 * falls below the best success of its edge: it can then neither win nor tie,
 * so every result is unchanged and only the walker-move count drops.
 * DYG_FLAG_EXHAUSTIVE runs every walker to its natural end, as the
 * reference does. */
#define DYG_FLAG_EXHAUSTIVE 1u

typedef struct dyg_walk_params {
    float threshold;            /* distortion threshold (incremental)           */
    uint32_t walkers;           /* walkers per edge: multiple of 32, <= 1024    */
    uint32_t max_steps;         /* the reference's max_steps (default 100)      */
    uint32_t transition;        /* DYG_TRANSITION_*                             */
    uint32_t heuristic_walkers; /* decremental fallback walkers per endpoint (16) */
    uint32_t flags;             /* DYG_FLAG_* bits (0 = default)                */
    uint64_t seed;              /* Philox key                                   */
} dyg_walk_params;

typedef struct dyg_graph_opts {
    uint32_t slack_per_row;     /* free slots reserved after each row (default 2)       */
    uint32_t reserved;
    double arena_headroom;      /* extra arena capacity as a fraction of slots (0.5)    */
    int32_t device;             /* CUDA device ordinal, -1 = current device             */
    int32_t pad;
} dyg_graph_opts;

/* Decremental status codes, per deletion (otherwise: path length >= 1). */
#define DYG_DEL_NOT_IN_G (-3)  /* edge absent from G: skipped (gpu_graph.cuh:345-347)   */
#define DYG_DEL_NOT_IN_H (-2)  /* removed from G only; H unchanged, no walk             */
#define DYG_DEL_NO_PATH (-1)   /* no walker reached the other end: fallback recovery    */

/* Stream-file operations and insertion status codes (otherwise: found_at). */
#define DYG_STREAM_INSERT 0u
#define DYG_STREAM_DELETE 1u
#define DYG_INS_MERGED (-4)     /* edge already in G (or repeated in the file): weight
                                   added to G and H (dynamic_update/gpu_graph.cuh:374-382) */
#define DYG_INS_SELF_LOOP (-5)  /* u == v: ignored                                        */

/* Kinds of recovered edges. */
#define DYG_REC_PATH 0u
#define DYG_REC_FALLBACK 1u

const char *dyg_version(void);
/* Message of the last failing call on this host thread ("" if none). */
const char *dyg_last_error_string(void);
void dyg_walk_params_default(dyg_walk_params *p);
void dyg_graph_opts_default(dyg_graph_opts *o);
/* Batch size the reference uses for a stream of n updates: ceil(n / 10)
 * (random_walk_incremental/gpu_graph.cuh:135). */
uint32_t dyg_reference_batch_size(uint32_t n);

/* Build a device graph from an edge list in file order.  Rows keep the
 * reference's order: line (s, d, w) appends d to row s, then s to row d
 * (random_walk_incremental/functions.cpp:168-232).  Weights must be finite
 * and > 0.  Host pointers only. */
dyg_status dyg_graph_create_from_edges(uint32_t n_vertices, uint64_t n_edges,
                                       const uint32_t *src, const uint32_t *dst,
                                       const float *w, const dyg_graph_opts *opts,
                                       dyg_graph **out);
/* A graph from rows as given: row v holds col/w[row_ptr[v] .. row_ptr[v+1]),
 * in that order; no reverse slots are added.  This is how the mixed
 * updater's loader fills rows from a full (both-direction) matrix file, each
 * record filling its source's row only (dynamic_update/functions.cpp:525-562).
 * Weights must be finite and > 0.  Host pointers only. */
dyg_status dyg_graph_create_from_csr(uint32_t n_vertices, const uint64_t *row_ptr,
                                     const uint32_t *col, const float *w,
                                     const dyg_graph_opts *opts, dyg_graph **out);
/* Deep copy on the same device (used to restore a snapshot). */
dyg_status dyg_graph_clone(const dyg_graph *g, dyg_graph **out);
/* Overwrite dst's rows with src's (same vertex count); stream-ordered. */
dyg_status dyg_graph_copy_from(dyg_graph *dst, const dyg_graph *src, dyg_stream_t stream);
dyg_status dyg_graph_destroy(dyg_graph *g);
/* Vertex count, live directed slots, arena slots used / allocated. */
dyg_status dyg_graph_info(const dyg_graph *g, uint32_t *n_vertices, uint64_t *n_slots,
                          uint64_t *arena_used, uint64_t *arena_cap);
/* Copy the rows to host CSR arrays: row_ptr[n+1], col/w[slot_cap]. */
dyg_status dyg_graph_export(dyg_graph *g, uint64_t *row_ptr, uint32_t *col, float *w,
                            uint64_t slot_cap);
/* Repack rows into a fresh arena with the configured slack (stream-ordered). */
dyg_status dyg_graph_compact(dyg_graph *g, dyg_stream_t stream);
/* Walker moves (neighbour draws) executed on this handle since creation. */
dyg_status dyg_graph_counters(const dyg_graph *g, uint64_t *walker_moves, uint64_t *walks);

/* One incremental batch on the snapshot H: every edge is tested by
 * p->walkers walks on the same H, then edges that no walker connected are
 * appended to H in input order.  If G is not NULL every edge of the batch is
 * appended to G too (G = dense graph after insertions).  Update ids
 * first_update_id + e key the random streams.  Outputs (any may be NULL):
 * found_at[e] = winner's step count or -1, conductance[e] = winner's 1/R,
 * accepted[e] = 1 iff the edge was added to H. */
dyg_status dyg_incremental_batch(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                 const uint32_t *dst, const float *w, uint32_t n,
                                 uint64_t first_update_id, const dyg_walk_params *p,
                                 int32_t *found_at, float *conductance, uint8_t *accepted,
                                 dyg_stream_t stream);
/* The whole insertion stream in batches of batch_size (0 = the reference's
 * ceil(n/10)); update ids are stream positions. */
dyg_status dyg_incremental_stream(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                  const uint32_t *dst, const float *w, uint32_t n,
                                  uint32_t batch_size, const dyg_walk_params *p,
                                  int32_t *found_at, float *conductance, uint8_t *accepted,
                                  dyg_stream_t stream);

/* One decremental batch: delete each edge from G (swap with the row's last
 * slot, in input order), erase the ones also in H, walk G from min(u,v) to
 * max(u,v), append the winning path's edges absent from H to H (in order),
 * and run the 2-step fallback walks for edges without a path.
 * status[e] = path length or DYG_DEL_*; conductance[e] = winner's 1/R.
 * Recovered edges (x, y, kind) go to rec_src/rec_dst/rec_kind in commit
 * order, at most rec_cap of them; *n_rec gets the total (DYG_ERANGE if it
 * exceeds rec_cap; the graph update itself is complete). */
dyg_status dyg_decremental_batch(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                 const uint32_t *dst, uint32_t n, uint64_t first_update_id,
                                 const dyg_walk_params *p, int32_t *status, float *conductance,
                                 uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind,
                                 uint64_t rec_cap, uint64_t *n_rec, dyg_stream_t stream);
dyg_status dyg_decremental_stream(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                  const uint32_t *dst, uint32_t n, uint32_t batch_size,
                                  const dyg_walk_params *p, int32_t *status, float *conductance,
                                  uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind,
                                  uint64_t rec_cap, uint64_t *n_rec, dyg_stream_t stream);

/* Recovered edges [first, first + count) of the last decremental call on G
 * (dyg_decremental_batch / _stream / _batch_ids, dyg_stream_file with
 * DYG_STREAM_DELETE, dyg_decremental_commit_keys); they stay readable until
 * the next such call on G.  Lets a caller pass rec_cap = 0 (no record
 * buffers), learn the total from *n_rec, and then read exactly that many
 * instead of sizing buffers for the worst case up front.  Host or device
 * outputs; blocking.  DYG_ERANGE if the range is not inside the last call's
 * records.  The reference writes these edges to added_edges.mtx
 * (random_walk_decremental/gpu_graph.cuh:633-646). */
dyg_status dyg_recovered_read(const dyg_graph *G, uint64_t first, uint64_t count,
                              uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind);

/* dyg_incremental_batch / dyg_decremental_batch with an explicit update id
 * per edge (update_ids[e] in place of first_update_id + e; host or device
 * array).  With a union of independent graphs (each graph's vertices at its
 * own offset), one call tests the current batch of every graph in a single
 * launch and gives each graph exactly what its own call with those ids would
 * (walks never leave a graph; rows are updated in list order per row).
 * Extends the batch entry points (random_walk_incremental/main.cu:301-328,
 * random_walk_decremental/main.cu:392-408) to many graphs at once. */
dyg_status dyg_incremental_batch_ids(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                     const uint32_t *dst, const float *w,
                                     const uint64_t *update_ids, uint32_t n,
                                     const dyg_walk_params *p, int32_t *found_at,
                                     float *conductance, uint8_t *accepted, dyg_stream_t stream);
dyg_status dyg_decremental_batch_ids(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                     const uint32_t *dst, const uint64_t *update_ids, uint32_t n,
                                     const dyg_walk_params *p, int32_t *status,
                                     float *conductance, uint32_t *rec_src, uint32_t *rec_dst,
                                     uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec,
                                     dyg_stream_t stream);
/* A batch sharded over processes holding replicas of G and H (one per GPU):
 * each rank computes the winner keys of a contiguous range of the batch, the
 * ranks combine their key arrays (element-wise max; entries outside a rank's
 * range are left as they were, so arrays that start at zero combine
 * exactly), and every rank commits the whole batch.  Together they give what
 * dyg_incremental_batch / dyg_decremental_batch give for the same ids.  Keys
 * are device arrays of n (incremental) or n_walk (decremental) u64.
 * Incremental: dyg_walk_keys on H (incremental = 1) for [lo, hi), then
 * dyg_incremental_commit_keys (outputs device arrays).  Decremental:
 * dyg_decremental_delete (status / conductance device arrays, kept for the
 * commit; *n_walk = edges to walk), dyg_decremental_walk_keys for [lo, hi) of
 * that walk list, then dyg_decremental_commit_keys with the same status /
 * conductance arrays; no other call on G may come in between.  Splits
 * random_walk_incremental/main.cu:301-328 and random_walk_decremental/main.cu:
 * 392-408 at the point where the reference reads the kernel's results back. */
dyg_status dyg_walk_keys(dyg_graph *X, const uint32_t *src, const uint32_t *dst, const float *w,
                         const uint64_t *update_ids, uint64_t first_update_id, uint32_t n,
                         uint32_t lo, uint32_t hi, uint32_t incremental,
                         const dyg_walk_params *p, uint64_t *keys, dyg_stream_t stream);
dyg_status dyg_incremental_commit_keys(dyg_graph *H, dyg_graph *G, const uint32_t *src,
                                       const uint32_t *dst, const float *w, uint32_t n,
                                       const uint64_t *keys, int32_t *found_at,
                                       float *conductance, uint8_t *accepted,
                                       dyg_stream_t stream);
dyg_status dyg_decremental_delete(dyg_graph *G, dyg_graph *H, const uint32_t *src,
                                  const uint32_t *dst, const uint64_t *update_ids,
                                  uint64_t first_update_id, uint32_t n, int32_t *status,
                                  float *conductance, uint32_t *n_walk, dyg_stream_t stream);
dyg_status dyg_decremental_walk_keys(dyg_graph *G, uint32_t lo, uint32_t hi,
                                     const dyg_walk_params *p, uint64_t *keys,
                                     dyg_stream_t stream);
dyg_status dyg_decremental_commit_keys(dyg_graph *G, dyg_graph *H, const dyg_walk_params *p,
                                       const uint64_t *keys, uint32_t n_walk, int32_t *status,
                                       float *conductance, uint32_t *rec_src, uint32_t *rec_dst,
                                       uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec,
                                       dyg_stream_t stream);

/* Launch shape of the walk kernel for this process (an autotuner's knobs;
 * results do not depend on them): walkers each warp takes per fetch (a
 * multiple of 32 dividing the walker count; 0 = 32) and resident blocks per
 * SM (0 or more than fit = as many as fit).  Replaces the reference's fixed
 * one-block-per-edge launch (random_walk_incremental/main.cu:316). */
void dyg_tune_set(uint32_t walk_chunk, uint32_t blocks_per_sm);

/* Walk iterations (of four moves) between a walker's reads of its edge's best
 * result, against which it is pruned: 1 (the default; 0 = 1), 2 or 4.  A
 * bound read less often is only lower, so results do not depend on it; an
 * autotuner's knob like the two above. */
void dyg_tune_set_prune_interval(uint32_t iterations);

/* Walk-list chunk of the mixed updater: 5% of |V|, at least 10000
 * (dynamic_update/main.cu:83-84). */
uint32_t dyg_stream_default_chunk(uint32_t n_vertices);
/* One file of the mixed insert/delete stream (dynamic_update).
 * op DYG_STREAM_INSERT, in file order: an edge already in G (or repeated
 * earlier in the file) adds its weight to G and, if there, to H
 * (status DYG_INS_MERGED); a new edge enters G at once.  The new edges are
 * then walked on H from src to dst in chunks of `chunk` (0 =
 * dyg_stream_default_chunk(|V|)); after each chunk its accepted edges
 * (status -1) enter H with their stream weight; otherwise status = found_at.
 * op DYG_STREAM_DELETE: the whole file is deleted from G and H first (status
 * DYG_DEL_*), then the edges that were in H are walked on G from src to dst in
 * chunks, recovering as dyg_decremental_batch does; w may be NULL.
 * Update ids are first_update_id + file position.  Recovered edges (delete
 * files) as in dyg_decremental_batch; *n_rec = 0 for insert files. */
dyg_status dyg_stream_file(dyg_graph *G, dyg_graph *H, uint32_t op, const uint32_t *src,
                           const uint32_t *dst, const float *w, uint32_t n,
                           uint64_t first_update_id, uint32_t chunk, const dyg_walk_params *p,
                           int32_t *status, float *conductance, uint32_t *rec_src,
                           uint32_t *rec_dst, uint8_t *rec_kind, uint64_t rec_cap,
                           uint64_t *n_rec, dyg_stream_t stream);

/* No counterpart in the reference.  Incremental walk decision for one batch
 * (found_at / conductance / accepted exactly as dyg_incremental_batch reports
 * them for the same H and update ids) without any device allocation, for
 * callers that cannot call cudaMalloc: a serving loop that reserves its device
 * memory at start-up and allows no allocation afterwards, or a plugin inside a
 * host framework that owns all device allocations.  Accepted edges are NOT
 * appended to H.  All array arguments must be device pointers on H's device
 * (memory of another GPU is rejected with DYG_EINVAL); found_at is -2
 * for an edge whose endpoint is not a vertex of H.  Scratch lives in a static
 * device array of DYG_NOALLOC_MAX_EDGES 64-bit keys (512 KiB) plus counters,
 * held by every device that loads the library until exit; batches larger than
 * DYG_NOALLOC_MAX_EDGES are rejected with DYG_EINVAL.  Calls share that array:
 * calls that overlap on the GPU race and must be serialized by the caller.
 * The first call on a device looks up the array's address (set-up), and so
 * does the first call after the device's context is replaced (for example by
 * cudaDeviceReset, which frees the array with the context); make those calls
 * before any stream capture.  Stream-ordered; returns before the results are
 * ready. */
#define DYG_NOALLOC_MAX_EDGES 65536u
dyg_status dyg_incremental_walk_noalloc(const dyg_graph *H, const uint32_t *src,
                                        const uint32_t *dst, const float *w, uint32_t n,
                                        uint64_t first_update_id, const dyg_walk_params *p,
                                        int32_t *found_at, float *conductance,
                                        uint8_t *accepted, dyg_stream_t stream);

/* Kernel timing for benchmarks: while enabled, CUDA events are recorded on
 * the launching stream around every walk-kernel launch of this process.
 * dyg_profile_read synchronizes those events and returns the totals since
 * the last reset (milliseconds, launches, walker moves are not split). */
typedef struct dyg_profile {
    double incr_walk_ms;
    double decr_walk_ms;
    double other_walk_ms;      /* winner replays and fallback walks */
    uint64_t incr_walk_launches;
    uint64_t decr_walk_launches;
    uint64_t other_walk_launches;
} dyg_profile;
dyg_status dyg_profile_enable(int on);
dyg_status dyg_profile_reset(void);
dyg_status dyg_profile_read(dyg_profile *out);
/* Number of this library's own kernel launches so far in this process. */
uint64_t dyg_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif
