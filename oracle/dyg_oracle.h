/*
 * dyg_oracle.h -- CPU oracle for the dyGRASS update path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference's incremental walk (random_walk_incremental/main.cu:70-211),
 * its host commit (random_walk_incremental/gpu_graph.cuh:292-336), its
 * decremental walk / recovery (random_walk_decremental/main.cu:77-290,
 * random_walk_decremental/gpu_graph.cuh:328-615), with the reference's
 * cuRAND draws replaced by the counter-based Philox4x32-10 stream that the
 * CUDA path also uses.  Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py may load it, and only as the checker or the
 * timed host baseline; the product never calls it.
 *
 * Parity pins: the Philox stream is pinned by the published Random123
 * known-answer vectors; walk/commit semantics by known-answer graphs whose
 * outcome does not depend on the random stream (tests/golden).
 */
#ifndef DYG_ORACLE_H
#define DYG_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_graph orc_graph;

typedef struct orc_params {
    float threshold;      /* distortion threshold (incremental only)          */
    uint32_t walkers;     /* walkers per edge                                 */
    uint32_t max_steps;   /* the reference's max_steps: walk ends when the
                             step counter reaches it (main.cu:44, 116)        */
    uint32_t transition;  /* 0 = uniform non-backtracking (reference),
                             1 = weight-proportional (opt-in, not reference)  */
    uint32_t heuristic_walkers; /* decremental fallback walkers per endpoint */
    uint32_t pad;
    uint64_t seed;
} orc_params;

/* Philox4x32-10 block: out[4] = philox(ctr[4], key[2]). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* The d-th 32-bit draw of walker `walker` of update `uid` in `domain`. */
uint32_t orc_draw(uint64_t seed, uint64_t uid, uint32_t domain, uint32_t walker, uint32_t d);

/* Graph built in the reference's row order: for each input line (s, d, w)
 * row s gets d appended, then row d gets s (functions.cpp:168-232). */
orc_graph *orc_graph_from_edges(uint32_t n, uint64_t m, const uint32_t *src,
                                const uint32_t *dst, const float *w);
void orc_graph_free(orc_graph *g);
/* A deep copy (rows in the same order). */
orc_graph *orc_graph_clone(const orc_graph *g);
uint32_t orc_graph_num_vertices(const orc_graph *g);
uint64_t orc_graph_num_slots(const orc_graph *g);
/* row_ptr[n+1], col[slots], w[slots]; any of the outputs may be NULL. */
uint64_t orc_graph_export(const orc_graph *g, uint64_t *row_ptr, uint32_t *col, float *w);
int orc_graph_has_edge(const orc_graph *g, uint32_t a, uint32_t b);

/* One incremental batch against the current snapshot of H.  Every edge is
 * walked on the same H; then accepted edges (no walker succeeded) are
 * appended to H in input order.  If G is non-NULL every edge of the batch is
 * appended to G as well (G = dense graph after insertions).
 * found_at[e] = winner's step count or -1; cond[e] = winner's 1/R (0 if none);
 * accepted[e] = 1 iff the edge was added to H.  Returns total walker moves. */
uint64_t orc_incremental_batch(orc_graph *H, orc_graph *G, const uint32_t *src,
                               const uint32_t *dst, const float *w, uint32_t n,
                               uint64_t first_uid, const orc_params *p, int threads,
                               int32_t *found_at, float *cond, uint8_t *accepted);

/* The reference batching: batches of ceil(n/10) (gpu_graph.cuh:135) unless
 * batch_size != 0.  Update ids are stream positions. */
uint64_t orc_incremental_stream(orc_graph *H, orc_graph *G, const uint32_t *src,
                                const uint32_t *dst, const float *w, uint32_t n,
                                uint32_t batch_size, const orc_params *p, int threads,
                                int32_t *found_at, float *cond, uint8_t *accepted);

/* Deletion status codes (per input deletion). */
#define ORC_DEL_NOT_IN_G  (-3)
#define ORC_DEL_NOT_IN_H  (-2)
#define ORC_DEL_NO_PATH   (-1)

/* One decremental batch: delete every edge from G (swap-with-last), erase the
 * ones also in H, walk G from min(u,v) to max(u,v) for those, add the
 * winner's path edges not in H to H (in order), and run the 2-step fallback
 * walks for edges without a path.  status[e] = path length or one of the
 * codes above; cond[e] = winner's 1/R.  Recovered edges are written to
 * rec_src/rec_dst/rec_kind (0 = path, 1 = fallback) up to rec_cap entries;
 * *n_rec gets the full count.  Returns total walker moves. */
uint64_t orc_decremental_batch(orc_graph *G, orc_graph *H, const uint32_t *src,
                               const uint32_t *dst, uint32_t n, uint64_t first_uid,
                               const orc_params *p, int threads, int32_t *status,
                               float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                               uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec);

uint64_t orc_decremental_stream(orc_graph *G, orc_graph *H, const uint32_t *src,
                                const uint32_t *dst, uint32_t n, uint32_t batch_size,
                                const orc_params *p, int threads, int32_t *status,
                                float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                                uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec);

/* One file of the mixed insert/delete stream
 * (dynamic_update/main.cu:96-126, gpu_graph.cuh:361-465, 620-723).
 * op ORC_STREAM_INSERT: in file order, an edge already in G adds its weight
 * to G (and to H if H has it) and gets status ORC_STREAM_MERGED; a new edge
 * enters G at once and is then walked on H from src to dst, in chunks of
 * `chunk` walked edges (0 = orc_stream_default_chunk(|V|)); a chunk's
 * accepted edges (status -1) enter H with their stream weight before the
 * next chunk walks; found_at >= 0 otherwise.  A self-loop is ignored
 * (ORC_STREAM_SELF_LOOP).
 * op ORC_STREAM_DELETE: the whole file is deleted from G and H first, then
 * the edges that were in H are walked on G from src to dst in chunks, with
 * the status / conductance / recovered-edge outputs of the batch functions. */
#define ORC_STREAM_INSERT 0u
#define ORC_STREAM_DELETE 1u
#define ORC_STREAM_MERGED (-4)
#define ORC_STREAM_SELF_LOOP (-5)
uint32_t orc_stream_default_chunk(uint32_t n_vertices);
uint64_t orc_stream_file(orc_graph *G, orc_graph *H, uint32_t op, const uint32_t *src,
                         const uint32_t *dst, const float *w, uint32_t n, uint64_t first_uid,
                         uint32_t chunk, const orc_params *p, int threads, int32_t *status,
                         float *cond, uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind,
                         uint64_t rec_cap, uint64_t *n_rec);

/* The batch functions in two halves, for a batch sharded over processes:
 * winner keys of edges [lo, hi) (incr: walks on H with the distortion test,
 * else on the graph given, endpoints as given), then the commit from a full
 * key array.  Decremental: the deletion stage lists the edges to walk
 * (returns their count), keys for [lo, hi) of that list (min -> max), then
 * the commit (winner paths, recovery, fallback) from the full key array. */
void orc_walk_keys(const orc_graph *g, const uint32_t *src, const uint32_t *dst, const float *w,
                   uint64_t first_uid, uint32_t lo, uint32_t hi, int incr, const orc_params *p,
                   int threads, uint64_t *keys, uint64_t *moves);
/* orc_decremental_batch with each deletion's update id read from uids[e]
 * (a union of graphs served together, as the server does). */
uint64_t orc_decremental_batch_ids(orc_graph *G, orc_graph *H, const uint32_t *src,
                                   const uint32_t *dst, const uint64_t *uids, uint32_t n,
                                   const orc_params *p, int threads, int32_t *status,
                                   float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                                   uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec);
/* orc_walk_keys with each edge's update id read from uids[e] (the batched
 * many-graph mode: a union of graphs at vertex offsets, every edge carrying
 * its position in its own graph's stream), incremental walks on g. */
void orc_walk_keys_ids(const orc_graph *g, const uint32_t *src, const uint32_t *dst,
                       const float *w, const uint64_t *uids, uint32_t n, const orc_params *p,
                       int threads, uint64_t *keys, uint64_t *moves);
void orc_incremental_commit_keys(orc_graph *H, orc_graph *G, const uint32_t *src,
                                 const uint32_t *dst, const float *w, uint32_t n,
                                 const uint64_t *keys, int32_t *found_at, float *cond,
                                 uint8_t *accepted);
uint32_t orc_decremental_delete(orc_graph *G, orc_graph *H, const uint32_t *src,
                                const uint32_t *dst, uint32_t n, int32_t *status, float *cond,
                                uint32_t *walk_list);
void orc_decremental_walk_list_keys(const orc_graph *G, const uint32_t *src, const uint32_t *dst,
                                    const uint32_t *walk_list, uint32_t lo, uint32_t hi,
                                    uint64_t first_uid, const orc_params *p, int threads,
                                    uint64_t *keys);
void orc_decremental_commit_keys(orc_graph *G, orc_graph *H, const uint32_t *src,
                                 const uint32_t *dst, const uint32_t *walk_list, uint32_t nf,
                                 uint64_t first_uid, const orc_params *p, const uint64_t *keys,
                                 int32_t *status, float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                                 uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec);

/* Path of one walker of a decremental walk (for tests): returns found_at or
 * -1 and writes up to max_steps+1 vertices into path. */
int32_t orc_decremental_walk_path(const orc_graph *G, uint32_t s, uint32_t t,
                                  uint64_t uid, uint32_t walker, const orc_params *p,
                                  uint32_t *path, float *R);

int orc_max_threads(void);

#ifdef __cplusplus
}
#endif
#endif
