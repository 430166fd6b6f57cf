/* dyg_serve.h -- continuous-batching server over many resident graphs.
 *
 * The reference updates one graph per process run (random_walk_incremental/
 * main.cu:240-362, random_walk_decremental/main.cu:318-468): it has no
 * request loop.  This server keeps many graphs resident as one union graph
 * (every graph at its own vertex offset, created by the caller with
 * dyg_graph_create_*), queues update requests per graph, and runs them in
 * scheduler steps: each step takes the oldest pending request of every graph
 * that has one, runs all insertion requests of the step as one incremental
 * batch and then all deletion requests as one decremental batch
 * (dyg_incremental_batch_ids / dyg_decremental_batch_ids semantics), and
 * completes them.  A graph's requests run in arrival order, one per step, and
 * its update ids count its own updates only (the first update of a graph is
 * id 0), so every request gets exactly the result it gets when run alone on
 * that graph's own handles with dyg_incremental_batch / dyg_decremental_batch
 * and first_update_id = the count of the graph's earlier updates.
 *
 * Requests are copied at submission; results stay in the server until
 * fetched.  Steps run either in the caller's thread (dyg_server_step) or in
 * the server's own loop thread (dyg_server_start), which runs a step whenever
 * a request is pending: requests submitted while a step runs join the next.
 * While a server exists its graphs must not be used by other calls, except
 * when it is idle (nothing pending, no step running, see dyg_server_drain).
 */
#ifndef DYG_SERVE_H
#define DYG_SERVE_H

#include "dyg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct dyg_server dyg_server;

/* One completed request, as reported by dyg_server_poll. */
typedef struct dyg_server_done {
    uint64_t tag;              /* the caller's id given at submission            */
    uint32_t graph;            /* graph index                                    */
    uint32_t op;               /* DYG_STREAM_INSERT or DYG_STREAM_DELETE         */
    uint32_t n;                /* updates in the request                         */
    int32_t status;            /* DYG_OK, or the status of the step that ran it  */
    uint64_t first_update_id;  /* id of its first update within its graph        */
    uint64_t n_rec;            /* recovered edges (deletion requests)            */
    uint64_t step;             /* index of the scheduler step that ran it        */
    uint64_t t_submit_ns;      /* server clock (dyg_server_now_ns)               */
    uint64_t t_start_ns;
    uint64_t t_done_ns;
} dyg_server_done;

/* G and H hold n_graphs graphs; graph k owns vertices
 * [vertex_offsets[k], vertex_offsets[k+1]) of both (offsets ascending,
 * vertex_offsets[n_graphs] <= the vertex count).  Request vertex ids are local
 * to their graph.  stream: the CUDA stream of the server's work (NULL = the
 * default stream). */
dyg_status dyg_server_create(dyg_graph *G, dyg_graph *H, uint32_t n_graphs,
                             const uint32_t *vertex_offsets,
                             const dyg_walk_params *insert_params,
                             const dyg_walk_params *delete_params, dyg_stream_t stream,
                             dyg_server **out);

/* Stops the loop thread (after its current step) and frees the server; the
 * graphs stay the caller's and must outlive the server (destroy it first). */
dyg_status dyg_server_destroy(dyg_server *s);

/* Queues a request: op DYG_STREAM_INSERT (w required, finite and > 0) or
 * DYG_STREAM_DELETE (w ignored); n may be 0.  Host arrays, copied.  tag must
 * not be held by an unfetched request.  DYG_EINVAL for a bad graph, op, tag,
 * vertex id or weight, DYG_ENOMEM if the copy cannot be allocated (nothing is
 * queued then). */
dyg_status dyg_server_submit(dyg_server *s, uint64_t tag, uint32_t graph, uint32_t op,
                             const uint32_t *src, const uint32_t *dst, const float *w,
                             uint32_t n);

/* Queues n_req requests at once, in order: request j has tags[j], graphs[j],
 * ops[j] and the updates [offsets[j], offsets[j+1]) of src, dst and w (w is
 * read for insertions only and may be NULL when there are none).  Every
 * request is checked first: on DYG_EINVAL nothing is queued. */
dyg_status dyg_server_submit_many(dyg_server *s, uint32_t n_req, const uint64_t *tags,
                                  const uint32_t *graphs, const uint32_t *ops,
                                  const uint64_t *offsets, const uint32_t *src,
                                  const uint32_t *dst, const float *w);

/* Runs one scheduler step in the calling thread; *n_done (may be NULL) gets
 * the number of requests it completed (0 when nothing is pending).
 * DYG_EINVAL while the loop thread runs.  A failed step completes its
 * requests with its status and returns it. */
dyg_status dyg_server_step(dyg_server *s, uint32_t *n_done);

/* Starts / stops the loop thread.  stop returns after the current step. */
dyg_status dyg_server_start(dyg_server *s);
dyg_status dyg_server_stop(dyg_server *s);

/* Waits until no request is pending and no step runs (timeout_s < 0: no
 * limit); DYG_ESTATE on timeout.  With the loop stopped and requests pending
 * it returns DYG_ESTATE at once. */
dyg_status dyg_server_drain(dyg_server *s, double timeout_s);

/* Requests queued and not yet run. */
uint32_t dyg_server_pending(dyg_server *s);

/* Moves up to cap completion records (oldest first) into out. */
dyg_status dyg_server_poll(dyg_server *s, dyg_server_done *out, uint32_t cap, uint32_t *n);

/* Copies the result of a completed request and releases it.  Insertion:
 * found_or_status[i] = found_at, conductance, accepted (as
 * dyg_incremental_batch).  Deletion: found_or_status = status, conductance,
 * and the recovered edges in commit order with local vertex ids (as
 * dyg_decremental_batch), at most rec_cap of them: DYG_ERANGE if there are
 * more (the result is kept then).  Any pointer may be NULL.  DYG_EINVAL for
 * an unknown or unfinished tag. */
dyg_status dyg_server_fetch(dyg_server *s, uint64_t tag, int32_t *found_or_status,
                            float *conductance, uint8_t *accepted, uint32_t *rec_src,
                            uint32_t *rec_dst, uint8_t *rec_kind, uint64_t rec_cap);

/* Back to update id 0 for every graph, with no results or completion records
 * kept (for a caller that restores the graphs to an earlier state).
 * DYG_ESTATE unless idle. */
dyg_status dyg_server_reset(dyg_server *s);

/* Steps run so far (since creation or reset). */
uint64_t dyg_server_steps(const dyg_server *s);

/* The server clock: nanoseconds since its creation (steady). */
uint64_t dyg_server_now_ns(const dyg_server *s);

/* Message of the last failed step or call on this server ("" if none). */
const char *dyg_server_last_error(dyg_server *s);

#ifdef __cplusplus
}
#endif

#endif /* DYG_SERVE_H */
