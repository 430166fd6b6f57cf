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

/* Pool mode: the server owns its union graphs (vertex_capacity vertices) and
 * admits registered graphs by footprint.  hbm_budget_bytes bounds the sum of
 * the resident graphs' estimated footprints (per slot 12 B with the arena's
 * 50 % headroom and 2 slack slots per row, plus 24 B per vertex, for G and H).
 * A registered graph stays in host memory until a request for it is
 * scheduled; at the start of each step, graphs with pending requests that are
 * not resident are admitted, oldest pending request first, into a free vertex
 * range while their footprint fits the budget; to make room, resident graphs
 * are evicted (their rows copied back to host memory, row order kept): idle
 * ones least recently used first; busy ones (requests pending), whose oldest
 * pending request is younger than the waiting graph's, only after the waiting
 * graph's oldest request has waited 32 steps, so that an oversubscribed
 * server rotates graphs as their queues drain.  Every request still gets the result it
 * gets alone on its graph's own handles.  device < 0: the current device.
 * keep_initial: keep a host copy of each graph as registered, so that
 * dyg_server_reset can restore it.  The reference keeps one graph per process
 * and has no counterpart. */
dyg_status dyg_server_create_pool(uint32_t vertex_capacity, uint64_t hbm_budget_bytes,
                                  const dyg_walk_params *insert_params,
                                  const dyg_walk_params *delete_params, int device,
                                  uint32_t keep_initial, dyg_stream_t stream, dyg_server **out);

/* Registers a graph with a pool server: its dense graph G and sparsifier H as
 * edge lists with local ids (rows are built as dyg_graph_create_from_edges
 * builds them), copied to host memory; *graph gets its index.  Not resident
 * until a request for it is scheduled (or dyg_server_prefetch).  DYG_ENOMEM
 * if its footprint alone exceeds the budget; DYG_EINVAL for bad ids or
 * weights, or more vertices than the pool holds. */
dyg_status dyg_server_add_graph(dyg_server *s, uint32_t n_vertices, uint64_t g_edges,
                                const uint32_t *g_src, const uint32_t *g_dst, const float *g_w,
                                uint64_t h_edges, const uint32_t *h_src, const uint32_t *h_dst,
                                const float *h_w, uint32_t *graph);

/* Admits a pool graph now if it fits (evicting idle graphs least recently
 * used first); *resident (may be NULL) tells whether it is resident.  Needs an
 * idle server (DYG_ESTATE otherwise). */
dyg_status dyg_server_prefetch(dyg_server *s, uint32_t graph, uint32_t *resident);

typedef struct dyg_server_stats {
    uint32_t graphs;           /* given (static) or registered (pool)           */
    uint32_t resident;         /* graphs on the device                          */
    uint32_t waiting;          /* graphs with pending requests, not resident    */
    uint32_t pending;          /* requests queued and not yet run               */
    uint64_t resident_bytes;   /* estimated footprint of the resident graphs    */
    uint64_t budget_bytes;     /* 0 for a static server                         */
    uint64_t admissions, evictions;
    uint64_t steps;
    /* host wall time of the steps so far, by phase (ns; reset by
     * dyg_server_reset): admitting graphs, staging the requests, the
     * insertion run and the deletion run (each with its device work and
     * synchronize), fetching the results, splitting them per request     */
    uint64_t ns_admit, ns_stage, ns_insert, ns_delete, ns_fetch, ns_split;
} dyg_server_stats;
dyg_status dyg_server_stats_read(dyg_server *s, dyg_server_stats *out);

typedef struct dyg_server_graph_info {
    uint32_t n_vertices;
    uint32_t resident;
    uint32_t vertex_offset;    /* first vertex in the union while resident      */
    uint32_t pad;
    uint64_t footprint_bytes;  /* pool: estimate used for admission             */
    uint64_t updates;          /* updates run so far (its next update id)       */
    uint64_t admissions, evictions;
    uint64_t pending;          /* its queued requests                           */
} dyg_server_graph_info;
dyg_status dyg_server_graph_info_read(dyg_server *s, uint32_t graph, dyg_server_graph_info *out);

/* The current rows of a graph's G (which = 0) or H (which = 1) with local
 * ids: row_ptr[n_vertices + 1], col / w up to slot_cap slots (DYG_ERANGE if
 * there are more; row_ptr is complete then).  From the device while resident,
 * else from the host copy.  Needs an idle server (DYG_ESTATE otherwise). */
dyg_status dyg_server_graph_export(dyg_server *s, uint32_t graph, uint32_t which,
                                   uint64_t *row_ptr, uint32_t *col, float *w, uint64_t slot_cap);

/* Walker moves so far on the sparsifier (insertion walks) and on the dense
 * graph (deletion walks) of the server's union graphs.  Needs an idle server. */
dyg_status dyg_server_counters(dyg_server *s, uint64_t *incr_moves, uint64_t *decr_moves);

/* Stops the loop thread (after its current step) and frees the server; the
 * graphs of a static server stay the caller's and must outlive the server
 * (destroy it first); a pool server frees its own. */
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

/* Runs one scheduler step in the calling thread (pool: admissions first);
 * *n_done (may be NULL) gets the number of requests it completed (0 when
 * nothing is pending; requests of a graph that cannot be admitted, because
 * it outgrew the budget, complete with DYG_ENOMEM).
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
 * kept (for a caller that restores the graphs to an earlier state; a pool
 * server created with keep_initial restores every graph to its registered
 * rows itself, none resident).  DYG_ESTATE unless idle. */
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
