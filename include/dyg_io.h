/*
 * dyg_io.h -- MatrixMarket-style edge files with the reference's conventions.
 *
 * The reference reads whitespace-separated "src dst [weight]" lines with
 * atoi/atof (random_walk_incremental/functions.cpp:58-239, 261-370;
 * random_walk_decremental/functions.cpp:69-420).  Which files are 0-based
 * and which 1-based is per file: adj_sparse.mtx is read raw (no offset),
 * ext.mtx, updated_*.mtx and del.mtx have 1 subtracted.  Weights are parsed
 * as double and rounded to float, as atof into a float does.  Lines that
 * start with '%' are skipped.  Output lines are "u v w" with the weight in
 * C++ ostream default format (%g, 6 significant digits), as
 * saveCurrentMtx writes them (random_walk_incremental/gpu_graph.cuh:427-454).
 */
#ifndef DYG_IO_H
#define DYG_IO_H
#include <stdint.h>

#include "dyg.h"
#ifdef __cplusplus
extern "C" {
#endif

/* Reads an edge file; ids have id_offset subtracted (0 = raw, 1 = 1-based).
 * *src, *dst and (if weighted) *w are malloc'ed; free them with dyg_mtx_free.
 * *max_id is the largest id after the offset (0 for an empty file). */
dyg_status dyg_mtx_read(const char *path, uint32_t id_offset, int weighted, uint64_t *n_edges,
                        uint32_t **src, uint32_t **dst, float **w, uint32_t *max_id);
void dyg_mtx_free(void *p);
/* Appends (append != 0) or writes lines "src+id_offset dst+id_offset[ w]". */
dyg_status dyg_mtx_write(const char *path, int append, uint64_t n_edges, const uint32_t *src,
                         const uint32_t *dst, const float *w, uint32_t id_offset);

/* What the mixed updater's format detection finds in a graph file
 * (auto_detect_graph_info, dynamic_update/functions.cpp:35-291). */
typedef struct dyg_mtx_info {
    int64_t skip_lines;        /* leading lines that are not records            */
    int32_t has_header;        /* leading '%' lines                             */
    int32_t has_dimensions;    /* an "n n m" line that matches the ids          */
    int32_t weighted;          /* records have a third (weight) column          */
    int32_t laplacian;         /* some weight is negative                       */
    int32_t triangular;        /* each undirected edge is listed once           */
    int32_t base;              /* smallest id: 0 or 1                           */
    uint32_t v_max, v_min;     /* largest / smallest id as written              */
} dyg_mtx_info;

/* Format detection with the reference's rules.  DYG_EIO (message in
 * dyg_last_error_string) where the reference exits: a line that is neither
 * 2 nor 3 numbers where the weight column is decided, ids neither 0- nor
 * 1-based. */
dyg_status dyg_mtx_detect(const char *path, dyg_mtx_info *info);
/* Detects, then reads the records as the mixed updater's graph loader does
 * (dynamic_update/functions.cpp:308-587): 0-based ids, weight 1 without a
 * weight column, a Laplacian's diagonal dropped and its weights negated.
 * Arrays are malloc'ed (free with dyg_mtx_free).  A triangular file lists
 * each undirected edge once (build with dyg_graph_create_from_edges); a full
 * one lists both directions (each record fills its source's row only:
 * dyg_graph_create_from_csr). */
dyg_status dyg_mtx_read_auto(const char *path, dyg_mtx_info *info, uint64_t *n_records,
                             uint32_t **src, uint32_t **dst, float **w);

/* One stream file of the mixed updater (EdgeStream::loadBatchFromFile,
 * dynamic_update/functions.cpp:717-838): its first line decides the weight
 * column (3 numbers: weighted; 2: not; a '%' line or anything else is
 * DYG_EIO); records "src dst [w]" with `base` subtracted (the dense graph's
 * base), weight 1 without the column.  Arrays are malloc'ed. */
dyg_status dyg_stream_read(const char *path, uint32_t base, uint64_t *n_records,
                           uint32_t **src, uint32_t **dst, float **w, int32_t *weighted);
/* Operation of a stream file from its name (functions.cpp:688-692): a name
 * containing "insert" or "inc" inserts, else one containing "delete" or "dec"
 * deletes, else the previous file's operation (prev_op). */
uint32_t dyg_stream_op_from_name(const char *name, uint32_t prev_op);

/* Writes a device graph as the mixed updater saves adj_dense.mtx /
 * adj_sparse.mtx (GPU_Dual_Graph::save_result,
 * dynamic_update/gpu_graph.cuh:725-763): one line "u+1 v+1 w" per undirected
 * edge, sorted by (u, v), u <= v, with the weight of u's first slot holding
 * v (the reference's order is its hash map's). */
dyg_status dyg_graph_save(dyg_graph *g, const char *path);

#ifdef __cplusplus
}
#endif
#endif
