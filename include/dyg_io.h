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

#ifdef __cplusplus
}
#endif
#endif
