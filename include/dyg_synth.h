/*
 * dyg_synth.h -- seeded synthetic workloads for the update path.
 *
 * The reference's datasets (G2, fe_*, del*, ...) are downloaded from a
 * private drive (datasetdownload.py) and are not available; these generators
 * produce graphs with the shapes, sizes and weight distributions of the
 * benchmark configurations instead.  Host-only; no device needed.
 * Every generator is deterministic in its seed.
 */
#ifndef DYG_SYNTH_H
#define DYG_SYNTH_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* Weight distributions. */
#define DYG_W_UNIFORM 0u     /* U[lo, hi)             */
#define DYG_W_LOGUNIFORM 1u  /* 10^U[log10 lo, log10 hi) */

/* Number of edges of an nx*ny*nz lattice with axis neighbours (nz = 1: 2-D). */
uint64_t dyg_synth_lattice_edges(uint32_t nx, uint32_t ny, uint32_t nz);
/* Lattice edges in vertex order, each vertex's +x, +y, +z edge in turn;
 * v = x + nx*(y + ny*z). */
void dyg_synth_lattice(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t wdist, float lo, float hi,
                       uint64_t seed, uint32_t *src, uint32_t *dst, float *w);

/* Maximum-weight spanning forest (Kruskal, ties by edge index) plus
 * floor(frac * #off-tree) off-tree edges chosen uniformly without
 * replacement.  Selected edge indices are written in increasing order to
 * out_idx (capacity m); returns their count. */
uint64_t dyg_synth_sparsifier(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                              const float *w, double frac, uint64_t seed, uint64_t *out_idx);

/* `count` new edges on the lattice: u uniform, hop distance d uniform in
 * [hop_lo, hop_hi], a lattice point at L1 distance d from u, rejecting pairs
 * outside the lattice, already in the edge list (src, dst, m) or already
 * drawn.  Returns the number produced (== count unless the lattice is too
 * small). */
uint64_t dyg_synth_lattice_inserts(uint32_t nx, uint32_t ny, uint32_t nz, uint64_t m,
                                   const uint32_t *src, const uint32_t *dst, uint64_t count,
                                   uint32_t hop_lo, uint32_t hop_hi, uint32_t wdist, float lo,
                                   float hi, uint64_t seed, uint32_t *out_src, uint32_t *out_dst,
                                   float *out_w);

/* R-MAT graph (Chakrabarti, Zhan, Faloutsos, SDM'04): 2^scale ids,
 * edge_factor * 2^scale generated pairs, quadrant probabilities a, b, c
 * (d = 1 - a - b - c), symmetrised (u < v), deduplicated, self-loops dropped,
 * restricted to the largest connected component and relabelled 0..n-1 in id
 * order; weights U[wlo, whi).  Edges are sorted by (u, v).  *src, *dst, *w and
 * *id_map (2^scale entries: new id or 0xFFFFFFFF) are malloc'ed (free with
 * dyg_mtx_free).  Returns the edge count; *n_out = vertex count. */
uint64_t dyg_synth_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                        float wlo, float whi, uint64_t seed, uint32_t *n_out, uint32_t **src,
                        uint32_t **dst, float **w, uint32_t **id_map);
/* `count` further R-MAT pairs in the original id space (no filtering). */
void dyg_synth_rmat_pairs(uint32_t scale, uint64_t count, double a, double b, double c,
                          uint64_t seed, uint32_t *src, uint32_t *dst);

/* Mixed update stream on an R-MAT graph from dyg_synth_rmat (id_map, and
 * its m edges src/dst): n_updates updates in files of file_size edges; file
 * f deletes iff floor((f+1)*del_frac) > floor(f*del_frac), so a fraction
 * del_frac of the files delete.  An insertion is a further R-MAT pair mapped
 * through id_map (pairs leaving the component or self-loops are redrawn; an
 * edge already present is kept: it merges its weight), weight U[wlo, whi).
 * A deletion is an edge drawn uniformly from the edges present at that point
 * (min, max order, weight 1).  Writes file_op[f] (0 insert, 1 delete) and
 * the updates in order; returns the number of files. */
uint64_t dyg_synth_rmat_stream(uint32_t scale, double a, double b, double c,
                               const uint32_t *id_map, uint64_t m, const uint32_t *src,
                               const uint32_t *dst, uint64_t n_updates, uint32_t file_size,
                               double del_frac, float wlo, float whi, uint64_t seed,
                               uint8_t *file_op, uint32_t *out_src, uint32_t *out_dst,
                               float *out_w);

/* Random geometric graph: n points uniform in the unit square, an edge
 * between two points closer than r = sqrt(avg_deg / (pi n)) (mean degree
 * avg_deg), weight 1/distance; restricted to the largest connected component,
 * relabelled in point order (*n_out vertices).  Then n_ins new edges: u
 * uniform over the component, v uniform among its points at distance in
 * [r, 3r) from u not yet adjacent to u, weight 1/distance (*n_ins_out may fall
 * short on tiny graphs).  Arrays are malloc'ed (free with dyg_mtx_free).
 * Returns the edge count. */
uint64_t dyg_synth_rgg(uint32_t n, double avg_deg, uint32_t n_ins, uint64_t seed,
                       uint32_t *n_out, uint32_t **src, uint32_t **dst, float **w,
                       uint32_t *n_ins_out, uint32_t **isrc, uint32_t **idst, float **iw);

/* k distinct indices of [0, m) in uniformly random order. */
void dyg_synth_sample(uint64_t m, uint64_t k, uint64_t seed, uint64_t *out_idx);

#ifdef __cplusplus
}
#endif
#endif
