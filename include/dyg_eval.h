/*
 * dyg_eval.h -- spectral quality of a sparsifier, host only.
 *
 * Replaces the reference's Julia evaluation of an updated sparsifier
 * (dyGRASS.jl:54-64 create_laplacian, 164-166 check_density, 361-362 the
 * condition number by eigs on the pencil, 558-588 pcg_test):
 *   kappa      largest eigenvalue of the pencil (L_G + offset I, L_H + offset I),
 *              offset 1e-6 as the reference adds; FP64 Lanczos in the L_H
 *              inner product with solves by a sparse LDL^T of L_H
 *   density    |E_H| / |V|
 *   pcg_iters  conjugate-gradient iterations on L_G x = b (b random, zero
 *              mean; x0 random) preconditioned by the L_H factorization, until
 *              ||r|| <= pcg_rtol * ||r_0||
 * Edge lists give each undirected edge once (either orientation); self-loops
 * are ignored; repeated edges add up.  The random vectors come from `seed`.
 */
#ifndef DYG_EVAL_H
#define DYG_EVAL_H
#include <stdint.h>

#include "dyg.h"
#ifdef __cplusplus
extern "C" {
#endif

typedef struct dyg_kappa_opts {
    double offset;          /* added to every diagonal entry (1e-6)             */
    double tol;             /* Lanczos: relative change of the estimate (1e-10) */
    uint32_t max_iter;      /* Lanczos steps (300)                              */
    uint32_t pcg_max_iter;  /* (10000)                                          */
    double pcg_rtol;        /* (1e-8)                                           */
    uint64_t seed;
} dyg_kappa_opts;

typedef struct dyg_kappa_result {
    double kappa;
    double density;
    uint32_t lanczos_iters;
    uint32_t pcg_iters;
    double pcg_relres;
    uint64_t factor_nnz;    /* off-diagonal entries of the L_H factor          */
} dyg_kappa_result;

void dyg_kappa_opts_default(dyg_kappa_opts *o);
/* DYG_EINVAL for an id >= n or a weight that is not > 0; DYG_ERANGE if
 * L_H + offset I is not positive definite. */
dyg_status dyg_kappa(uint32_t n, uint64_t m_g, const uint32_t *g_src, const uint32_t *g_dst,
                     const float *g_w, uint64_t m_h, const uint32_t *h_src, const uint32_t *h_dst,
                     const float *h_w, const dyg_kappa_opts *opts, dyg_kappa_result *out);

#ifdef __cplusplus
}
#endif
#endif
