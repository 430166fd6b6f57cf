/*
 * dyg_oracle.c -- CPU oracle for the dyGRASS update path (TEST INFRASTRUCTURE).
 *
 * Restates, in plain C, the arithmetic and control flow of:
 *   - the incremental walk kernel   random_walk_incremental/main.cu:70-211
 *   - the incremental host commit   random_walk_incremental/gpu_graph.cuh:292-336
 *   - the batching of the stream    random_walk_incremental/gpu_graph.cuh:135, 395-413
 *   - the decremental delete/filter random_walk_decremental/gpu_graph.cuh:328-477
 *   - the decremental walk kernel   random_walk_decremental/main.cu:77-220
 *   - the path commit               random_walk_decremental/gpu_graph.cuh:509-559
 *   - the 2-step fallback walks     random_walk_decremental/main.cu:243-290,
 *                                   random_walk_decremental/gpu_graph.cuh:577-615
 * with cuRAND's per-thread XORWOW stream replaced by Philox4x32-10 keyed by
 * (seed; draw block, walker, update id, domain).  Deviations from the
 * reference are the ones the CUDA path makes too:
 * a walker whose source has degree 0 fails instead of computing `x % 0`,
 * the winner is (max 1/R, lowest walker id) for every walker count, and the
 * fallback walk's second step reads the row of the vertex it stands on.
 *
 * Floating point: compiled with -ffp-contract=off; every operation is a
 * single IEEE binary32 operation, matching the CUDA path bit for bit.
 */
#include "dyg_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------ Philox */

#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

/* Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
 * SC'11: Philox-4x32 with 10 rounds. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PHILOX_M0 * c0;
        uint64_t p1 = (uint64_t)PHILOX_M1 * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

typedef struct {
    uint32_t key[2];
    uint32_t ctr1, ctr2, ctr3;
    uint32_t blk;
    uint32_t buf[4];
} rng_t;

static void rng_init(rng_t *r, uint64_t seed, uint64_t uid, uint32_t domain, uint32_t walker) {
    r->key[0] = (uint32_t)seed;
    r->key[1] = (uint32_t)(seed >> 32);
    r->ctr1 = walker;
    r->ctr2 = (uint32_t)uid;
    r->ctr3 = ((uint32_t)(uid >> 32) & 0x00FFFFFFu) | (domain << 24);
    r->blk = 0xFFFFFFFFu;
}

static inline uint32_t rng_get(rng_t *r, uint32_t d) {
    uint32_t b = d >> 2;
    if (b != r->blk) {
        uint32_t c[4] = {b, r->ctr1, r->ctr2, r->ctr3};
        orc_philox4x32_10(c, r->key, r->buf);
        r->blk = b;
    }
    return r->buf[d & 3u];
}

uint32_t orc_draw(uint64_t seed, uint64_t uid, uint32_t domain, uint32_t walker, uint32_t d) {
    rng_t r;
    rng_init(&r, seed, uid, domain, walker);
    return rng_get(&r, d);
}

#define DOMAIN_INCR 0u
#define DOMAIN_DECR 1u
#define DOMAIN_HEUR 2u

/* ------------------------------------------------------------------- graph */

struct orc_graph {
    uint32_t n;
    uint32_t *deg;
    uint32_t *cap;
    uint32_t **col;
    float **w;
};

static void row_reserve(orc_graph *g, uint32_t x, uint32_t need) {
    if (need <= g->cap[x]) return;
    uint32_t c = g->cap[x] ? g->cap[x] : 4;
    while (c < need) c *= 2;
    g->col[x] = (uint32_t *)realloc(g->col[x], (size_t)c * sizeof(uint32_t));
    g->w[x] = (float *)realloc(g->w[x], (size_t)c * sizeof(float));
    g->cap[x] = c;
}

static void row_append(orc_graph *g, uint32_t x, uint32_t y, float w) {
    row_reserve(g, x, g->deg[x] + 1);
    g->col[x][g->deg[x]] = y;
    g->w[x][g->deg[x]] = w;
    g->deg[x]++;
}

/* Swap-with-last delete of the first slot of row x holding y
 * (random_walk_decremental/gpu_graph.cuh:359-399). */
static int row_remove(orc_graph *g, uint32_t x, uint32_t y) {
    uint32_t d = g->deg[x];
    for (uint32_t j = 0; j < d; ++j) {
        if (g->col[x][j] == y) {
            g->col[x][j] = g->col[x][d - 1];
            g->w[x][j] = g->w[x][d - 1];
            g->deg[x] = d - 1;
            return 1;
        }
    }
    return 0;
}

int orc_graph_has_edge(const orc_graph *g, uint32_t a, uint32_t b) {
    if (a >= g->n) return 0;
    for (uint32_t j = 0; j < g->deg[a]; ++j)
        if (g->col[a][j] == b) return 1;
    return 0;
}

orc_graph *orc_graph_from_edges(uint32_t n, uint64_t m, const uint32_t *src,
                                const uint32_t *dst, const float *w) {
    orc_graph *g = (orc_graph *)calloc(1, sizeof(orc_graph));
    g->n = n;
    g->deg = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    g->cap = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    g->col = (uint32_t **)calloc(n ? n : 1, sizeof(uint32_t *));
    g->w = (float **)calloc(n ? n : 1, sizeof(float *));
    for (uint64_t i = 0; i < m; ++i) {
        row_append(g, src[i], dst[i], w[i]);
        row_append(g, dst[i], src[i], w[i]);
    }
    return g;
}

void orc_graph_free(orc_graph *g) {
    if (!g) return;
    for (uint32_t x = 0; x < g->n; ++x) {
        free(g->col[x]);
        free(g->w[x]);
    }
    free(g->deg); free(g->cap); free(g->col); free(g->w);
    free(g);
}

orc_graph *orc_graph_clone(const orc_graph *g) {
    orc_graph *c = (orc_graph *)calloc(1, sizeof(orc_graph));
    const uint32_t n = g->n;
    c->n = n;
    c->deg = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    c->cap = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    c->col = (uint32_t **)calloc(n ? n : 1, sizeof(uint32_t *));
    c->w = (float **)calloc(n ? n : 1, sizeof(float *));
    for (uint32_t x = 0; x < n; ++x) {
        c->deg[x] = g->deg[x];
        c->cap[x] = g->cap[x];
        if (g->cap[x]) {
            c->col[x] = (uint32_t *)malloc(sizeof(uint32_t) * g->cap[x]);
            c->w[x] = (float *)malloc(sizeof(float) * g->cap[x]);
            memcpy(c->col[x], g->col[x], sizeof(uint32_t) * g->deg[x]);
            memcpy(c->w[x], g->w[x], sizeof(float) * g->deg[x]);
        }
    }
    return c;
}

uint32_t orc_graph_num_vertices(const orc_graph *g) { return g->n; }

uint64_t orc_graph_num_slots(const orc_graph *g) {
    uint64_t s = 0;
    for (uint32_t x = 0; x < g->n; ++x) s += g->deg[x];
    return s;
}

uint64_t orc_graph_export(const orc_graph *g, uint64_t *row_ptr, uint32_t *col, float *w) {
    uint64_t o = 0;
    for (uint32_t x = 0; x < g->n; ++x) {
        if (row_ptr) row_ptr[x] = o;
        for (uint32_t j = 0; j < g->deg[x]; ++j) {
            if (col) col[o + j] = g->col[x][j];
            if (w) w[o + j] = g->w[x][j];
        }
        o += g->deg[x];
    }
    if (row_ptr) row_ptr[g->n] = o;
    return o;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------- transitions */

static inline uint64_t wq(float w) {
    /* fixed-point weight for the weight-proportional mode: exact w * 2^32,
       truncated; integer sums make the choice associative. */
    double v = (double)w * 4294967296.0;
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551615.0) return 0xFFFFFFFFFFFFFFFFull;
    return (uint64_t)v;
}

/* Weight-proportional choice among the slots of a row whose column differs
 * from `excl` (when has_excl).  Returns deg when no slot is eligible. */
static uint32_t pick_weighted(const uint32_t *col, const float *w, uint32_t deg,
                              uint32_t excl, int has_excl, uint32_t r) {
    uint64_t total = 0;
    for (uint32_t j = 0; j < deg; ++j)
        if (!(has_excl && col[j] == excl)) total += wq(w[j]);
    if (total == 0) return deg;
    uint64_t target = (uint64_t)(((unsigned __int128)r * total) >> 32);
    uint64_t acc = 0;
    uint32_t last = deg;
    for (uint32_t j = 0; j < deg; ++j) {
        if (has_excl && col[j] == excl) continue;
        acc += wq(w[j]);
        last = j;
        if (acc > target) return j;
    }
    return last;
}

/* ------------------------------------------------------------------- walks */

/* One walker.  `incr` selects the incremental variant (distortion test,
 * main.cu:144-146); the decremental variant has none (main.cu:124-165).
 * Returns the step at which the target was found, or -1.  `path`, if not
 * NULL, receives path[0..found] (random_walk_decremental/main.cu:106, 114, 152). */
static int32_t walk_one(const orc_graph *g, uint32_t s, uint32_t t, float we, int incr,
                        const orc_params *p, rng_t *rng, float *R_out, uint32_t *path,
                        float *pathw, uint64_t *moves) {
    float R = 0.0f;
    uint32_t cur = s, prev = 0, nxt, idx;
    int32_t found = -1;
    uint32_t step = 1;
    float w;
    if (path) path[0] = s;
    uint32_t deg = g->deg[cur];
    if (deg == 0) { *R_out = 0.0f; return -1; }
    /* first step: any neighbour (main.cu:99-106) */
    uint32_t r = rng_get(rng, 0);
    if (p->transition == 1) {
        idx = pick_weighted(g->col[cur], g->w[cur], deg, 0, 0, r);
        if (idx == deg) { *R_out = 0.0f; return -1; }   /* no weight in the row: no move */
    } else {
        idx = r % deg;
    }
    nxt = g->col[cur][idx];
    w = g->w[cur][idx];
    R = R + 1.0f / w;
    (*moves)++;
    if (path) { path[1] = nxt; pathw[1] = w; }
    if (nxt == t) {
        found = 1;                                   /* main.cu:160-163 */
    } else {
        prev = cur; cur = nxt; step = 2;             /* main.cu:112-114 */
        while (step < p->max_steps) {                /* main.cu:116 */
            deg = g->deg[cur];
            if (deg <= 1) break;                     /* dead end, main.cu:119-121 */
            r = rng_get(rng, step - 1);
            if (p->transition == 1) {
                idx = pick_weighted(g->col[cur], g->w[cur], deg, prev, 1, r);
                if (idx == deg) break;
                nxt = g->col[cur][idx];
                w = g->w[cur][idx];
            } else {
                /* non-backtracking uniform choice, main.cu:126-137 */
                idx = r % (deg - 1);
                nxt = g->col[cur][idx];
                if (nxt == prev) {
                    nxt = g->col[cur][deg - 1];
                    w = g->w[cur][deg - 1];
                } else {
                    w = g->w[cur][idx];
                }
            }
            R = R + 1.0f / w;                        /* main.cu:139 */
            (*moves)++;
            if (path) { path[step] = nxt; pathw[step] = w; }
            if (incr && R * we >= p->threshold) break;   /* main.cu:144-146 */
            if (nxt == t) { found = (int32_t)step; break; }  /* main.cu:149-152 */
            prev = cur; cur = nxt; step++;
        }
    }
    *R_out = R;
    return found;
}

/* Winner key: max conductance 1/R, then lowest walker id; 0 = nobody found
 * the target (main.cu:166-210 reduce the same quantity). */
static inline uint64_t pack_key(float cond, uint32_t walker, int32_t found) {
    uint32_t cb;
    memcpy(&cb, &cond, 4);
    return ((uint64_t)cb << 32) | ((uint64_t)(1023u - walker) << 22) | ((uint64_t)found & 0x3FFFFFu);
}

static inline float key_cond(uint64_t k) {
    uint32_t cb = (uint32_t)(k >> 32);
    float f;
    memcpy(&f, &cb, 4);
    return f;
}

static uint64_t best_key(const orc_graph *g, uint32_t s, uint32_t t, float we, int incr,
                         const orc_params *p, uint64_t uid, uint32_t domain, uint64_t *moves) {
    uint64_t best = 0;
    for (uint32_t k = 0; k < p->walkers; ++k) {
        rng_t rng;
        rng_init(&rng, p->seed, uid, domain, k);
        float R;
        int32_t f = walk_one(g, s, t, we, incr, p, &rng, &R, NULL, NULL, moves);
        if (f > 0) {
            float cond = 1.0f / R;
            uint64_t key = pack_key(cond, k, f);
            if (key > best) best = key;
        }
    }
    return best;
}

/* ------------------------------------------------------------- incremental */

void orc_walk_keys(const orc_graph *g, const uint32_t *src, const uint32_t *dst, const float *w,
                   uint64_t first_uid, uint32_t lo, uint32_t hi, int incr, const orc_params *p,
                   int threads, uint64_t *keys, uint64_t *moves) {
    uint64_t mv_total = 0;
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) reduction(+ : mv_total)
    for (int64_t e = lo; e < (int64_t)hi; ++e) {
        uint64_t mv = 0;
        keys[e] = best_key(g, src[e], dst[e], incr ? w[e] : 0.0f, incr, p, first_uid + (uint64_t)e,
                           incr ? DOMAIN_INCR : DOMAIN_DECR, &mv);
        mv_total += mv;
    }
    if (moves) *moves = mv_total;
}

void orc_walk_keys_ids(const orc_graph *g, const uint32_t *src, const uint32_t *dst,
                       const float *w, const uint64_t *uids, uint32_t n, const orc_params *p,
                       int threads, uint64_t *keys, uint64_t *moves) {
    uint64_t mv_total = 0;
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) reduction(+ : mv_total)
    for (int64_t e = 0; e < (int64_t)n; ++e) {
        uint64_t mv = 0;
        keys[e] = best_key(g, src[e], dst[e], w[e], 1, p, uids[e], DOMAIN_INCR, &mv);
        mv_total += mv;
    }
    if (moves) *moves = mv_total;
}

/* commit in input order (gpu_graph.cuh:297-329): add iff no path */
void orc_incremental_commit_keys(orc_graph *H, orc_graph *G, const uint32_t *src,
                                 const uint32_t *dst, const float *w, uint32_t n,
                                 const uint64_t *keys, int32_t *found_at, float *cond,
                                 uint8_t *accepted) {
    for (uint32_t e = 0; e < n; ++e) {
        uint64_t k = keys[e];
        if (found_at) found_at[e] = k ? (int32_t)(k & 0x3FFFFFu) : -1;
        if (cond) cond[e] = k ? key_cond(k) : 0.0f;
        if (accepted) accepted[e] = k ? 0 : 1;
        if (!k) {
            row_append(H, src[e], dst[e], w[e]);
            row_append(H, dst[e], src[e], w[e]);
        }
    }
    if (G) {
        for (uint32_t e = 0; e < n; ++e) {
            row_append(G, src[e], dst[e], w[e]);
            row_append(G, dst[e], src[e], w[e]);
        }
    }
}

uint64_t orc_incremental_batch(orc_graph *H, orc_graph *G, const uint32_t *src,
                               const uint32_t *dst, const float *w, uint32_t n,
                               uint64_t first_uid, const orc_params *p, int threads,
                               int32_t *found_at, float *cond, uint8_t *accepted) {
    uint64_t moves = 0;
    uint64_t *keys = (uint64_t *)malloc((size_t)(n ? n : 1) * sizeof(uint64_t));
    orc_walk_keys(H, src, dst, w, first_uid, 0, n, 1, p, threads, keys, &moves);
    orc_incremental_commit_keys(H, G, src, dst, w, n, keys, found_at, cond, accepted);
    free(keys);
    return moves;
}

static uint32_t ref_batch(uint32_t n, uint32_t batch_size) {
    if (batch_size) return batch_size;
    uint32_t b = (n + 9u) / 10u;          /* gpu_graph.cuh:135 */
    return b ? b : 1u;
}

uint64_t orc_incremental_stream(orc_graph *H, orc_graph *G, const uint32_t *src,
                                const uint32_t *dst, const float *w, uint32_t n,
                                uint32_t batch_size, const orc_params *p, int threads,
                                int32_t *found_at, float *cond, uint8_t *accepted) {
    uint32_t B = ref_batch(n, batch_size);
    uint64_t moves = 0;
    for (uint32_t b0 = 0; b0 < n; b0 += B) {
        uint32_t nb = (n - b0 < B) ? n - b0 : B;
        moves += orc_incremental_batch(H, G, src + b0, dst + b0, w + b0, nb, b0, p, threads,
                                       found_at ? found_at + b0 : NULL, cond ? cond + b0 : NULL,
                                       accepted ? accepted + b0 : NULL);
    }
    return moves;
}

/* ------------------------------------------------------------- decremental */

static int32_t decr_walk_path(const orc_graph *G, uint32_t s, uint32_t t, uint64_t uid,
                              uint32_t walker, const orc_params *p, uint32_t *path,
                              float *pathw, float *R) {
    rng_t rng;
    uint64_t mv = 0;
    rng_init(&rng, p->seed, uid, DOMAIN_DECR, walker);
    return walk_one(G, s, t, 0.0f, 0, p, &rng, R, path, pathw, &mv);
}

int32_t orc_decremental_walk_path(const orc_graph *G, uint32_t s, uint32_t t, uint64_t uid,
                                  uint32_t walker, const orc_params *p, uint32_t *path,
                                  float *R) {
    uint32_t n = p->max_steps > 2 ? p->max_steps : 2;
    float *pw = (float *)malloc((size_t)n * sizeof(float));
    int32_t f = decr_walk_path(G, s, t, uid, walker, p, path, pw, R);
    free(pw);
    return f;
}

typedef struct {
    uint32_t *a, *b;
    uint8_t *kind;
    uint64_t n, cap_out;
    uint32_t *out_a, *out_b;
    uint8_t *out_kind;
} rec_t;

/* Append (x, y, w) to H unless already present (gpu_graph.cuh:534-538,
 * 599-601) and record it. */
static void rec_add(orc_graph *H, rec_t *rc, uint32_t x, uint32_t y, float w, uint8_t kind) {
    if (x == y) return;
    if (orc_graph_has_edge(H, x, y)) return;
    row_append(H, x, y, w);
    row_append(H, y, x, w);
    if (rc->n < rc->cap_out) {
        if (rc->out_a) rc->out_a[rc->n] = x;
        if (rc->out_b) rc->out_b[rc->n] = y;
        if (rc->out_kind) rc->out_kind[rc->n] = kind;
    }
    rc->n++;
}

/* Deletion stage: delete every edge from G (swap with the row's last slot),
 * erase the ones also in H, and list those (gpu_graph.cuh:338-458;
 * dynamic_update/gpu_graph.cuh:398-431).  Endpoints are ordered min -> max
 * for the row operations (gpu_graph.cuh:342). */
static uint32_t decr_delete(orc_graph *G, orc_graph *H, const uint32_t *src, const uint32_t *dst,
                            uint32_t n, int32_t *status, float *cond, uint32_t *filt) {
    uint32_t nf = 0;
    for (uint32_t e = 0; e < n; ++e) {
        uint32_t a = src[e], b = dst[e];
        if (a > b) { uint32_t t = a; a = b; b = t; }
        int32_t st;
        if (!orc_graph_has_edge(G, a, b)) {
            st = ORC_DEL_NOT_IN_G;
        } else {
            row_remove(G, a, b);
            row_remove(G, b, a);
            if (orc_graph_has_edge(H, a, b)) {
                row_remove(H, a, b);
                row_remove(H, b, a);
                filt[nf++] = e;
                st = ORC_DEL_NO_PATH;   /* provisional */
            } else {
                st = ORC_DEL_NOT_IN_H;
            }
        }
        if (status) status[e] = st;
        if (cond) cond[e] = 0.0f;
    }
    return nf;
}

/* Walk endpoints of listed deletion e: min -> max for the standalone
 * decremental updater (random_walk_decremental/gpu_graph.cuh:342), file
 * orientation for stream files (dynamic_update/gpu_graph.cuh:874-875). */
static void walk_ends(const uint32_t *src, const uint32_t *dst, uint32_t e, int file_orient,
                      uint32_t *s, uint32_t *t) {
    uint32_t a = src[e], b = dst[e];
    if (!file_orient && a > b) { uint32_t x = a; a = b; b = x; }
    *s = a;
    *t = b;
}

/* Walk-and-recover stage for listed deletions filt[0..nf): walks on G, winner
 * paths into H in order (gpu_graph.cuh:514-552), then the 2-step fallback
 * walks from both walk endpoints (main.cu:243-290). */
static uint64_t decr_walk(orc_graph *G, orc_graph *H, const uint32_t *src, const uint32_t *dst,
                          const uint32_t *filt, uint32_t nf, uint64_t first_uid, int file_orient,
                          const orc_params *p, int threads, int32_t *status, float *cond,
                          rec_t *rc, const uint64_t *keys_in, const uint64_t *uids) {
#define DECR_UID(e) (uids ? uids[e] : first_uid + (e))
    uint64_t moves = 0;
    uint64_t *keys = (uint64_t *)malloc((size_t)(nf ? nf : 1) * sizeof(uint64_t));
    if (threads < 1) threads = 1;
    if (keys_in) memcpy(keys, keys_in, (size_t)nf * sizeof(uint64_t));
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) reduction(+ : moves)
    for (int64_t f = 0; f < (int64_t)(keys_in ? 0 : nf); ++f) {
        uint32_t e = filt[f], a, b;
        walk_ends(src, dst, e, file_orient, &a, &b);
        uint64_t mv = 0;
        keys[f] = best_key(G, a, b, 0.0f, 0, p, DECR_UID(e), DOMAIN_DECR, &mv);
        moves += mv;
    }
    uint32_t pathlen = p->max_steps > 2 ? p->max_steps : 2;
    uint32_t *path = (uint32_t *)malloc((size_t)pathlen * sizeof(uint32_t));
    float *pathw = (float *)malloc((size_t)pathlen * sizeof(float));
    uint32_t *nop = (uint32_t *)malloc((size_t)(nf ? nf : 1) * sizeof(uint32_t));
    uint32_t nnop = 0;
    for (uint32_t f = 0; f < nf; ++f) {
        uint32_t e = filt[f], a, b;
        walk_ends(src, dst, e, file_orient, &a, &b);
        uint64_t k = keys[f];
        if (k) {
            uint32_t walker = 1023u - (uint32_t)((k >> 22) & 0x3FFu);
            float R;
            int32_t found = decr_walk_path(G, a, b, DECR_UID(e), walker, p, path, pathw, &R);
            if (status) status[e] = found;
            if (cond) cond[e] = key_cond(k);
            for (int32_t j = 0; j < found; ++j) rec_add(H, rc, path[j], path[j + 1], pathw[j + 1], 0);
        } else {
            nop[nnop++] = f;
        }
    }
    for (uint32_t q = 0; q < nnop; ++q) {
        uint32_t e = filt[nop[q]];
        uint32_t ends[2];
        walk_ends(src, dst, e, file_orient, &ends[0], &ends[1]);
        for (uint32_t side = 0; side < 2; ++side) {
            for (uint32_t j = 0; j < p->heuristic_walkers; ++j) {
                rng_t rng;
                rng_init(&rng, p->seed, DECR_UID(e), DOMAIN_HEUR, side * p->heuristic_walkers + j);
                uint32_t s0 = ends[side];
                uint32_t d0 = G->deg[s0];
                if (d0 == 0) continue;
                uint32_t i0 = rng_get(&rng, 0) % d0;
                uint32_t x1 = G->col[s0][i0];
                float w1 = G->w[s0][i0];
                uint32_t d1 = G->deg[x1];
                uint32_t x2 = x1;
                float w2 = 0.0f;
                if (d1 > 0) {
                    uint32_t i1 = rng_get(&rng, 1) % d1;
                    if (G->col[x1][i1] == s0) i1 = d1 - 1;
                    x2 = G->col[x1][i1];
                    w2 = G->w[x1][i1];
                }
                rec_add(H, rc, s0, x1, w1, 1);
                rec_add(H, rc, x1, x2, w2, 1);
            }
        }
    }
    free(path); free(pathw); free(nop); free(keys);
    return moves;
}
#undef DECR_UID

uint64_t orc_decremental_batch(orc_graph *G, orc_graph *H, const uint32_t *src,
                               const uint32_t *dst, uint32_t n, uint64_t first_uid,
                               const orc_params *p, int threads, int32_t *status,
                               float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                               uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec) {
    uint32_t *filt = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t nf = decr_delete(G, H, src, dst, n, status, cond, filt);
    rec_t rc = {0};
    rc.cap_out = rec_cap; rc.out_a = rec_src; rc.out_b = rec_dst; rc.out_kind = rec_kind;
    uint64_t moves = decr_walk(G, H, src, dst, filt, nf, first_uid, 0, p, threads, status, cond, &rc,
                               NULL, NULL);
    if (n_rec) *n_rec = rc.n;
    free(filt);
    return moves;
}

/* orc_decremental_batch with each deletion's update id read from uids[e] */
uint64_t orc_decremental_batch_ids(orc_graph *G, orc_graph *H, const uint32_t *src,
                                   const uint32_t *dst, const uint64_t *uids, uint32_t n,
                                   const orc_params *p, int threads, int32_t *status,
                                   float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                                   uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec) {
    uint32_t *filt = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t nf = decr_delete(G, H, src, dst, n, status, cond, filt);
    rec_t rc = {0};
    rc.cap_out = rec_cap; rc.out_a = rec_src; rc.out_b = rec_dst; rc.out_kind = rec_kind;
    uint64_t moves = decr_walk(G, H, src, dst, filt, nf, 0, 0, p, threads, status, cond, &rc,
                               NULL, uids);
    if (n_rec) *n_rec = rc.n;
    free(filt);
    return moves;
}

/* ----------------------------------------------------------- stream files */

uint32_t orc_stream_default_chunk(uint32_t n_vertices) {
    /* 5% of |V|, at least 10000 (dynamic_update/main.cu:83-84) */
    uint32_t c = (uint32_t)((double)n_vertices * 0.05);
    return c < 10000u ? 10000u : c;
}

/* Adds `w` to the weight of the first slot of row x holding y
 * (dynamic_update/gpu_graph.cuh:452-465). */
static void row_add_weight(orc_graph *g, uint32_t x, uint32_t y, float w) {
    for (uint32_t j = 0; j < g->deg[x]; ++j)
        if (g->col[x][j] == y) {
            g->w[x][j] = g->w[x][j] + w;
            return;
        }
}

uint64_t orc_stream_file(orc_graph *G, orc_graph *H, uint32_t op, const uint32_t *src,
                         const uint32_t *dst, const float *w, uint32_t n, uint64_t first_uid,
                         uint32_t chunk, const orc_params *p, int threads, int32_t *status,
                         float *cond, uint32_t *rec_src, uint32_t *rec_dst, uint8_t *rec_kind,
                         uint64_t rec_cap, uint64_t *n_rec) {
    uint64_t moves = 0;
    uint32_t *list = (uint32_t *)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
    uint32_t nl = 0;
    if (chunk == 0) chunk = orc_stream_default_chunk(G->n);
    if (threads < 1) threads = 1;
    if (n_rec) *n_rec = 0;
    if (op == ORC_STREAM_INSERT) {
        /* preprocessing in file order (dynamic_update/gpu_graph.cuh:373-396):
           an edge already in G adds its weight to G and, if there, to H; a
           new edge enters G at once and is walked later */
        for (uint32_t i = 0; i < n; ++i) {
            uint32_t a = src[i] < dst[i] ? src[i] : dst[i];
            uint32_t b = src[i] < dst[i] ? dst[i] : src[i];
            if (cond) cond[i] = 0.0f;
            if (a == b) {
                if (status) status[i] = ORC_STREAM_SELF_LOOP;
            } else if (orc_graph_has_edge(G, a, b)) {
                row_add_weight(G, a, b, w[i]);
                row_add_weight(G, b, a, w[i]);
                if (orc_graph_has_edge(H, a, b)) {
                    row_add_weight(H, a, b, w[i]);
                    row_add_weight(H, b, a, w[i]);
                }
                if (status) status[i] = ORC_STREAM_MERGED;
            } else {
                row_append(G, a, b, w[i]);
                row_append(G, b, a, w[i]);
                list[nl++] = i;
            }
        }
        /* walks on H in chunks, each chunk's accepted edges entering H with
           their stream weight before the next chunk walks
           (dynamic_update/main.cu:107-126, gpu_graph.cuh:632-636) */
        uint64_t *keys = (uint64_t *)malloc((size_t)(nl ? nl : 1) * sizeof(uint64_t));
        for (uint32_t c0 = 0; c0 < nl; c0 += chunk) {
            uint32_t c1 = nl - c0 < chunk ? nl : c0 + chunk;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads) reduction(+ : moves)
            for (int64_t k = c0; k < (int64_t)c1; ++k) {
                uint32_t i = list[k];
                uint64_t mv = 0;
                keys[k] = best_key(H, src[i], dst[i], w[i], 1, p, first_uid + i, DOMAIN_INCR, &mv);
                moves += mv;
            }
            for (uint32_t k = c0; k < c1; ++k) {
                uint32_t i = list[k];
                uint64_t kk = keys[k];
                if (status) status[i] = kk ? (int32_t)(kk & 0x3FFFFFu) : -1;
                if (cond) cond[i] = kk ? key_cond(kk) : 0.0f;
                if (!kk) {
                    row_append(H, src[i], dst[i], w[i]);
                    row_append(H, dst[i], src[i], w[i]);
                }
            }
        }
        free(keys);
    } else {
        /* the whole file is deleted first (dynamic_update/gpu_graph.cuh:398-431),
           then the listed edges are walked on G in chunks, each chunk's
           recovered edges entering H before the next */
        nl = decr_delete(G, H, src, dst, n, status, cond, list);
        rec_t rc = {0};
        rc.cap_out = rec_cap; rc.out_a = rec_src; rc.out_b = rec_dst; rc.out_kind = rec_kind;
        for (uint32_t c0 = 0; c0 < nl; c0 += chunk) {
            uint32_t c1 = nl - c0 < chunk ? nl : c0 + chunk;
            moves += decr_walk(G, H, src, dst, list + c0, c1 - c0, first_uid, 1, p, threads,
                               status, cond, &rc, NULL, NULL);
        }
        if (n_rec) *n_rec = rc.n;
    }
    free(list);
    return moves;
}

uint32_t orc_decremental_delete(orc_graph *G, orc_graph *H, const uint32_t *src,
                                const uint32_t *dst, uint32_t n, int32_t *status, float *cond,
                                uint32_t *walk_list) {
    return decr_delete(G, H, src, dst, n, status, cond, walk_list);
}

void orc_decremental_walk_list_keys(const orc_graph *G, const uint32_t *src, const uint32_t *dst,
                                    const uint32_t *walk_list, uint32_t lo, uint32_t hi,
                                    uint64_t first_uid, const orc_params *p, int threads,
                                    uint64_t *keys) {
    if (threads < 1) threads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads)
    for (int64_t f = lo; f < (int64_t)hi; ++f) {
        uint32_t e = walk_list[f], a, b;
        walk_ends(src, dst, e, 0, &a, &b);
        uint64_t mv = 0;
        keys[f] = best_key(G, a, b, 0.0f, 0, p, first_uid + e, DOMAIN_DECR, &mv);
    }
}

void orc_decremental_commit_keys(orc_graph *G, orc_graph *H, const uint32_t *src,
                                 const uint32_t *dst, const uint32_t *walk_list, uint32_t nf,
                                 uint64_t first_uid, const orc_params *p, const uint64_t *keys,
                                 int32_t *status, float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                                 uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec) {
    rec_t rc = {0};
    rc.cap_out = rec_cap; rc.out_a = rec_src; rc.out_b = rec_dst; rc.out_kind = rec_kind;
    decr_walk(G, H, src, dst, walk_list, nf, first_uid, 0, p, 1, status, cond, &rc, keys, NULL);
    if (n_rec) *n_rec = rc.n;
}

uint64_t orc_decremental_stream(orc_graph *G, orc_graph *H, const uint32_t *src,
                                const uint32_t *dst, uint32_t n, uint32_t batch_size,
                                const orc_params *p, int threads, int32_t *status,
                                float *cond, uint32_t *rec_src, uint32_t *rec_dst,
                                uint8_t *rec_kind, uint64_t rec_cap, uint64_t *n_rec) {
    uint32_t B = ref_batch(n, batch_size);
    uint64_t moves = 0, total = 0;
    for (uint32_t b0 = 0; b0 < n; b0 += B) {
        uint32_t nb = (n - b0 < B) ? n - b0 : B;
        uint64_t got = 0;
        uint64_t room = total < rec_cap ? rec_cap - total : 0;
        moves += orc_decremental_batch(G, H, src + b0, dst + b0, nb, b0, p, threads,
                                       status ? status + b0 : NULL, cond ? cond + b0 : NULL,
                                       rec_src ? rec_src + total : NULL,
                                       rec_dst ? rec_dst + total : NULL,
                                       rec_kind ? rec_kind + total : NULL, room, &got);
        total += got;
    }
    if (n_rec) *n_rec = total;
    return moves;
}
