// synth.cpp -- seeded synthetic workloads (include/dyg_synth.h).
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <unordered_set>
#include <vector>

#include "../../include/dyg_synth.h"

namespace {

struct SplitMix {
    uint64_t s;
    explicit SplitMix(uint64_t seed) : s(seed) {}
    uint64_t next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
    uint64_t below(uint64_t n) { return n ? next() % n : 0; }
};

float draw_weight(SplitMix &r, uint32_t dist, float lo, float hi) {
    const double u = r.unit();
    if (dist == DYG_W_LOGUNIFORM) {
        const double a = log10((double)lo), b = log10((double)hi);
        return (float)pow(10.0, a + (b - a) * u);
    }
    return (float)((double)lo + ((double)hi - (double)lo) * u);
}

struct DSU {
    std::vector<uint32_t> p;
    explicit DSU(uint32_t n) : p(n) { std::iota(p.begin(), p.end(), 0u); }
    uint32_t find(uint32_t x) {
        while (p[x] != x) {
            p[x] = p[p[x]];
            x = p[x];
        }
        return x;
    }
    bool unite(uint32_t a, uint32_t b) {
        a = find(a);
        b = find(b);
        if (a == b) return false;
        p[a] = b;
        return true;
    }
};

inline uint64_t pair_key(uint32_t a, uint32_t b) {
    if (a > b) std::swap(a, b);
    return ((uint64_t)a << 32) | b;
}

}  // namespace

extern "C" {

uint64_t dyg_synth_lattice_edges(uint32_t nx, uint32_t ny, uint32_t nz) {
    const uint64_t X = nx, Y = ny, Z = nz ? nz : 1;
    return (X - 1) * Y * Z + X * (Y - 1) * Z + X * Y * (Z - 1);
}

void dyg_synth_lattice(uint32_t nx, uint32_t ny, uint32_t nz, uint32_t wdist, float lo, float hi,
                       uint64_t seed, uint32_t *src, uint32_t *dst, float *w) {
    if (nz == 0) nz = 1;
    SplitMix r(seed);
    uint64_t k = 0;
    for (uint32_t z = 0; z < nz; ++z)
        for (uint32_t y = 0; y < ny; ++y)
            for (uint32_t x = 0; x < nx; ++x) {
                const uint32_t v = x + nx * (y + ny * z);
                if (x + 1 < nx) {
                    src[k] = v; dst[k] = v + 1; w[k] = draw_weight(r, wdist, lo, hi); ++k;
                }
                if (y + 1 < ny) {
                    src[k] = v; dst[k] = v + nx; w[k] = draw_weight(r, wdist, lo, hi); ++k;
                }
                if (z + 1 < nz) {
                    src[k] = v; dst[k] = v + nx * ny; w[k] = draw_weight(r, wdist, lo, hi); ++k;
                }
            }
}

uint64_t dyg_synth_sparsifier(uint32_t n, uint64_t m, const uint32_t *src, const uint32_t *dst,
                              const float *w, double frac, uint64_t seed, uint64_t *out_idx) {
    std::vector<uint64_t> order(m);
    std::iota(order.begin(), order.end(), 0ull);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint64_t a, uint64_t b) { return w[a] > w[b]; });
    DSU dsu(n);
    std::vector<uint8_t> in_tree(m, 0);
    std::vector<uint64_t> off;
    off.reserve(m);
    for (uint64_t i : order) {
        if (src[i] != dst[i] && dsu.unite(src[i], dst[i])) in_tree[i] = 1;
    }
    for (uint64_t i = 0; i < m; ++i)
        if (!in_tree[i]) off.push_back(i);
    const uint64_t k = (uint64_t)floor(frac * (double)off.size());
    SplitMix r(seed);
    for (uint64_t i = 0; i < k; ++i) {  // partial Fisher-Yates
        const uint64_t j = i + r.below(off.size() - i);
        std::swap(off[i], off[j]);
    }
    for (uint64_t i = 0; i < k; ++i) in_tree[off[i]] = 1;
    uint64_t c = 0;
    for (uint64_t i = 0; i < m; ++i)
        if (in_tree[i]) out_idx[c++] = i;
    return c;
}

uint64_t dyg_synth_lattice_inserts(uint32_t nx, uint32_t ny, uint32_t nz, uint64_t m,
                                   const uint32_t *src, const uint32_t *dst, uint64_t count,
                                   uint32_t hop_lo, uint32_t hop_hi, uint32_t wdist, float lo,
                                   float hi, uint64_t seed, uint32_t *out_src, uint32_t *out_dst,
                                   float *out_w) {
    if (nz == 0) nz = 1;
    const bool three = nz > 1;
    std::unordered_set<uint64_t> seen;
    seen.reserve((size_t)(m + count) * 2);
    for (uint64_t i = 0; i < m; ++i) seen.insert(pair_key(src[i], dst[i]));
    SplitMix r(seed);
    const uint64_t nv = (uint64_t)nx * ny * nz;
    uint64_t k = 0, tries = 0;
    const uint64_t max_tries = count * 1000 + 1000000;
    while (k < count && tries < max_tries) {
        ++tries;
        const uint32_t u = (uint32_t)r.below(nv);
        const int64_t d = (int64_t)hop_lo + (int64_t)r.below((uint64_t)(hop_hi - hop_lo + 1));
        const int64_t ux = u % nx, uy = (u / nx) % ny, uz = u / ((uint64_t)nx * ny);
        int64_t dx = (int64_t)r.below((uint64_t)(2 * d + 1)) - d;
        int64_t rem = d - (dx < 0 ? -dx : dx);
        int64_t dy, dz = 0;
        if (three) {
            dy = (int64_t)r.below((uint64_t)(2 * rem + 1)) - rem;
            const int64_t rz = rem - (dy < 0 ? -dy : dy);
            dz = (r.next() & 1) ? rz : -rz;
        } else {
            dy = (r.next() & 1) ? rem : -rem;
        }
        const int64_t vx = ux + dx, vy = uy + dy, vz = uz + dz;
        if (vx < 0 || vy < 0 || vz < 0 || vx >= nx || vy >= ny || vz >= nz) continue;
        const uint32_t v = (uint32_t)(vx + (int64_t)nx * (vy + (int64_t)ny * vz));
        if (v == u) continue;
        if (!seen.insert(pair_key(u, v)).second) continue;
        out_src[k] = u;
        out_dst[k] = v;
        out_w[k] = draw_weight(r, wdist, lo, hi);
        ++k;
    }
    return k;
}

static inline void rmat_pair(SplitMix &r, uint32_t scale, double a, double b, double c,
                             uint32_t *u, uint32_t *v) {
    uint32_t x = 0, y = 0;
    for (uint32_t l = 0; l < scale; ++l) {
        const double p = r.unit();
        uint32_t bx = 0, by = 0;
        if (p < a) {
        } else if (p < a + b) {
            by = 1;
        } else if (p < a + b + c) {
            bx = 1;
        } else {
            bx = by = 1;
        }
        x = (x << 1) | bx;
        y = (y << 1) | by;
    }
    *u = x;
    *v = y;
}

void dyg_synth_rmat_pairs(uint32_t scale, uint64_t count, double a, double b, double c,
                          uint64_t seed, uint32_t *src, uint32_t *dst) {
    SplitMix r(seed);
    for (uint64_t i = 0; i < count; ++i) rmat_pair(r, scale, a, b, c, &src[i], &dst[i]);
}

uint64_t dyg_synth_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                        float wlo, float whi, uint64_t seed, uint32_t *n_out, uint32_t **src,
                        uint32_t **dst, float **w, uint32_t **id_map) {
    const uint64_t nv = 1ull << scale;
    const uint64_t m0 = (uint64_t)edge_factor * nv;
    SplitMix r(seed);
    std::vector<uint64_t> keys;
    keys.reserve(m0);
    for (uint64_t i = 0; i < m0; ++i) {
        uint32_t u, v;
        rmat_pair(r, scale, a, b, c, &u, &v);
        if (u == v) continue;
        if (u > v) std::swap(u, v);
        keys.push_back(((uint64_t)u << 32) | v);
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    DSU dsu((uint32_t)nv);
    for (uint64_t k : keys) dsu.unite((uint32_t)(k >> 32), (uint32_t)k);
    std::vector<uint32_t> size(nv, 0);
    std::vector<uint8_t> touched(nv, 0);
    for (uint64_t k : keys) {
        touched[k >> 32] = 1;
        touched[(uint32_t)k] = 1;
    }
    for (uint64_t v = 0; v < nv; ++v)
        if (touched[v]) size[dsu.find((uint32_t)v)]++;
    uint32_t best = 0;
    for (uint64_t v = 0; v < nv; ++v)
        if (size[v] > size[best]) best = (uint32_t)v;
    uint32_t *map = (uint32_t *)malloc(sizeof(uint32_t) * nv);
    uint32_t n = 0;
    for (uint64_t v = 0; v < nv; ++v)
        map[v] = (touched[v] && dsu.find((uint32_t)v) == best) ? n++ : 0xFFFFFFFFu;
    uint64_t m = 0;
    for (uint64_t k : keys)
        if (map[k >> 32] != 0xFFFFFFFFu) ++m;
    *src = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    *dst = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    *w = (float *)malloc(sizeof(float) * (m ? m : 1));
    SplitMix rw(seed ^ 0x5bd1e995ull);
    uint64_t j = 0;
    for (uint64_t k : keys) {
        const uint32_t u = map[k >> 32], v = map[(uint32_t)k];
        if (u == 0xFFFFFFFFu) continue;
        (*src)[j] = u;
        (*dst)[j] = v;
        (*w)[j] = draw_weight(rw, DYG_W_UNIFORM, wlo, whi);
        ++j;
    }
    *n_out = n;
    *id_map = map;
    return m;
}

uint64_t dyg_synth_rmat_stream(uint32_t scale, double a, double b, double c,
                               const uint32_t *id_map, uint64_t m, const uint32_t *src,
                               const uint32_t *dst, uint64_t n_updates, uint32_t file_size,
                               double del_frac, float wlo, float whi, uint64_t seed,
                               uint8_t *file_op, uint32_t *out_src, uint32_t *out_dst,
                               float *out_w) {
    if (file_size == 0) return 0;
    std::unordered_set<uint64_t> live;
    live.reserve((size_t)(m + n_updates) * 2);
    std::vector<uint64_t> alive;
    alive.reserve((size_t)(m + n_updates));
    for (uint64_t i = 0; i < m; ++i) {
        const uint64_t k = pair_key(src[i], dst[i]);
        if (live.insert(k).second) alive.push_back(k);
    }
    SplitMix r(seed);
    const uint64_t nfiles = (n_updates + file_size - 1) / file_size;
    uint64_t o = 0;
    for (uint64_t f = 0; f < nfiles; ++f) {
        const uint64_t cnt = std::min<uint64_t>(file_size, n_updates - o);
        const bool del = (uint64_t)floor((double)(f + 1) * del_frac) > (uint64_t)floor((double)f * del_frac);
        file_op[f] = del ? 1 : 0;
        for (uint64_t k = 0; k < cnt; ++k, ++o) {
            if (del && !alive.empty()) {
                const uint64_t j = r.below(alive.size());
                const uint64_t key = alive[j];
                alive[j] = alive.back();
                alive.pop_back();
                live.erase(key);
                out_src[o] = (uint32_t)(key >> 32);
                out_dst[o] = (uint32_t)key;
                out_w[o] = 1.0f;
                continue;
            }
            uint32_t u = 0, v = 0;
            for (int tries = 0; tries < 1000000; ++tries) {
                uint32_t x, y;
                rmat_pair(r, scale, a, b, c, &x, &y);
                u = id_map[x];
                v = id_map[y];
                if (u != 0xFFFFFFFFu && v != 0xFFFFFFFFu && u != v) break;
                u = v = 0xFFFFFFFFu;
            }
            out_src[o] = u;
            out_dst[o] = v;
            out_w[o] = draw_weight(r, DYG_W_UNIFORM, wlo, whi);
            const uint64_t key = pair_key(u, v);
            if (u != 0xFFFFFFFFu && live.insert(key).second) alive.push_back(key);
        }
    }
    return nfiles;
}

uint64_t dyg_synth_rgg(uint32_t n, double avg_deg, uint32_t n_ins, uint64_t seed,
                       uint32_t *n_out, uint32_t **src, uint32_t **dst, float **w,
                       uint32_t *n_ins_out, uint32_t **isrc, uint32_t **idst, float **iw) {
    SplitMix r(seed);
    std::vector<double> px(n), py(n);
    for (uint32_t i = 0; i < n; ++i) {
        px[i] = r.unit();
        py[i] = r.unit();
    }
    const double rad = sqrt(avg_deg / (3.141592653589793 * (double)(n ? n : 1)));
    const uint32_t gdim = std::max<uint32_t>(1, (uint32_t)(1.0 / rad));
    auto cell = [&](double x) { return std::min<uint32_t>(gdim - 1, (uint32_t)(x * gdim)); };
    std::vector<std::vector<uint32_t>> grid((size_t)gdim * gdim);
    for (uint32_t i = 0; i < n; ++i) grid[(size_t)cell(py[i]) * gdim + cell(px[i])].push_back(i);
    // cells are at least rad wide, so neighbours lie in the 3x3 block
    std::vector<std::pair<uint32_t, uint32_t>> e;
    for (uint32_t i = 0; i < n; ++i) {
        const int cx = (int)cell(px[i]), cy = (int)cell(py[i]);
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int x = cx + dx, y = cy + dy;
                if (x < 0 || y < 0 || x >= (int)gdim || y >= (int)gdim) continue;
                for (uint32_t j : grid[(size_t)y * gdim + x]) {
                    if (j <= i) continue;
                    const double d = hypot(px[i] - px[j], py[i] - py[j]);
                    if (d < rad && d > 0) e.emplace_back(i, j);
                }
            }
    }
    std::sort(e.begin(), e.end());
    DSU dsu(n);
    for (auto &p : e) dsu.unite(p.first, p.second);
    std::vector<uint32_t> size(n, 0);
    for (uint32_t i = 0; i < n; ++i) size[dsu.find(i)]++;
    uint32_t best = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (size[i] > size[best]) best = i;
    std::vector<uint32_t> map(n, 0xFFFFFFFFu);
    uint32_t nn = 0;
    for (uint32_t i = 0; i < n; ++i)
        if (dsu.find(i) == best) map[i] = nn++;
    std::vector<uint32_t> vs, vd;
    std::vector<float> vw;
    std::unordered_set<uint64_t> present;
    for (auto &p : e) {
        if (map[p.first] == 0xFFFFFFFFu) continue;
        vs.push_back(map[p.first]);
        vd.push_back(map[p.second]);
        vw.push_back((float)(1.0 / hypot(px[p.first] - px[p.second], py[p.first] - py[p.second])));
        present.insert(pair_key(map[p.first], map[p.second]));
    }
    std::vector<uint32_t> back(nn);
    for (uint32_t i = 0; i < n; ++i)
        if (map[i] != 0xFFFFFFFFu) back[map[i]] = i;
    // insertions: pairs of component points at distance in [rad, 3 rad)
    std::vector<uint32_t> is, id;
    std::vector<float> iwv;
    std::vector<uint32_t> cand;
    uint64_t tries = 0;
    while (is.size() < n_ins && nn > 1 && tries < (uint64_t)n_ins * 1000 + 1000) {
        ++tries;
        const uint32_t u = (uint32_t)r.below(nn);
        const uint32_t pu = back[u];
        const int cx = (int)cell(px[pu]), cy = (int)cell(py[pu]);
        cand.clear();
        for (int dy = -3; dy <= 3; ++dy)
            for (int dx = -3; dx <= 3; ++dx) {
                const int x = cx + dx, y = cy + dy;
                if (x < 0 || y < 0 || x >= (int)gdim || y >= (int)gdim) continue;
                for (uint32_t j : grid[(size_t)y * gdim + x]) {
                    if (map[j] == 0xFFFFFFFFu || j == pu) continue;
                    const double d = hypot(px[pu] - px[j], py[pu] - py[j]);
                    if (d >= rad && d < 3 * rad && !present.count(pair_key(u, map[j])))
                        cand.push_back(j);
                }
            }
        if (cand.empty()) continue;
        const uint32_t pv = cand[r.below(cand.size())];
        const uint32_t v = map[pv];
        present.insert(pair_key(u, v));
        is.push_back(u);
        id.push_back(v);
        iwv.push_back((float)(1.0 / hypot(px[pu] - px[pv], py[pu] - py[pv])));
    }
    auto out_u32 = [](const std::vector<uint32_t> &v) {
        uint32_t *p = (uint32_t *)malloc(sizeof(uint32_t) * (v.size() ? v.size() : 1));
        if (p && !v.empty()) memcpy(p, v.data(), sizeof(uint32_t) * v.size());
        return p;
    };
    auto out_f32 = [](const std::vector<float> &v) {
        float *p = (float *)malloc(sizeof(float) * (v.size() ? v.size() : 1));
        if (p && !v.empty()) memcpy(p, v.data(), sizeof(float) * v.size());
        return p;
    };
    *n_out = nn;
    *src = out_u32(vs);
    *dst = out_u32(vd);
    *w = out_f32(vw);
    *n_ins_out = (uint32_t)is.size();
    *isrc = out_u32(is);
    *idst = out_u32(id);
    *iw = out_f32(iwv);
    return vs.size();
}

void dyg_synth_sample(uint64_t m, uint64_t k, uint64_t seed, uint64_t *out_idx) {
    if (k > m) k = m;
    SplitMix r(seed);
    if (k * 4 >= m) {
        std::vector<uint64_t> a(m);
        std::iota(a.begin(), a.end(), 0ull);
        for (uint64_t i = 0; i < k; ++i) {
            const uint64_t j = i + r.below(m - i);
            std::swap(a[i], a[j]);
            out_idx[i] = a[i];
        }
        return;
    }
    std::unordered_set<uint64_t> used;
    used.reserve((size_t)k * 2);
    uint64_t c = 0;
    while (c < k) {
        const uint64_t j = r.below(m);
        if (used.insert(j).second) out_idx[c++] = j;
    }
}

}  // extern "C"
