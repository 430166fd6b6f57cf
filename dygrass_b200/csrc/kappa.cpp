// kappa.cpp -- spectral quality of a sparsifier (include/dyg_eval.h): the
// relative condition number kappa(L_G, L_H) and the PCG iteration count, the
// two figures the reference's Julia evaluation reports (dyGRASS.jl:54-64,
// 361-362, 558-588).  Host only, FP64.
//
//   L_X      = Laplacian of X (off-diagonal -w, diagonal = weighted degree;
//              self-loops ignored) + offset * I (the reference adds 1e-6)
//   kappa    = largest eigenvalue of the pencil (L_G, L_H), by Lanczos in
//              the L_H inner product, each step solving with L_H
//   L_H      = P L D L^T P^T, eliminated in greedy minimum-degree order on the
//              graph itself (a sparsifier is a tree plus few edges: leaves and
//              chains eliminate without fill)
//   pcg      = conjugate-gradient iterations on L_G x = b (b of zero mean),
//              preconditioned by that factorization, until
//              ||r|| <= rtol * ||r_0||
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <queue>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/dyg_eval.h"

namespace dyg {
void set_error(const std::string &msg);
}

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
    double unit() { return ((double)(next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); }
    double normal() {   // Box-Muller
        const double u = unit(), v = unit();
        return sqrt(-2.0 * log(u)) * cos(6.283185307179586 * v);
    }
};

// Symmetric matrix in full CSR.
struct Csr {
    uint32_t n = 0;
    std::vector<uint64_t> rp;
    std::vector<uint32_t> ci;
    std::vector<double> v;
};

Csr laplacian(uint32_t n, uint64_t m, const uint32_t *s, const uint32_t *d, const float *w,
              double offset) {
    std::vector<double> diag(n, offset);
    std::vector<std::vector<std::pair<uint32_t, double>>> rows(n);
    for (uint64_t i = 0; i < m; ++i) {
        const uint32_t a = s[i], b = d[i];
        if (a == b) continue;
        const double x = (double)w[i];
        diag[a] += x;
        diag[b] += x;
        rows[a].emplace_back(b, -x);
        rows[b].emplace_back(a, -x);
    }
    Csr L;
    L.n = n;
    L.rp.assign((size_t)n + 1, 0);
    for (uint32_t r = 0; r < n; ++r) {
        auto &row = rows[r];
        std::sort(row.begin(), row.end(),
                  [](const auto &p, const auto &q) { return p.first < q.first; });
        bool diag_done = false;
        size_t k = 0;
        while (k < row.size()) {
            const uint32_t c = row[k].first;
            double sum = 0;
            while (k < row.size() && row[k].first == c) sum += row[k++].second;
            if (!diag_done && c > r) {
                L.ci.push_back(r);
                L.v.push_back(diag[r]);
                diag_done = true;
            }
            L.ci.push_back(c);
            L.v.push_back(sum);
        }
        if (!diag_done) {
            L.ci.push_back(r);
            L.v.push_back(diag[r]);
        }
        L.rp[r + 1] = L.ci.size();
        std::vector<std::pair<uint32_t, double>>().swap(row);
    }
    return L;
}

void spmv(const Csr &A, const std::vector<double> &x, std::vector<double> &y) {
    for (uint32_t r = 0; r < A.n; ++r) {
        double acc = 0;
        for (uint64_t j = A.rp[r]; j < A.rp[r + 1]; ++j) acc += A.v[j] * x[A.ci[j]];
        y[r] = acc;
    }
}

double dot(const std::vector<double> &a, const std::vector<double> &b) {
    double s = 0;
    for (size_t i = 0; i < a.size(); ++i) s += a[i] * b[i];
    return s;
}

// LDL^T by elimination on the matrix graph: the vertex of least current
// degree goes next; eliminating v subtracts a_iv a_jv / d_v from every pair
// of its remaining neighbours (the fill) and leaves column v of L.
struct Ldl {
    uint32_t n = 0;
    std::vector<uint32_t> order;                      // elimination order
    std::vector<double> dpiv;                         // pivots, by vertex
    std::vector<std::vector<std::pair<uint32_t, double>>> col;   // L(i, v) by vertex v
    uint64_t nnz = 0;

    bool factor(const Csr &A) {
        n = A.n;
        std::vector<std::unordered_map<uint32_t, double>> adj(n);
        std::vector<double> dg(n, 0.0);
        for (uint32_t r = 0; r < n; ++r)
            for (uint64_t j = A.rp[r]; j < A.rp[r + 1]; ++j) {
                if (A.ci[j] == r) dg[r] += A.v[j];
                else if (A.v[j] != 0.0) adj[r][A.ci[j]] += A.v[j];
            }
        std::vector<uint8_t> done(n, 0);
        using Item = std::pair<size_t, uint32_t>;
        std::priority_queue<Item, std::vector<Item>, std::greater<Item>> pq;
        for (uint32_t v = 0; v < n; ++v) pq.emplace(adj[v].size(), v);
        order.reserve(n);
        dpiv.assign(n, 0.0);
        col.assign(n, {});
        std::vector<std::pair<uint32_t, double>> nb;
        while (!pq.empty()) {
            const auto [deg, v] = pq.top();
            pq.pop();
            if (done[v] || deg != adj[v].size()) continue;
            const double dv = dg[v];
            if (!(dv > 0.0)) return false;
            done[v] = 1;
            order.push_back(v);
            dpiv[v] = dv;
            nb.assign(adj[v].begin(), adj[v].end());
            std::sort(nb.begin(), nb.end());
            auto &cv = col[v];
            cv.reserve(nb.size());
            for (const auto &[i, a] : nb) cv.emplace_back(i, a / dv);
            nnz += nb.size();
            for (size_t p = 0; p < nb.size(); ++p) {
                const uint32_t i = nb[p].first;
                const double ai = nb[p].second;
                adj[i].erase(v);
                dg[i] -= ai * ai / dv;
                for (size_t q = 0; q < nb.size(); ++q) {
                    if (q == p) continue;
                    auto it = adj[i].emplace(nb[q].first, 0.0).first;
                    it->second -= ai * nb[q].second / dv;
                }
            }
            for (const auto &e : nb) pq.emplace(adj[e.first].size(), e.first);
            std::unordered_map<uint32_t, double>().swap(adj[v]);
        }
        return order.size() == n;
    }

    // x = A^{-1} b
    void solve(const std::vector<double> &b, std::vector<double> &x) const {
        x = b;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t v = order[k];
            const double yv = x[v];
            for (const auto &[i, l] : col[v]) x[i] -= l * yv;
        }
        for (uint32_t k = 0; k < n; ++k) x[order[k]] /= dpiv[order[k]];
        for (uint32_t k = n; k-- > 0;) {
            const uint32_t v = order[k];
            double s = x[v];
            for (const auto &[i, l] : col[v]) s -= l * x[i];
            x[v] = s;
        }
    }
};

// Largest eigenvalue of the symmetric tridiagonal (a, b) by bisection on the
// Sturm count (Gershgorin bounds).
double tridiag_max(const std::vector<double> &a, const std::vector<double> &b) {
    const size_t k = a.size();
    double lo = a[0], hi = a[0];
    for (size_t i = 0; i < k; ++i) {
        const double r = (i ? fabs(b[i - 1]) : 0.0) + (i + 1 < k ? fabs(b[i]) : 0.0);
        lo = std::min(lo, a[i] - r);
        hi = std::max(hi, a[i] + r);
    }
    auto count_below = [&](double x) {   // eigenvalues < x
        size_t c = 0;
        double q = a[0] - x;
        if (q < 0) ++c;
        for (size_t i = 1; i < k; ++i) {
            const double den = q != 0.0 ? q : 1e-300;
            q = a[i] - x - b[i - 1] * b[i - 1] / den;
            if (q < 0) ++c;
        }
        return c;
    };
    for (int it = 0; it < 200 && hi - lo > 1e-15 * std::max(1.0, fabs(hi)); ++it) {
        const double mid = 0.5 * (lo + hi);
        if (count_below(mid) >= k) hi = mid;   // every eigenvalue is below mid
        else lo = mid;
    }
    return 0.5 * (lo + hi);
}

}  // namespace

extern "C" {

void dyg_kappa_opts_default(dyg_kappa_opts *o) {
    if (!o) return;
    o->offset = 1e-6;
    o->tol = 1e-10;
    o->max_iter = 300;
    o->pcg_max_iter = 10000;
    o->pcg_rtol = 1e-8;
    o->seed = 20251203ull;
}

dyg_status dyg_kappa(uint32_t n, uint64_t m_g, const uint32_t *g_src, const uint32_t *g_dst,
                     const float *g_w, uint64_t m_h, const uint32_t *h_src, const uint32_t *h_dst,
                     const float *h_w, const dyg_kappa_opts *opts, dyg_kappa_result *out) {
    if (!out || n == 0 || (m_g && (!g_src || !g_dst || !g_w)) ||
        (m_h && (!h_src || !h_dst || !h_w))) {
        dyg::set_error("dyg_kappa: NULL argument or empty graph");
        return DYG_EINVAL;
    }
    dyg_kappa_opts o;
    dyg_kappa_opts_default(&o);
    if (opts) o = *opts;
    for (uint64_t i = 0; i < m_g; ++i)
        if (g_src[i] >= n || g_dst[i] >= n || !(g_w[i] > 0.0f)) {
            dyg::set_error("dyg_kappa: G edge " + std::to_string(i) + " has a bad id or weight");
            return DYG_EINVAL;
        }
    for (uint64_t i = 0; i < m_h; ++i)
        if (h_src[i] >= n || h_dst[i] >= n || !(h_w[i] > 0.0f)) {
            dyg::set_error("dyg_kappa: H edge " + std::to_string(i) + " has a bad id or weight");
            return DYG_EINVAL;
        }
    memset(out, 0, sizeof *out);
    const Csr A = laplacian(n, m_g, g_src, g_dst, g_w, o.offset);
    const Csr B = laplacian(n, m_h, h_src, h_dst, h_w, o.offset);
    Ldl F;
    if (!F.factor(B)) {
        dyg::set_error("dyg_kappa: L_H + offset*I is not positive definite");
        return DYG_ERANGE;
    }
    out->factor_nnz = F.nnz;
    out->density = (double)m_h / (double)n;

    // Lanczos for the pencil (A, B) in the B inner product, full
    // reorthogonalisation while the basis fits in 1 GiB.
    SplitMix rng(o.seed);
    std::vector<double> v(n), vprev(n, 0.0), u(n), w(n), Bw(n);
    for (auto &x : v) x = rng.normal();
    spmv(B, v, Bw);
    double nb = sqrt(dot(v, Bw));
    for (auto &x : v) x /= nb;
    const bool full = (double)n * o.max_iter * 16.0 < 1073741824.0;
    std::vector<std::vector<double>> V, BV;
    std::vector<double> al, be;
    double theta = 0, theta_prev = -1;
    uint32_t stable = 0, it = 0;
    for (it = 0; it < o.max_iter; ++it) {
        spmv(A, v, u);
        const double alpha = dot(v, u);
        F.solve(u, w);
        for (uint32_t i = 0; i < n; ++i)
            w[i] -= alpha * v[i] + (be.empty() ? 0.0 : be.back() * vprev[i]);
        if (full) {
            spmv(B, v, Bw);
            V.push_back(v);
            BV.push_back(Bw);
            for (int pass = 0; pass < 2; ++pass)
                for (size_t q = 0; q < V.size(); ++q) {
                    const double c = dot(BV[q], w);
                    for (uint32_t i = 0; i < n; ++i) w[i] -= c * V[q][i];
                }
        }
        al.push_back(alpha);
        theta = tridiag_max(al, be);
        if (fabs(theta - theta_prev) <= o.tol * fabs(theta)) {
            if (++stable >= 3) break;
        } else {
            stable = 0;
        }
        theta_prev = theta;
        spmv(B, w, Bw);
        const double beta = sqrt(std::max(dot(w, Bw), 0.0));
        if (beta <= 1e-14 * std::max(1.0, fabs(theta))) break;   // invariant subspace
        be.push_back(beta);
        vprev.swap(v);
        for (uint32_t i = 0; i < n; ++i) v[i] = w[i] / beta;
    }
    out->kappa = theta;
    out->lanczos_iters = std::min(it + 1, o.max_iter);

    // PCG on A x = b, preconditioned by B's factorization
    std::vector<double> b(n), x(n), r(n), z(n), p(n), q(n);
    for (auto &e : b) e = rng.normal();
    double mean = 0;
    for (double e : b) mean += e;
    mean /= n;
    for (auto &e : b) e -= mean;
    for (auto &e : x) e = rng.normal();
    spmv(A, x, q);
    for (uint32_t i = 0; i < n; ++i) r[i] = b[i] - q[i];
    const double r0 = sqrt(dot(r, r));
    F.solve(r, z);
    p = z;
    double rz = dot(r, z), rn = r0;
    uint32_t k = 0;
    while (k < o.pcg_max_iter && rn > o.pcg_rtol * r0) {
        spmv(A, p, q);
        const double a = rz / dot(p, q);
        for (uint32_t i = 0; i < n; ++i) {
            x[i] += a * p[i];
            r[i] -= a * q[i];
        }
        ++k;
        rn = sqrt(dot(r, r));
        F.solve(r, z);
        const double rz2 = dot(r, z);
        const double bt = rz2 / rz;
        rz = rz2;
        for (uint32_t i = 0; i < n; ++i) p[i] = z[i] + bt * p[i];
    }
    out->pcg_iters = k;
    out->pcg_relres = r0 > 0 ? rn / r0 : 0.0;
    return DYG_OK;
}

}  // extern "C"
