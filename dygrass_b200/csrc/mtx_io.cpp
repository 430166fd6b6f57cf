// mtx_io.cpp -- edge-file reader/writer with the reference's conventions
// (include/dyg_io.h).
#include <errno.h>
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/dyg_io.h"

namespace dyg {
void set_error(const std::string &msg);
}

namespace {

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

// A read-only mapping of a whole file (empty files map to nothing).
struct Mapped {
    const char *p = nullptr;
    size_t n = 0;
    int fd = -1;
    ~Mapped() {
        if (p) munmap((void *)p, n);
        if (fd >= 0) close(fd);
    }
    dyg_status open_file(const char *path) {
        fd = open(path, O_RDONLY);
        if (fd < 0) {
            dyg::set_error(std::string("cannot open ") + path + ": " + strerror(errno));
            return DYG_EIO;
        }
        struct stat stt;
        if (fstat(fd, &stt) != 0) {
            dyg::set_error(std::string("cannot stat ") + path);
            return DYG_EIO;
        }
        n = (size_t)stt.st_size;
        if (n) {
            void *m = mmap(nullptr, n, PROT_READ, MAP_PRIVATE, fd, 0);
            if (m == MAP_FAILED) {
                n = 0;
                dyg::set_error(std::string("cannot mmap ") + path);
                return DYG_EIO;
            }
            p = (const char *)m;
        }
        return DYG_OK;
    }
};

// Parses the line at [b, e) (at most 254 characters, like the reference's
// 256-byte line buffer) with sscanf("%lf %lf %lf"); returns the count parsed,
// 0 for a longer line.
int scan3(const char *b, const char *e, double *x) {
    const size_t len = (size_t)(e - b);
    if (len >= 255) return 0;
    char line[256];
    memcpy(line, b, len);
    line[len] = 0;
    return sscanf(line, "%lf %lf %lf", &x[0], &x[1], &x[2]);
}

// Advances past a "line" the way the detector's first two steps do: to the
// next newline or tab, then past every newline and tab that follows.
size_t skip_record(const char *d, size_t i, size_t n) {
    while (i < n && d[i] != '\n' && d[i] != '\t') ++i;
    while (i < n && (d[i] == '\n' || d[i] == '\t')) ++i;
    return i;
}

const char *line_end(const char *d, size_t i, size_t n) {
    while (i < n && d[i] != '\n') ++i;
    return d + i;
}

// Vertex ids go through the reference's (vertex_t)double conversion.
inline uint32_t as_vertex(double v) { return (uint32_t)(long long)v; }

}  // namespace

extern "C" {

dyg_status dyg_mtx_read(const char *path, uint32_t id_offset, int weighted, uint64_t *n_edges,
                        uint32_t **src, uint32_t **dst, float **w, uint32_t *max_id) {
    if (!path || !n_edges || !src || !dst || (weighted && !w)) {
        dyg::set_error("dyg_mtx_read: NULL argument");
        return DYG_EINVAL;
    }
    *n_edges = 0;
    *src = *dst = nullptr;
    if (w) *w = nullptr;
    if (max_id) *max_id = 0;
    int fd = open(path, O_RDONLY);
    if (fd < 0) {
        dyg::set_error(std::string("cannot open ") + path + ": " + strerror(errno));
        return DYG_EIO;
    }
    struct stat stt;
    if (fstat(fd, &stt) != 0) {
        close(fd);
        dyg::set_error(std::string("cannot stat ") + path);
        return DYG_EIO;
    }
    const size_t size = (size_t)stt.st_size;
    const char *buf = nullptr;
    if (size) {
        void *m = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (m == MAP_FAILED) {
            close(fd);
            dyg::set_error(std::string("cannot mmap ") + path);
            return DYG_EIO;
        }
        buf = (const char *)m;
    }
    std::vector<uint32_t> vs, vd;
    std::vector<float> vw;
    size_t p = 0;
    uint32_t mx = 0;
    uint64_t line_no = 0;
    dyg_status rc = DYG_OK;
    std::string tok;
    while (p < size) {
        // one line
        size_t e = p;
        while (e < size && buf[e] != '\n') ++e;
        ++line_no;
        size_t q = p;
        while (q < e && is_ws(buf[q])) ++q;
        if (q < e && buf[q] != '%') {
            long long ids[2] = {0, 0};
            double wt = 1.0;
            int got = 0;
            const int want = weighted ? 3 : 2;
            while (q < e && got < want) {
                size_t t = q;
                while (t < e && !is_ws(buf[t])) ++t;
                tok.assign(buf + q, t - q);
                if (got < 2) ids[got] = atoll(tok.c_str());
                else wt = atof(tok.c_str());
                ++got;
                q = t;
                while (q < e && is_ws(buf[q])) ++q;
            }
            if (got < want) {
                dyg::set_error(std::string(path) + ":" + std::to_string(line_no) +
                               ": expected " + std::to_string(want) + " fields");
                rc = DYG_EIO;
                break;
            }
            const long long a = ids[0] - (long long)id_offset, b = ids[1] - (long long)id_offset;
            if (a < 0 || b < 0 || a > 0xFFFFFFFELL || b > 0xFFFFFFFELL) {
                dyg::set_error(std::string(path) + ":" + std::to_string(line_no) +
                               ": vertex id out of range for this file's base");
                rc = DYG_EIO;
                break;
            }
            vs.push_back((uint32_t)a);
            vd.push_back((uint32_t)b);
            if (weighted) vw.push_back((float)wt);
            if ((uint32_t)a > mx) mx = (uint32_t)a;
            if ((uint32_t)b > mx) mx = (uint32_t)b;
        }
        p = e + 1;
    }
    if (buf) munmap((void *)buf, size);
    close(fd);
    if (rc != DYG_OK) return rc;
    const uint64_t m = vs.size();
    *src = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    *dst = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    if (weighted) *w = (float *)malloc(sizeof(float) * (m ? m : 1));
    if (!*src || !*dst || (weighted && !*w)) {
        free(*src);
        free(*dst);
        if (weighted) free(*w);
        dyg::set_error("host allocation failed");
        return DYG_ENOMEM;
    }
    if (m) {
        memcpy(*src, vs.data(), sizeof(uint32_t) * m);
        memcpy(*dst, vd.data(), sizeof(uint32_t) * m);
        if (weighted) memcpy(*w, vw.data(), sizeof(float) * m);
    }
    *n_edges = m;
    if (max_id) *max_id = mx;
    return DYG_OK;
}

void dyg_mtx_free(void *p) { free(p); }

dyg_status dyg_mtx_write(const char *path, int append, uint64_t n_edges, const uint32_t *src,
                         const uint32_t *dst, const float *w, uint32_t id_offset) {
    FILE *f = fopen(path, append ? "a" : "w");
    if (!f) {
        dyg::set_error(std::string("cannot open ") + path + " for writing: " + strerror(errno));
        return DYG_EIO;
    }
    char line[96];
    for (uint64_t i = 0; i < n_edges; ++i) {
        int k;
        if (w)
            k = snprintf(line, sizeof line, "%llu %llu %g\n",
                         (unsigned long long)src[i] + id_offset,
                         (unsigned long long)dst[i] + id_offset, (double)w[i]);
        else
            k = snprintf(line, sizeof line, "%llu %llu\n", (unsigned long long)src[i] + id_offset,
                         (unsigned long long)dst[i] + id_offset);
        if (fwrite(line, 1, (size_t)k, f) != (size_t)k) {
            fclose(f);
            dyg::set_error(std::string("write failed: ") + path);
            return DYG_EIO;
        }
    }
    if (fclose(f) != 0) {
        dyg::set_error(std::string("close failed: ") + path);
        return DYG_EIO;
    }
    return DYG_OK;
}

// Restates auto_detect_graph_info (dynamic_update/functions.cpp:35-291):
//  - leading lines starting with '%' are header lines (each ends at a newline
//    or a tab, functions.cpp:59-70);
//  - the first other line is a dimensions line when it holds three numbers
//    "n n m" with m an integer > 1, n*n > m and m >= n - 1 (96-110); it is
//    skipped even if its n later disagrees with the ids (246-258);
//  - the next line decides weighted (three numbers) or not (two) (139-170);
//  - a later line with a negative third number marks a Laplacian (207-211);
//  - the file is triangular unless the first off-diagonal edge after the
//    first line appears again, in either orientation, on a later line (214-226);
//  - the smallest id (0 or 1) is the base (237-244).
dyg_status dyg_mtx_detect(const char *path, dyg_mtx_info *info) {
    if (!path || !info) {
        dyg::set_error("dyg_mtx_detect: NULL argument");
        return DYG_EINVAL;
    }
    Mapped f;
    dyg_status rc = f.open_file(path);
    if (rc != DYG_OK) return rc;
    const char *d = f.p;
    const size_t n = f.n;
    dyg_mtx_info r;
    memset(&r, 0, sizeof r);
    uint32_t vmax = 0, vmin = 1u << 30;
    size_t pos = 0;
    while (pos < n && d[pos] == '%') {
        r.has_header = 1;
        r.skip_lines++;
        pos = skip_record(d, pos, n);
    }
    // first non-header line
    double x[3] = {0, 0, 0};
    size_t cur = pos;
    pos = skip_record(d, pos, n);
    int k = scan3(d + cur, line_end(d, cur, n), x);
    double dims = 0;
    if (k == 3 && x[2] == (double)(long)x[2] && x[2] > 1 && x[0] == x[1] && x[0] * x[1] > x[2] &&
        x[2] >= x[0] - 1) {
        r.has_dimensions = 1;
        dims = x[0];
        r.skip_lines++;
    }
    if (!r.has_dimensions) {
        if (k < 2) {
            dyg::set_error(std::string(path) + ": the first data line does not hold two numbers");
            return DYG_EIO;
        }
        vmax = std::max(vmax, as_vertex(x[0]));
        vmin = std::min(vmin, as_vertex(x[0]));
        vmax = std::max(vmax, as_vertex(x[1]));
        vmin = std::min(vmin, as_vertex(x[1]));
    }
    // the line that decides the weight column
    bool loaded = false, checked = false;
    double ea = 0, eb = 0;
    r.triangular = 1;
    cur = pos;
    pos = skip_record(d, pos, n);
    k = scan3(d + cur, line_end(d, cur, n), x);
    if (k == 3) {
        r.weighted = 1;
        if (x[0] != x[1]) {
            ea = std::max(x[0], x[1]);
            eb = std::min(x[0], x[1]);
            loaded = true;
        }
    } else if (k != 2) {
        dyg::set_error(std::string(path) + ": invalid line format (expected 2 or 3 numbers)");
        return DYG_EIO;
    }
    vmax = std::max(vmax, as_vertex(x[0]));
    vmin = std::min(vmin, as_vertex(x[0]));
    vmax = std::max(vmax, as_vertex(x[1]));
    vmin = std::min(vmin, as_vertex(x[1]));
    // every later line
    while (pos < n) {
        size_t c = pos;
        while (c < n && (d[c] == ' ' || d[c] == '\t')) ++c;
        if (c >= n) break;
        {
            // ids of the line's first two numbers (strtod, as the reference)
            char *e1 = nullptr, *e2 = nullptr;
            const double a = strtod(d + c, &e1);
            if (e1 > d + c) {
                const double b = strtod(e1, &e2);
                if (e2 > e1) {
                    vmax = std::max(vmax, as_vertex(a));
                    vmin = std::min(vmin, as_vertex(a));
                    vmax = std::max(vmax, as_vertex(b));
                    vmin = std::min(vmin, as_vertex(b));
                }
            }
        }
        const char *le = line_end(d, c, n);
        const size_t len = (size_t)(le - (d + c));
        if (len > 0 && len < 255) {
            char line[256];
            memcpy(line, d + c, len);
            line[len] = 0;
            if (r.weighted) {
                k = sscanf(line, "%lf %lf %lf", &x[0], &x[1], &x[2]);
                if (k >= 3 && x[2] < 0) r.laplacian = 1;
            } else {
                k = sscanf(line, "%lf %lf", &x[0], &x[1]);
            }
            if (k >= 2) {
                if (!loaded && x[0] != x[1]) {
                    ea = std::max(x[0], x[1]);
                    eb = std::min(x[0], x[1]);
                    loaded = true;
                } else if (!checked && loaded) {
                    if (std::max(x[0], x[1]) == ea && std::min(x[0], x[1]) == eb) {
                        r.triangular = 0;
                        checked = true;
                    }
                }
            }
        }
        while (pos < n && d[pos] != '\n') ++pos;
        ++pos;
        while (pos < n && d[pos] == '\n') ++pos;
    }
    if (vmin == 1) {
        r.base = 1;
    } else if (vmin == 0) {
        r.base = 0;
    } else {
        dyg::set_error(std::string(path) + ": vertex ids are neither 0- nor 1-based");
        return DYG_EIO;
    }
    if (r.has_dimensions && (double)vmax + (r.base ? 0.0 : 1.0) != dims) r.has_dimensions = 0;
    r.v_max = vmax;
    r.v_min = vmin;
    *info = r;
    return DYG_OK;
}

// Reads the records the way the mixed updater's CSRGraph constructor does
// (dynamic_update/functions.cpp:308-587): skip info.skip_lines lines, then
// whitespace-separated "src dst [w]" records (w = 1 without a weight column),
// ids minus the base; a Laplacian's diagonal records are dropped and its
// weights negated.
dyg_status dyg_mtx_read_auto(const char *path, dyg_mtx_info *info, uint64_t *n_records,
                             uint32_t **src, uint32_t **dst, float **w) {
    if (!path || !info || !n_records || !src || !dst || !w) {
        dyg::set_error("dyg_mtx_read_auto: NULL argument");
        return DYG_EINVAL;
    }
    *n_records = 0;
    *src = *dst = nullptr;
    *w = nullptr;
    dyg_status rc = dyg_mtx_detect(path, info);
    if (rc != DYG_OK) return rc;
    Mapped f;
    rc = f.open_file(path);
    if (rc != DYG_OK) return rc;
    const char *d = f.p;
    const size_t n = f.n;
    size_t pos = 0;
    for (int64_t skipped = 0; skipped < info->skip_lines && pos < n;)
        if (d[pos++] == '\n') ++skipped;
    auto is_sep = [](char c) { return c == ' ' || c == '\n' || c == '\t'; };
    std::vector<uint32_t> vs, vd;
    std::vector<float> vw;
    std::string tok;
    auto next_token = [&](size_t &i) -> const char * {
        const char *t = d + i;
        size_t j = i;
        while (j < n && !is_sep(d[j])) ++j;
        tok.assign(t, j - i);
        while (j < n && is_sep(d[j])) ++j;
        i = j;
        return tok.c_str();
    };
    while (pos < n) {
        const long a = atol(next_token(pos)) - info->base;
        const long b = pos < n ? atol(next_token(pos)) - info->base : -1;
        float wt = 1.0f;
        if (info->weighted && pos < n) {
            wt = (float)atof(next_token(pos));
            if (info->laplacian) wt = -wt;
        }
        if (a < 0 || b < 0) {
            dyg::set_error(std::string(path) + ": record " + std::to_string(vs.size() + 1) +
                           " has an id below the base");
            return DYG_EIO;
        }
        if (info->laplacian && a == b) continue;
        vs.push_back((uint32_t)a);
        vd.push_back((uint32_t)b);
        vw.push_back(wt);
    }
    const size_t m = vs.size();
    *src = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    *dst = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    *w = (float *)malloc(sizeof(float) * (m ? m : 1));
    if (!*src || !*dst || !*w) {
        free(*src); free(*dst); free(*w);
        *src = *dst = nullptr;
        *w = nullptr;
        dyg::set_error("host allocation failed");
        return DYG_ENOMEM;
    }
    if (m) {
        memcpy(*src, vs.data(), sizeof(uint32_t) * m);
        memcpy(*dst, vd.data(), sizeof(uint32_t) * m);
        memcpy(*w, vw.data(), sizeof(float) * m);
    }
    *n_records = m;
    return DYG_OK;
}

// Restates EdgeStream::autoDetectWeightExist and loadBatchFromFile
// (dynamic_update/functions.cpp:717-838): the first line decides the weight
// column (three numbers: weighted, two: not; a '%' line or anything else is
// an error); then whitespace-separated records "src dst [w]", ids minus
// `base`, weight 1 without the column.
dyg_status dyg_stream_read(const char *path, uint32_t base, uint64_t *n_records,
                           uint32_t **src, uint32_t **dst, float **w, int32_t *weighted) {
    if (!path || !n_records || !src || !dst || !w) {
        dyg::set_error("dyg_stream_read: NULL argument");
        return DYG_EINVAL;
    }
    *n_records = 0;
    *src = *dst = nullptr;
    *w = nullptr;
    Mapped f;
    dyg_status rc = f.open_file(path);
    if (rc != DYG_OK) return rc;
    const char *d = f.p;
    const size_t n = f.n;
    if (n == 0) {
        dyg::set_error(std::string(path) + ": cannot read the first line");
        return DYG_EIO;
    }
    if (d[0] == '%') {
        dyg::set_error(std::string(path) + ": comment lines are not supported in stream files");
        return DYG_EIO;
    }
    const std::string first(d, line_end(d, 0, n));
    double x[3];
    const int k = sscanf(first.c_str(), "%lf %lf %lf", &x[0], &x[1], &x[2]);
    if (k != 2 && k != 3) {
        dyg::set_error(std::string(path) + ": invalid first line (expected 2 or 3 numbers)");
        return DYG_EIO;
    }
    const bool wt = k == 3;
    if (weighted) *weighted = wt ? 1 : 0;
    auto is_sep = [](char c) { return c == ' ' || c == '\n' || c == '\t'; };
    std::vector<std::string> toks;
    for (size_t i = 0; i < n;) {
        while (i < n && is_sep(d[i])) ++i;
        if (i >= n) break;
        size_t j = i;
        while (j < n && !is_sep(d[j])) ++j;
        toks.emplace_back(d + i, j - i);
        i = j;
    }
    const size_t per = wt ? 3 : 2;
    const size_t m = toks.size() / per;
    *src = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    *dst = (uint32_t *)malloc(sizeof(uint32_t) * (m ? m : 1));
    *w = (float *)malloc(sizeof(float) * (m ? m : 1));
    if (!*src || !*dst || !*w) {
        free(*src); free(*dst); free(*w);
        *src = *dst = nullptr;
        *w = nullptr;
        dyg::set_error("host allocation failed");
        return DYG_ENOMEM;
    }
    for (size_t r = 0; r < m; ++r) {
        const long a = atol(toks[r * per].c_str()) - (long)base;
        const long b = atol(toks[r * per + 1].c_str()) - (long)base;
        if (a < 0 || b < 0) {
            free(*src); free(*dst); free(*w);
            *src = *dst = nullptr;
            *w = nullptr;
            dyg::set_error(std::string(path) + ": record " + std::to_string(r + 1) +
                           " has an id below the base");
            return DYG_EIO;
        }
        (*src)[r] = (uint32_t)a;
        (*dst)[r] = (uint32_t)b;
        (*w)[r] = wt ? (float)atof(toks[r * per + 2].c_str()) : 1.0f;
    }
    *n_records = m;
    return DYG_OK;
}

uint32_t dyg_stream_op_from_name(const char *name, uint32_t prev_op) {
    if (!name) return prev_op;
    if (strstr(name, "insert") || strstr(name, "inc")) return DYG_STREAM_INSERT;
    if (strstr(name, "delete") || strstr(name, "dec")) return DYG_STREAM_DELETE;
    return prev_op;
}

// Snapshot of a device graph in the mixed updater's save format
// (GPU_Dual_Graph::save_result, dynamic_update/gpu_graph.cuh:725-763): one
// line "u+1 v+1 w" per undirected edge, here sorted by (u, v) with u <= v and
// the weight of u's first slot holding v (the reference writes its hash map
// in iteration order).
dyg_status dyg_graph_save(dyg_graph *g, const char *path) {
    if (!g || !path) {
        dyg::set_error("dyg_graph_save: NULL argument");
        return DYG_EINVAL;
    }
    uint32_t n = 0;
    uint64_t slots = 0;
    dyg_status s = dyg_graph_info(g, &n, &slots, nullptr, nullptr);
    if (s) return s;
    std::vector<uint64_t> rp((size_t)n + 1);
    std::vector<uint32_t> col(slots ? slots : 1);
    std::vector<float> w(slots ? slots : 1);
    s = dyg_graph_export(g, rp.data(), col.data(), w.data(), slots);
    if (s) return s;
    struct E {
        uint32_t u, v;
        float w;
    };
    std::vector<E> e;
    for (uint32_t u = 0; u < n; ++u)
        for (uint64_t j = rp[u]; j < rp[u + 1]; ++j)
            if (col[j] >= u) e.push_back({u, col[j], w[j]});
    std::stable_sort(e.begin(), e.end(), [](const E &a, const E &b) {
        return a.u != b.u ? a.u < b.u : a.v < b.v;
    });
    std::vector<uint32_t> ou, ov;
    std::vector<float> ow;
    for (size_t i = 0; i < e.size(); ++i) {
        if (i && e[i].u == e[i - 1].u && e[i].v == e[i - 1].v) continue;   // self-loop: 2 slots
        ou.push_back(e[i].u);
        ov.push_back(e[i].v);
        ow.push_back(e[i].w);
    }
    return dyg_mtx_write(path, 0, ou.size(), ou.data(), ov.data(), ow.data(), 1);
}

}  // extern "C"
