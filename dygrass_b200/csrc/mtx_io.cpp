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

#include <string>
#include <vector>

#include "../../include/dyg_io.h"

namespace dyg {
void set_error(const std::string &msg);
}

namespace {

inline bool is_ws(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r'; }

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

}  // extern "C"
