// Host-side readers of the reference's input files, with the reference's acceptance rules:
//   graph.txt               src/graph.h:29-97
//   sorted_eigens_<w>.txt   src/aesc.h:51-64
#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "internal.hpp"

namespace tgtp {
namespace {

struct MappedFile {
    const char* data = nullptr;
    size_t size = 0;
    int fd = -1;
    explicit MappedFile(const char* path) {
        fd = ::open(path, O_RDONLY);
        if (fd < 0) return;
        struct stat st;
        if (fstat(fd, &st) != 0) return;
        size = size_t(st.st_size);
        if (size == 0) {
            data = "";
            return;
        }
        void* p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (p == MAP_FAILED) {
            size = 0;
            return;
        }
        data = static_cast<const char*>(p);
    }
    ~MappedFile() {
        if (data && size) munmap(const_cast<char*>(data), size);
        if (fd >= 0) ::close(fd);
    }
    bool ok() const { return data != nullptr; }
};

inline bool is_ws(char c) {
    return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r';
}

// istream >> int64_t on [p, end): optional sign and at least one digit, no range wrap.
bool parse_i64(const char*& p, const char* end, int64_t& out) {
    while (p < end && is_ws(*p)) ++p;
    const char* q = p;
    bool neg = false;
    if (q < end && (*q == '+' || *q == '-')) {
        neg = *q == '-';
        ++q;
    }
    if (q >= end || *q < '0' || *q > '9') return false;
    unsigned __int128 v = 0;
    while (q < end && *q >= '0' && *q <= '9') {
        v = v * 10 + unsigned(*q - '0');
        if (v > (unsigned __int128)INT64_MAX + 1) return false;
        ++q;
    }
    if (!neg && v > (unsigned __int128)INT64_MAX) return false;
    out = neg ? int64_t(-(__int128)v) : int64_t(v);
    p = q;
    return true;
}

// Length of the decimal floating-point prefix at p ([+-]d*[.d*][(e|E)[+-]d+]), 0 if none.
size_t float_prefix(const char* p, const char* end) {
    const char* q = p;
    if (q < end && (*q == '+' || *q == '-')) ++q;
    size_t digits = 0;
    while (q < end && *q >= '0' && *q <= '9') ++q, ++digits;
    if (q < end && *q == '.') {
        ++q;
        while (q < end && *q >= '0' && *q <= '9') ++q, ++digits;
    }
    if (!digits) return 0;
    if (q < end && (*q == 'e' || *q == 'E')) {
        const char* r = q + 1;
        if (r < end && (*r == '+' || *r == '-')) ++r;
        const char* s = r;
        while (r < end && *r >= '0' && *r <= '9') ++r;
        if (r > s) q = r;
    }
    return size_t(q - p);
}

}  // namespace
}  // namespace tgtp

using namespace tgtp;

extern "C" {

tgtp_status tgtp_load_graph_txt(const char* path, uint32_t** idx_out, uint32_t** adj_out,
                                uint64_t* n_out, uint64_t* m_out) {
    return guarded([&] {
        if (!path || !idx_out || !adj_out || !n_out || !m_out)
            fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        *idx_out = nullptr;
        *adj_out = nullptr;
        MappedFile f(path);
        if (!f.ok()) fail(TGTP_ERR_IO, std::string("cannot open graph: ") + path);
        const char* p = f.data;
        const char* end = f.data + f.size;
        std::vector<uint32_t> src, dst;
        uint64_t n = 0;
        while (p < end) {
            const char* line_end = static_cast<const char*>(memchr(p, '\n', size_t(end - p)));
            if (!line_end) line_end = end;
            const char* q = p;
            // comment lines: first character '#' or '%' (src/graph.h:41-42)
            if (q < line_end && (*q == '#' || *q == '%')) {
                p = line_end + 1;
                continue;
            }
            const char* r = q;
            while (r < line_end && is_ws(*r)) ++r;
            if (r == line_end || *r == '#' || *r == '%') {  // src/graph.h:49-50
                p = line_end + 1;
                continue;
            }
            int64_t s, t;
            const char* cur = r;
            if (!parse_i64(cur, line_end, s) || !parse_i64(cur, line_end, t) || s < 0 || t < 0 ||
                s >= int64_t(UINT32_MAX) || t >= int64_t(UINT32_MAX)) {
                std::string line(q, line_end);
                fail(TGTP_ERR_IO, std::string("invalid edge in ") + path + ": " + line);
            }
            src.push_back(uint32_t(s));
            dst.push_back(uint32_t(t));
            n = std::max<uint64_t>(n, uint64_t(std::max(s, t)) + 1);
            p = line_end + 1;
        }
        if (src.empty()) fail(TGTP_ERR_IO, std::string("empty graph: ") + path);
        const uint64_t m = 2 * uint64_t(src.size());
        if (m > UINT32_MAX) fail(TGTP_ERR_INVALID_ARGUMENT, "graph exceeds CSR index capacity");
        // mirrored edges, rows sorted ascending, duplicates and self-loops kept (src/graph.h:58-95)
        uint32_t* idx = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (n + 1)));
        uint32_t* adj = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (m ? m : 1)));
        if (!idx || !adj) {
            std::free(idx);
            std::free(adj);
            fail(TGTP_ERR_OUT_OF_MEMORY, "host allocation failed");
        }
        std::vector<uint64_t> cnt(n + 1, 0);
        for (size_t e = 0; e < src.size(); ++e) {
            cnt[src[e]]++;
            cnt[dst[e]]++;
        }
        idx[0] = 0;
        for (uint64_t v = 0; v < n; ++v) idx[v + 1] = idx[v] + uint32_t(cnt[v]);
        std::vector<uint32_t> fill(idx, idx + n);
        for (size_t e = 0; e < src.size(); ++e) {
            adj[fill[src[e]]++] = dst[e];
            adj[fill[dst[e]]++] = src[e];
        }
        for (uint64_t v = 0; v < n; ++v) std::sort(adj + idx[v], adj + idx[v + 1]);
        *idx_out = idx;
        *adj_out = adj;
        *n_out = n;
        *m_out = m;
    });
}

tgtp_status tgtp_load_eigens_txt(const char* path, uint64_t n, uint32_t omega, double* values,
                                 float* vec_f32, double* vec_f64) {
    return guarded([&] {
        if (!path || !values) fail(TGTP_ERR_INVALID_ARGUMENT, "null argument");
        MappedFile f(path);
        if (!f.ok()) fail(TGTP_ERR_IO, std::string("cannot open eigenpairs: ") + path);
        const char* p = f.data;
        const char* end = f.data + f.size;
        std::string tok;
        auto next = [&](double* d, float* fl) -> bool {
            while (p < end && is_ws(*p)) ++p;
            const size_t len = float_prefix(p, end);
            if (!len) return false;
            tok.assign(p, len);
            p += len;
            if (d) *d = std::strtod(tok.c_str(), nullptr);
            if (fl) *fl = std::strtof(tok.c_str(), nullptr);
            return (!d || std::isfinite(*d)) && (!fl || std::isfinite(*fl));
        };
        for (uint32_t i = 0; i < omega; ++i) {
            if (!next(&values[i], nullptr))
                fail(TGTP_ERR_IO, std::string("invalid eigenvalue in ") + path);
            for (uint64_t j = 0; j < n; ++j) {
                double d;
                float fl;
                if (!next(vec_f64 ? &d : nullptr, vec_f32 ? &fl : (vec_f64 ? nullptr : &fl)))
                    fail(TGTP_ERR_IO, std::string("invalid eigenvector in ") + path);
                if (vec_f32) vec_f32[j * omega + i] = fl;
                if (vec_f64) vec_f64[j * omega + i] = d;
            }
        }
    });
}

}  // extern "C"
