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
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <thread>
#include <utility>
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


// ---- opt-in binary cache of parsed inputs (TGTP_INPUT_CACHE=1) ----------------------------------
// Parsing the text inputs dominates a run's wall time on large graphs (a 10^6-vertex eigen file is
// gigabytes of decimal text).  With TGTP_INPUT_CACHE=1 the loaders keep what they parsed in
// "<text file>.tgtpcache" beside it and reuse it while the text file's size and modification time
// are unchanged; a cache that cannot be written (read-only folder) is skipped silently.  Off by
// default: the reference writes nothing beside its inputs.
struct CacheHeader {
    char magic[8];
    uint64_t text_size;
    int64_t text_mtime_ns;
    uint64_t a, b;  // graph: n, m; eigens: n, omega
};

bool cache_enabled() {
    const char* e = std::getenv("TGTP_INPUT_CACHE");
    return e && std::string(e) == "1";
}

bool text_stamp(const char* path, uint64_t& size, int64_t& mtime) {
    struct stat st;
    if (stat(path, &st) != 0) return false;
    size = uint64_t(st.st_size);
    mtime = int64_t(st.st_mtim.tv_sec) * 1000000000LL + int64_t(st.st_mtim.tv_nsec);
    return true;
}

// Opens the cache of `path` if it matches the text file (magic, size, mtime); the header is read.
FILE* cache_open(const char* path, const char* magic, CacheHeader& h) {
    uint64_t size;
    int64_t mtime;
    if (!cache_enabled() || !text_stamp(path, size, mtime)) return nullptr;
    FILE* f = std::fopen((std::string(path) + ".tgtpcache").c_str(), "rb");
    if (!f) return nullptr;
    if (std::fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, magic, 8) != 0 ||
        h.text_size != size || h.text_mtime_ns != mtime) {
        std::fclose(f);
        return nullptr;
    }
    return f;
}

// Writes the cache of `path` through a temporary file renamed into place; any failure is ignored.
void cache_write(const char* path, const char* magic, uint64_t a, uint64_t b,
                 const std::vector<std::pair<const void*, size_t>>& parts) {
    CacheHeader h;
    std::memcpy(h.magic, magic, 8);
    h.a = a;
    h.b = b;
    if (!cache_enabled() || !text_stamp(path, h.text_size, h.text_mtime_ns)) return;
    const std::string dst = std::string(path) + ".tgtpcache";
    const std::string tmp = dst + ".tmp" + std::to_string(getpid());
    FILE* f = std::fopen(tmp.c_str(), "wb");
    if (!f) return;
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1;
    for (const auto& part : parts)
        ok = ok && (part.second == 0 || std::fwrite(part.first, part.second, 1, f) == 1);
    ok = std::fclose(f) == 0 && ok;
    if (!ok || std::rename(tmp.c_str(), dst.c_str()) != 0) std::remove(tmp.c_str());
}

// ---- parallel reader of decimal numbers ----------------------------------------------------------
// The eigen file of a 10^6-vertex graph holds ~1.3e8 numbers; read one after another they take
// tens of seconds.  read_numbers gives the result of the sequential reader (skip whitespace, take
// the longest decimal prefix, repeat; stop at the first spot that starts no number) on several
// threads: the text is cut into chunks at whitespace, so no number spans two chunks; a first pass
// counts the numbers of each chunk up to its first unreadable spot, a second pass converts each
// chunk's numbers with their global index k.  Numbers past the `need` first are not examined, as
// the sequential reader never reaches them.
struct NumberChunk {
    const char* begin;
    const char* end;
    uint64_t count = 0;    // numbers before the chunk's first unreadable spot (or its end)
    bool stopped = false;  // an unreadable spot was met
    uint64_t first = 0;    // global index of the chunk's first number
};

unsigned reader_threads(size_t bytes) {
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const size_t by_size = bytes / (size_t(4) << 20) + 1;  // at least 4 MB of text per thread
    return unsigned(std::min<size_t>({size_t(hw), size_t(32), by_size}));
}

template <class F>
void parallel_for(size_t count, unsigned threads, F&& body) {
    if (threads <= 1 || count <= 1) {
        for (size_t i = 0; i < count; ++i) body(i);
        return;
    }
    std::vector<std::thread> pool;
    const unsigned t = unsigned(std::min<size_t>(threads, count));
    pool.reserve(t);
    for (unsigned w = 0; w < t; ++w) {
        auto share = [&, w] {
            for (size_t i = w; i < count; i += t) body(i);
        };
        if (w + 1 == t) {  // the calling thread takes the last share
            share();
            break;
        }
        try {
            pool.emplace_back(share);
        } catch (...) {  // no thread to be had: this share runs here
            share();
        }
    }
    for (auto& th : pool) th.join();
}

// convert(k, token, len) converts number k (a NUL-terminated copy of its text) and returns false
// when the value is not acceptable.  Returns the index of the first number the sequential reader
// rejects or cannot find (the file's end included), or `need` when the first `need` numbers are
// all read and accepted.
template <class Convert>
uint64_t read_numbers(const char* data, size_t size, uint64_t need, Convert&& convert) {
    const char* end = data + size;
    const unsigned threads = reader_threads(size);
    std::vector<NumberChunk> chunks;
    const size_t target = std::max<size_t>(size / (size_t(threads) * 4) + 1, size_t(1) << 20);
    for (const char* b = data; b < end;) {
        const char* e = b + std::min(target, size_t(end - b));
        while (e < end && !is_ws(*e)) ++e;  // cut at whitespace
        chunks.push_back(NumberChunk{b, e});
        b = e;
    }
    parallel_for(chunks.size(), threads, [&](size_t c) {
        NumberChunk& ch = chunks[c];
        for (const char* p = ch.begin;;) {
            while (p < ch.end && is_ws(*p)) ++p;
            if (p >= ch.end) break;
            const size_t len = float_prefix(p, ch.end);
            if (!len) {
                ch.stopped = true;
                break;
            }
            ++ch.count;
            p += len;
        }
    });
    // limit: the index where the sequential reader stops (first unreadable spot, end of file or
    // `need`); chunks behind an unreadable spot start at or past it and are not converted
    uint64_t upto = 0, limit = UINT64_MAX;
    for (NumberChunk& ch : chunks) {
        ch.first = upto;
        upto += ch.count;
        if (ch.stopped && limit == UINT64_MAX) limit = upto;
    }
    limit = std::min({limit, upto, need});
    std::vector<uint64_t> bad(chunks.size(), UINT64_MAX);
    parallel_for(chunks.size(), threads, [&](size_t c) {
        const NumberChunk& ch = chunks[c];
        if (ch.first >= limit) return;
        std::string tok;
        uint64_t k = ch.first;
        for (const char* p = ch.begin; k < limit;) {
            while (p < ch.end && is_ws(*p)) ++p;
            if (p >= ch.end) break;
            const size_t len = float_prefix(p, ch.end);
            if (!len) break;
            tok.assign(p, len);
            p += len;
            if (!convert(k, tok.c_str())) {
                bad[c] = k;
                return;
            }
            ++k;
        }
    });
    uint64_t first_bad = limit;
    for (uint64_t b : bad) first_bad = std::min(first_bad, b);
    return first_bad;
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
        CacheHeader ch;
        if (FILE* cf = cache_open(path, "TGTPCSR1", ch)) {
            const uint64_t n = ch.a, m = ch.b;
            uint32_t* idx = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (n + 1)));
            uint32_t* adj = static_cast<uint32_t*>(std::malloc(sizeof(uint32_t) * (m ? m : 1)));
            const bool ok = idx && adj && std::fread(idx, sizeof(uint32_t), n + 1, cf) == n + 1 &&
                            (m == 0 || std::fread(adj, sizeof(uint32_t), m, cf) == m);
            std::fclose(cf);
            if (ok) {
                *idx_out = idx;
                *adj_out = adj;
                *n_out = n;
                *m_out = m;
                return;
            }
            std::free(idx);
            std::free(adj);
        }
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
        cache_write(path, "TGTPCSR1", n, m,
                    {{idx, sizeof(uint32_t) * (n + 1)}, {adj, sizeof(uint32_t) * m}});
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
        // the cache holds values, FP32 and FP64 vectors of the first `omega` pairs of an n-vertex
        // file, parsed as below
        CacheHeader ch;
        if (FILE* cf = cache_open(path, "TGTPEIG1", ch)) {
            bool ok = ch.a == n && ch.b == omega &&
                      std::fread(values, sizeof(double), omega, cf) == omega;
            const size_t cnt = size_t(n) * omega;
            if (ok) {
                if (vec_f32) ok = std::fread(vec_f32, sizeof(float), cnt, cf) == cnt;
                else ok = fseeko(cf, off_t(sizeof(float) * cnt), SEEK_CUR) == 0;
            }
            if (ok && vec_f64) ok = std::fread(vec_f64, sizeof(double), cnt, cf) == cnt;
            std::fclose(cf);
            if (ok) return;
        }
        MappedFile f(path);
        if (!f.ok()) fail(TGTP_ERR_IO, std::string("cannot open eigenpairs: ") + path);
        // with the cache on, both precisions are parsed so that one cache serves every form
        std::vector<float> keep32;
        std::vector<double> keep64;
        float* out32 = vec_f32;
        double* out64 = vec_f64;
        if (cache_enabled()) {
            if (!out32) {
                keep32.resize(size_t(n) * omega);
                out32 = keep32.data();
            }
            if (!out64) {
                keep64.resize(size_t(n) * omega);
                out64 = keep64.data();
            }
        }
        // number k of the file: k = i (n + 1) is eigenvalue i, the n after it its vector; the
        // vector entries are stored vertex-major (entry j of pair i at j * omega + i)
        const uint64_t row = n + 1;
        const uint64_t need = uint64_t(omega) * row;
        const uint64_t stop = read_numbers(f.data, f.size, need, [&](uint64_t k, const char* tok) {
            const uint64_t i = k / row, j = k % row;
            if (j == 0) {
                values[i] = std::strtod(tok, nullptr);
                return bool(std::isfinite(values[i]));
            }
            const size_t at = size_t(j - 1) * omega + i;
            bool ok = true;
            if (out64) {
                out64[at] = std::strtod(tok, nullptr);
                ok = std::isfinite(out64[at]);
            }
            if (out32 || !out64) {
                const float fl = std::strtof(tok, nullptr);
                if (out32) out32[at] = fl;
                ok = ok && std::isfinite(fl);
            }
            return ok;
        });
        if (stop < need)
            fail(TGTP_ERR_IO, std::string(stop % row == 0 ? "invalid eigenvalue in "
                                                           : "invalid eigenvector in ") + path);
        if (cache_enabled())
            cache_write(path, "TGTPEIG1", n, omega,
                        {{values, sizeof(double) * omega},
                         {out32, sizeof(float) * size_t(n) * omega},
                         {out64, sizeof(double) * size_t(n) * omega}});
    });
}

}  // extern "C"
