// io.cpp -- graph file readers: the reference drivers' input formats (host side).
//
//   MatrixMarket coordinate files, as the MST driver reads them
//     (getGraphInfo + mmapPopulateEdgeArray, MST/src/utils.cu:160-180, 896-1036):
//     '%' comment lines, a "rows cols nnz" header, then nnz lines "u v [w]"
//     with 1-based ids; an edge is stored (min - 1, max - 1, w); without
//     weights in the file, w = ((u - 1) * (v - 1) mod rows) + 1 in 32-bit
//     arithmetic.  Only decimal digits are parsed, as in the reference.
//   ECL binary CSR, as the CC driver reads it (readECLgraph, CC/graph.cu:90-121):
//     int64 n, int64 nnz, int64 offsets[n + 1], int32 cols[nnz].
//   Text edge lists, as the CC driver reads them (readEdgeList, CC/graph.cu:45-88):
//     "n m" then m directed lines "u v" (0-based); each undirected edge is
//     kept once, from its u < v line.
// phem_read_graph_pairs dispatches on the file extension the way the CC
// driver does (CC/graph.cu:25-43): ".edges", ".eg2" and ".txt" are edge
// lists; every other name is read as ECL binary (the reference's test
// `ext == ".egr" || ext == ".bin" || ".csr"` is always true).
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fcntl.h>
#include <string>
#include <sys/mman.h>
#include <sys/stat.h>
#include <thread>
#include <unistd.h>
#include <vector>

#include "../../include/phem.h"

namespace {

thread_local char g_io_error[256] = "";

phem_status io_error(phem_status st, const char *fmt, const char *path)
{
    snprintf(g_io_error, sizeof(g_io_error), fmt, path);
    return st;
}

// Read-only mapping of a whole file.
struct Mapped {
    const char *data = nullptr;
    size_t size = 0;
    int fd = -1;
    explicit Mapped(const char *path)
    {
        fd = open(path, O_RDONLY);
        if (fd < 0)
            return;
        struct stat sb;
        if (fstat(fd, &sb) != 0)
            return;
        size = (size_t)sb.st_size;
        if (size == 0) {
            data = "";
            return;
        }
        void *p = mmap(nullptr, size, PROT_READ, MAP_PRIVATE, fd, 0);
        if (p != MAP_FAILED)
            data = static_cast<const char *>(p);
    }
    ~Mapped()
    {
        if (data && size)
            munmap(const_cast<char *>(data), size);
        if (fd >= 0)
            close(fd);
    }
};

inline bool is_blank(char c) { return c == ' ' || c == '\t'; }

// Decimal digits at *p (stops at the first non-digit), 32-bit wrap-around.
inline uint32_t parse_u32(const char *&p, const char *end)
{
    uint32_t x = 0;
    while (p < end && *p >= '0' && *p <= '9')
        x = x * 10u + (uint32_t)(*p++ - '0');
    return x;
}

inline uint64_t parse_u64(const char *&p, const char *end)
{
    uint64_t x = 0;
    while (p < end && *p >= '0' && *p <= '9')
        x = x * 10u + (uint64_t)(*p++ - '0');
    return x;
}

inline void skip_blanks(const char *&p, const char *end)
{
    while (p < end && is_blank(*p))
        p++;
}

// Start of the line after the one containing p (or end).
inline const char *next_line(const char *p, const char *end)
{
    const void *nl = memchr(p, '\n', (size_t)(end - p));
    return nl ? static_cast<const char *>(nl) + 1 : end;
}

template <class F>
void parallel_for(uint64_t count, F &&f)
{
    unsigned T = std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
    if (count < (1u << 16))
        T = 1;
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < T; t++)
        pool.emplace_back([&, t] { f(count * t / T, count * (t + 1) / T); });
    for (auto &th : pool)
        th.join();
}

}  // namespace

extern "C" {

const char *phem_io_last_error(void) { return g_io_error; }

phem_status phem_read_mtx(const char *path, int generate_weights, phem_edge *out, uint64_t capacity, uint32_t *n_out,
                          uint64_t *m_out)
{
    if (!path || !n_out || !m_out)
        return io_error(PHEM_ERR_INVALID, "read_mtx: null argument%s", "");
    Mapped f(path);
    if (!f.data)
        return io_error(PHEM_ERR_INVALID, "read_mtx: cannot read %s", path);
    const char *p = f.data, *end = f.data + f.size;
    while (p < end && *p == '%')
        p = next_line(p, end);
    if (p >= end)
        return io_error(PHEM_ERR_INVALID, "read_mtx: %s has no size line", path);
    const char *q = p;
    skip_blanks(q, end);
    const uint64_t rows = parse_u64(q, end);
    skip_blanks(q, end);
    parse_u64(q, end);
    skip_blanks(q, end);
    const uint64_t nnz = parse_u64(q, end);
    if (rows == 0 || rows >= (1ull << 32))
        return io_error(PHEM_ERR_INVALID, "read_mtx: %s: bad vertex count", path);
    *n_out = (uint32_t)rows;
    *m_out = nnz;
    if (!out)
        return PHEM_OK;
    if (capacity < nnz)
        return io_error(PHEM_ERR_INVALID, "read_mtx: output too small for %s", path);
    p = next_line(p, end);
    // line starts of the data section (at most nnz lines are used)
    std::vector<const char *> starts;
    starts.reserve((size_t)std::min<uint64_t>(nnz, 1ull << 26));
    for (const char *s = p; s < end && starts.size() < nnz; s = next_line(s, end))
        starts.push_back(s);
    const uint32_t n32 = (uint32_t)rows;
    parallel_for(nnz, [&](uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; i++) {
            phem_edge e{0, 0, 0};  // a missing or empty line reads as a self-loop at vertex 0
            if (i < starts.size()) {
                const char *s = starts[i];
                const char *le = i + 1 < starts.size() ? starts[i + 1] : end;
                if (le - s > 1 || (le - s == 1 && *s != '\n')) {
                    skip_blanks(s, le);
                    const uint32_t u = parse_u32(s, le);
                    skip_blanks(s, le);
                    const uint32_t v = parse_u32(s, le);
                    uint32_t w;
                    if (generate_weights) {
                        w = ((u - 1u) * (v - 1u)) % n32 + 1u;
                    } else {
                        skip_blanks(s, le);
                        w = parse_u32(s, le);
                    }
                    e.u = (u > v ? v : u) - 1u;
                    e.v = (u > v ? u : v) - 1u;
                    e.w = w;
                }
            }
            out[i] = e;
        }
    });
    return PHEM_OK;
}

phem_status phem_read_ecl(const char *path, int64_t *offsets, uint32_t *cols, uint64_t cols_capacity, uint32_t *n_out,
                          uint64_t *nnz_out)
{
    if (!path || !n_out || !nnz_out)
        return io_error(PHEM_ERR_INVALID, "read_ecl: null argument%s", "");
    Mapped f(path);
    if (!f.data || f.size < 16)
        return io_error(PHEM_ERR_INVALID, "read_ecl: cannot read the sizes of %s", path);
    int64_t n = 0, nnz = 0;
    memcpy(&n, f.data, 8);
    memcpy(&nnz, f.data + 8, 8);
    if (n <= 0 || n >= (1ll << 31) || nnz < 0 || f.size < 16 + 8 * (uint64_t)(n + 1) + 4 * (uint64_t)nnz)
        return io_error(PHEM_ERR_INVALID, "read_ecl: %s is not an ECL CSR file of the sizes it states", path);
    *n_out = (uint32_t)n;
    *nnz_out = (uint64_t)nnz;
    if (!offsets || !cols)
        return PHEM_OK;
    if (cols_capacity < (uint64_t)nnz)
        return io_error(PHEM_ERR_INVALID, "read_ecl: output too small for %s", path);
    memcpy(offsets, f.data + 16, 8 * (size_t)(n + 1));
    memcpy(cols, f.data + 16 + 8 * (size_t)(n + 1), 4 * (size_t)nnz);
    return PHEM_OK;
}

phem_status phem_read_graph_pairs(const char *path, uint64_t *pairs, uint64_t capacity, uint32_t *n_out,
                                  uint64_t *m_out)
{
    if (!path || !n_out || !m_out)
        return io_error(PHEM_ERR_INVALID, "read_graph_pairs: null argument%s", "");
    const std::string name(path);
    const size_t dot = name.find_last_of('.');
    const std::string ext = dot == std::string::npos ? "" : name.substr(dot);
    if (ext == ".edges" || ext == ".eg2" || ext == ".txt") {
        Mapped f(path);
        if (!f.data)
            return io_error(PHEM_ERR_INVALID, "read_graph_pairs: cannot read %s", path);
        const char *p = f.data, *end = f.data + f.size;
        auto skip_space = [&] {
            while (p < end && (*p == ' ' || *p == '\t' || *p == '\n' || *p == '\r'))
                p++;
        };
        skip_space();
        const uint64_t n = parse_u64(p, end);
        skip_space();
        const uint64_t lines = parse_u64(p, end);
        if (n == 0 || n >= (1ull << 31))
            return io_error(PHEM_ERR_INVALID, "read_graph_pairs: %s: bad vertex count", path);
        *n_out = (uint32_t)n;
        uint64_t k = 0;
        for (uint64_t i = 0; i < lines; i++) {
            skip_space();
            if (p >= end)
                break;
            const uint32_t u = parse_u32(p, end);
            skip_space();
            const uint32_t v = parse_u32(p, end);
            if (u < v) {
                if (pairs) {
                    if (k >= capacity)
                        return io_error(PHEM_ERR_INVALID, "read_graph_pairs: output too small for %s", path);
                    pairs[k] = ((uint64_t)u << 32) | v;
                }
                k++;
            }
        }
        *m_out = k;
        return PHEM_OK;
    }
    uint32_t n = 0;
    uint64_t nnz = 0;
    phem_status st = phem_read_ecl(path, nullptr, nullptr, 0, &n, &nnz);
    if (st != PHEM_OK)
        return st;
    std::vector<int64_t> off(n + 1);
    std::vector<uint32_t> cols(nnz ? nnz : 1);
    st = phem_read_ecl(path, off.data(), cols.data(), nnz, &n, &nnz);
    if (st != PHEM_OK)
        return st;
    // csr_to_coo (CC/graph.cu:149-196): row-major, entries with row < col
    uint64_t k = 0;
    for (uint32_t i = 0; i < n; i++)
        for (int64_t j = off[i]; j < off[i + 1]; j++)
            if ((int32_t)i < (int32_t)cols[j]) {
                if (pairs) {
                    if (k >= capacity)
                        return io_error(PHEM_ERR_INVALID, "read_graph_pairs: output too small for %s", path);
                    pairs[k] = ((uint64_t)i << 32) | cols[j];
                }
                k++;
            }
    *n_out = n;
    *m_out = k;
    return PHEM_OK;
}

}  // extern "C"
