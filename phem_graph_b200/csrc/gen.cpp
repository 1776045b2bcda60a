// gen.cpp -- seeded synthetic graph generators (host side).
//
// The reference benchmarks on files that are not shipped with it; these
// generators stand in for them with seeded inputs of the same shapes.  Every
// random value is a pure function of (seed, stream tag, counter): SplitMix64
// (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
// OOPSLA 2014) evaluated at counter i, reduced to a range with Lemire's
// multiply-shift.  Output is therefore identical for any thread count, and the
// CPU oracle and the GPU tests see the same graphs.
//
// Edge formats produced:
//   - packed CC edges: uint64 (u << 32 | v) with u < v, the format
//     CC/graph.cu:76,176 builds;
//   - MSF edges: {u, v, w} uint32 records (MST/src/constants.h:15-19);
//   - symmetrised CSR: int64 offsets[n + 1], uint32 cols[2m], rows sorted by
//     column (the ECL .egr layout read by CC/graph.cu:90-121).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

#include "../../include/phem.h"

namespace {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ull;

inline uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Base of the stream `tag` under `seed`; value i of the stream is
// mix64(base + (i + 1) * gamma), i.e. the i-th output of a SplitMix64
// generator whose state starts at base.
inline uint64_t stream_base(uint64_t seed, uint64_t tag) { return mix64(seed * kGamma + tag); }
inline uint64_t stream_at(uint64_t base, uint64_t i) { return mix64(base + (i + 1) * kGamma); }
inline uint32_t lemire(uint32_t x, uint32_t range) { return (uint32_t)(((uint64_t)x * range) >> 32); }

constexpr uint64_t kTagER = 0x45522D45444745ull;    // "ER-EDGE"
constexpr uint64_t kTagRMAT = 0x524D41542D4544ull;  // "RMAT-ED"
constexpr uint64_t kTagW = 0x5745494748542Dull;     // "WEIGHT-"
constexpr uint64_t kTagRGG = 0x5247472D505453ull;   // "RGG-PTS"

int num_threads()
{
    unsigned t = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(t, 64u));
}

template <class F>
void parallel_ranges(uint64_t count, F &&f)
{
    int T = num_threads();
    if (count < (1u << 16))
        T = 1;
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++) {
        uint64_t lo = count * t / T, hi = count * (t + 1) / T;
        pool.emplace_back([&, t, lo, hi] { f(t, lo, hi); });
    }
    for (auto &th : pool)
        th.join();
}

// Generic two-pass "emit if" over draws [0, draws): produce(i, &value) returns
// whether draw i yields a value.  Output keeps draw order.
template <class P>
uint64_t emit_in_draw_order(uint64_t draws, uint64_t *out, P &&produce)
{
    int T = (draws < (1u << 16)) ? 1 : num_threads();
    std::vector<uint64_t> counts(T + 1, 0);
    std::vector<std::thread> pool;
    for (int t = 0; t < T; t++)
        pool.emplace_back([&, t] {
            uint64_t lo = draws * t / T, hi = draws * (t + 1) / T, c = 0, v;
            for (uint64_t i = lo; i < hi; i++)
                c += produce(i, &v) ? 1 : 0;
            counts[t + 1] = c;
        });
    for (auto &th : pool)
        th.join();
    pool.clear();
    for (int t = 0; t < T; t++)
        counts[t + 1] += counts[t];
    if (out)
        for (int t = 0; t < T; t++)
            pool.emplace_back([&, t] {
                uint64_t lo = draws * t / T, hi = draws * (t + 1) / T, k = counts[t], v;
                for (uint64_t i = lo; i < hi; i++)
                    if (produce(i, &v))
                        out[k++] = v;
            });
    for (auto &th : pool)
        th.join();
    return counts[T];
}

// Parallel LSD radix sort of keys that fit in `bits` bits, 11-bit digits.
void radix_sort(uint64_t *keys, uint64_t count, int bits)
{
    if (count < 2)
        return;
    constexpr int D = 11, B = 1 << D;
    std::vector<uint64_t> tmp(count);
    uint64_t *src = keys, *dst = tmp.data();
    int T = (count < (1u << 18)) ? 1 : num_threads();
    std::vector<uint64_t> hist((size_t)T * B);
    for (int shift = 0; shift < bits; shift += D) {
        std::fill(hist.begin(), hist.end(), 0);
        std::vector<std::thread> pool;
        for (int t = 0; t < T; t++)
            pool.emplace_back([&, t] {
                uint64_t lo = count * t / T, hi = count * (t + 1) / T;
                uint64_t *h = &hist[(size_t)t * B];
                for (uint64_t i = lo; i < hi; i++)
                    h[(src[i] >> shift) & (B - 1)]++;
            });
        for (auto &th : pool)
            th.join();
        pool.clear();
        uint64_t sum = 0;
        for (int d = 0; d < B; d++)
            for (int t = 0; t < T; t++) {
                uint64_t c = hist[(size_t)t * B + d];
                hist[(size_t)t * B + d] = sum;
                sum += c;
            }
        for (int t = 0; t < T; t++)
            pool.emplace_back([&, t] {
                uint64_t lo = count * t / T, hi = count * (t + 1) / T;
                uint64_t *h = &hist[(size_t)t * B];
                for (uint64_t i = lo; i < hi; i++)
                    dst[h[(src[i] >> shift) & (B - 1)]++] = src[i];
            });
        for (auto &th : pool)
            th.join();
        std::swap(src, dst);
    }
    if (src != keys)
        std::memcpy(keys, src, count * sizeof(uint64_t));
}

// Draw i of an R-MAT stream: `scale` quadrant choices, each from 32 random
// bits compared against integer thresholds; (lo, hi) with lo < hi, or false
// for a self-loop.
struct RmatDraw {
    uint32_t scale, words;
    uint64_t base, tA, tAB, tABC;
    RmatDraw(uint32_t s, double a, double b, double c, uint64_t seed)
        : scale(s), words((s + 1) / 2), base(stream_base(seed, kTagRMAT))
    {
        const double two32 = 4294967296.0;
        tA = (uint64_t)std::floor(a * two32);
        tAB = (uint64_t)std::floor((a + b) * two32);
        tABC = (uint64_t)std::floor((a + b + c) * two32);
    }
    bool operator()(uint64_t i, uint32_t *lo, uint32_t *hi) const
    {
        uint32_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; l++) {
            const uint64_t word = stream_at(base, i * words + l / 2);
            const uint64_t r = (l & 1) ? (word >> 32) : (word & 0xffffffffu);
            const uint32_t ubit = r >= tAB;                          // quadrants c, d
            const uint32_t vbit = (r >= tA && r < tAB) || r >= tABC;  // quadrants b, d
            u = (u << 1) | ubit;
            v = (v << 1) | vbit;
        }
        if (u == v)
            return false;
        *lo = u < v ? u : v;
        *hi = u < v ? v : u;
        return true;
    }
};

}  // namespace

extern "C" {

uint64_t phem_gen_mix64(uint64_t seed, uint64_t tag, uint64_t i)
{
    return stream_at(stream_base(seed, tag), i);
}

phem_status phem_gen_er(uint32_t n, uint64_t draws, uint64_t seed, uint64_t *out, uint64_t *out_m)
{
    if (n < 2 || !out_m)
        return PHEM_ERR_INVALID;
    const uint64_t base = stream_base(seed, kTagER);
    *out_m = emit_in_draw_order(draws, out, [&](uint64_t i, uint64_t *val) {
        uint64_t r = stream_at(base, i);
        uint32_t a = lemire((uint32_t)(r >> 32), n), b = lemire((uint32_t)r, n);
        if (a == b)
            return false;  // self-loops are dropped, duplicates kept
        uint32_t lo = a < b ? a : b, hi = a < b ? b : a;
        *val = ((uint64_t)lo << 32) | hi;
        return true;
    });
    return PHEM_OK;
}

phem_status phem_gen_rmat(uint32_t scale, uint64_t draws, double a, double b, double c, uint64_t seed,
                          uint64_t *out, uint64_t *out_m)
{
    if (scale < 1 || scale > 31 || !out_m || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
        return PHEM_ERR_INVALID;
    const RmatDraw draw(scale, a, b, c, seed);
    // Pairs are emitted compactly as (lo << scale | hi) so the sort runs on 2*scale bits.
    uint64_t m = emit_in_draw_order(draws, out, [&](uint64_t i, uint64_t *val) {
        uint32_t lo, hi;
        if (!draw(i, &lo, &hi))
            return false;
        *val = ((uint64_t)lo << scale) | hi;
        return true;
    });
    if (out) {
        radix_sort(out, m, 2 * (int)scale);
        const uint64_t mask = (1ull << scale) - 1;
        parallel_ranges(m, [&](int, uint64_t lo, uint64_t hi) {
            for (uint64_t i = lo; i < hi; i++)
                out[i] = ((out[i] >> scale) << 32) | (out[i] & mask);
        });
    }
    *out_m = m;
    return PHEM_OK;
}

phem_status phem_gen_weights(uint64_t m, uint64_t seed, uint32_t bits, uint32_t *w)
{
    if (!w || bits < 1 || bits > 31)
        return PHEM_ERR_INVALID;
    const uint64_t base = stream_base(seed, kTagW);
    const uint64_t mask = (1ull << bits) - 1;
    parallel_ranges(m, [&](int, uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; i++)
            w[i] = (uint32_t)(1 + (stream_at(base, i) & mask));
    });
    return PHEM_OK;
}

phem_status phem_pack_msf_edges(const uint64_t *pairs, const uint32_t *w, uint64_t m, phem_edge *out)
{
    if (!pairs || !out)
        return PHEM_ERR_INVALID;
    parallel_ranges(m, [&](int, uint64_t lo, uint64_t hi) {
        for (uint64_t i = lo; i < hi; i++) {
            out[i].u = (uint32_t)(pairs[i] >> 32);
            out[i].v = (uint32_t)pairs[i];
            out[i].w = w ? w[i] : 0;
        }
    });
    return PHEM_OK;
}

// Symmetrised CSR from pairs sorted by (u, v) with u < v: row x holds every
// partner of x, ascending (partners below x come from pairs (y, x), those above
// from pairs (x, y)), duplicates kept.  offsets has n + 1 entries, cols 2m.
phem_status phem_csr_from_sorted_pairs(const uint64_t *pairs, uint64_t m, uint32_t n, int64_t *offsets,
                                       uint32_t *cols)
{
    if (!pairs || !offsets || !cols)
        return PHEM_ERR_INVALID;
    std::vector<uint64_t> low(n + 1, 0), high(n + 1, 0);  // partners below / above each row
    for (uint64_t i = 0; i < m; i++) {
        uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
        if (u >= v || v >= n)
            return PHEM_ERR_INVALID;
        high[u]++;
        low[v]++;
    }
    offsets[0] = 0;
    for (uint32_t x = 0; x < n; x++)
        offsets[x + 1] = offsets[x] + (int64_t)(low[x] + high[x]);
    // fill cursors: partners below x land first, in increasing y because pairs are sorted by u
    std::vector<int64_t> lowpos(n), highpos(n);
    for (uint32_t x = 0; x < n; x++) {
        lowpos[x] = offsets[x];
        highpos[x] = offsets[x] + (int64_t)low[x];
    }
    for (uint64_t i = 0; i < m; i++) {
        uint32_t u = (uint32_t)(pairs[i] >> 32), v = (uint32_t)pairs[i];
        cols[lowpos[v]++] = u;
        cols[highpos[u]++] = v;
    }
    return PHEM_OK;
}

// Draws [first, first + count) of the same R-MAT stream as phem_gen_rmat,
// unsorted: packed (lo << 32 | hi), self-loops dropped, draw order kept.  A
// streaming consumer generates a huge graph batch by batch this way.
phem_status phem_gen_rmat_range(uint32_t scale, uint64_t first, uint64_t count, double a, double b, double c,
                                uint64_t seed, uint64_t *out, uint64_t *out_m)
{
    if (scale < 1 || scale > 31 || !out_m || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
        return PHEM_ERR_INVALID;
    const RmatDraw draw(scale, a, b, c, seed);
    *out_m = emit_in_draw_order(count, out, [&](uint64_t i, uint64_t *val) {
        uint32_t lo, hi;
        if (!draw(first + i, &lo, &hi))
            return false;
        *val = ((uint64_t)lo << 32) | hi;
        return true;
    });
    return PHEM_OK;
}

// 2-D random geometric k-nearest-neighbour graph.  Point i is
// (x, y) = (value 2i, value 2i + 1) of the stream, each scaled from its top 53
// bits to [0, 1).  Every point links to its k nearest other points (distance
// ties broken by the lower index); a pair chosen from both sides is emitted
// once.  Weights are floor(distance * 2^24) in double precision on the host
// (IEEE sqrt is correctly rounded, so the weights are the same everywhere).
// Pairs come out packed (min << 32 | max), sorted; out and w need n * k
// entries (NULL to count).
phem_status phem_gen_rgg(uint32_t n, uint32_t k, uint64_t seed, uint64_t *out, uint32_t *w, uint64_t *out_m)
{
    if (n < 2 || k < 1 || k >= n || !out_m)
        return PHEM_ERR_INVALID;
    const uint64_t base = stream_base(seed, kTagRGG);
    std::vector<double> px(n), py(n);
    for (uint32_t i = 0; i < n; i++) {
        px[i] = (double)(stream_at(base, 2ull * i) >> 11) * 0x1.0p-53;
        py[i] = (double)(stream_at(base, 2ull * i + 1) >> 11) * 0x1.0p-53;
    }
    // uniform grid with about four points per cell: the 3 x 3 block around a
    // point usually holds its 8 nearest neighbours
    const uint32_t side = std::max(1u, (uint32_t)std::sqrt((double)n / 4.0));
    std::vector<uint32_t> cell_start((size_t)side * side + 1, 0), cell_pts(n);
    auto cell_of = [&](uint32_t i) {
        const uint32_t cx = std::min(side - 1, (uint32_t)(px[i] * side));
        const uint32_t cy = std::min(side - 1, (uint32_t)(py[i] * side));
        return cy * side + cx;
    };
    for (uint32_t i = 0; i < n; i++)
        cell_start[cell_of(i) + 1]++;
    for (uint32_t c = 0; c < side * side; c++)
        cell_start[c + 1] += cell_start[c];
    {
        std::vector<uint32_t> fill(cell_start.begin(), cell_start.end() - 1);
        for (uint32_t i = 0; i < n; i++)
            cell_pts[fill[cell_of(i)]++] = i;
    }
    std::vector<uint64_t> pairs((uint64_t)n * k);
    parallel_ranges(n, [&](int, uint64_t lo, uint64_t hi) {
        std::vector<std::pair<double, uint32_t>> cand;
        for (uint64_t i = lo; i < hi; i++) {
            const int cx = (int)std::min(side - 1, (uint32_t)(px[i] * side));
            const int cy = (int)std::min(side - 1, (uint32_t)(py[i] * side));
            // grow the searched square ring by ring until k candidates are
            // strictly closer than anything outside it could be
            for (int ring = 1;; ring++) {
                cand.clear();
                for (int y = std::max(0, cy - ring); y <= std::min((int)side - 1, cy + ring); y++)
                    for (int x = std::max(0, cx - ring); x <= std::min((int)side - 1, cx + ring); x++) {
                        const uint32_t c = (uint32_t)y * side + (uint32_t)x;
                        for (uint32_t q = cell_start[c]; q < cell_start[c + 1]; q++) {
                            const uint32_t j = cell_pts[q];
                            if (j == i)
                                continue;
                            const double dx = px[i] - px[j], dy = py[i] - py[j];
                            cand.emplace_back(dx * dx + dy * dy, j);
                        }
                    }
                const bool all = ring >= (int)side;
                if (cand.size() < k && !all)
                    continue;
                std::partial_sort(cand.begin(), cand.begin() + std::min<size_t>(k, cand.size()), cand.end());
                const double reach = (double)ring / side;  // every point closer than this was searched
                if (all || cand[k - 1].first < reach * reach)
                    break;
            }
            for (uint32_t t = 0; t < k; t++) {
                const uint32_t j = cand[t].second;
                const uint32_t a = (uint32_t)i < j ? (uint32_t)i : j, b = (uint32_t)i < j ? j : (uint32_t)i;
                pairs[i * k + t] = ((uint64_t)a << 32) | b;
            }
        }
    });
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    *out_m = pairs.size();
    if (out)
        std::copy(pairs.begin(), pairs.end(), out);
    if (w)
        for (uint64_t e = 0; e < pairs.size(); e++) {
            const uint32_t a = (uint32_t)(pairs[e] >> 32), b = (uint32_t)pairs[e];
            const double dx = px[a] - px[b], dy = py[a] - py[b];
            w[e] = (uint32_t)std::floor(std::sqrt(dx * dx + dy * dy) * 16777216.0);
        }
    return PHEM_OK;
}

}  // extern "C"
