// graphgen.cpp -- seeded synthetic graph generators (host C++).
//
// The reference is evaluated on an external 57-graph collection that is not
// available here; these generators produce the seeded stand-ins with the shapes
// the workloads are quoted on:
//   * planted-partition SBM (equal blocks, expected intra / inter degree),
//   * degree-corrected SBM with power-law degrees and power-law community sizes,
//     mixing parameter mu and optional FP32 weights uniform in [wlo, whi),
//   * R-MAT (Chakrabarti, Zhan, Faloutsos 2004) with quadrant probabilities a,b,c.
// Every output is a symmetric CSR with int64 row offsets, int32 columns sorted
// ascending within each row, no self-loops and no duplicate edges.  Results are
// identical for any thread count: each independent task draws from its own
// splitmix64 stream and rows are canonicalised by sorting.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

using i32 = int32_t;
using i64 = int64_t;
using u32 = uint32_t;
using u64 = uint64_t;

inline u64 mix64(u64 z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {  // splitmix64 stream
    u64 s;
    explicit Rng(u64 seed) : s(mix64(seed + 0x9E3779B97F4A7C15ull)) {}
    u64 next() { return mix64(s += 0x9E3779B97F4A7C15ull); }
    double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

int num_threads() {
    unsigned t = std::thread::hardware_concurrency();
    return t == 0 ? 4 : (int)std::min(t, 64u);
}

template <class F>
void parallel_tasks(i64 ntasks, F f) {
    int nt = (int)std::min<i64>(num_threads(), std::max<i64>(ntasks, 1));
    std::atomic<i64> next(0);
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&]() {
            while (true) {
                i64 k = next.fetch_add(1);
                if (k >= ntasks) break;
                f(k);
            }
        });
    for (auto& x : th) x.join();
}

struct Csr {
    i64 n = 0, nnz = 0;
    std::vector<i64> rowptr;
    std::vector<i32> col;
    std::vector<float> w;
};

// Symmetrise a list of undirected pairs into a canonical CSR.
void build_csr(i64 n, std::vector<std::vector<std::pair<i32, i32>>>& chunks, Csr& out) {
    std::vector<std::atomic<i64>> deg(n);
    for (i64 i = 0; i < n; i++) deg[i].store(0, std::memory_order_relaxed);
    parallel_tasks((i64)chunks.size(), [&](i64 k) {
        for (auto& e : chunks[k]) {
            deg[e.first].fetch_add(1, std::memory_order_relaxed);
            deg[e.second].fetch_add(1, std::memory_order_relaxed);
        }
    });
    std::vector<i64> rp(n + 1, 0);
    for (i64 i = 0; i < n; i++) rp[i + 1] = rp[i] + deg[i].load(std::memory_order_relaxed);
    std::vector<i32> col(rp[n]);
    std::vector<std::atomic<i64>> pos(n);
    for (i64 i = 0; i < n; i++) pos[i].store(rp[i], std::memory_order_relaxed);
    parallel_tasks((i64)chunks.size(), [&](i64 k) {
        for (auto& e : chunks[k]) {
            col[pos[e.first].fetch_add(1, std::memory_order_relaxed)] = e.second;
            col[pos[e.second].fetch_add(1, std::memory_order_relaxed)] = e.first;
        }
        std::vector<std::pair<i32, i32>>().swap(chunks[k]);
    });
    // sort + unique each row
    std::vector<i64> newdeg(n);
    const i64 RB = 4096;
    parallel_tasks((n + RB - 1) / RB, [&](i64 k) {
        i64 lo = k * RB, hi = std::min(n, lo + RB);
        for (i64 i = lo; i < hi; i++) {
            auto b = col.begin() + rp[i], e = col.begin() + rp[i + 1];
            std::sort(b, e);
            newdeg[i] = std::unique(b, e) - b;
        }
    });
    out.n = n;
    out.rowptr.assign(n + 1, 0);
    for (i64 i = 0; i < n; i++) out.rowptr[i + 1] = out.rowptr[i] + newdeg[i];
    out.nnz = out.rowptr[n];
    out.col.resize(out.nnz);
    parallel_tasks((n + RB - 1) / RB, [&](i64 k) {
        i64 lo = k * RB, hi = std::min(n, lo + RB);
        for (i64 i = lo; i < hi; i++)
            std::copy(col.begin() + rp[i], col.begin() + rp[i] + newdeg[i], out.col.begin() + out.rowptr[i]);
    });
}

// Symmetric pair weight in [lo, hi): a function of the unordered pair and the seed.
void pair_weights(Csr& g, u64 seed, float lo, float hi) {
    g.w.resize(g.nnz);
    const i64 RB = 4096;
    parallel_tasks((g.n + RB - 1) / RB, [&](i64 k) {
        i64 a = k * RB, b = std::min(g.n, a + RB);
        for (i64 i = a; i < b; i++)
            for (i64 j = g.rowptr[i]; j < g.rowptr[i + 1]; j++) {
                u64 x = (u64)std::min<i64>(i, g.col[j]), y = (u64)std::max<i64>(i, g.col[j]);
                u64 h = mix64(mix64(seed ^ 0xA5A5A5A5ull) ^ (x << 32 | y));
                double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
                g.w[j] = (float)(lo + (hi - lo) * u);
            }
    });
}

}  // namespace

extern "C" {

void* pggc_gen_free(void* h) {
    delete (Csr*)h;
    return nullptr;
}

void pggc_gen_dims(void* h, int64_t* n, int64_t* nnz, int* has_w) {
    auto* g = (Csr*)h;
    *n = g->n;
    *nnz = g->nnz;
    *has_w = g->w.empty() ? 0 : 1;
}

void pggc_gen_read(void* h, int64_t* rowptr, int32_t* col, float* w) {
    auto* g = (Csr*)h;
    if (rowptr) std::copy(g->rowptr.begin(), g->rowptr.end(), rowptr);
    if (col) std::copy(g->col.begin(), g->col.end(), col);
    if (w && !g->w.empty()) std::copy(g->w.begin(), g->w.end(), w);
}

// Planted-partition SBM: `blocks` equal blocks (vertex v in block v / (n/blocks)),
// expected intra-block degree deg_in and inter-block degree deg_out.  Pairs are
// sampled independently by geometric skipping inside each block pair.
void* pggc_gen_sbm(int64_t n, int64_t blocks, double deg_in, double deg_out, uint64_t seed, int weighted, float wlo,
                   float whi) {
    i64 bs = n / blocks;
    double p_in = deg_in / (double)(bs - 1);
    double p_out = deg_out / (double)(n - bs);
    i64 npairs = blocks * (blocks + 1) / 2;
    std::vector<std::vector<std::pair<i32, i32>>> chunks(npairs);
    parallel_tasks(npairs, [&](i64 task) {
        // task -> (a, b), a <= b
        i64 a = 0, rem = task;
        while (rem >= blocks - a) {
            rem -= blocks - a;
            a++;
        }
        i64 b = a + rem;
        i64 a0 = a * bs, a1 = (a == blocks - 1) ? n : a0 + bs;
        i64 b0 = b * bs, b1 = (b == blocks - 1) ? n : b0 + bs;
        double p = (a == b) ? p_in : p_out;
        if (p <= 0) return;
        Rng rng(mix64(seed) ^ mix64((u64)task + 1));
        i64 sa = a1 - a0, sb = b1 - b0;
        i64 total = (a == b) ? sa * (sa - 1) / 2 : sa * sb;
        double lq = std::log1p(-std::min(p, 0.999999999));
        auto& out = chunks[task];
        i64 idx = -1;
        while (true) {
            double u = rng.uniform();
            i64 skip = (p >= 0.999999999) ? 1 : 1 + (i64)std::floor(std::log(1.0 - u) / lq);
            idx += skip;
            if (idx >= total) break;
            i64 u0, v0;
            if (a == b) {
                // idx -> (r, c) with r < c over the upper triangle, row-major
                i64 r = (i64)((2.0 * sa - 1 - std::sqrt((2.0 * sa - 1) * (2.0 * sa - 1) - 8.0 * idx)) / 2.0);
                if (r < 0) r = 0;
                auto rowstart = [&](i64 rr) { return rr * (2 * sa - rr - 1) / 2; };
                while (r > 0 && rowstart(r) > idx) r--;
                while (rowstart(r + 1) <= idx) r++;
                i64 c = r + 1 + (idx - rowstart(r));
                u0 = a0 + r;
                v0 = a0 + c;
            } else {
                u0 = a0 + idx / sb;
                v0 = b0 + idx % sb;
            }
            out.push_back({(i32)u0, (i32)v0});
        }
    });
    auto* g = new Csr();
    build_csr(n, chunks, *g);
    if (weighted) pair_weights(*g, seed, wlo, whi);
    return g;
}

// Degree-corrected SBM.  Community sizes ~ power law (exponent comm_exp) on
// [cmin, cmax], assigned to contiguous vertex ranges.  Expected degrees theta ~
// Pareto(min_deg, deg_exp - 1) capped at max_deg, rescaled to mean mean_deg.
// Vertex u emits round(theta_u / 2) edge stubs; each stub's other end is drawn
// proportional to theta inside u's community with probability 1 - mu, else over
// the whole graph.
void* pggc_gen_dcsbm(int64_t n, double deg_exp, double min_deg, double mean_deg, double max_deg, double comm_exp,
                     int64_t cmin, int64_t cmax, double mu, uint64_t seed, int weighted, float wlo, float whi) {
    Rng rng(seed ^ 0x5eed0001ull);
    // communities
    std::vector<i64> cstart;
    i64 covered = 0;
    const double g1 = 1.0 - comm_exp;
    const double lo = std::pow((double)cmin, g1), hi = std::pow((double)cmax + 1.0, g1);
    while (covered < n) {
        double s = std::pow(lo + rng.uniform() * (hi - lo), 1.0 / g1);
        i64 sz = std::max<i64>(cmin, std::min<i64>(cmax, (i64)s));
        if (covered + sz > n) sz = n - covered;
        if (sz < cmin && !cstart.empty()) break;  // merge the remainder into the last community
        cstart.push_back(covered);
        covered += sz;
    }
    cstart.push_back(n);
    i64 ncomm = (i64)cstart.size() - 1;
    std::vector<i32> comm(n);
    for (i64 c = 0; c < ncomm; c++)
        for (i64 v = cstart[c]; v < cstart[c + 1]; v++) comm[v] = (i32)c;
    // expected degrees
    std::vector<double> theta(n);
    const double alpha = deg_exp - 1.0;
    {
        const i64 RB = 65536;
        parallel_tasks((n + RB - 1) / RB, [&](i64 k) {
            Rng r(mix64(seed ^ 0xD0D0ull) ^ mix64((u64)k + 7));
            for (i64 v = k * RB; v < std::min(n, (k + 1) * RB); v++) {
                double t = min_deg * std::pow(1.0 - r.uniform(), -1.0 / alpha);
                theta[v] = std::min(t, max_deg);
            }
        });
    }
    double s = 0;
    for (i64 v = 0; v < n; v++) s += theta[v];
    double scale = mean_deg / (s / (double)n);
    for (i64 v = 0; v < n; v++) theta[v] *= scale;
    // cumulative sums: global and (implicitly) per community since communities are contiguous
    std::vector<double> cum(n + 1, 0.0);
    for (i64 v = 0; v < n; v++) cum[v + 1] = cum[v] + theta[v];
    auto draw = [&](Rng& r, i64 lo_v, i64 hi_v) -> i64 {
        double t = cum[lo_v] + r.uniform() * (cum[hi_v] - cum[lo_v]);
        i64 pos = std::upper_bound(cum.begin() + lo_v + 1, cum.begin() + hi_v + 1, t) - cum.begin() - 1;
        return std::min(std::max(pos, lo_v), hi_v - 1);
    };
    const i64 RB = 16384;
    i64 ntask = (n + RB - 1) / RB;
    std::vector<std::vector<std::pair<i32, i32>>> chunks(ntask);
    parallel_tasks(ntask, [&](i64 k) {
        Rng r(mix64(seed ^ 0xE0E0ull) ^ mix64((u64)k + 11));
        auto& out = chunks[k];
        for (i64 u = k * RB; u < std::min(n, (k + 1) * RB); u++) {
            double half = theta[u] * 0.5;
            i64 stubs = (i64)half + (r.uniform() < (half - std::floor(half)) ? 1 : 0);
            i64 c = comm[u];
            for (i64 t = 0; t < stubs; t++) {
                i64 v = (r.uniform() < mu) ? draw(r, 0, n) : draw(r, cstart[c], cstart[c + 1]);
                if (v != u) out.push_back({(i32)u, (i32)v});
            }
        }
    });
    auto* g = new Csr();
    build_csr(n, chunks, *g);
    if (weighted) pair_weights(*g, seed, wlo, whi);
    return g;
}

// R-MAT: 2^scale vertices, edge_factor * 2^scale generated edges, quadrant
// probabilities a, b, c (d = 1 - a - b - c); self-loops and duplicates removed.
void* pggc_gen_rmat(int64_t scale, int64_t edge_factor, double a, double b, double c, uint64_t seed, int weighted,
                    float wlo, float whi) {
    i64 n = (i64)1 << scale;
    i64 m = edge_factor * n;
    const i64 RB = 1 << 20;
    i64 ntask = (m + RB - 1) / RB;
    std::vector<std::vector<std::pair<i32, i32>>> chunks(ntask);
    const double ab = a + b, abc = a + b + c;
    parallel_tasks(ntask, [&](i64 k) {
        Rng r(mix64(seed ^ 0x4A4A4Aull) ^ mix64((u64)k + 3));
        auto& out = chunks[k];
        i64 cnt = std::min(m, (k + 1) * RB) - k * RB;
        out.reserve(cnt);
        for (i64 e = 0; e < cnt; e++) {
            i64 u = 0, v = 0;
            for (i64 l = 0; l < scale; l++) {
                double x = r.uniform();
                int ub = 0, vb = 0;
                if (x < a) {
                } else if (x < ab) vb = 1;
                else if (x < abc) ub = 1;
                else {
                    ub = 1;
                    vb = 1;
                }
                u = (u << 1) | ub;
                v = (v << 1) | vb;
            }
            if (u != v) out.push_back({(i32)u, (i32)v});
        }
    });
    auto* g = new Csr();
    build_csr(n, chunks, *g);
    if (weighted) pair_weights(*g, seed, wlo, whi);
    return g;
}

}  // extern "C"
