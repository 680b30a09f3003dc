// pggc_oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU restatement of the PGGC clustering hot path (local-move sweep, hashed
// contraction, Leiden refinement, degree-bucket ordering, and the multilevel
// V-cycles that drive them).  It is the parity oracle for the CUDA library in
// pennsylvaniagpugraphclustering_b200/: only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline / reference leg may load it, and never as the thing
// measured or shipped.
//
// Every function cites the reference file:line it restates (paths relative to
// the reference project root).  The reference is non-deterministic (hash slot
// order, atomics order, std::random_device seeds), so this restatement pins a
// canonical form of each of those choices; the CUDA library implements the same
// canonical form, which is what makes GPU-vs-oracle parity bit-exact:
//
//  * DeltaQ argmax ties go to the smallest cluster id (team-path rule,
//    src/local_mover.cpp:557-561); a real destination beats NEW_PART (thread
//    path, src/local_mover.cpp:506-512).
//  * FP32 gain arithmetic is kept operation by operation (no FMA contraction),
//    including the int->float conversions the reference performs implicitly.
//  * Floating-point accumulations that the reference does in FP32 (afterburner
//    change, strict prefix) are done in FP64 in a fixed association:
//      - per-vertex edge sums: 32 lane-strided sequential partial sums combined
//        by an xor butterfly (1024 thread-strided partials, butterfly per warp,
//        butterfly over warps for vertices of degree >= 15000);
//      - array reductions / scans: groups of 32 reduced by xor butterfly /
//        scanned Kogge-Stone, recursively over group totals.
//  * Weight sums that the reference keeps in int32 are int64 (integer graphs) or
//    FP64 (FP32-weighted graphs, which the reference cannot represent).
//  * Random picks use MurmurHash3_x86_32 of the 4-byte key with seed 0 (the hash
//    behind Kokkos::pod_hash, used at src/leidenR.cpp:37,302-303,406-407,421,484);
//    seeds come from an explicit splitmix64 stream instead of std::random_device.
//  * Leiden in-cluster order ties are broken by vertex id (the reference leaves
//    them to KokkosKernels sort_crs_matrix, src/leidenR.cpp:75).
//  * Coarse CSR rows are sorted by column (the reference emits hash-slot order,
//    src/contract.cpp:310-328).
//
// Built by oracle/Makefile into oracle/_build/libpggc_oracle.so.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <deque>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace orc {

using i32 = int32_t;
using i64 = int64_t;
using u32 = uint32_t;
using u64 = uint64_t;

// src/local_mover.cpp:74-80
constexpr float OBJ_MIN = std::numeric_limits<float>::lowest();
constexpr i32 NULL_PART = -1;
constexpr i32 NO_MOVE = -3;
constexpr i32 NEW_PART = -4;
constexpr float AFTERBURNER_EPS = 0.1f;
// Test switch: 0 (default) sums the afterburner's change and the strict
// prefix's gains canonically in FP64, as the CUDA library does; 1 accumulates
// them in FP32 in the reference's order with its separately rounded updates
// (src/local_mover.cpp:145-204, 318-326), to compare this oracle with the
// reference's own code (oracle/_ref) step by step.
static int g_afterburner_reference_order = 0;
// src/header/ordering.h:17-19
constexpr i64 MID_CUTOFF = 64;
constexpr i64 LARGE_CUTOFF = 128;
constexpr i64 MASSIVE_CUTOFF = 15000;
// src/leidenR.cpp:38-39
constexpr i32 ORD_MAX = std::numeric_limits<i32>::max();
constexpr i32 SPLIT = 1000000000;

// src/local_mover.cpp:82-87 (Marsaglia xorshift32, 13/17/5)
inline u32 xorshift32(u32 x) {
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    return x;
}

inline u32 rotl32(u32 x, int r) { return (x << r) | (x >> (32 - r)); }

// MurmurHash3_x86_32 (Appleby, public domain) of one 4-byte little-endian key,
// seed 0: the published algorithm behind Kokkos::pod_hash<int32_t>.
inline u32 murmur3_32(u32 key) {
    const u32 c1 = 0xcc9e2d51u, c2 = 0x1b873593u;
    u32 h = 0;
    u32 k = key;
    k *= c1;
    k = rotl32(k, 15);
    k *= c2;
    h ^= k;
    h = rotl32(h, 13);
    h = h * 5u + 0xe6546b64u;
    h ^= 4u;
    h ^= h >> 16;
    h *= 0x85ebca6bu;
    h ^= h >> 13;
    h *= 0xc2b2ae35u;
    h ^= h >> 16;
    return h;
}

// splitmix64 (Steele, Lea, Flood 2014): the seed stream replacing std::random_device.
struct SplitMix64 {
    u64 s;
    explicit SplitMix64(u64 seed) : s(seed) {}
    u64 next() {
        u64 z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
};

// ---------------------------------------------------------------------------
// Fixed-association FP64 arithmetic shared (by definition) with the CUDA code.
// ---------------------------------------------------------------------------
inline void butterfly32(double* v) {
    double t[32];
    for (int d = 16; d >= 1; d >>= 1) {
        for (int l = 0; l < 32; l++) t[l] = v[l] + v[l ^ d];
        for (int l = 0; l < 32; l++) v[l] = t[l];
    }
}

// Reduction of a[0..k): groups of 32 -> butterfly -> recurse on group totals.
double det_reduce(const double* a, i64 k) {
    std::vector<double> cur(a, a + k);
    if (k == 0) return 0.0;
    do {
        i64 groups = (i64)((cur.size() + 31) / 32);
        std::vector<double> nxt(groups);
        for (i64 g = 0; g < groups; g++) {
            double v[32];
            for (int l = 0; l < 32; l++) {
                i64 idx = g * 32 + l;
                v[l] = idx < (i64)cur.size() ? cur[idx] : 0.0;
            }
            butterfly32(v);
            nxt[g] = v[0];
        }
        cur.swap(nxt);
    } while (cur.size() > 1);
    return cur[0];
}

// Inclusive scan of a[0..k): Kogge-Stone within groups of 32, recursive scan of
// group totals, then S[g-1] + element for groups g >= 1.
void det_scan_incl(const double* a, double* out, i64 k) {
    if (k == 0) return;
    i64 groups = (k + 31) / 32;
    std::vector<double> tot(groups);
    for (i64 g = 0; g < groups; g++) {
        double v[32], t[32];
        for (int l = 0; l < 32; l++) {
            i64 idx = g * 32 + l;
            v[l] = idx < k ? a[idx] : 0.0;
        }
        for (int d = 1; d < 32; d <<= 1) {
            for (int l = 0; l < 32; l++) t[l] = (l >= d) ? v[l] + v[l - d] : v[l];
            for (int l = 0; l < 32; l++) v[l] = t[l];
        }
        for (int l = 0; l < 32; l++) {
            i64 idx = g * 32 + l;
            if (idx < k) out[idx] = v[l];
        }
        tot[g] = v[31];
    }
    if (groups > 1) {
        std::vector<double> S(groups);
        det_scan_incl(tot.data(), S.data(), groups);
        for (i64 g = 1; g < groups; g++)
            for (int l = 0; l < 32; l++) {
                i64 idx = g * 32 + l;
                if (idx < k) out[idx] = S[g - 1] + out[idx];
            }
    }
}

// Per-vertex edge reduction in the canonical association.  term(j) is the
// double contribution of edge j; deg < MASSIVE_CUTOFF uses 32 lanes, larger
// degrees 1024 threads (32 warps).
template <class F>
double canon_vertex_sum(i64 begin, i64 end, F term) {
    i64 deg = end - begin;
    if (deg < MASSIVE_CUTOFF) {
        double v[32];
        for (int l = 0; l < 32; l++) v[l] = 0.0;
        for (i64 j = begin; j < end; j++) v[(j - begin) & 31] += term(j);
        butterfly32(v);
        return v[0];
    }
    std::vector<double> p(1024, 0.0);
    for (i64 j = begin; j < end; j++) p[(j - begin) & 1023] += term(j);
    double wt[32];
    for (int w = 0; w < 32; w++) {
        double v[32];
        for (int l = 0; l < 32; l++) v[l] = p[w * 32 + l];
        butterfly32(v);
        wt[w] = v[0];
    }
    butterfly32(wt);
    return wt[0];
}

template <class V>
inline float to_f(V x) { return static_cast<float>(x); }

// ---------------------------------------------------------------------------
// Types: weighted_graph (interface/weighted_graph.h:10-19) and cluster_data
// (interface/cluster_data.hpp:9-181).
// ---------------------------------------------------------------------------
template <class W> struct Traits;
template <> struct Traits<i32> { using V = i64; };
template <> struct Traits<float> { using V = double; };

template <class W>
struct Graph {
    using V = typename Traits<W>::V;
    using Weight = W;
    i64 n = 0, nnz = 0;
    std::vector<i64> rowptr;
    std::vector<i32> col;
    std::vector<W> w;  // empty when uniform
    bool uniform = true;
    std::vector<V> vtx_w;
    W wgt(i64 j) const { return uniform ? W(1) : w[j]; }
    i64 deg(i64 i) const { return rowptr[i + 1] - rowptr[i]; }
};

enum ObjKind { OBJ_MOD = 0, OBJ_WMOD = 1, OBJ_CPM = 2, OBJ_NLCC = 3, OBJ_LCC = 4 };

template <class V>
struct ClusterData {
    std::vector<V> total_deg;
    V uncut = 0;
    i64 top_nnz = 0;
    double obj = -1.0;
    i64 label_count = 0;
    V last_pval = 0;
    double lambda = 1.0;
    int kind = OBJ_LCC;
    double inv_gdeg = 0.0;   // modularity normalisation
    double v_total = 0.0;    // CPM
    double g_deg = 0.0;      // NLCC

    // interface/cluster_data.hpp:76-87
    void update_objective() {
        double m = 0;
        if constexpr (std::is_same<V, i64>::value) {
            i64 ss = 0;
            for (i64 l = 0; l < label_count; l++) ss += total_deg[l] * total_deg[l];
            m = static_cast<double>(uncut);
            m = m - lambda * static_cast<double>(ss);
        } else {
            std::vector<double> sq(label_count);
            for (i64 l = 0; l < label_count; l++) sq[l] = total_deg[l] * total_deg[l];
            double ss = det_reduce(sq.data(), label_count);
            m = uncut;
            m = m - lambda * ss;
        }
        obj = m;
    }
    // interface/cluster_data.hpp:124-126,146-148,172-174
    double get_objective() const {
        switch (kind) {
            case OBJ_MOD:
            case OBJ_WMOD: return obj * inv_gdeg;
            case OBJ_CPM: return obj + lambda * v_total;
            case OBJ_NLCC: return obj / g_deg;
            default: return obj;
        }
    }
    // interface/cluster_data.hpp:56-65
    void copy(const ClusterData& rhs) {
        if ((i64)total_deg.size() < rhs.label_count) total_deg.resize(rhs.total_deg.size());
        std::copy(rhs.total_deg.begin(), rhs.total_deg.begin() + rhs.label_count, total_deg.begin());
        top_nnz = rhs.top_nnz;
        uncut = rhs.uncut;
        obj = rhs.obj;
        label_count = rhs.label_count;
        lambda = rhs.lambda;
        kind = rhs.kind;
        inv_gdeg = rhs.inv_gdeg;
        v_total = rhs.v_total;
        g_deg = rhs.g_deg;
    }
    void ensure_capacity(i64 c) {
        if ((i64)total_deg.size() < c) total_deg.resize(c, V(0));
    }
};

template <class V>
V sum_exact(const std::vector<V>& a, i64 k) {
    if constexpr (std::is_same<V, i64>::value) {
        i64 s = 0;
        for (i64 i = 0; i < k; i++) s += a[i];
        return s;
    } else {
        return det_reduce(a.data(), k);
    }
}

// interface/cluster_data.hpp:38-46 + :109-181, app/objective_helpers.hpp:9-22
template <class W>
ClusterData<typename Graph<W>::V> make_objective(const Graph<W>& g, int kind, double mult) {
    using V = typename Graph<W>::V;
    ClusterData<V> cd;
    cd.total_deg.assign(2 * std::max<i64>(g.n, 1), V(0));
    for (i64 i = 0; i < g.n; i++) cd.total_deg[i] = g.vtx_w[i];
    cd.top_nnz = g.nnz;
    cd.uncut = 0;
    cd.label_count = g.n;
    cd.kind = kind;
    cd.lambda = 1.0;
    if (kind == OBJ_MOD || kind == OBJ_WMOD) {
        double gdeg;
        if (g.uniform) gdeg = (double)g.nnz;
        else gdeg = (double)sum_exact(g.vtx_w, g.n);
        cd.inv_gdeg = 1.0 / gdeg;
        cd.lambda = mult * cd.inv_gdeg;
    } else if (kind == OBJ_CPM) {
        cd.v_total = (double)g.n;
        cd.lambda = mult * 0.5;
    } else if (kind == OBJ_NLCC) {
        double gd;
        if (g.uniform) gd = (double)g.nnz;
        else {
            if constexpr (std::is_same<V, i64>::value) {
                i64 s = 0;
                for (i64 j = 0; j < g.nnz; j++) s += g.w[j];
                gd = (double)s;
            } else {
                std::vector<double> tmp(g.w.begin(), g.w.end());
                gd = det_reduce(tmp.data(), g.nnz);
            }
        }
        cd.g_deg = gd;
        double denom;
        if constexpr (std::is_same<V, i64>::value) {
            u64 vt = (u64)sum_exact(g.vtx_w, g.n);
            denom = static_cast<double>(vt * vt);
        } else {
            double vt = sum_exact(g.vtx_w, g.n);
            denom = vt * vt;
        }
        cd.lambda = mult * gd / denom;
    } else {
        cd.lambda = mult;
    }
    cd.update_objective();
    return cd;
}

// ---------------------------------------------------------------------------
// src/ordering.cpp:131-164 -- two stable degree-bucket permutations.
// ---------------------------------------------------------------------------
struct Ordering {
    std::vector<i32> order1, order2;
    i64 offset_large = 0, offset_large2 = 0, offset_mid = 0, offset_mid2 = 0;
};

inline Ordering generate_orderings(const i64* rowptr, i64 n) {
    Ordering o;
    o.order1.resize(n);
    o.order2.resize(n);
    i64 c[5] = {0, 0, 0, 0, 0};
    for (i64 i = 0; i < n; i++) {
        i64 d = rowptr[i + 1] - rowptr[i];
        if (d < LARGE_CUTOFF) c[0]++;
        else if (d < MASSIVE_CUTOFF) c[1]++;
        else c[4]++;
        if (d < MID_CUTOFF) c[2]++;
        else if (d < MASSIVE_CUTOFF) c[3]++;
    }
    i64 off[5] = {0, c[0], 0, c[2], c[0] + c[1]};
    o.offset_large = off[1];
    o.offset_mid = off[3];
    o.offset_large2 = off[4];
    o.offset_mid2 = off[4];
    i64 u[5] = {0, 0, 0, 0, 0};
    for (i64 i = 0; i < n; i++) {
        i64 d = rowptr[i + 1] - rowptr[i];
        if (d < LARGE_CUTOFF) o.order1[off[0] + u[0]++] = (i32)i;
        else if (d < MASSIVE_CUTOFF) o.order1[off[1] + u[1]++] = (i32)i;
        else {
            o.order1[off[4] + u[4]] = (i32)i;
            o.order2[off[4] + u[4]] = (i32)i;
            u[4]++;
        }
        if (d < MID_CUTOFF) o.order2[off[2] + u[2]++] = (i32)i;
        else if (d < MASSIVE_CUTOFF) o.order2[off[3] + u[3]++] = (i32)i;
    }
    return o;
}

// ---------------------------------------------------------------------------
// The clustering engine for one weight type.
// ---------------------------------------------------------------------------
template <class W>
struct Engine {
    using V = typename Traits<W>::V;
    using G = Graph<W>;
    using CD = ClusterData<V>;

    static constexpr bool IS_INT = std::is_same<V, i64>::value;

    // per-vertex memory (interface/memory_store.hpp:20-31)
    std::vector<i32> part, dest, best_part;
    std::vector<float> gain;
    std::vector<V> pvals, pvals_clone;
    Ordering ord;
    bool cdata_init = false;
    int sweep_limit = -1;   // test hook: cap on sweeps per local_move call (<0: none)
    int sweeps_done = 0;
    i64 total_sweeps = 0, total_moves = 0;

    // own-cluster weight of i (the pvals of update_cdata, src/local_mover.cpp:858-886)
    static V own_weight(const G& g, const i32* lab, i64 i) {
        i64 b = g.rowptr[i], e = g.rowptr[i + 1];
        i32 li = lab[i];
        if constexpr (IS_INT) {
            i64 s = 0;
            for (i64 j = b; j < e; j++)
                if (lab[g.col[j]] == li) s += g.wgt(j);
            return s;
        } else {
            return canon_vertex_sum(b, e, [&](i64 j) -> double {
                return lab[g.col[j]] == li ? (double)g.wgt(j) : 0.0;
            });
        }
    }

    void recompute_pvals_all(const G& g) {
        i64 n = g.n;
#pragma omp parallel for schedule(dynamic, 2048)
        for (i64 i = 0; i < n; i++) pvals[i] = own_weight(g, part.data(), i);
    }

    // ---- select_destinations / candidates_and_destinations
    // src/local_mover.cpp:435-634.  Returns the candidate list in order1 order.
    void select(const G& g, CD& cd, float filter_ratio, bool constrained, const i32* constraint,
                std::vector<i32>& candidates) {
        i64 n = g.n;
        const float pm = (float)cd.lambda;
        const bool initial = !cdata_init;
        i64 cap = std::max<i64>(cd.label_count, n) + 1;
#pragma omp parallel
        {
            std::vector<V> acc(initial ? 0 : cap, V(0));
            std::vector<char> seen(initial ? 0 : cap, 0);
            std::vector<i32> touched;
#pragma omp for schedule(dynamic, 1024)
            for (i64 x = 0; x < n; x++) {
                i32 i = ord.order1[x];
                if (dest[i] == NO_MOVE) continue;
                V w = g.vtx_w[i];
                float multi = to_f(w) * pm;
                i32 p = part[i];
                float p_conn = to_f(pvals[i]) - to_f(V(cd.total_deg[p] - w)) * multi;
                float thr = p_conn < 0 ? 0.0f : (float)((double)p_conn * (1.0 - (double)filter_ratio));
                i32 best = NO_MOVE;
                float bconn = thr;
                auto consider = [&](i32 px, V jv) {
                    if (!(jv > 0)) return;
                    if (!(to_f(jv) >= thr)) return;
                    if (constrained && constraint[px] != constraint[p]) return;
                    float jc = to_f(jv) - to_f(cd.total_deg[px]) * multi;
                    if (jc >= thr) {
                        if (best == NO_MOVE || jc > bconn || (jc == bconn && px < best)) {
                            best = px;
                            bconn = jc;
                        }
                    }
                };
                i64 b = g.rowptr[i], e = g.rowptr[i + 1];
                if (initial) {
                    // the input graph stands in for the conn graph (src/local_mover.cpp:1392-1395)
                    for (i64 j = b; j < e; j++) consider(g.col[j], V(g.wgt(j)));
                } else {
                    touched.clear();
                    for (i64 j = b; j < e; j++) {
                        i32 c = part[g.col[j]];
                        if (c == p) continue;
                        if (!seen[c]) {
                            seen[c] = 1;
                            touched.push_back(c);
                        }
                        acc[c] += g.wgt(j);
                    }
                    for (i32 c : touched) {
                        consider(c, acc[c]);
                        acc[c] = V(0);
                        seen[c] = 0;
                    }
                }
                float gn;
                if (best != NO_MOVE) {
                    gn = bconn - p_conn;
                } else if (p_conn < 0) {
                    gn = -p_conn;
                    best = NEW_PART;
                } else {
                    gn = OBJ_MIN;
                }
                gain[i] = gn;
                dest[i] = best;
            }
        }
        candidates.clear();
        for (i64 x = 0; x < n; x++) {
            i32 i = ord.order1[x];
            if (dest[i] != NO_MOVE) candidates.push_back(i);
        }
    }

    // ---- afterburner_kernel / afterburner_filter, src/local_mover.cpp:280-433
    void afterburner(const G& g, CD& cd, const std::vector<i32>& cand, std::vector<i32>& moves) {
        const float pm = (float)cd.lambda;
        i64 k = (i64)cand.size();
        std::vector<char> keep(k, 0);
#pragma omp parallel for schedule(dynamic, 512)
        for (i64 x = 0; x < k; x++) {
            i32 i = cand[x];
            i32 best = dest[i];
            i32 p = part[i];
            float multi = to_f(g.vtx_w[i]) * pm;
            float igain = gain[i];
            i32 hi = (i32)xorshift32((u32)i);
            if (g_afterburner_reference_order) {
                float change = 0;
                for (i64 j = g.rowptr[i]; j < g.rowptr[i + 1]; j++) {
                    i32 v = g.col[j];
                    float vgain = gain[v];
                    if ((vgain - igain) >= AFTERBURNER_EPS ||
                        (std::fabs(vgain - igain) < AFTERBURNER_EPS && (i32)xorshift32((u32)v) < hi)) {
                        float q = (float)g.wgt(j) - multi * to_f(g.vtx_w[v]);
                        i32 vp = dest[v];
                        change -= (vp == p) ? q : 0.0f;
                        change += (vp == best && best != NEW_PART) ? q : 0.0f;
                        vp = part[v];
                        change += (vp == p) ? q : 0.0f;
                        change -= (vp == best) ? q : 0.0f;
                    }
                }
                keep[x] = igain + change >= 0.0f;
                continue;
            }
            double change = canon_vertex_sum(g.rowptr[i], g.rowptr[i + 1], [&](i64 j) -> double {
                i32 v = g.col[j];
                float vgain = gain[v];
                float d = vgain - igain;
                if (d >= AFTERBURNER_EPS || (std::fabs(d) < AFTERBURNER_EPS && (i32)xorshift32((u32)v) < hi)) {
                    float q = (float)g.wgt(j) - multi * to_f(g.vtx_w[v]);
                    int coef = 0;
                    i32 vp = dest[v];
                    if (vp == p) coef--;
                    if (vp == best && best != NEW_PART) coef++;
                    vp = part[v];
                    if (vp == p) coef++;
                    if (vp == best) coef--;
                    return (double)coef * (double)q;
                }
                return 0.0;
            });
            float total = igain + (float)change;
            keep[x] = total >= 0.0f;
        }
        moves.clear();
        for (i64 x = 0; x < k; x++)
            if (keep[x]) moves.push_back(cand[x]);
    }

    // ---- set_new_cluster_ids, src/local_mover.cpp:217-274
    void set_new_cluster_ids(const G& g, CD& cd, const std::vector<i32>& moves, bool constrained,
                             std::vector<i32>* constraint) {
        std::vector<i32> newl;
        for (i32 i : moves)
            if (dest[i] == NEW_PART) newl.push_back(i);
        i64 new_parts = (i64)newl.size();
        if (new_parts == 0) return;
        i64 curr = cd.label_count;
        std::vector<char> has(curr, 0);
        for (i64 i = 0; i < g.n; i++) has[part[i]] = 1;
        i64 avail = 0;
        for (i64 l = 0; l < curr; l++) {
            if (!has[l]) {
                if (avail < new_parts) {
                    i32 x = newl[avail];
                    dest[x] = (i32)l;
                    if (constrained) (*constraint)[l] = (*constraint)[part[x]];
                }
                avail++;
            }
        }
        if (avail < new_parts) {
            i64 needed = new_parts - avail;
            cd.label_count += needed;
            cd.ensure_capacity(cd.label_count);
            if (constrained && (i64)constraint->size() < cd.label_count) constraint->resize(cd.label_count, 0);
            for (i64 x = avail; x < new_parts; x++) {
                i32 i = newl[x];
                i32 d = (i32)((x - avail) + curr);
                dest[i] = d;
                if (constrained) (*constraint)[d] = (*constraint)[part[i]];
            }
            for (i64 l = curr; l < cd.label_count; l++) cd.total_deg[l] = V(0);
        }
    }

    // ---- perform_moves, src/local_mover.cpp:1241-1279 (tables replaced by exact pvals)
    void perform_moves(const G& g, CD& cd, const std::vector<i32>& moves) {
        for (i32 i : moves) {
            i32 b = dest[i], p = part[i];
            if (b < 0) {
                std::fprintf(stderr, "oracle: unresolved destination %d for vertex %d\n", b, i);
                std::abort();
            }
            cd.total_deg[p] = cd.total_deg[p] - g.vtx_w[i];
            cd.total_deg[b] = cd.total_deg[b] + g.vtx_w[i];
        }
        for (i32 i : moves) part[i] = dest[i];
        if (!cdata_init) {
            cdata_init = true;
            recompute_pvals_all(g);
            std::fill(dest.begin(), dest.begin() + g.n, NULL_PART);
        } else {
            std::vector<char> aff(g.n, 0);
            for (i32 i : moves) {
                aff[i] = 1;
                for (i64 j = g.rowptr[i]; j < g.rowptr[i + 1]; j++) aff[g.col[j]] = 1;
            }
#pragma omp parallel for schedule(dynamic, 2048)
            for (i64 v = 0; v < g.n; v++)
                if (aff[v]) {
                    pvals[v] = own_weight(g, part.data(), v);
                    dest[v] = NULL_PART;
                }
        }
        V curr_pval = sum_exact(pvals, g.n);
        V cut_change = curr_pval - cd.last_pval;
        cd.last_pval = curr_pval;
        cd.uncut = cd.uncut + cut_change;
        cd.update_objective();
        total_moves += (i64)moves.size();
    }

    // ---- relabel_contiguously, src/local_mover.cpp:100-129
    static void relabel_contiguously(std::vector<i32>& labels, i64 n, CD& cd) {
        i64 L = cd.label_count;
        std::vector<i32> used(L, 0);
        for (i64 i = 0; i < n; i++) used[labels[i]] = 1;
        i32 t = 0;
        std::vector<V> td(L);
        for (i64 l = 0; l < L; l++)
            if (used[l] > 0) {
                used[l] = t;
                td[t] = cd.total_deg[l];
                t++;
            }
        for (i64 l = 0; l < t; l++) cd.total_deg[l] = td[l];
        for (i64 i = 0; i < n; i++) labels[i] = used[labels[i]];
        cd.label_count = t;
    }

    // truncate_and_init_mem + init (src/local_mover.cpp:1322-1352, 1369-1380)
    void begin_local_move(const G& g, const std::vector<i32>& in_part, CD& best, CD& curr, bool is_initial) {
        i64 n = g.n;
        curr = best;
        curr.copy(best);
        part.assign(in_part.begin(), in_part.begin() + n);
        dest.assign(n, NULL_PART);
        gain.assign(n, 0.0f);
        pvals.assign(n, V(0));
        if (!is_initial) {
            cdata_init = true;
            recompute_pvals_all(g);
            curr.last_pval = sum_exact(pvals, n);
        } else {
            cdata_init = false;
            curr.last_pval = 0;
        }
        pvals_clone = pvals;
    }

    bool sweep_budget_left() { return sweep_limit < 0 || sweeps_done < sweep_limit; }

    // ---- local_move<constrained>, src/local_mover.cpp:1361-1417
    void local_move(const G& g, std::vector<i32>& best_part_io, CD& best, bool is_initial, bool constrained,
                    std::vector<i32>* constraint, bool sa) {
        CD curr;
        begin_local_move(g, best_part_io, best, curr, is_initial);
        std::vector<i32> cand, moves;
        const float ratios[2] = {0.75f, 0.25f};
        const int limits[2] = {4, 2};
        int iter_count = 0;
        for (int x = 0; x < 2; x++) {
            float fr = sa ? ratios[x] : 0.0f;
            int count = 0;
            while (count++ < limits[x]) {
                if (!sweep_budget_left()) break;
                sweeps_done++;
                total_sweeps++;
                iter_count++;
                select(g, curr, fr, constrained, constraint ? constraint->data() : nullptr, cand);
                if (cand.empty()) break;
                afterburner(g, curr, cand, moves);
                if (moves.empty()) break;
                if (iter_count > 1 || !is_initial) set_new_cluster_ids(g, curr, moves, constrained, constraint);
                perform_moves(g, curr, moves);
                if (curr.obj > best.obj) {
                    best.copy(curr);
                    std::copy(part.begin(), part.begin() + g.n, best_part_io.begin());
                    pvals_clone = pvals;
                }
            }
        }
        relabel_contiguously(best_part_io, g.n, best);
    }

    // ---- afterburner_filter_strict, src/local_mover.cpp:131-213.  The O(k^2) inner
    // loop (:168-177) is restated as -multi * S where S is the exact prefix sum of
    // vtx_w(v) * indicator over earlier moves.
    void afterburner_strict(const G& g, CD& cd, std::vector<i32>& moves) {
        const float pm = (float)cd.lambda;
        i64 n = g.n;
        i64 k = (i64)moves.size();
        std::vector<i64> prio(n, n + 1);
        for (i64 x = 0; x < k; x++) prio[moves[x]] = x;
        if (g_afterburner_reference_order) {
            // the reference's FP32 arithmetic in its order: per move the
            // separately rounded updates over edges then earlier moves, an FP32
            // inclusive scan, and the first maximum (src/local_mover.cpp:145-204)
            std::vector<float> oc32(k);
            for (i64 x = 0; x < k; x++) {
                i32 i = moves[x];
                i32 best = dest[i];
                i32 p = part[i];
                float w = to_f(g.vtx_w[i]);
                float multi = w * pm;
                float obj_change = gain[i];
                for (i64 j = g.rowptr[i]; j < g.rowptr[i + 1]; j++) {
                    i32 v = g.col[j];
                    if (prio[v] < prio[i]) {
                        const float wgt = (float)g.wgt(j);
                        i32 vp = dest[v];
                        obj_change -= (vp == p) ? wgt : 0.0f;
                        obj_change += (vp == best && best != NEW_PART) ? wgt : 0.0f;
                        vp = part[v];
                        obj_change += (vp == p) ? wgt : 0.0f;
                        obj_change -= (vp == best) ? wgt : 0.0f;
                    }
                }
                for (i64 jx = 0; jx < x; jx++) {
                    i32 v = moves[jx];
                    i32 vp = dest[v];
                    float wgt = -multi * to_f(g.vtx_w[v]);
                    obj_change -= (vp == p) ? wgt : 0.0f;
                    obj_change += (vp == best && best != NEW_PART) ? wgt : 0.0f;
                    vp = part[v];
                    obj_change += (vp == p) ? wgt : 0.0f;
                    obj_change -= (vp == best) ? wgt : 0.0f;
                }
                oc32[x] = obj_change;
            }
            float run = 0.0f, bv32 = std::numeric_limits<float>::lowest();
            i64 bl32 = n;
            for (i64 x = 0; x < k; x++) {
                run += oc32[x];
                if (run > bv32) {
                    bv32 = run;
                    bl32 = x;
                }
            }
            i64 truncate = 0;
            if (bl32 < k && bv32 > 0) truncate = bl32 + 1;
            moves.resize(truncate);
            return;
        }
        std::vector<double> oc(k);
        for (i64 x = 0; x < k; x++) {
            i32 i = moves[x];
            i32 best = dest[i];
            i32 p = part[i];
            float multi = to_f(g.vtx_w[i]) * pm;
            V nb = 0;
            for (i64 j = g.rowptr[i]; j < g.rowptr[i + 1]; j++) {
                i32 v = g.col[j];
                if (prio[v] < prio[i]) {
                    int coef = 0;
                    i32 vp = dest[v];
                    if (vp == p) coef--;
                    if (vp == best && best != NEW_PART) coef++;
                    vp = part[v];
                    if (vp == p) coef++;
                    if (vp == best) coef--;
                    nb += (V)coef * (V)g.wgt(j);
                }
            }
            V S = 0;
            for (i64 jx = 0; jx < x; jx++) {
                i32 v = moves[jx];
                int coef = 0;
                i32 vp = dest[v];
                if (vp == p) coef--;
                if (vp == best && best != NEW_PART) coef++;
                vp = part[v];
                if (vp == p) coef++;
                if (vp == best) coef--;
                S += (V)coef * g.vtx_w[v];
            }
            double t2 = -(double)multi * (double)S;
            oc[x] = ((double)gain[i] + (double)nb) + t2;
        }
        std::vector<double> pre(k);
        det_scan_incl(oc.data(), pre.data(), k);
        // MaxFirstLoc over the prefix values: largest value, first position among ties
        double bv = -std::numeric_limits<double>::infinity();
        i64 bl = n;
        for (i64 x = 0; x < k; x++)
            if (pre[x] > bv) {
                bv = pre[x];
                bl = x;
            }
        i64 truncate = 0;
        if (bl < k && bv > 0) truncate = bl + 1;
        moves.resize(truncate);
    }

    // ---- local_move_strict<constrained>, src/local_mover.cpp:1422-1483
    void local_move_strict(const G& g, std::vector<i32>& best_part_io, CD& best, bool is_initial, bool constrained,
                           std::vector<i32>* constraint) {
        CD curr;
        begin_local_move(g, best_part_io, best, curr, is_initial);
        std::vector<i32> cand;
        for (int it = 0; it < 6; it++) {
            if (!sweep_budget_left()) break;
            sweeps_done++;
            total_sweeps++;
            select(g, curr, 0.0f, constrained, constraint ? constraint->data() : nullptr, cand);
            if (cand.empty()) break;
            if (it > 0 || !is_initial) set_new_cluster_ids(g, curr, cand, constrained, constraint);
            afterburner_strict(g, curr, cand);
            if (cand.empty()) break;
            perform_moves(g, curr, cand);
            if (curr.obj > best.obj) {
                best.copy(curr);
                std::copy(part.begin(), part.begin() + g.n, best_part_io.begin());
                pvals_clone = pvals;
            }
            std::fill(dest.begin(), dest.begin() + g.n, NULL_PART);
        }
        relabel_contiguously(best_part_io, g.n, best);
    }

    // ---- build_coarse_graph, src/contract.cpp:234-336 (rows sorted by column)
    static G build_coarse_graph(const G& g, const std::vector<i32>& vcmap, i64 nc) {
        G cg;
        cg.n = nc;
        cg.uniform = false;
        std::vector<i64> cnt(nc + 1, 0);
        for (i64 i = 0; i < g.n; i++) cnt[vcmap[i] + 1]++;
        for (i64 c = 0; c < nc; c++) cnt[c + 1] += cnt[c];
        std::vector<i32> members(g.n);
        {
            std::vector<i64> pos(cnt.begin(), cnt.end() - 1);
            for (i64 i = 0; i < g.n; i++) members[pos[vcmap[i]]++] = (i32)i;
        }
        std::vector<std::vector<std::pair<i32, V>>> rows(nc);
#pragma omp parallel
        {
            std::vector<V> acc(nc, V(0));
            std::vector<char> seen(nc, 0);
            std::vector<i32> touched;
#pragma omp for schedule(dynamic, 256)
            for (i64 c = 0; c < nc; c++) {
                touched.clear();
                for (i64 m = cnt[c]; m < cnt[c + 1]; m++) {
                    i32 i = members[m];
                    for (i64 j = g.rowptr[i]; j < g.rowptr[i + 1]; j++) {
                        i32 u = vcmap[g.col[j]];
                        if (u == c) continue;
                        if (!seen[u]) {
                            seen[u] = 1;
                            touched.push_back(u);
                        }
                        acc[u] += (V)g.wgt(j);
                    }
                }
                std::sort(touched.begin(), touched.end());
                auto& r = rows[c];
                r.reserve(touched.size());
                for (i32 u : touched) {
                    r.push_back({u, acc[u]});
                    acc[u] = V(0);
                    seen[u] = 0;
                }
            }
        }
        cg.rowptr.assign(nc + 1, 0);
        for (i64 c = 0; c < nc; c++) cg.rowptr[c + 1] = cg.rowptr[c] + (i64)rows[c].size();
        cg.nnz = cg.rowptr[nc];
        cg.col.resize(cg.nnz);
        cg.w.resize(cg.nnz);
        for (i64 c = 0; c < nc; c++) {
            i64 o = cg.rowptr[c];
            for (auto& pr : rows[c]) {
                cg.col[o] = pr.first;
                cg.w[o] = (W)pr.second;
                o++;
            }
        }
        return cg;
    }

    // coarsen_vtx_w, src/clustering_methods.cpp:33-38
    static void coarsen_vtx_w(const G& g, const std::vector<i32>& map, G& cg) {
        cg.vtx_w.assign(cg.n, V(0));
        for (i64 i = 0; i < g.n; i++) cg.vtx_w[map[i]] += g.vtx_w[i];
    }

    // ---- find_trees, src/leidenR.cpp:213-260
    static void find_trees(std::vector<i32>& vcmap, i64 n, const std::vector<i32>& hn, std::vector<i32>& order) {
        for (i64 i = 0; i < n; i++) {
            i32 now = (i32)i, then = hn[i];
            if (now == then) {
                vcmap[i] = (i32)i;
                continue;
            }
            while (order[now] > order[then]) {
                now = then;
                then = hn[then];
            }
            if (now != (i32)i) {
                vcmap[i] = now;
                vcmap[now] = now;
            }
        }
        for (i64 i = 0; i < n; i++)
            if (vcmap[i] == ORD_MAX) order[i] = 2 * SPLIT - order[i];
        std::vector<char> unassigned(n);
        for (i64 i = 0; i < n; i++) unassigned[i] = vcmap[i] == ORD_MAX;
        for (i64 i = 0; i < n; i++) {
            if (!unassigned[i]) continue;
            i32 now = (i32)i, then = hn[i];
            while (vcmap[now] == ORD_MAX && order[now] > order[then]) {
                now = then;
                then = hn[then];
            }
            vcmap[i] = vcmap[now];
        }
    }

    // ---- ensure_gamma_connectivity, src/leidenR.cpp:41-187
    static void ensure_gamma_connectivity(const G& g, std::vector<i32>& vcmap, const std::vector<i32>& constraint,
                                          const std::vector<i32>& order, const CD& cd, const std::vector<V>& pv) {
        i64 n = g.n;
        float gamma = (float)cd.lambda;
        const auto& vw = g.vtx_w;
        std::vector<i64> row_map(n + 1, 0);
        for (i64 i = 0; i < n; i++) row_map[vcmap[i] + 1]++;
        for (i64 c = 0; c < n; c++) row_map[c + 1] += row_map[c];
        std::vector<i32> ids(n);
        for (i64 i = 0; i < n; i++) ids[i] = (i32)i;
        std::sort(ids.begin(), ids.end(), [&](i32 a, i32 b) {
            if (vcmap[a] != vcmap[b]) return vcmap[a] < vcmap[b];
            if (order[a] != order[b]) return order[a] < order[b];
            return a < b;
        });
        // exclusive prefix of vtx_w over the sorted positions (src/leidenR.cpp:81-88)
        std::vector<V> ts(n);
        if constexpr (IS_INT) {
            i64 s = 0;
            for (i64 x = 0; x < n; x++) {
                ts[x] = s;
                s += vw[ids[x]];
            }
        } else {
            std::vector<double> a(n), inc(n);
            for (i64 x = 0; x < n; x++) a[x] = vw[ids[x]];
            det_scan_incl(a.data(), inc.data(), n);
            for (i64 x = 0; x < n; x++) ts[x] = x == 0 ? 0.0 : inc[x - 1];
        }
        // inner_conn (src/leidenR.cpp:96-133)
        std::vector<V> inner(n);
#pragma omp parallel for schedule(dynamic, 2048)
        for (i64 i = 0; i < n; i++) {
            i64 b = g.rowptr[i], e = g.rowptr[i + 1];
            if constexpr (IS_INT) {
                i64 s = 0;
                for (i64 j = b; j < e; j++) {
                    i32 v = g.col[j];
                    if (vcmap[i] == vcmap[v] && order[v] < order[i]) s += g.wgt(j);
                }
                inner[i] = s;
            } else {
                inner[i] = canon_vertex_sum(b, e, [&](i64 j) -> double {
                    i32 v = g.col[j];
                    return (vcmap[i] == vcmap[v] && order[v] < order[i]) ? (double)g.wgt(j) : 0.0;
                });
            }
        }
        std::vector<i64> breakers(n, n);
        // part 1 (src/leidenR.cpp:140-149)
        for (i64 x = 0; x < n; x++) {
            i32 i = ids[x];
            i32 c = vcmap[i];
            i64 cb = row_map[c];
            V prev = ts[x] - ts[cb];
            if (to_f(inner[i]) < (gamma * to_f(vw[i])) * to_f(prev)) breakers[c] = std::min(breakers[c], x);
        }
        // outer conn inclusive scan (src/leidenR.cpp:154-163)
        std::vector<V> oc(n);
        if constexpr (IS_INT) {
            i64 s = 0;
            for (i64 x = 0; x < n; x++) {
                i32 i = ids[x];
                s += pv[i] - 2 * inner[i];
                oc[i] = s;
            }
        } else {
            std::vector<double> a(n), inc(n);
            for (i64 x = 0; x < n; x++) {
                i32 i = ids[x];
                a[x] = pv[i] - 2.0 * inner[i];
            }
            det_scan_incl(a.data(), inc.data(), n);
            for (i64 x = 0; x < n; x++) oc[ids[x]] = inc[x];
        }
        // part 2 (src/leidenR.cpp:166-178)
        for (i64 x = 0; x < n; x++) {
            i32 i = ids[x];
            i32 c = vcmap[i];
            i64 cb = row_map[c];
            V curr_size = (ts[x] + vw[i]) - ts[cb];
            V other = cd.total_deg[constraint[i]] - curr_size;
            V outer = oc[i];
            if (cb > 0) outer = outer - oc[ids[cb - 1]];
            if (to_f(outer) < (gamma * to_f(curr_size)) * to_f(other)) breakers[c] = std::min(breakers[c], x + 1);
        }
        // break (src/leidenR.cpp:180-186)
        for (i64 x = 0; x < n; x++) {
            i32 i = ids[x];
            i32 c = vcmap[i];
            if (x >= breakers[c]) vcmap[i] = i;
        }
    }

    // ---- contigitize_clusters, src/leidenR.cpp:190-210
    static i64 contigitize(std::vector<i32>& vcmap, i64 n) {
        i32 nc = 0;
        for (i64 u = 0; u < n; u++) {
            if (vcmap[u] == (i32)u) vcmap[u] = nc++;
            else vcmap[u] = vcmap[u] + (i32)n;
        }
        for (i64 u = 0; u < n; u++)
            if (vcmap[u] >= (i32)n) vcmap[u] = vcmap[vcmap[u] - (i32)n];
        return nc;
    }

    // ---- coarsen_leidenR<top,uniform>, src/leidenR.cpp:263-500
    static i64 coarsen_leidenR(const G& g, const std::vector<i32>& constraint, const CD& cd, u32 seed_pick,
                               u32 seed_order, std::vector<i32>& vcmap) {
        i64 n = g.n;
        float gamma = (float)cd.lambda;
        const auto& vw = g.vtx_w;
        std::vector<V> pv(n);
#pragma omp parallel for schedule(dynamic, 2048)
        for (i64 i = 0; i < n; i++) pv[i] = own_weight(g, constraint.data(), i);
        std::vector<char> well(n);
        for (i64 i = 0; i < n; i++) {
            i32 c = constraint[i];
            V wd = vw[i];
            well[i] = to_f(pv[i]) >= (gamma * to_f(wd)) * to_f(V(cd.total_deg[c] - wd));
        }
        std::vector<i32> hn(n);
        if (g.uniform) {
            // select random edge (src/leidenR.cpp:296-393)
#pragma omp parallel for schedule(dynamic, 2048)
            for (i64 i = 0; i < n; i++) {
                i64 b = g.rowptr[i], e = g.rowptr[i + 1];
                i64 width = e - b;
                float multi = gamma * to_f(vw[i]);
                i32 jxs = (i32)murmur3_32(seed_pick + (u32)i);
                if (jxs % 1000 == 0 || !well[i] || width == 0) {
                    hn[i] = (i32)i;
                    continue;
                }
                i64 jx = b + (i64)((u32)jxs % (u32)width);
                i32 pick = (i32)i;
                bool found = false;
                for (i64 s = 0; s < width && !found; s++) {
                    i64 j = jx + s;
                    if (j >= e) j -= width;
                    i32 v = g.col[j];
                    if (constraint[i] != constraint[v]) continue;
                    if (!well[v]) continue;
                    if (1.0f >= multi * to_f(vw[v])) {
                        pick = v;
                        found = true;
                    }
                }
                hn[i] = pick;
            }
        } else {
            // select heaviest edge (src/leidenR.cpp:400-474)
#pragma omp parallel for schedule(dynamic, 2048)
            for (i64 i = 0; i < n; i++) {
                i64 b = g.rowptr[i], e = g.rowptr[i + 1];
                float multi = gamma * to_f(vw[i]);
                u32 h = murmur3_32(seed_pick + (u32)i);
                if (h % 10000u == 0 || !well[i]) {
                    hn[i] = (i32)i;
                    continue;
                }
                float m = 0.0f;
                i64 am = e;
                for (i64 j = b; j < e; j++) {
                    i32 v = g.col[j];
                    if (constraint[i] != constraint[v]) continue;
                    if (!well[v]) continue;
                    float val = (float)g.wgt(j) - multi * to_f(vw[v]);
                    if (val >= 0) {
                        float sample = std::fabs((float)murmur3_32(seed_pick + (u32)(u64)j) / (float)ORD_MAX);
                        float v2 = val * val;
                        sample = sample * (v2 * v2);
                        if (sample >= m) {
                            m = sample;
                            am = j;
                        }
                    }
                }
                hn[i] = (am >= b && am < e && m >= 0) ? g.col[am] : (i32)i;
            }
        }
        // set order / unselect equal order edges (src/leidenR.cpp:482-494)
        std::vector<i32> order(n);
        for (i64 i = 0; i < n; i++) {
            i32 o = (i32)murmur3_32((u32)i + seed_order);
            order[i] = std::abs(o % SPLIT);
        }
        for (i64 i = 0; i < n; i++)
            if (order[i] == order[hn[i]]) hn[i] = (i32)i;
        vcmap.assign(n, ORD_MAX);
        find_trees(vcmap, n, hn, order);
        ensure_gamma_connectivity(g, vcmap, constraint, order, cd, pv);
        return contigitize(vcmap, n);
    }

    // ---- leiden_part<plus,improve>, src/clustering_methods.cpp:47-137
    std::vector<i32> leiden_part(const G& top, CD& rfd, bool plus, bool improve, const i32* input, u64 seed,
                                 i64* level_count, i64* total_nnz) {
        std::deque<G> coarse;  // owned coarse graphs; a deque keeps references stable
        std::vector<const G*> levels;
        std::vector<std::vector<i32>> parts;
        levels.push_back(&top);
        std::vector<i32> part(top.n);
        if (!improve)
            for (i64 x = 0; x < top.n; x++) part[x] = (i32)x;
        else
            std::copy(input, input + top.n, part.begin());
        SplitMix64 rng(seed);
        while (true) {
            const G& c = *levels.back();
            if ((i64)levels.size() > 4096) throw std::runtime_error("multilevel hierarchy exceeded 4096 levels");
            double old_obj = rfd.obj;
            bool init = !improve && levels.size() == 1;
            ord = generate_orderings(c.rowptr.data(), c.n);
            local_move(c, part, rfd, init, false, nullptr, true);
            if (c.nnz > 100000 && old_obj == rfd.obj) local_move(c, part, rfd, init, false, nullptr, false);
            if (old_obj == rfd.obj) local_move_strict(c, part, rfd, init, false, nullptr);
            if (rfd.label_count == c.n) {
                parts.push_back(part);
                break;
            }
            std::vector<i32> louv = part;
            u32 s_pick = (u32)rng.next();
            u32 s_order = (u32)rng.next();
            std::vector<i32> cmap;
            i64 nc = coarsen_leidenR(c, louv, rfd, s_pick, s_order, cmap);
            parts.push_back(cmap);
            if (nc < c.n) {
                coarse.push_back(build_coarse_graph(c, cmap, nc));
                G& next = coarse.back();
                coarsen_vtx_w(c, cmap, next);
                part.assign(nc, 0);
                for (i64 i = 0; i < c.n; i++) part[cmap[i]] = louv[i];
                levels.push_back(&next);
            } else {
                levels.push_back(&c);
            }
        }
        if (level_count) *level_count = (i64)levels.size();
        if (total_nnz) {
            i64 t = 0;
            for (auto* l : levels) t += l->nnz;
            *total_nnz = t;
        }
        for (i64 i = (i64)levels.size() - 2; i >= 0; i--) {
            const G& c = *levels[i];
            auto& fine = parts[i];
            const auto& cp = parts[i + 1];
            for (i64 x = 0; x < c.n; x++) fine[x] = cp[fine[x]];
            if (plus) {
                ord = generate_orderings(c.rowptr.data(), c.n);
                local_move(c, fine, rfd, false, false, nullptr, true);
            }
        }
        return parts[0];
    }

    // ---- louvain_part<constrained>, src/clustering_methods.cpp:139-222
    std::vector<i32> louvain_part(const G& top, CD& rfd, bool constrained, std::vector<i32> constraint,
                                  i64* level_count, i64* total_nnz) {
        if (constrained) {
            for (i64 i = 0; i < top.n; i++) rfd.total_deg[i] = top.vtx_w[i];
            rfd.uncut = 0;
            rfd.label_count = top.n;
            rfd.update_objective();
        }
        std::deque<G> coarse;  // owned coarse graphs; a deque keeps references stable
        std::vector<const G*> levels;
        std::vector<std::vector<i32>> parts;
        levels.push_back(&top);
        bool drop = constrained;
        while (true) {
            const G& c = *levels.back();
            if ((i64)levels.size() > 4096) throw std::runtime_error("multilevel hierarchy exceeded 4096 levels");
            std::vector<i32> part(c.n);
            for (i64 x = 0; x < c.n; x++) part[x] = (i32)x;
            ord = generate_orderings(c.rowptr.data(), c.n);
            if (constrained && (i64)constraint.size() < 2 * c.n) constraint.resize(2 * c.n, 0);
            local_move(c, part, rfd, true, constrained, constrained ? &constraint : nullptr, true);
            if (constrained && rfd.label_count == c.n)
                local_move_strict(c, part, rfd, true, constrained, &constraint);
            parts.push_back(part);
            if (rfd.label_count < c.n) {
                coarse.push_back(build_coarse_graph(c, part, rfd.label_count));
                G& next = coarse.back();
                next.vtx_w.assign(rfd.total_deg.begin(), rfd.total_deg.begin() + rfd.label_count);
                levels.push_back(&next);
                if (constrained) {
                    std::vector<i32> nxt(rfd.label_count, 0);
                    for (i64 i = 0; i < c.n; i++) nxt[part[i]] = constraint[i];
                    constraint = nxt;
                }
            } else if (drop) {
                std::fill(constraint.begin(), constraint.end(), 0);
                parts.pop_back();
                drop = false;
            } else {
                break;
            }
        }
        if (level_count) *level_count = (i64)levels.size();
        if (total_nnz) {
            i64 t = 0;
            for (auto* l : levels) t += l->nnz;
            *total_nnz = t;
        }
        if (levels.size() > 1) {
            levels.pop_back();
            parts.pop_back();
        }
        for (i64 i = (i64)levels.size() - 2; i >= 0; i--) {
            const G& c = *levels[i];
            auto& p = parts[i];
            const auto& cp = parts[i + 1];
            for (i64 x = 0; x < c.n; x++) p[x] = cp[p[x]];
            ord = generate_orderings(c.rowptr.data(), c.n);
            local_move(c, p, rfd, false, false, nullptr, true);
        }
        return parts[0];
    }
};

// verify_objective<uniform>, app/verify_objective.cpp:64-89 (int64 / FP64 sums)
template <class W>
double verify_objective(const Graph<W>& g, const i32* labels, int kind, double mult, double* raw_obj) {
    using V = typename Graph<W>::V;
    auto cd = make_objective<W>(g, kind, mult);
    i64 n = g.n;
    std::vector<V> total(2 * std::max<i64>(n, 1), V(0));
    V uncut = 0;
    if constexpr (std::is_same<V, i64>::value) {
        for (i64 i = 0; i < n; i++) {
            for (i64 j = g.rowptr[i]; j < g.rowptr[i + 1]; j++)
                if (labels[g.col[j]] == labels[i]) uncut += g.wgt(j);
            total[labels[i]] += g.vtx_w[i];
        }
    } else {
        std::vector<double> own(n);
        for (i64 i = 0; i < n; i++) {
            own[i] = canon_vertex_sum(g.rowptr[i], g.rowptr[i + 1], [&](i64 j) -> double {
                return labels[g.col[j]] == labels[i] ? (double)g.wgt(j) : 0.0;
            });
            total[labels[i]] += g.vtx_w[i];
        }
        uncut = det_reduce(own.data(), n);
    }
    cd.total_deg = total;
    cd.uncut = uncut;
    cd.label_count = n;
    cd.update_objective();
    if (raw_obj) *raw_obj = cd.obj;
    return cd.get_objective();
}

}  // namespace orc

// ===========================================================================
// C API for the Python test harness (ctypes).  Weight kinds: 0 uniform, 1 int32,
// 2 float32.  Vertex weights: int64 for kinds 0/1, float64 for kind 2.
// ===========================================================================
using namespace orc;

struct OrcGraph {
    int kind = 0;
    Graph<i32> gi;
    Graph<float> gf;
};

struct OrcCD {
    int kind = 0;
    ClusterData<i64> ci;
    ClusterData<double> cf;
};

struct OrcStats {
    int64_t levels;
    int64_t total_nnz;
    int64_t sweeps;
    int64_t moves;
    double objective;
    double raw_obj;
    int64_t label_count;
};

template <class W>
static void fill_graph(Graph<W>& g, int kind, int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col,
                       const void* w, const void* vtx_w, int objective) {
    using V = typename Graph<W>::V;
    g.n = n;
    g.nnz = nnz;
    g.rowptr.assign(rowptr, rowptr + n + 1);
    g.col.assign(col, col + nnz);
    g.uniform = (kind == 0);
    if (!g.uniform) {
        const W* ww = (const W*)w;
        g.w.assign(ww, ww + nnz);
    }
    g.vtx_w.assign(n, V(0));
    if (vtx_w) {
        const V* vv = (const V*)vtx_w;
        g.vtx_w.assign(vv, vv + n);
    } else {
        // app/io/vertex_weighting.cpp:27-42
        for (int64_t i = 0; i < n; i++) {
            if (objective == OBJ_MOD) g.vtx_w[i] = (V)(rowptr[i + 1] - rowptr[i]);
            else if (objective == OBJ_WMOD) {
                if constexpr (std::is_same<V, i64>::value) {
                    i64 s = 0;
                    for (i64 j = rowptr[i]; j < rowptr[i + 1]; j++) s += g.wgt(j);
                    g.vtx_w[i] = s;
                } else {
                    double s = canon_vertex_sum(rowptr[i], rowptr[i + 1], [&](i64 j) -> double { return (double)g.wgt(j); });
                    g.vtx_w[i] = (double)(float)s;
                }
            } else g.vtx_w[i] = V(1);
        }
    }
}

// the level loops throw when a hierarchy passes 4096 levels; the C entry points
// turn exceptions into -1 and keep the message for orc_last_error
static thread_local std::string orc_error;
template <class F>
static int orc_guard(F f) {
    try {
        return f();
    } catch (const std::exception& e) {
        orc_error = e.what();
        return -1;
    }
}

extern "C" {

const char* orc_last_error() { return orc_error.c_str(); }

void* orc_graph_new(int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col, const void* w, int wkind,
                    const void* vtx_w, int objective) {
    auto* g = new OrcGraph();
    g->kind = wkind;
    if (wkind == 2) fill_graph<float>(g->gf, wkind, n, nnz, rowptr, col, w, vtx_w, objective);
    else fill_graph<i32>(g->gi, wkind, n, nnz, rowptr, col, w, vtx_w, objective);
    return g;
}

void orc_graph_free(void* h) { delete (OrcGraph*)h; }

void orc_graph_dims(void* h, int64_t* n, int64_t* nnz, int* wkind) {
    auto* g = (OrcGraph*)h;
    if (g->kind == 2) {
        *n = g->gf.n;
        *nnz = g->gf.nnz;
    } else {
        *n = g->gi.n;
        *nnz = g->gi.nnz;
    }
    *wkind = g->kind;
}

void orc_graph_read(void* h, int64_t* rowptr, int32_t* col, void* w, void* vtx_w) {
    auto* g = (OrcGraph*)h;
    auto rd = [&](auto& gg) {
        using GW = typename std::decay<decltype(gg.w)>::type::value_type;
        using GV = typename std::decay<decltype(gg.vtx_w)>::type::value_type;
        if (rowptr) std::copy(gg.rowptr.begin(), gg.rowptr.end(), rowptr);
        if (col) std::copy(gg.col.begin(), gg.col.end(), col);
        if (w && !gg.uniform) std::copy(gg.w.begin(), gg.w.end(), (GW*)w);
        if (vtx_w) std::copy(gg.vtx_w.begin(), gg.vtx_w.end(), (GV*)vtx_w);
    };
    if (g->kind == 2) rd(g->gf);
    else rd(g->gi);
}

void* orc_cd_new(void* gh, int objective, double mult) {
    auto* g = (OrcGraph*)gh;
    auto* cd = new OrcCD();
    cd->kind = g->kind == 2 ? 2 : 1;
    if (g->kind == 2) cd->cf = make_objective<float>(g->gf, objective, mult);
    else cd->ci = make_objective<i32>(g->gi, objective, mult);
    return cd;
}

void orc_cd_free(void* h) { delete (OrcCD*)h; }

// out: [obj, objective(), lambda, uncut(as double), label_count]
void orc_cd_get(void* h, double* out) {
    auto* cd = (OrcCD*)h;
    if (cd->kind == 2) {
        out[0] = cd->cf.obj;
        out[1] = cd->cf.get_objective();
        out[2] = cd->cf.lambda;
        out[3] = cd->cf.uncut;
        out[4] = (double)cd->cf.label_count;
    } else {
        out[0] = cd->ci.obj;
        out[1] = cd->ci.get_objective();
        out[2] = cd->ci.lambda;
        out[3] = (double)cd->ci.uncut;
        out[4] = (double)cd->ci.label_count;
    }
}

void orc_cd_total_deg(void* h, void* out) {
    auto* cd = (OrcCD*)h;
    if (cd->kind == 2) std::copy(cd->cf.total_deg.begin(), cd->cf.total_deg.begin() + cd->cf.label_count, (double*)out);
    else std::copy(cd->ci.total_deg.begin(), cd->ci.total_deg.begin() + cd->ci.label_count, (int64_t*)out);
}

// Overwrite the state of a cluster_data (labels 0..label_count-1).
void orc_cd_set(void* h, int64_t label_count, const void* total_deg, double uncut) {
    auto* cd = (OrcCD*)h;
    if (cd->kind == 2) {
        cd->cf.ensure_capacity(label_count);
        std::copy((const double*)total_deg, (const double*)total_deg + label_count, cd->cf.total_deg.begin());
        cd->cf.label_count = label_count;
        cd->cf.uncut = uncut;
        cd->cf.update_objective();
    } else {
        cd->ci.ensure_capacity(label_count);
        std::copy((const int64_t*)total_deg, (const int64_t*)total_deg + label_count, cd->ci.total_deg.begin());
        cd->ci.label_count = label_count;
        cd->ci.uncut = (int64_t)uncut;
        cd->ci.update_objective();
    }
}

void orc_generate_orderings(int64_t n, const int64_t* rowptr, int32_t* order1, int32_t* order2, int64_t* offsets4) {
    Ordering o = generate_orderings(rowptr, n);
    std::copy(o.order1.begin(), o.order1.end(), order1);
    std::copy(o.order2.begin(), o.order2.end(), order2);
    offsets4[0] = o.offset_large;
    offsets4[1] = o.offset_large2;
    offsets4[2] = o.offset_mid;
    offsets4[3] = o.offset_mid2;
}

void* orc_build_coarse_graph(void* gh, const int32_t* vcmap, int64_t nc) {
    auto* g = (OrcGraph*)gh;
    auto* out = new OrcGraph();
    std::vector<i32> m(vcmap, vcmap + (g->kind == 2 ? g->gf.n : g->gi.n));
    if (g->kind == 2) {
        out->kind = 2;
        out->gf = Engine<float>::build_coarse_graph(g->gf, m, nc);
        Engine<float>::coarsen_vtx_w(g->gf, m, out->gf);
    } else {
        out->kind = 1;
        out->gi = Engine<i32>::build_coarse_graph(g->gi, m, nc);
        Engine<i32>::coarsen_vtx_w(g->gi, m, out->gi);
    }
    return out;
}

// One select pass (candidates_and_destinations) on a given state.
// dest_io: dest cache in / destinations out; gain_io: save_gains in/out (entries
// of skipped NO_MOVE vertices keep their input values, as save_gains does).
int64_t orc_select(void* gh, void* cdh, const int32_t* part, const void* pvals, int32_t* dest_io, float* gain_io,
                   float filter_ratio, int initial, int constrained, const int32_t* constraint) {
    auto* g = (OrcGraph*)gh;
    auto* cd = (OrcCD*)cdh;
    auto run = [&](auto& eng, auto& gg, auto& c) {
        using V = typename std::decay<decltype(c.total_deg)>::type::value_type;
        i64 n = gg.n;
        eng.ord = generate_orderings(gg.rowptr.data(), n);
        eng.part.assign(part, part + n);
        eng.dest.assign(dest_io, dest_io + n);
        eng.gain.assign(gain_io, gain_io + n);
        eng.pvals.assign((const V*)pvals, (const V*)pvals + n);
        eng.cdata_init = !initial;
        std::vector<i32> cand;
        eng.select(gg, c, filter_ratio, constrained != 0, constraint, cand);
        std::copy(eng.dest.begin(), eng.dest.end(), dest_io);
        std::copy(eng.gain.begin(), eng.gain.end(), gain_io);
        return (int64_t)cand.size();
    };
    if (g->kind == 2) {
        Engine<float> e;
        return run(e, g->gf, cd->cf);
    }
    Engine<i32> e;
    return run(e, g->gi, cd->ci);
}

// local_move / local_move_strict on (graph, cluster_data, part).
// mode 0: local_move (SA per enable_sa), mode 1: local_move_strict.
int orc_local_move(void* gh, void* cdh, int32_t* part_io, int is_initial, int constrained, int32_t* constraint_io,
                   int64_t constraint_len, int enable_sa, int mode, int sweep_limit, OrcStats* st) {
    auto* g = (OrcGraph*)gh;
    auto* cd = (OrcCD*)cdh;
    auto run = [&](auto& eng, auto& gg, auto& c) {
        i64 n = gg.n;
        eng.ord = generate_orderings(gg.rowptr.data(), n);
        eng.sweep_limit = sweep_limit;
        std::vector<i32> part(part_io, part_io + n);
        std::vector<i32> con;
        if (constrained) con.assign(constraint_io, constraint_io + constraint_len);
        if (mode == 0) eng.local_move(gg, part, c, is_initial != 0, constrained != 0, constrained ? &con : nullptr, enable_sa != 0);
        else eng.local_move_strict(gg, part, c, is_initial != 0, constrained != 0, constrained ? &con : nullptr);
        std::copy(part.begin(), part.end(), part_io);
        if (constrained) std::copy(con.begin(), con.begin() + std::min<i64>(constraint_len, (i64)con.size()), constraint_io);
        if (st) {
            st->sweeps = eng.total_sweeps;
            st->moves = eng.total_moves;
            st->objective = c.get_objective();
            st->raw_obj = c.obj;
            st->label_count = c.label_count;
        }
        return 0;
    };
    if (g->kind == 2) {
        Engine<float> e;
        return run(e, g->gf, cd->cf);
    }
    Engine<i32> e;
    return run(e, g->gi, cd->ci);
}

int64_t orc_coarsen_leidenR(void* gh, void* cdh, const int32_t* constraint, uint32_t seed_pick, uint32_t seed_order,
                            int32_t* vcmap_out) {
    auto* g = (OrcGraph*)gh;
    auto* cd = (OrcCD*)cdh;
    std::vector<i32> vcmap;
    i64 nc;
    if (g->kind == 2) {
        std::vector<i32> con(constraint, constraint + g->gf.n);
        nc = Engine<float>::coarsen_leidenR(g->gf, con, cd->cf, seed_pick, seed_order, vcmap);
    } else {
        std::vector<i32> con(constraint, constraint + g->gi.n);
        nc = Engine<i32>::coarsen_leidenR(g->gi, con, cd->ci, seed_pick, seed_order, vcmap);
    }
    std::copy(vcmap.begin(), vcmap.end(), vcmap_out);
    return nc;
}

// method: 0 louvain (plouvain), 1 leiden (pleiden), 2 leiden+ (pleiden+).
// ex_iters as in app/cluster_main.cpp:101-114 (negative: until the objective stops rising).
int orc_run_clustering(void* gh, void* cdh, int method, int ex_iters, uint64_t seed, int32_t* labels_out, OrcStats* st) {
    return orc_guard([&]() -> int {
        auto* g = (OrcGraph*)gh;
        auto* cd = (OrcCD*)cdh;
        auto run = [&](auto& eng, auto& gg, auto& c) {
            i64 lv = 0, tn = 0;
            std::vector<i32> part;
            u64 pass = 0;
            auto one = [&](bool improve, const std::vector<i32>* input) {
                if (method == 0) {
                    std::vector<i32> con;
                    if (improve) con = *input;
                    return eng.louvain_part(gg, c, improve, con, &lv, &tn);
                }
                u64 s = seed + 0x9E3779B97F4A7C15ull * pass;
                pass++;
                return eng.leiden_part(gg, c, method == 2, improve, improve ? input->data() : nullptr, s, &lv, &tn);
            };
            part = one(false, nullptr);
            double last = -std::numeric_limits<double>::infinity();
            int counter = 0;
            while (true) {
                bool terminate = true;
                if (ex_iters < 0) {
                    if (c.get_objective() > last) terminate = false;
                    last = c.get_objective();
                } else {
                    if (counter++ < ex_iters) terminate = false;
                }
                if (terminate) break;
                std::vector<i32> con = part;
                part = one(true, &con);
            }
            std::copy(part.begin(), part.end(), labels_out);
            if (st) {
                st->levels = lv;
                st->total_nnz = tn;
                st->sweeps = eng.total_sweeps;
                st->moves = eng.total_moves;
                st->objective = c.get_objective();
                st->raw_obj = c.obj;
                st->label_count = c.label_count;
            }
            return 0;
        };
        if (g->kind == 2) {
            Engine<float> e;
            return run(e, g->gf, cd->cf);
        }
        Engine<i32> e;
        return run(e, g->gi, cd->ci);
    });
}

// leiden_part / louvain_part, one call (no ex_iters loop).
int orc_leiden_part(void* gh, void* cdh, int plus, int improve, const int32_t* input, uint64_t seed, int32_t* labels_out,
                    OrcStats* st) {
    return orc_guard([&]() -> int {
        auto* g = (OrcGraph*)gh;
        auto* cd = (OrcCD*)cdh;
        auto run = [&](auto& eng, auto& gg, auto& c) {
            i64 lv = 0, tn = 0;
            auto part = eng.leiden_part(gg, c, plus != 0, improve != 0, input, seed, &lv, &tn);
            std::copy(part.begin(), part.end(), labels_out);
            if (st) {
                st->levels = lv;
                st->total_nnz = tn;
                st->sweeps = eng.total_sweeps;
                st->moves = eng.total_moves;
                st->objective = c.get_objective();
                st->raw_obj = c.obj;
                st->label_count = c.label_count;
            }
            return 0;
        };
        if (g->kind == 2) {
            Engine<float> e;
            return run(e, g->gf, cd->cf);
        }
        Engine<i32> e;
        return run(e, g->gi, cd->ci);
    });
}

int orc_louvain_part(void* gh, void* cdh, int constrained, const int32_t* constraint, int32_t* labels_out, OrcStats* st) {
    return orc_guard([&]() -> int {
        auto* g = (OrcGraph*)gh;
        auto* cd = (OrcCD*)cdh;
        auto run = [&](auto& eng, auto& gg, auto& c) {
            i64 lv = 0, tn = 0;
            std::vector<i32> con;
            if (constrained) con.assign(constraint, constraint + gg.n);
            auto part = eng.louvain_part(gg, c, constrained != 0, con, &lv, &tn);
            std::copy(part.begin(), part.end(), labels_out);
            if (st) {
                st->levels = lv;
                st->total_nnz = tn;
                st->sweeps = eng.total_sweeps;
                st->moves = eng.total_moves;
                st->objective = c.get_objective();
                st->raw_obj = c.obj;
                st->label_count = c.label_count;
            }
            return 0;
        };
        if (g->kind == 2) {
            Engine<float> e;
            return run(e, g->gf, cd->cf);
        }
        Engine<i32> e;
        return run(e, g->gi, cd->ci);
    });
}

// ---- memetic driver, app/memetic_clustering.cpp:27-219 ---------------------
// intersection_cluster (:27-62) with canonical ids: ranks of the distinct
// (c1, c2) pairs in ascending order (the reference's ids follow hash-slot order)
int64_t orc_intersect(const int32_t* c1, const int32_t* c2, int64_t n, int32_t* out) {
    std::vector<std::pair<u64, i32>> kv((size_t)n);
    for (int64_t i = 0; i < n; i++) kv[i] = {((u64)(u32)c1[i] << 32) | (u64)(u32)c2[i], (i32)i};
    std::sort(kv.begin(), kv.end());
    int64_t r = -1;
    for (int64_t x = 0; x < n; x++) {
        if (x == 0 || kv[x].first != kv[x - 1].first) r++;
        out[kv[x].second] = (i32)r;
    }
    return r + 1;
}

// gen_signature (:64-104): bit j set when edge j joins two clusters
void orc_signature(void* gh, const int32_t* labels, uint32_t* sign) {
    auto* g = (OrcGraph*)gh;
    auto run = [&](auto& gg) {
        const int64_t words = (std::max<int64_t>(gg.nnz, 1) + 31) / 32;
        std::fill(sign, sign + words, 0u);
        for (int64_t i = 0; i < gg.n; i++)
            for (int64_t j = gg.rowptr[i]; j < gg.rowptr[i + 1]; j++)
                if (labels[i] != labels[gg.col[j]]) sign[j / 32] |= 1u << (j % 32);
    };
    if (g->kind == 2) run(g->gf);
    else run(g->gi);
}

struct OrcMemeStats {
    double objective;
    int64_t label_count;
    int64_t offspring;
    int64_t replaced;
    double best_initial;
};

static inline int64_t orc_uniform_below(SplitMix64& r, int64_t m) {
    return (int64_t)(((unsigned __int128)r.next() * (u64)m) >> 64);
}

// meme_cluster (:118-219) with `offspring` children instead of the time limit;
// the random stream matches the GPU driver's call for call
int orc_meme_cluster(void* gh, int objective, double mult, int pop_size, int64_t offspring, uint64_t seed,
                     int32_t* labels_out, OrcMemeStats* st) {
    return orc_guard([&]() -> int {
        auto* g = (OrcGraph*)gh;
        auto run = [&](auto& eng, auto& gg) {
            using W = typename std::remove_reference_t<decltype(gg)>::Weight;
            const int64_t n = gg.n;
            const int64_t words = (std::max<int64_t>(gg.nnz, 1) + 31) / 32;
            struct Member {
                std::vector<i32> clusters;
                std::vector<uint32_t> sign;
                double obj = 0;
                int64_t labels = 0;
            };
            std::vector<Member> pop((size_t)pop_size);
            SplitMix64 rng(seed);
            double best_initial = -std::numeric_limits<double>::infinity();
            auto signature = [&](const std::vector<i32>& c, std::vector<uint32_t>& s) {
                s.assign((size_t)words, 0u);
                for (int64_t i = 0; i < n; i++)
                    for (int64_t j = gg.rowptr[i]; j < gg.rowptr[i + 1]; j++)
                        if (c[i] != c[gg.col[j]]) s[j / 32] |= 1u << (j % 32);
            };
            i64 lv = 0, tn = 0;
            for (int p = 0; p < pop_size; p++) {
                auto cd = make_objective<W>(gg, objective, mult);
                pop[p].clusters = eng.leiden_part(gg, cd, true, false, nullptr, rng.next(), &lv, &tn);
                pop[p].obj = cd.get_objective();
                pop[p].labels = cd.label_count;
                signature(pop[p].clusters, pop[p].sign);
                best_initial = std::max(best_initial, pop[p].obj);
            }
            auto pick = [&]() {
                const int64_t a = orc_uniform_below(rng, pop_size);
                const int64_t b = (a + orc_uniform_below(rng, pop_size - 1)) % pop_size;
                return pop[a].obj > pop[b].obj ? a : b;
            };
            int64_t made = 0, replaced = 0;
            std::vector<i32> constraint((size_t)n);
            std::vector<uint32_t> csign;
            while (made < offspring) {
                const int64_t p1 = pick();
                int64_t p2 = p1;
                while (p2 == p1) p2 = pick();
                orc_intersect(pop[p1].clusters.data(), pop[p2].clusters.data(), n, constraint.data());
                auto cd = make_objective<W>(gg, objective, mult);
                std::vector<i32> child = eng.louvain_part(gg, cd, true, constraint, &lv, &tn);
                for (int x = 0; x < 5; x++) {
                    std::vector<i32> in = child;
                    child = eng.leiden_part(gg, cd, true, true, in.data(), rng.next(), &lv, &tn);
                }
                made++;
                const double obj = cd.get_objective();
                signature(child, csign);
                int64_t am = -1;
                int64_t min_diff = std::numeric_limits<int64_t>::max();
                for (int p = 0; p < pop_size; p++) {
                    if (pop[p].obj < obj) {
                        int64_t d = 0;
                        for (int64_t w = 0; w < words; w++) d += __builtin_popcount(csign[w] ^ pop[p].sign[w]);
                        if (d < min_diff) {
                            min_diff = d;
                            am = p;
                        }
                    }
                }
                if (am >= 0) {
                    pop[am].clusters = child;
                    pop[am].sign = csign;
                    pop[am].obj = obj;
                    pop[am].labels = cd.label_count;
                    replaced++;
                }
            }
            int am = 0;
            for (int p = 1; p < pop_size; p++)
                if (pop[p].obj > pop[am].obj) am = p;
            std::copy(pop[am].clusters.begin(), pop[am].clusters.end(), labels_out);
            if (st) {
                st->objective = pop[am].obj;
                st->label_count = pop[am].labels;
                st->offspring = made;
                st->replaced = replaced;
                st->best_initial = best_initial;
            }
            return 0;
        };
        if (g->kind == 2) {
            Engine<float> e;
            return run(e, g->gf);
        }
        Engine<i32> e;
        return run(e, g->gi);
    });
}

double orc_verify_objective(void* gh, const int32_t* labels, int objective, double mult, double* raw_obj) {
    auto* g = (OrcGraph*)gh;
    if (g->kind == 2) return verify_objective<float>(g->gf, labels, objective, mult, raw_obj);
    return verify_objective<i32>(g->gi, labels, objective, mult, raw_obj);
}

// connected_comps (app/cluster_main.cpp:67-99): number of components after
// deleting the cut edges of `labels`.
int64_t orc_connected_components(int64_t n, const int64_t* rowptr, const int32_t* col, const int32_t* labels) {
    std::vector<i32> comp(n, -1);
    std::vector<i32> q;
    q.reserve(n);
    i64 t = 0;
    for (i64 i = 0; i < n; i++) {
        if (comp[i] != -1) continue;
        q.clear();
        q.push_back((i32)i);
        comp[i] = (i32)t;
        for (size_t h = 0; h < q.size(); h++) {
            i32 u = q[h];
            for (i64 j = rowptr[u]; j < rowptr[u + 1]; j++) {
                i32 v = col[j];
                if (comp[v] == -1 && labels[v] == labels[u]) {
                    comp[v] = (i32)t;
                    q.push_back(v);
                }
            }
        }
        t++;
    }
    return t;
}

void orc_det_scan(const double* a, double* out, int64_t k) { det_scan_incl(a, out, k); }
double orc_det_reduce(const double* a, int64_t k) { return det_reduce(a, k); }
uint32_t orc_murmur3(uint32_t k) { return murmur3_32(k); }

void orc_set_afterburner_reference_order(int on) { g_afterburner_reference_order = on ? 1 : 0; }

int orc_num_threads() {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
