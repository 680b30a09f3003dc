// graph_io.cu -- graph input (app/io/io_mtx.cpp:95-345, app/io/io_metis.cpp:64-181).
//
// The text is parsed on the host (one pass, the reference's number rules:
// digits only, 1-based ids); the CSR of a Matrix Market file is built on the
// GPU from its edge list (construct_from_edgelist, io_mtx.cpp:95-201): self
// loops and zero-weight entries are dropped, every entry is stored in both
// directions, entries of a non-symmetric file are de-duplicated as unordered
// pairs, and rows are sorted by column.  Here the rows come out of one stable
// LSD radix sort of the directed (row, column) keys, so rows are sorted and
// duplicate entries of a symmetric file keep their input order -- the CSR is
// deterministic (the reference writes rows with atomics, then sorts with an
// unstable sort).  METIS files are CSR already: ids go 1-based to 0-based.
#include <cctype>
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>
#include "kernels.cuh"
#include "graph_io.cuh"

namespace pggc {

namespace {

std::vector<char> read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary | std::ios::ate);
    if (!f.is_open()) throw InvalidArg("could not open graph file " + path);
    std::streamsize sz = f.tellg();
    f.seekg(0);
    std::vector<char> buf((size_t)sz + 1);
    if (sz > 0 && !f.read(buf.data(), sz)) throw InvalidArg("could not read graph file " + path);
    buf[(size_t)sz] = '\n';  // a trailing newline keeps the scanner inside the buffer
    return buf;
}

// io_common.hpp fast_atoi: digits only; saturates at 2^58 instead of wrapping,
// so an oversized number is rejected by the range checks
template <class T>
T read_uint(const char*& s) {
    T v = 0;
    while (std::isdigit((unsigned char)*s)) {
        if (v < ((T)1 << 58)) v = v * 10 + (T)(*s - '0');
        s++;
    }
    return v;
}

// 1-based id in the file -> 0-based vertex
i32 vertex_id(i64 v, i64 n) {
    if (v < 1 || v > n) throw InvalidArg("vertex id " + std::to_string(v) + " outside [1, " + std::to_string(n) + "]");
    return (i32)(v - 1);
}

void skip_line(const char*& s, const char* end) {
    while (s < end && *s != '\n') s++;
    if (s < end) s++;
}

}  // namespace

// io_mtx.cpp:204-333
void parse_mtx(const std::string& path, bool& uniform, EdgeList& el) {
    std::vector<char> buf = read_file(path);
    const char* f = buf.data();
    const char* end = buf.data() + buf.size();
    // banner: %%MatrixMarket matrix <coordinate> <pattern|integer|real> <general|symmetric>
    std::string fields[5];
    {
        int k = 0;
        const char* s = f;
        while (s < end && *s != '\n') {
            while (s < end && *s != '\n' && !std::isalnum((unsigned char)*s)) s++;
            const char* b = s;
            while (s < end && std::isalnum((unsigned char)*s)) s++;
            if (s > b && k < 5) fields[k++].assign(b, s);
        }
    }
    const bool coordinate = fields[2] == "coordinate";
    const bool pattern = fields[3] == "pattern";
    const bool integer = fields[3] == "integer";
    el.symmetric = fields[4] == "symmetric";
    if (!coordinate) throw InvalidArg("only coordinate Matrix Market files are supported");
    if (!pattern && !integer) uniform = true;  // non-integer weights are ignored
    if (!el.symmetric) uniform = true;          // weights of non-symmetric files are ignored
    while (f < end && *f == '%') skip_line(f, end);
    while (f < end && !std::isdigit((unsigned char)*f)) f++;
    u64 hdr[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        hdr[i] = read_uint<u64>(f);
        while (f < end && !std::isdigit((unsigned char)*f)) {
            if (*f == '\n') {
                i = 4;
                f++;
                break;
            }
            f++;
        }
    }
    if (hdr[0] != hdr[1]) throw InvalidArg("bipartite (non-square) Matrix Market files are not supported");
    if (hdr[0] >= 2147483647ull) throw InvalidArg("too many vertices");
    el.n = (i64)hdr[0];
    const i64 m = (i64)hdr[2];
    el.src.resize((size_t)m);
    el.dst.resize((size_t)m);
    el.weighted = !uniform && !pattern;
    if (el.weighted) el.w.resize((size_t)m);
    i64 read = 0;
    int state = 0;  // 0 source, 1 destination, 2 weight
    while (f < end) {
        while (f < end && !std::isdigit((unsigned char)*f)) {
            if (*f == '%') {
                skip_line(f, end);
                continue;
            }
            if (*f == '\n' && state != 0) throw InvalidArg("Matrix Market line with exactly one value");
            f++;
        }
        if (f >= end) break;
        if (read >= m) throw InvalidArg("more Matrix Market entries than the header states");
        if (state == 0) {
            el.src[(size_t)read] = vertex_id(read_uint<i64>(f), el.n);
            state = 1;
        } else if (state == 1) {
            el.dst[(size_t)read] = vertex_id(read_uint<i64>(f), el.n);
            if (!el.weighted) {
                state = 0;
                read++;
                skip_line(f, end);
            } else {
                state = 2;
            }
        } else {
            el.w[(size_t)read] = (i32)read_uint<i64>(f);
            read++;
            state = 0;
            skip_line(f, end);
        }
    }
    if (read != m) throw InvalidArg("Matrix Market entry count differs from the header");
}

// io_metis.cpp:64-181
void parse_metis(const std::string& path, bool& uniform, CsrHost& g) {
    std::vector<char> buf = read_file(path);
    const char* f = buf.data();
    const char* end = buf.data() + buf.size();
    while (f < end && *f == '%') skip_line(f, end);
    while (f < end && !std::isdigit((unsigned char)*f)) f++;
    u64 hdr[4] = {0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        hdr[i] = read_uint<u64>(f);
        while (f < end && !std::isdigit((unsigned char)*f)) {
            if (*f == '\n') {
                i = 4;
                f++;
                break;
            }
            f++;
        }
    }
    const i64 n = (i64)hdr[0], m = (i64)hdr[1];
    const int fmt = (int)hdr[2], ncon = (int)hdr[3];
    if (fmt != 0 && fmt != 1) throw InvalidArg("unsupported METIS format flags (vertex weights)");
    if (ncon != 0) throw InvalidArg("unsupported METIS ncon (vertex weights)");
    if (n >= 2147483647) throw InvalidArg("too many vertices");
    const bool has_ew = fmt == 1;
    if (!has_ew) uniform = true;
    g.n = n;
    g.rowptr.assign((size_t)n + 1, 0);
    g.col.resize((size_t)(2 * m));
    g.weighted = has_ew && !uniform;
    if (g.weighted) g.w.resize((size_t)(2 * m));
    i64 edges = 0, rows = 0;
    bool is_value = false;
    while (f < end) {
        while (f < end && !std::isdigit((unsigned char)*f)) {
            if (*f == '%') {
                skip_line(f, end);
                continue;
            }
            if (*f == '\n' && rows < n) g.rowptr[(size_t)++rows] = edges;
            f++;
        }
        if (f >= end) break;
        const i64 v = read_uint<i64>(f);
        if (!is_value) {
            if (edges >= 2 * m) throw InvalidArg("more METIS adjacency entries than the header states");
            g.col[(size_t)edges] = vertex_id(v, n);
            if (!has_ew) edges++;
        } else {
            if (g.weighted) g.w[(size_t)edges] = (i32)v;
            edges++;
        }
        if (has_ew) is_value = !is_value;
    }
    if (rows != n || edges != 2 * m)
        throw InvalidArg("METIS line or adjacency count differs from the header (" + std::to_string(rows) + " lines, " +
                         std::to_string(edges) + " entries; expected " + std::to_string(n) + " and " +
                         std::to_string(2 * m) + ")");
}

// ---------------------------------------------------------------------------
// GPU CSR construction from an edge list
// ---------------------------------------------------------------------------
// directed keys (row << cb | col) of both directions of every kept entry;
// dropped entries get the all-ones key and sort last
__global__ void k_edge_keys(const i32* src, const i32* dst, const i32* w, i64 m, int cb, u64 drop, u64* keys,
                            i32* vals) {
    for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < m; j += (i64)gridDim.x * blockDim.x) {
        const i32 u = src[j], v = dst[j];
        const i32 x = w ? w[j] : 1;
        const bool keep = u != v && x != 0;
        keys[2 * j] = keep ? (((u64)(u32)u << cb) | (u64)(u32)v) : drop;
        keys[2 * j + 1] = keep ? (((u64)(u32)v << cb) | (u64)(u32)u) : drop;
        vals[2 * j] = x;
        vals[2 * j + 1] = x;
    }
}

// entry x survives: not dropped, and (symmetric file) or first of its key
struct KeepIn {
    const u64* keys;
    u64 drop;
    int dedupe;
    __device__ i64 operator()(i64 x) const {
        const u64 k = keys[x];
        if (k == drop) return 0;
        if (dedupe && x > 0 && keys[x - 1] == k) return 0;
        return 1;
    }
};
struct KeepEpi {
    const u64* keys;
    const i32* vals;
    u64 cmask;
    int cb;
    i32* col;
    i32* w;
    unsigned long long* deg;
    __device__ void operator()(i64 x, i64 excl, i64 v) const {
        if (!v) return;
        const u64 k = keys[x];
        col[excl] = (i32)(k & cmask);
        if (w) w[excl] = vals[x];
        atomicAdd(&deg[k >> cb], 1ull);
    }
};
struct DegIn {
    const unsigned long long* deg;
    i64 n;
    __device__ i64 operator()(i64 i) const { return i < n ? (i64)deg[i] : 0; }
};
struct RowptrOutIO {
    i64* rp;
    __device__ void operator()(i64 i, i64 excl, i64) const { rp[i] = excl; }
};

__global__ void k_check_edge_ids(const i32* src, const i32* dst, i64 m, i64 n, int* bad) {
    for (i64 j = blockIdx.x * (i64)blockDim.x + threadIdx.x; j < m; j += (i64)gridDim.x * blockDim.x)
        if (src[j] < 0 || src[j] >= n || dst[j] < 0 || dst[j] >= n) atomicExch(bad, 1);
}

void check_edge_ids(Context& ctx, const i32* src, const i32* dst, i64 m, i64 n, int* d_bad) {
    PGGC_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(int), ctx.stream));
    if (m <= 0) return;
    const int grid = (int)std::min<i64>(ceil_div(m, 256), (i64)ctx.num_sms * 16);
    k_check_edge_ids<<<grid, 256, 0, ctx.stream>>>(src, dst, m, n, d_bad);
    PGGC_LAUNCH_CHECK();
}

i64 build_csr_from_edges(Context& ctx, i64 n, i64 m, const i32* src, const i32* dst, const i32* w, bool symmetric,
                         DBuf<i64>& rowptr, DBuf<i32>& col, DBuf<i32>& wout) {
    rowptr = DBuf<i64>(ctx, n + 1);
    if (m <= 0 || n <= 0) {
        PGGC_CUDA(cudaMemsetAsync(rowptr.p, 0, sizeof(i64) * (n + 1), ctx.stream));
        col = DBuf<i32>(ctx, 1);
        if (w) wout = DBuf<i32>(ctx, 1);
        return 0;
    }
    const int cb = std::max(1, bits_for((u64)(n - 1)));
    const u64 drop = (cb * 2 >= 64) ? ~0ull : ((1ull << (2 * cb)) - 1);
    const i64 k = 2 * m;
    DBuf<u64> keys(ctx, k), keys2(ctx, k);
    DBuf<i32> vals(ctx, k), vals2(ctx, k);
    const int grid = (int)std::min<i64>(ceil_div(m, 256), (i64)ctx.num_sms * 16);
    k_edge_keys<<<grid, 256, 0, ctx.stream>>>(src, dst, w, m, cb, drop, keys.p, vals.p);
    PGGC_LAUNCH_CHECK();
    radix_sort_pairs<i32>(ctx, keys.p, vals.p, k, 0, 2 * cb, keys2.p, vals2.p);
    DBuf<unsigned long long> deg(ctx, n);
    PGGC_CUDA(cudaMemsetAsync(deg.p, 0, sizeof(unsigned long long) * n, ctx.stream));
    col = DBuf<i32>(ctx, k);
    if (w) wout = DBuf<i32>(ctx, k);
    DBuf<i64> total(ctx, 1);
    scan_apply(ctx, KeepIn{keys.p, drop, symmetric ? 0 : 1},
               KeepEpi{keys.p, vals.p, (1ull << cb) - 1, cb, col.p, w ? wout.p : nullptr, deg.p}, k, nullptr,
               total.p);
    scan_apply(ctx, DegIn{deg.p, n}, RowptrOutIO{rowptr.p}, n + 1, nullptr, nullptr);
    return ctx.read1(total.p);
}

}  // namespace pggc
