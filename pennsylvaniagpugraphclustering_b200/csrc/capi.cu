// capi.cu -- the extern "C" boundary declared in include/pggc.h.
#include <algorithm>
#include <cstring>
#include <string>
#include <thread>
#include "kernels.cuh"
#include "graph_io.cuh"
#include "mlp_train.cuh"
#include "pggc.h"

using namespace pggc;

namespace pggc {
std::atomic<unsigned long long> g_kernel_launches{0};
}

// The context is reference counted: every graph and cluster_data created on it
// holds a reference, so the device buffers they own are released on a live
// stream whatever order the caller destroys things in.
struct pggc_context {
    std::unique_ptr<Context> ctx;
    std::atomic<int> refs{1};
    // extra streams for pggc_batch_run, created on first use and kept
    std::mutex workers_mu;
    std::vector<std::unique_ptr<Context>> workers;
    // held for a whole pggc_batch_run: two batches on one context would
    // otherwise drive the same worker contexts at once
    std::mutex batch_mu;
};

static void ctx_retain(pggc_context* c) { c->refs.fetch_add(1); }
static void ctx_release(pggc_context* c) {
    if (c && c->refs.fetch_sub(1) == 1) delete c;
}

struct pggc_graph {
    pggc_context* owner = nullptr;
    int kind = PGGC_W_UNIFORM;
    std::unique_ptr<Graph<i32>> gi;
    std::unique_ptr<Graph<float>> gf;
    bool is_float() const { return kind == PGGC_W_FLOAT32; }
    explicit pggc_graph(pggc_context* o) : owner(o) { ctx_retain(o); }
    ~pggc_graph() {
        gi.reset();
        gf.reset();
        ctx_release(owner);
    }
};

struct pggc_cluster_data {
    pggc_context* owner = nullptr;
    bool is_float = false;
    ClusterState<i64> ci;
    ClusterState<double> cf;
    explicit pggc_cluster_data(pggc_context* o) : owner(o) { ctx_retain(o); }
    ~pggc_cluster_data() {
        ci.total_deg.reset();
        cf.total_deg.reset();
        ctx_release(owner);
    }
};

namespace {

thread_local std::string g_last_error;

pggc_status fail(pggc_status s, const std::string& msg) {
    g_last_error = msg;
    return s;
}

template <class F>
pggc_status guarded(F f) {
    try {
        f();
        return PGGC_OK;
    } catch (const InvalidArg& e) {
        return fail(PGGC_ERR_INVALID, e.what());
    } catch (const DeviceFault& e) {
        return fail(PGGC_ERR_DEVICE, e.what());
    } catch (const CudaError& e) {
        return fail(PGGC_ERR_CUDA, e.what());
    } catch (const std::exception& e) {
        return fail(PGGC_ERR_INTERNAL, e.what());
    }
}

void need(bool cond, const char* what) {
    if (!cond) throw InvalidArg(what);
}

// caller array -> device pointer (copied in for host memory)
template <class T>
struct In {
    DBuf<T> tmp;
    const T* p = nullptr;
    In(Context& ctx, const T* src, i64 count, int mem_kind) {
        if (!src || count <= 0) {
            p = src;
            return;
        }
        if (mem_kind == PGGC_MEM_DEVICE) {
            p = src;
        } else {
            tmp = DBuf<T>(ctx, count);
            PGGC_CUDA(cudaMemcpyAsync(tmp.p, src, sizeof(T) * (size_t)count, cudaMemcpyHostToDevice, ctx.stream));
            p = tmp.p;
        }
    }
};

// caller output array: device pointer for the kernels, copied out by finish()
template <class T>
struct Out {
    Context& ctx;
    DBuf<T> tmp;
    T* user;
    T* p;
    i64 count;
    int mem_kind;
    Out(Context& c, T* dst, i64 n, int mk, bool copy_in) : ctx(c), user(dst), p(dst), count(n), mem_kind(mk) {
        if (mem_kind != PGGC_MEM_DEVICE && dst && n > 0) {
            tmp = DBuf<T>(ctx, n);
            p = tmp.p;
            if (copy_in)
                PGGC_CUDA(cudaMemcpyAsync(tmp.p, dst, sizeof(T) * (size_t)n, cudaMemcpyHostToDevice, ctx.stream));
        }
    }
    void finish() {
        if (mem_kind != PGGC_MEM_DEVICE && user && count > 0)
            PGGC_CUDA(cudaMemcpyAsync(user, p, sizeof(T) * (size_t)count, cudaMemcpyDeviceToHost, ctx.stream));
    }
};

__global__ void k_labels_in_range(const i32* labels, i64 n, i64 hi, int* bad) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        if (labels[i] < 0 || labels[i] >= hi) atomicExch(bad, 1);
}

// rejects label arrays with entries outside [0, hi) before any kernel indexes by them
void check_labels(Context& c, const i32* labels, i64 n, i64 hi, const char* what) {
    if (n <= 0) return;
    DBuf<int> bad(c, 1);
    PGGC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), c.stream));
    k_labels_in_range<<<(int)std::min<i64>(ceil_div(n, 256), 4096), 256, 0, c.stream>>>(labels, n, hi, bad.p);
    PGGC_LAUNCH_CHECK();
    need(c.read1(bad.p) == 0, what);
}

void check_mem_kind(int mk) { need(mk == PGGC_MEM_HOST || mk == PGGC_MEM_DEVICE, "mem_kind must be PGGC_MEM_HOST or PGGC_MEM_DEVICE"); }

// CSR checks on the device copy: bit 0 bad offsets, bit 1 column out of range,
// bit 2 self-loop.  Columns are only checked inside well-formed rows.
__global__ void k_validate_csr(const i64* rowptr, const i32* col, i64 n, i64 nnz, int* bad) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x) {
        i64 b = rowptr[i], e = rowptr[i + 1];
        if (b < 0 || e < b || e > nnz || (i == 0 && b != 0) || (i == n - 1 && e != nnz)) {
            atomicOr(bad, 1);
            continue;
        }
        for (i64 j = b; j < e; j++) {
            i32 v = col[j];
            if (v < 0 || v >= n) atomicOr(bad, 2);
            else if (v == (i32)i) atomicOr(bad, 4);
        }
    }
}

void validate_csr_device(Context& c, const i64* rowptr, const i32* col, i64 n, i64 nnz) {
    DBuf<int> bad(c, 1);
    PGGC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), c.stream));
    if (n > 0) {
        k_validate_csr<<<(int)std::min<i64>(ceil_div(n, 256), (i64)c.num_sms * 16), 256, 0, c.stream>>>(rowptr, col, n,
                                                                                                       nnz, bad.p);
        PGGC_LAUNCH_CHECK();
    }
    int b = c.read1(bad.p);
    if (n == 0) {
        i64 r0 = c.read1(rowptr);
        need(r0 == 0 && nnz == 0, "an empty graph must have rowptr = {0} and nnz = 0");
    }
    need(!(b & 1), "rowptr must start at 0, be non-decreasing and end at nnz");
    need(!(b & 2), "column index out of range");
    need(!(b & 4), "self-loops are not supported");
}

template <class W>
std::unique_ptr<Graph<W>> make_graph(Context& ctx, int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col,
                                     const void* weights, int kind, const void* vtx_w, int objective, int mem_kind) {
    using V = typename Traits<W>::V;
    auto g = std::make_unique<Graph<W>>();
    g->n = n;
    g->nnz = nnz;
    g->uniform = kind == PGGC_W_UNIFORM;
    g->rowptr = DBuf<i64>(ctx, n + 1);
    g->col = DBuf<i32>(ctx, std::max<i64>(nnz, 1));
    auto kindc = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    PGGC_CUDA(cudaMemcpyAsync(g->rowptr.p, rowptr, sizeof(i64) * (n + 1), kindc, ctx.stream));
    if (nnz > 0) PGGC_CUDA(cudaMemcpyAsync(g->col.p, col, sizeof(i32) * nnz, kindc, ctx.stream));
    validate_csr_device(ctx, g->rowptr.p, g->col.p, n, nnz);
    if (!g->uniform) {
        need(weights != nullptr, "weights required for a non-uniform graph");
        g->w = DBuf<W>(ctx, std::max<i64>(nnz, 1));
        if (nnz > 0) PGGC_CUDA(cudaMemcpyAsync(g->w.p, weights, sizeof(W) * nnz, kindc, ctx.stream));
    }
    if (vtx_w) {
        g->vtx_w = DBuf<V>(ctx, std::max<i64>(n, 1));
        if (n > 0) PGGC_CUDA(cudaMemcpyAsync(g->vtx_w.p, vtx_w, sizeof(V) * n, kindc, ctx.stream));
    } else {
        default_vertex_weights<W>(ctx, *g, objective);
    }
    row_sums<W>(ctx, *g);
    ctx.sync();
    return g;
}

// a graph whose CSR already lives in device buffers of `ctx` (graph input):
// the buffers move in, nothing is copied
std::unique_ptr<Graph<i32>> adopt_graph(Context& ctx, i64 n, i64 nnz, DBuf<i64>&& rowptr, DBuf<i32>&& col,
                                        DBuf<i32>&& w, bool uniform, int objective) {
    auto g = std::make_unique<Graph<i32>>();
    g->n = n;
    g->nnz = nnz;
    g->uniform = uniform;
    g->rowptr = std::move(rowptr);
    g->col = std::move(col);
    if (!uniform) g->w = std::move(w);
    validate_csr_device(ctx, g->rowptr.p, g->col.p, n, nnz);
    default_vertex_weights<i32>(ctx, *g, objective);
    row_sums<i32>(ctx, *g);
    ctx.sync();
    return g;
}

template <class F>
void dispatch(const pggc_graph* g, F f) {
    if (g->is_float()) f(*g->gf, (double*)nullptr);
    else f(*g->gi, (i64*)nullptr);
}

template <class V>
ClusterState<V>& cstate(pggc_cluster_data* cd);
template <>
ClusterState<i64>& cstate<i64>(pggc_cluster_data* cd) {
    return cd->ci;
}
template <>
ClusterState<double>& cstate<double>(pggc_cluster_data* cd) {
    return cd->cf;
}

void fill_stats(pggc_stats* st, const RunStats& rs, double objective, double raw, i64 L) {
    if (!st) return;
    st->levels = rs.levels;
    st->total_nnz = rs.total_nnz;
    st->sweeps = rs.sweeps;
    st->moves = rs.moves;
    st->passes = rs.passes;
    st->objective = objective;
    st->raw_obj = raw;
    st->label_count = L;
    st->filtered_passes = rs.filtered_passes;
    st->exact_passes = rs.exact_passes;
    st->judge_gain = rs.judge_gain;
    st->fell_back = rs.fell_back;
}

// verify_objective kernels
template <class W>
__global__ void k_verify_totals(DGraph<W> g, const i32* labels, typename Traits<W>::V* total) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < g.n; i += (i64)gridDim.x * blockDim.x) {
        if constexpr (std::is_same<typename Traits<W>::V, double>::value) ::atomicAdd(&total[labels[i]], g.vtx_w[i]);
        else ::atomicAdd((unsigned long long*)&total[labels[i]], (unsigned long long)g.vtx_w[i]);
    }
}
__global__ void k_check_labels(const i32* labels, i64 n, int* bad) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        if (labels[i] < 0 || labels[i] >= n) atomicExch(bad, 1);
}
struct I64Arr {
    const i64* a;
    __device__ i64 operator()(i64 i) const { return a[i]; }
};

}  // namespace

// shared with entry points defined next to their kernels in other files
void pggc_set_last_error(const char* msg) { g_last_error = msg; }

extern "C" {

const char* pggc_last_error(void) { return g_last_error.c_str(); }

uint64_t pggc_launch_count(void) { return (uint64_t)pggc::g_kernel_launches.load(); }

pggc_status pggc_debug_set_probe_limit(pggc_context* ctx, int limit) {
    return guarded([&] {
        need(ctx != nullptr, "NULL context");
        need(limit >= 0, "limit must be >= 0");
        ctx->ctx->probe_cap = (u32)limit;
    });
}

pggc_status pggc_profile_enable(pggc_context* ctx, int on) {
    return guarded([&] {
        need(ctx != nullptr, "NULL context");
        ctx->ctx->prof_flush();
        ctx->ctx->profiling = on != 0;
        ctx->ctx->prof_by_level = on == 2;
    });
}

pggc_status pggc_profile_reset(pggc_context* ctx) {
    return guarded([&] {
        need(ctx != nullptr, "NULL context");
        ctx->ctx->prof_reset();
    });
}

pggc_status pggc_profile_names(pggc_context* ctx, char* buf, int64_t cap, int64_t* needed) {
    return guarded([&] {
        need(ctx != nullptr, "NULL context");
        ctx->ctx->prof_flush();
        std::string all;
        for (auto& kv : ctx->ctx->prof) {
            all += kv.first;
            all += '\n';
        }
        if (needed) *needed = (int64_t)all.size() + 1;
        if (buf && cap > 0) {
            const size_t k = std::min<size_t>(all.size(), (size_t)cap - 1);
            std::memcpy(buf, all.data(), k);
            buf[k] = 0;
        }
    });
}

pggc_status pggc_profile_read(pggc_context* ctx, const char* family, int64_t* launches, double* ms, double* bytes) {
    return guarded([&] {
        need(ctx && family, "NULL argument");
        ctx->ctx->prof_flush();
        auto it = ctx->ctx->prof.find(family);
        ProfStat st;
        if (it != ctx->ctx->prof.end()) st = it->second;
        if (launches) *launches = st.launches;
        if (ms) *ms = st.ms;
        if (bytes) *bytes = st.bytes;
    });
}
const char* pggc_version(void) { return "pggc-b200 0.1 sm_100a"; }

pggc_status pggc_context_create(int device, pggc_context** out) {
    return guarded([&] {
        need(out != nullptr, "out is NULL");
        int count = 0;
        PGGC_CUDA(cudaGetDeviceCount(&count));
        need(device >= 0 && device < count, "device index out of range");
        auto* c = new pggc_context();
        try {
            c->ctx = std::make_unique<Context>(device);
        } catch (...) {
            delete c;
            throw;
        }
        *out = c;
    });
}

pggc_status pggc_context_destroy(pggc_context* ctx) {
    return guarded([&] { ctx_release(ctx); });
}

pggc_status pggc_context_stream(pggc_context* ctx, void** stream_out) {
    return guarded([&] {
        need(ctx && stream_out, "NULL argument");
        *stream_out = (void*)ctx->ctx->stream;
    });
}

pggc_status pggc_graph_create(pggc_context* ctx, int64_t n, int64_t nnz, const int64_t* rowptr, const int32_t* col,
                              const void* weights, int weight_kind, const void* vtx_w, int objective, int mem_kind,
                              pggc_graph** out) {
    return guarded([&] {
        need(ctx && out && rowptr, "NULL argument");
        need(n >= 0 && n < 2147483647 && nnz >= 0, "n must be in [0, 2^31-1) and nnz >= 0");
        need(nnz == 0 || col != nullptr, "col is NULL");
        need(weight_kind >= PGGC_W_UNIFORM && weight_kind <= PGGC_W_FLOAT32, "unknown weight kind");
        need(objective >= PGGC_OBJ_MOD && objective <= PGGC_OBJ_LCC, "unknown objective");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        c.sync();
        auto* g = new pggc_graph(ctx);
        g->kind = weight_kind;
        try {
            if (weight_kind == PGGC_W_FLOAT32)
                g->gf = make_graph<float>(c, n, nnz, rowptr, col, weights, weight_kind, vtx_w, objective, mem_kind);
            else
                g->gi = make_graph<i32>(c, n, nnz, rowptr, col, weights, weight_kind, vtx_w, objective, mem_kind);
        } catch (...) {
            delete g;
            throw;
        }
        *out = g;
    });
}

pggc_status pggc_graph_from_edges(pggc_context* ctx, int64_t n, int64_t m, const int32_t* src, const int32_t* dst,
                                  const int32_t* weights, int symmetric, int objective, int mem_kind,
                                  pggc_graph** out) {
    return guarded([&] {
        need(ctx && out, "NULL argument");
        need(n >= 0 && n < 2147483647 && m >= 0, "n must be in [0, 2^31-1) and m >= 0");
        need(m == 0 || (src && dst), "src or dst is NULL");
        need(weights == nullptr || symmetric, "weights are only kept for symmetric edge lists");
        need(objective >= PGGC_OBJ_MOD && objective <= PGGC_OBJ_LCC, "unknown objective");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        c.sync();
        DBuf<i32> ds, dd, dw;
        const i32 *ps = src, *pd = dst, *pw = weights;
        if (mem_kind == PGGC_MEM_HOST && m > 0) {
            ds = DBuf<i32>(c, m);
            dd = DBuf<i32>(c, m);
            PGGC_CUDA(cudaMemcpyAsync(ds.p, src, sizeof(i32) * m, cudaMemcpyHostToDevice, c.stream));
            PGGC_CUDA(cudaMemcpyAsync(dd.p, dst, sizeof(i32) * m, cudaMemcpyHostToDevice, c.stream));
            ps = ds.p;
            pd = dd.p;
            if (weights) {
                dw = DBuf<i32>(c, m);
                PGGC_CUDA(cudaMemcpyAsync(dw.p, weights, sizeof(i32) * m, cudaMemcpyHostToDevice, c.stream));
                pw = dw.p;
            }
        }
        if (m > 0) {
            DBuf<int> bad(c, 1);
            check_edge_ids(c, ps, pd, m, n, bad.p);
            need(c.read1(bad.p) == 0, "edge endpoint out of range");
        }
        DBuf<i64> rp;
        DBuf<i32> col, w;
        const i64 nnz = build_csr_from_edges(c, n, m, ps, pd, pw, symmetric != 0, rp, col, w);
        ds.reset();
        dd.reset();
        dw.reset();
        const bool uniform = pw == nullptr;
        auto* g = new pggc_graph(ctx);
        g->kind = uniform ? PGGC_W_UNIFORM : PGGC_W_INT32;
        try {
            g->gi = adopt_graph(c, n, nnz, std::move(rp), std::move(col), std::move(w), uniform, objective);
        } catch (...) {
            delete g;
            throw;
        }
        *out = g;
    });
}

pggc_status pggc_graph_load(pggc_context* ctx, const char* path, int objective, int* edge_uniform_out,
                            pggc_graph** out) {
    return guarded([&] {
        need(ctx && path && out, "NULL argument");
        need(objective >= PGGC_OBJ_MOD && objective <= PGGC_OBJ_LCC, "unknown objective");
        Context& c = *ctx->ctx;
        c.sync();
        // Mod and CPM read no edge weights (app/objective_helpers.hpp:24-29)
        bool uniform = objective == PGGC_OBJ_MOD || objective == PGGC_OBJ_CPM;
        const std::string p(path);
        const bool mtx = p.size() >= 4 && p.compare(p.size() - 4, 4, ".mtx") == 0;
        auto* g = new pggc_graph(ctx);
        try {
            if (mtx) {
                EdgeList el;
                parse_mtx(p, uniform, el);
                const i64 m = (i64)el.src.size();
                DBuf<i32> ds(c, std::max<i64>(m, 1)), dd(c, std::max<i64>(m, 1)), dw;
                if (m > 0) {
                    PGGC_CUDA(cudaMemcpyAsync(ds.p, el.src.data(), sizeof(i32) * m, cudaMemcpyHostToDevice, c.stream));
                    PGGC_CUDA(cudaMemcpyAsync(dd.p, el.dst.data(), sizeof(i32) * m, cudaMemcpyHostToDevice, c.stream));
                }
                if (el.weighted) {
                    dw = DBuf<i32>(c, std::max<i64>(m, 1));
                    if (m > 0)
                        PGGC_CUDA(cudaMemcpyAsync(dw.p, el.w.data(), sizeof(i32) * m, cudaMemcpyHostToDevice, c.stream));
                }
                DBuf<i64> rp;
                DBuf<i32> col, w;
                const i64 nnz =
                    build_csr_from_edges(c, el.n, m, ds.p, dd.p, el.weighted ? dw.p : nullptr, el.symmetric, rp, col, w);
                c.sync();  // the host edge list is released next
                g->kind = el.weighted ? PGGC_W_INT32 : PGGC_W_UNIFORM;
                g->gi = adopt_graph(c, el.n, nnz, std::move(rp), std::move(col), std::move(w), !el.weighted, objective);
            } else {
                CsrHost h;
                parse_metis(p, uniform, h);
                const i64 nnz = (i64)h.col.size();
                DBuf<i64> rp(c, h.n + 1);
                DBuf<i32> col(c, std::max<i64>(nnz, 1)), w;
                PGGC_CUDA(cudaMemcpyAsync(rp.p, h.rowptr.data(), sizeof(i64) * (h.n + 1), cudaMemcpyHostToDevice,
                                          c.stream));
                if (nnz > 0)
                    PGGC_CUDA(cudaMemcpyAsync(col.p, h.col.data(), sizeof(i32) * nnz, cudaMemcpyHostToDevice, c.stream));
                if (h.weighted) {
                    w = DBuf<i32>(c, std::max<i64>(nnz, 1));
                    if (nnz > 0)
                        PGGC_CUDA(cudaMemcpyAsync(w.p, h.w.data(), sizeof(i32) * nnz, cudaMemcpyHostToDevice, c.stream));
                }
                g->kind = h.weighted ? PGGC_W_INT32 : PGGC_W_UNIFORM;
                g->gi = adopt_graph(c, h.n, nnz, std::move(rp), std::move(col), std::move(w), !h.weighted, objective);
            }
        } catch (...) {
            delete g;
            throw;
        }
        if (edge_uniform_out) *edge_uniform_out = g->kind == PGGC_W_UNIFORM ? 1 : 0;
        *out = g;
    });
}

pggc_status pggc_graph_set_vertex_weights(pggc_context* ctx, pggc_graph* g, const void* vtx_w, int mem_kind) {
    return guarded([&] {
        need(ctx && g && vtx_w, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        auto kindc = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        c.sync();
        if (g->is_float()) {
            if (g->gf->n > 0)
                PGGC_CUDA(cudaMemcpyAsync(g->gf->vtx_w.p, vtx_w, sizeof(double) * g->gf->n, kindc, c.stream));
        } else {
            if (g->gi->n > 0)
                PGGC_CUDA(cudaMemcpyAsync(g->gi->vtx_w.p, vtx_w, sizeof(i64) * g->gi->n, kindc, c.stream));
        }
        c.sync();
    });
}

pggc_status pggc_graph_destroy(pggc_graph* g) {
    return guarded([&] { delete g; });
}

pggc_status pggc_graph_dims(const pggc_graph* g, int64_t* n, int64_t* nnz, int* weight_kind) {
    return guarded([&] {
        need(g != nullptr, "NULL graph");
        i64 nn = g->is_float() ? g->gf->n : g->gi->n;
        i64 mm = g->is_float() ? g->gf->nnz : g->gi->nnz;
        if (n) *n = nn;
        if (nnz) *nnz = mm;
        if (weight_kind) *weight_kind = g->kind;
    });
}

pggc_status pggc_graph_read(pggc_context* ctx, const pggc_graph* g, int64_t* rowptr, int32_t* col, void* weights,
                            void* vtx_w, int mem_kind) {
    return guarded([&] {
        need(ctx && g, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        auto kindc = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            using W = std::conditional_t<std::is_same<V, double>::value, float, i32>;
            auto gv = gr.view();
            if (rowptr) PGGC_CUDA(cudaMemcpyAsync(rowptr, gv.rowptr, sizeof(i64) * (gr.n + 1), kindc, c.stream));
            if (col && gr.nnz) PGGC_CUDA(cudaMemcpyAsync(col, gv.col, sizeof(i32) * gr.nnz, kindc, c.stream));
            if (weights && gv.w && gr.nnz) PGGC_CUDA(cudaMemcpyAsync(weights, gv.w, sizeof(W) * gr.nnz, kindc, c.stream));
            if (vtx_w && gr.n) PGGC_CUDA(cudaMemcpyAsync(vtx_w, gv.vtx_w, sizeof(V) * gr.n, kindc, c.stream));
        });
        c.sync();
    });
}

pggc_status pggc_cluster_data_create(pggc_context* ctx, const pggc_graph* g, int objective, double lambda_mult,
                                     pggc_cluster_data** out) {
    return guarded([&] {
        need(ctx && g && out, "NULL argument");
        need(objective >= PGGC_OBJ_MOD && objective <= PGGC_OBJ_LCC, "unknown objective");
        Context& c = *ctx->ctx;
        auto* cd = new pggc_cluster_data(ctx);
        try {
            cd->is_float = g->is_float();
            if (g->is_float()) make_cluster_state<float>(c, *g->gf, objective, lambda_mult, cd->cf);
            else make_cluster_state<i32>(c, *g->gi, objective, lambda_mult, cd->ci);
            c.sync();
        } catch (...) {
            delete cd;
            throw;
        }
        *out = cd;
    });
}

pggc_status pggc_cluster_data_destroy(pggc_cluster_data* cd) {
    return guarded([&] { delete cd; });
}

pggc_status pggc_cluster_data_get(const pggc_cluster_data* cd, double* obj, double* objective, double* lambda,
                                  double* uncut, int64_t* label_count) {
    return guarded([&] {
        need(cd != nullptr, "NULL cluster_data");
        auto get = [&](const auto& cs) {
            if (obj) *obj = cs.obj;
            if (objective) *objective = cs.get_objective();
            if (lambda) *lambda = cs.lambda;
            if (uncut) *uncut = (double)cs.uncut;
            if (label_count) *label_count = cs.label_count;
        };
        if (cd->is_float) get(cd->cf);
        else get(cd->ci);
    });
}

pggc_status pggc_cluster_data_total_deg(pggc_context* ctx, const pggc_cluster_data* cd, void* out, int mem_kind) {
    return guarded([&] {
        need(ctx && cd && out, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        auto kindc = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (cd->is_float)
            PGGC_CUDA(cudaMemcpyAsync(out, cd->cf.total_deg.p, sizeof(double) * cd->cf.label_count, kindc, c.stream));
        else
            PGGC_CUDA(cudaMemcpyAsync(out, cd->ci.total_deg.p, sizeof(i64) * cd->ci.label_count, kindc, c.stream));
        c.sync();
    });
}

pggc_status pggc_cluster_data_set(pggc_context* ctx, pggc_cluster_data* cd, int64_t label_count, const void* total_deg,
                                  double uncut, int mem_kind) {
    return guarded([&] {
        need(ctx && cd && total_deg, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        auto kindc = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        auto set = [&](auto& cs, size_t elem) {
            need(label_count >= 0 && label_count <= cs.capacity, "label_count exceeds capacity");
            PGGC_CUDA(cudaMemcpyAsync(cs.total_deg.p, total_deg, elem * label_count, kindc, c.stream));
            cs.label_count = label_count;
            using V = std::remove_reference_t<decltype(cs.uncut)>;
            cs.uncut = (V)uncut;
            update_objective(c, cs);
        };
        if (cd->is_float) set(cd->cf, sizeof(double));
        else set(cd->ci, sizeof(i64));
        c.sync();
    });
}

pggc_status pggc_generate_orderings(pggc_context* ctx, const pggc_graph* g, int32_t* order1, int32_t* order2,
                                    int64_t offsets[4], int mem_kind) {
    return guarded([&] {
        need(ctx && g, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        Ordering o;
        dispatch(g, [&](auto& gr, auto*) { generate_orderings(c, gr.view().rowptr, gr.n, o); });
        auto kindc = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (o.n > 0) {
            if (order1) PGGC_CUDA(cudaMemcpyAsync(order1, o.order1.p, sizeof(i32) * o.n, kindc, c.stream));
            if (order2) PGGC_CUDA(cudaMemcpyAsync(order2, o.order2.p, sizeof(i32) * o.n, kindc, c.stream));
        }
        if (offsets) {
            offsets[0] = o.off_large;
            offsets[1] = o.off_large2;
            offsets[2] = o.off_mid;
            offsets[3] = o.off_mid2;
        }
        c.sync();
    });
}

pggc_status pggc_local_move(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int32_t* part_io,
                            int is_initial, int constrained, int32_t* constraint_io, int64_t constraint_len,
                            int enable_sa, int strict, int sweep_limit, int mem_kind, pggc_stats* stats) {
    return guarded([&] {
        need(ctx && g && cd && part_io, "NULL argument");
        need(!constrained || constraint_io, "constraint required when constrained");
        need(cd->is_float == g->is_float(), "cluster_data / graph weight kinds differ");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            auto& cs = cstate<V>(cd);
            need(!constrained || (constraint_len >= cs.label_count && constraint_len <= cs.capacity),
                 "constraint_len must lie in [label_count, 2n + 64]");
            need(!constrained || constraint_len >= gr.n, "constraint_len must be >= n");
            Out<i32> part(c, part_io, gr.n, mem_kind, true);
            check_labels(c, part.p, gr.n, cs.label_count, "partition labels must lie in [0, label_count)");
            // cluster-indexed constraint with room for appended labels
            DBuf<i32> con;
            if (constrained) {
                con = DBuf<i32>(c, cs.capacity);
                PGGC_CUDA(cudaMemsetAsync(con.p, 0, sizeof(i32) * cs.capacity, c.stream));
                auto k = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
                PGGC_CUDA(cudaMemcpyAsync(con.p, constraint_io, sizeof(i32) * constraint_len, k, c.stream));
            }
            Ordering o;
            generate_orderings(c, gr.view().rowptr, gr.n, o);
            MoveStats ms;
            local_move(c, gr, o, part.p, cs, is_initial != 0, constrained != 0, constrained ? con.p : nullptr,
                       enable_sa != 0, strict != 0, sweep_limit, &ms);
            part.finish();
            if (constrained) {
                auto k = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
                PGGC_CUDA(cudaMemcpyAsync(constraint_io, con.p, sizeof(i32) * constraint_len, k, c.stream));
            }
            c.sync();
            RunStats rs;
            rs.sweeps = ms.sweeps;
            rs.moves = ms.moves;
            fill_stats(stats, rs, cs.get_objective(), cs.obj, cs.label_count);
        });
    });
}

pggc_status pggc_select_pass(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, const int32_t* part,
                             const void* pvals, int32_t* dest_io, float* gain_io, float filter_ratio, int initial,
                             int constrained, const int32_t* constraint, int mem_kind, int64_t* num_candidates) {
    return guarded([&] {
        need(ctx && g && cd && part && pvals && dest_io && gain_io, "NULL argument");
        need(cd->is_float == g->is_float(), "cluster_data / graph weight kinds differ");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            auto& cs = cstate<V>(cd);
            In<i32> pin(c, part, gr.n, mem_kind);
            In<V> pv(c, (const V*)pvals, gr.n, mem_kind);
            DBuf<i32> con;
            if (constrained) {
                con = DBuf<i32>(c, cs.capacity);
                PGGC_CUDA(cudaMemsetAsync(con.p, 0, sizeof(i32) * cs.capacity, c.stream));
                auto k = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
                PGGC_CUDA(cudaMemcpyAsync(con.p, constraint, sizeof(i32) * cs.label_count, k, c.stream));
            }
            check_labels(c, pin.p, gr.n, cs.label_count, "partition labels must lie in [0, label_count)");
            Out<i32> dest(c, dest_io, gr.n, mem_kind, true);
            Out<float> gain(c, gain_io, gr.n, mem_kind, true);
            Ordering o;
            generate_orderings(c, gr.view().rowptr, gr.n, o);
            i64 k = select_pass(c, gr, o, pin.p, pv.p, cs, dest.p, gain.p, filter_ratio, initial != 0,
                                constrained != 0, con.p);
            dest.finish();
            gain.finish();
            c.sync();
            if (num_candidates) *num_candidates = k;
        });
    });
}

pggc_status pggc_build_coarse_graph(pggc_context* ctx, const pggc_graph* g, const int32_t* vcmap, int64_t nc,
                                    int mem_kind, pggc_graph** out) {
    return guarded([&] {
        need(ctx && g && vcmap && out, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        auto* cg = new pggc_graph(ctx);
        try {
            dispatch(g, [&](auto& gr, auto* vtag) {
                using V = std::remove_pointer_t<decltype(vtag)>;
                need(nc >= 0 && nc <= gr.n, "nc out of range");
                In<i32> map(c, vcmap, gr.n, mem_kind);
                check_labels(c, map.p, gr.n, nc, "vcmap entries must lie in [0, nc)");
                auto next = build_coarse_graph(c, gr, map.p, nc);
                coarsen_vtx_w(c, gr, map.p, *next);
                c.sync();
                if constexpr (std::is_same<V, double>::value) {
                    cg->kind = PGGC_W_FLOAT32;
                    cg->gf = std::move(next);
                } else {
                    cg->kind = PGGC_W_INT32;
                    cg->gi = std::move(next);
                }
            });
        } catch (...) {
            delete cg;
            throw;
        }
        *out = cg;
    });
}

pggc_status pggc_coarsen_leidenR(pggc_context* ctx, const pggc_graph* g, const pggc_cluster_data* cd,
                                 const int32_t* constraint, uint32_t seed_pick, uint32_t seed_order,
                                 int32_t* vcmap_out, int64_t* nc_out, int mem_kind) {
    return guarded([&] {
        need(ctx && g && cd && constraint && vcmap_out, "NULL argument");
        need(cd->is_float == g->is_float(), "cluster_data / graph weight kinds differ");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            auto& cs = cstate<V>(const_cast<pggc_cluster_data*>(cd));
            In<i32> con(c, constraint, gr.n, mem_kind);
            check_labels(c, con.p, gr.n, cs.label_count, "constraint labels must lie in [0, label_count)");
            Out<i32> vc(c, vcmap_out, gr.n, mem_kind, false);
            Ordering o;
            generate_orderings(c, gr.view().rowptr, gr.n, o);
            i64 nc = coarsen_leidenR(c, gr, o, con.p, cs, seed_pick, seed_order, vc.p);
            vc.finish();
            c.sync();
            if (nc_out) *nc_out = nc;
        });
    });
}

pggc_status pggc_leiden_part(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int plus, int improve,
                             const int32_t* input, uint64_t seed, int32_t* labels_out, int mem_kind,
                             pggc_stats* stats) {
    return guarded([&] {
        need(ctx && g && cd && labels_out, "NULL argument");
        need(!improve || input, "input partition required when improve");
        need(cd->is_float == g->is_float(), "cluster_data / graph weight kinds differ");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            auto& cs = cstate<V>(cd);
            In<i32> inp(c, improve ? input : nullptr, gr.n, mem_kind);
            if (improve) check_labels(c, inp.p, gr.n, cs.label_count, "input labels must lie in [0, label_count)");
            Out<i32> lab(c, labels_out, gr.n, mem_kind, false);
            RunStats rs;
            rs.passes = 1;
            leiden_part(c, gr, cs, plus != 0, improve != 0, inp.p, seed, lab.p, &rs);
            lab.finish();
            c.sync();
            fill_stats(stats, rs, cs.get_objective(), cs.obj, cs.label_count);
        });
    });
}

pggc_status pggc_louvain_part(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int constrained,
                              const int32_t* constraint, int32_t* labels_out, int mem_kind, pggc_stats* stats) {
    return guarded([&] {
        need(ctx && g && cd && labels_out, "NULL argument");
        need(!constrained || constraint, "constraint required when constrained");
        need(cd->is_float == g->is_float(), "cluster_data / graph weight kinds differ");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            auto& cs = cstate<V>(cd);
            In<i32> con(c, constrained ? constraint : nullptr, gr.n, mem_kind);
            if (constrained) check_labels(c, con.p, gr.n, gr.n, "constraint labels must lie in [0, n)");
            Out<i32> lab(c, labels_out, gr.n, mem_kind, false);
            RunStats rs;
            rs.passes = 1;
            louvain_part(c, gr, cs, constrained != 0, con.p, lab.p, &rs);
            lab.finish();
            c.sync();
            fill_stats(stats, rs, cs.get_objective(), cs.obj, cs.label_count);
        });
    });
}

pggc_status pggc_run_clustering(pggc_context* ctx, const pggc_graph* g, pggc_cluster_data* cd, int method,
                                int ex_iters, uint64_t seed, int32_t* labels_out, int mem_kind, pggc_stats* stats) {
    return guarded([&] {
        need(ctx && g && cd && labels_out, "NULL argument");
        need(method >= PGGC_METHOD_LOUVAIN && method <= PGGC_METHOD_LEIDEN_PLUS, "unknown method");
        need(cd->is_float == g->is_float(), "cluster_data / graph weight kinds differ");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            using W = std::conditional_t<std::is_same<V, double>::value, float, i32>;
            auto& cs = cstate<V>(cd);
            Out<i32> lab(c, labels_out, gr.n, mem_kind, false);
            RunStats rs;
            run_clustering<W>(c, gr, cs, method, ex_iters, seed, lab.p, &rs);
            lab.finish();
            c.sync();
            fill_stats(stats, rs, cs.get_objective(), cs.obj, cs.label_count);
        });
    });
}

// validation shared by the batch entry points
static void check_batch_jobs(pggc_context* ctx, const pggc_batch_job* jobs, int64_t count) {
    need(ctx && (count == 0 || jobs), "NULL argument");
    need(count >= 0, "count must be >= 0");
    for (i64 k = 0; k < count; k++) {
        const auto& J = jobs[k];
        need(J.graph && J.labels_out, "a job has a NULL graph or labels_out");
        need(J.graph->owner == ctx, "a job's graph belongs to another context");
        need(J.method >= PGGC_METHOD_LOUVAIN && J.method <= PGGC_METHOD_LEIDEN_PLUS, "unknown method");
        need(J.objective >= PGGC_OBJ_MOD && J.objective <= PGGC_OBJ_LCC, "unknown objective");
        check_mem_kind(J.mem_kind);
    }
    need(ctx->ctx->filt.mode != 1, "sample logging is not supported in batched runs");
}

// The batch itself (jobs validated, ctx->batch_mu held by the caller).
static void batch_impl(pggc_context* ctx, pggc_batch_job* jobs, int64_t count, int streams) {
    Context& c = *ctx->ctx;
    if (count == 0) return;
    c.sync();
    const int nw = (int)std::min<i64>(streams, count);
    {
        std::lock_guard<std::mutex> lk(ctx->workers_mu);
        while ((int)ctx->workers.size() < nw) ctx->workers.push_back(std::make_unique<Context>(c.device));
    }
    // Device-side ordering of the batch against the context stream: the
    // workers start after the work queued on it so far, and it waits for
    // every worker, so CUDA events recorded on the context stream around
    // this call bracket the whole batch on the device.
    cudaEvent_t start_ev = nullptr;
    std::vector<cudaEvent_t> done_ev((size_t)nw, nullptr);
    PGGC_CUDA(cudaEventCreateWithFlags(&start_ev, cudaEventDisableTiming));
    for (auto& e : done_ev) PGGC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    PGGC_CUDA(cudaEventRecord(start_ev, c.stream));
    std::atomic<i64> next{0};
    std::vector<std::string> msgs((size_t)count);
    auto work = [&](int wi) {
        Context& wc = *ctx->workers[wi];
        cudaSetDevice(wc.device);
        cudaStreamWaitEvent(wc.stream, start_ev, 0);
        // the main context's kernel knobs and learned filter (network,
        // threshold, counters) are shared read-only
        wc.tune = c.tune;
        wc.filt.mode = c.filt.mode;
        wc.filt.net = c.filt.net;
        wc.filt.threshold = c.filt.threshold;
        wc.filt.stats = c.filt.stats;
        wc.filt.max_pass = c.filt.max_pass;
        wc.filt.min_level = c.filt.min_level;
        for (;;) {
            const i64 k = next.fetch_add(1);
            if (k >= count) break;
            pggc_batch_job& J = jobs[k];
            J.status = PGGC_ERR_INTERNAL;
            try {
                dispatch(J.graph, [&](auto& gr, auto* vtag) {
                    using V = std::remove_pointer_t<decltype(vtag)>;
                    using W = std::conditional_t<std::is_same<V, double>::value, float, i32>;
                    ClusterState<V> cs;
                    make_cluster_state<W>(wc, gr, J.objective, J.lambda_mult, cs);
                    Out<i32> lab(wc, J.labels_out, gr.n, J.mem_kind, false);
                    RunStats rs;
                    run_clustering<W>(wc, gr, cs, J.method, J.ex_iters, J.seed, lab.p, &rs);
                    lab.finish();
                    wc.sync();
                    fill_stats(&J.stats, rs, cs.get_objective(), cs.obj, cs.label_count);
                });
                J.status = PGGC_OK;
            } catch (const InvalidArg& e) {
                J.status = PGGC_ERR_INVALID;
                msgs[k] = e.what();
            } catch (const DeviceFault& e) {
                J.status = PGGC_ERR_DEVICE;
                msgs[k] = e.what();
            } catch (const CudaError& e) {
                J.status = PGGC_ERR_CUDA;
                msgs[k] = e.what();
            } catch (const std::exception& e) {
                msgs[k] = e.what();
            }
        }
        wc.filt.mode = 0;
        wc.filt.net = nullptr;
        wc.filt.stats = nullptr;
        cudaEventRecord(done_ev[wi], wc.stream);
    };
    std::vector<std::thread> th;
    for (int wi = 0; wi < nw; wi++) th.emplace_back(work, wi);
    for (auto& t : th) t.join();
    for (auto& e : done_ev) {
        cudaStreamWaitEvent(c.stream, e, 0);
        cudaEventDestroy(e);
    }
    cudaEventDestroy(start_ev);
    for (i64 k = 0; k < count; k++) {
        if (jobs[k].status == PGGC_OK) continue;
        std::string m = "batch job " + std::to_string(k) + ": " + msgs[k];
        if (jobs[k].status == PGGC_ERR_INVALID) throw InvalidArg(m);
        if (jobs[k].status == PGGC_ERR_DEVICE) throw DeviceFault(m);
        if (jobs[k].status == PGGC_ERR_CUDA) throw CudaError(cudaErrorUnknown, m);
        throw std::runtime_error(m);
    }
}

pggc_status pggc_batch_run(pggc_context* ctx, pggc_batch_job* jobs, int64_t count, int streams) {
    return guarded([&] {
        check_batch_jobs(ctx, jobs, count);
        need(streams >= 0 && streams <= 64, "streams must be in [0, 64]");
        std::lock_guard<std::mutex> batch_lock(ctx->batch_mu);
        batch_impl(ctx, jobs, count, streams == 0 ? ctx->ctx->tune.streams : streams);
    });
}

namespace {
TuneParams tune_from(const pggc_tune& t) {
    TuneParams p;
    p.thread_max_deg = t.thread_max_deg >= 24 ? 32 : t.thread_max_deg >= 12 ? 16 : t.thread_max_deg >= 4 ? 8 : 0;
    p.warp_max_deg = t.warp_max_deg >= 80 ? 127 : 32;
    p.load = t.load_factor >= 0.6 ? 0.7f : 0.5f;
    p.streams = std::max(1, std::min(64, t.streams));
    return p;
}
pggc_tune tune_to(const TuneParams& p) {
    pggc_tune t;
    t.thread_max_deg = p.thread_max_deg;
    t.warp_max_deg = p.warp_max_deg;
    t.load_factor = p.load;
    t.streams = p.streams;
    return t;
}
}  // namespace

pggc_status pggc_tune_set(pggc_context* ctx, const pggc_tune* t) {
    return guarded([&] {
        need(ctx && t, "NULL argument");
        ctx->ctx->tune = tune_from(*t);
    });
}

pggc_status pggc_tune_get(pggc_context* ctx, pggc_tune* out) {
    return guarded([&] {
        need(ctx && out, "NULL argument");
        *out = tune_to(ctx->ctx->tune);
    });
}

pggc_status pggc_batch_autotune(pggc_context* ctx, pggc_batch_job* jobs, int64_t count, pggc_tune_trial* trials,
                                int64_t trials_cap, int64_t* n_trials, pggc_tune* best) {
    return guarded([&] {
        check_batch_jobs(ctx, jobs, count);
        need(count > 0, "the autotuner needs at least one job");
        need(trials_cap >= 0 && (trials_cap == 0 || trials), "invalid trial buffer");
        std::lock_guard<std::mutex> batch_lock(ctx->batch_mu);
        Context& c = *ctx->ctx;
        double edges = 0;
        for (i64 k = 0; k < count; k++)
            edges += 0.5 * (double)(jobs[k].graph->is_float() ? jobs[k].graph->gf->nnz : jobs[k].graph->gi->nnz);
        cudaEvent_t e0, e1;
        PGGC_CUDA(cudaEventCreate(&e0));
        PGGC_CUDA(cudaEventCreate(&e1));
        i64 nt = 0;
        // a configuration's time is the better of two batches
        auto trial = [&](const TuneParams& p) -> double {
            c.tune = p;
            double sec = 1e300;
            for (int rep = 0; rep < 2; rep++) {
                PGGC_CUDA(cudaEventRecord(e0, c.stream));
                batch_impl(ctx, jobs, count, p.streams);
                PGGC_CUDA(cudaEventRecord(e1, c.stream));
                PGGC_CUDA(cudaEventSynchronize(e1));
                float ms = 0.f;
                PGGC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                sec = std::min(sec, ms / 1000.0);
            }
            if (nt < trials_cap) {
                trials[nt].config = tune_to(p);
                trials[nt].seconds = sec;
                trials[nt].edges_per_s = sec > 0 ? edges / sec : 0;
            }
            nt++;
            return sec;
        };
        try {
            TuneParams cur = c.tune;
            // warm-up at the widest batch width tried (creates the worker contexts)
            cur.streams = (int)std::min<i64>(32, count);
            c.tune = cur;
            batch_impl(ctx, jobs, count, cur.streams);
            TuneParams bestp = cur;
            double best_s = 1e300;
            // a challenger replaces the best only when more than 2 % faster,
            // so timing noise does not move the knobs
            auto consider = [&](TuneParams p) {
                const double sec = trial(p);
                if (best_s >= 1e299 || sec < 0.98 * best_s) {
                    best_s = sec;
                    bestp = p;
                }
            };
            std::vector<int> widths;
            for (int sw : {1, 4, 8, 16, 32}) {
                const int w = (int)std::min<i64>(sw, count);
                if (std::find(widths.begin(), widths.end(), w) != widths.end()) continue;
                widths.push_back(w);
                TuneParams p = cur;
                p.streams = w;
                consider(p);
            }
            cur = bestp;
            const int th[6][2] = {{32, 127}, {16, 127}, {8, 127}, {0, 127}, {32, 32}, {8, 32}};
            for (auto& t : th) {
                TuneParams p = cur;
                p.thread_max_deg = t[0];
                p.warp_max_deg = t[1];
                if (p.thread_max_deg == cur.thread_max_deg && p.warp_max_deg == cur.warp_max_deg) continue;
                consider(p);
            }
            cur = bestp;
            {
                TuneParams p = cur;
                p.load = cur.load >= 0.7f ? 0.5f : 0.7f;
                consider(p);
            }
            c.tune = bestp;
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (n_trials) *n_trials = nt;
        if (best) *best = tune_to(c.tune);
    });
}

pggc_status pggc_meme_cluster(pggc_context* ctx, const pggc_graph* g, int objective, double lambda_mult, int pop_size,
                              int64_t offspring, double time_limit_s, uint64_t seed, int32_t* labels_out,
                              int mem_kind, pggc_meme_stats* stats) {
    return guarded([&] {
        need(ctx && g && labels_out, "NULL argument");
        need(pop_size >= 2, "pop_size must be at least 2");
        need(offspring >= 0 || time_limit_s > 0, "set an offspring count or a time limit");
        need(objective >= PGGC_OBJ_MOD && objective <= PGGC_OBJ_LCC, "unknown objective");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            using W = std::conditional_t<std::is_same<V, double>::value, float, i32>;
            Out<i32> lab(c, labels_out, gr.n, mem_kind, false);
            MemeStats ms;
            meme_cluster<W>(c, gr, objective, lambda_mult, pop_size, offspring, time_limit_s, seed, lab.p, &ms);
            lab.finish();
            c.sync();
            if (stats) {
                stats->objective = ms.objective;
                stats->label_count = ms.label_count;
                stats->offspring = ms.offspring;
                stats->replaced = ms.replaced;
                stats->best_initial = ms.best_initial;
            }
        });
    });
}

pggc_status pggc_intersect_clusters(pggc_context* ctx, const int32_t* c1, const int32_t* c2, int64_t n, int32_t* out,
                                    int64_t* count_out, int mem_kind) {
    return guarded([&] {
        need(ctx && (n == 0 || (c1 && c2 && out)), "NULL argument");
        need(n >= 0, "n must be >= 0");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        In<i32> a(c, c1, n, mem_kind), b(c, c2, n, mem_kind);
        check_labels(c, a.p, n, std::max<i64>(n, 1), "labels must lie in [0, n)");
        check_labels(c, b.p, n, std::max<i64>(n, 1), "labels must lie in [0, n)");
        Out<i32> o(c, out, n, mem_kind, false);
        const i64 k = intersect_clusters(c, a.p, b.p, n, o.p);
        o.finish();
        c.sync();
        if (count_out) *count_out = k;
    });
}

pggc_status pggc_cut_signature(pggc_context* ctx, const pggc_graph* g, const int32_t* labels, uint32_t* sign_out,
                               int mem_kind) {
    return guarded([&] {
        need(ctx && g && labels && sign_out, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            using W = std::conditional_t<std::is_same<V, double>::value, float, i32>;
            In<i32> lab(c, labels, gr.n, mem_kind);
            check_labels(c, lab.p, gr.n, std::max<i64>(gr.n, 1), "labels must lie in [0, n)");
            const i64 words = ceil_div(std::max<i64>(gr.nnz, 1), 32);
            Out<u32> o(c, sign_out, words, mem_kind, false);
            cut_signature<W>(c, gr, lab.p, o.p);
            o.finish();
            c.sync();
        });
    });
}

pggc_status pggc_verify_objective(pggc_context* ctx, const pggc_graph* g, const int32_t* labels, int objective,
                                  double lambda_mult, int mem_kind, double* objective_out, double* raw_obj_out) {
    return guarded([&] {
        need(ctx && g && labels, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        dispatch(g, [&](auto& gr, auto* vtag) {
            using V = std::remove_pointer_t<decltype(vtag)>;
            using W = std::conditional_t<std::is_same<V, double>::value, float, i32>;
            const i64 n = gr.n;
            In<i32> lab(c, labels, n, mem_kind);
            DBuf<int> bad(c, 1);
            PGGC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), c.stream));
            if (n > 0) {
                k_check_labels<<<(int)std::min<i64>(ceil_div(n, 256), 4096), 256, 0, c.stream>>>(lab.p, n, bad.p);
                PGGC_LAUNCH_CHECK();
            }
            need(c.read1(bad.p) == 0, "labels must lie in [0, n)");
            ClusterState<V> cs;
            make_cluster_state<W>(c, gr, objective, lambda_mult, cs);
            PGGC_CUDA(cudaMemsetAsync(cs.total_deg.p, 0, sizeof(V) * cs.capacity, c.stream));
            if (n > 0) {
                k_verify_totals<W><<<(int)std::min<i64>(ceil_div(n, 256), 4096), 256, 0, c.stream>>>(gr.view(), lab.p,
                                                                                                     cs.total_deg.p);
                PGGC_LAUNCH_CHECK();
            }
            Ordering o;
            generate_orderings(c, gr.view().rowptr, n, o);
            DBuf<V> own(c, std::max<i64>(n, 1));
            own_weights<W>(c, gr, o, lab.p, own.p);
            DBuf<V> u(c, 1);
            if constexpr (std::is_same<V, double>::value) det_reduce(c, DArrIn{own.p}, n, u.p);
            else sum_i64(c, I64Arr{own.p}, n, u.p);
            cs.uncut = c.read1(u.p);
            cs.label_count = n;
            update_objective(c, cs);
            if (objective_out) *objective_out = cs.get_objective();
            if (raw_obj_out) *raw_obj_out = cs.obj;
        });
    });
}

// ---- learned move filter ---------------------------------------------------
static void filter_free_log(Context& c) {
    auto& F = c.filt;
    for (void* q : {(void*)F.log_x, (void*)F.log_y, (void*)F.log_v, (void*)F.log_cnt})
        if (q) PGGC_CUDA(cudaFreeAsync(q, c.stream));
    F.log_x = F.log_y = nullptr;
    F.log_v = nullptr;
    F.log_cnt = nullptr;
    F.log_cap = 0;
}

pggc_status pggc_mlp_infer(pggc_context* ctx, const float* params, const float* features, int64_t count, int mem_kind,
                           float* logits_out) {
    return guarded([&] {
        need(ctx && params && (count == 0 || (features && logits_out)), "NULL argument");
        need(count >= 0, "count must be >= 0");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        In<float> p(c, params, MLP_PARAMS, mem_kind);
        In<float> x(c, features, count * MLP_IN, mem_kind);
        Out<float> out(c, logits_out, count, mem_kind, false);
        DBuf<MlpDev> net(c, 1);
        mlp_pack(c, p.p, net.p);
        mlp_infer(c, net.p, x.p, count, out.p);
        out.finish();
        c.sync();
    });
}

pggc_status pggc_mlp_loss_grad(pggc_context* ctx, const float* params, const float* features, const float* labels,
                               int64_t count, float pos_weight, int mem_kind, float* grad_out, float* loss_out) {
    return guarded([&] {
        need(ctx && params && features && labels && grad_out && loss_out, "NULL argument");
        need(count > 0 && count <= (1 << 20), "count must be in [1, 1048576]");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        In<float> p(c, params, MLP_PARAMS, mem_kind);
        In<float> x(c, features, count * MLP_IN, mem_kind);
        In<float> y(c, labels, count, mem_kind);
        Out<float> g(c, grad_out, MLP_PARAMS, mem_kind, false);
        Out<float> l(c, loss_out, 1, mem_kind, false);
        mlp_loss_grad(c, p.p, x.p, y.p, nullptr, 0, (int)count, pos_weight, g.p, l.p);
        g.finish();
        l.finish();
        c.sync();
    });
}

pggc_status pggc_mlp_train(pggc_context* ctx, float* params_io, const float* features, const float* labels,
                           int64_t count, int mem_kind, int epochs, int batch, float lr, float pos_weight,
                           uint64_t seed, float* epoch_loss_out) {
    return guarded([&] {
        need(ctx && params_io && features && labels, "NULL argument");
        need(count > 0 && epochs >= 0 && batch > 0 && batch <= (1 << 20), "invalid training sizes");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        Out<float> p(c, params_io, MLP_PARAMS, mem_kind, true);
        In<float> x(c, features, count * MLP_IN, mem_kind);
        In<float> y(c, labels, count, mem_kind);
        std::vector<float> losses;
        mlp_train(c, p.p, x.p, y.p, count, epochs, batch, lr, pos_weight, seed, epoch_loss_out ? &losses : nullptr);
        p.finish();
        c.sync();
        if (epoch_loss_out)
            for (size_t i = 0; i < losses.size(); i++) epoch_loss_out[i] = losses[i];
    });
}

pggc_status pggc_filter_log_start(pggc_context* ctx, int64_t capacity, double sample_rate, uint64_t seed) {
    return guarded([&] {
        need(ctx != nullptr, "NULL argument");
        need(capacity > 0 && sample_rate > 0.0 && sample_rate <= 1.0, "capacity must be > 0, sample_rate in (0, 1]");
        Context& c = *ctx->ctx;
        need(c.filt.mode != 2, "the filter is enabled; disable it before logging");
        filter_free_log(c);
        auto& F = c.filt;
        F.log_x = c.alloc<float>(capacity * MLP_IN);
        F.log_y = c.alloc<float>(capacity);
        F.log_v = c.alloc<i32>(capacity);
        F.log_cnt = c.alloc<unsigned long long>(2);
        PGGC_CUDA(cudaMemsetAsync(F.log_cnt, 0, 2 * sizeof(unsigned long long), c.stream));
        F.log_cap = capacity;
        const double r = sample_rate * 4294967296.0;
        F.log_rate = r >= 4294967295.0 ? 0xFFFFFFFFu : (u32)r;
        F.log_seed = seed;
        F.mode = 1;
        c.sync();
    });
}

pggc_status pggc_filter_log_stop(pggc_context* ctx, float* features_out, float* labels_out, int64_t capacity,
                                 int mem_kind, int64_t* count_out) {
    return guarded([&] {
        need(ctx && count_out, "NULL argument");
        check_mem_kind(mem_kind);
        Context& c = *ctx->ctx;
        auto& F = c.filt;
        need(F.mode == 1 && F.log_cnt, "logging is not active");
        const i64 rows = std::min<i64>((i64)c.read1(F.log_cnt), F.log_cap);
        const i64 k = std::min<i64>(rows, std::max<i64>(capacity, 0));
        auto kind = mem_kind == PGGC_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        if (k > 0 && features_out)
            PGGC_CUDA(cudaMemcpyAsync(features_out, F.log_x, sizeof(float) * k * MLP_IN, kind, c.stream));
        if (k > 0 && labels_out) PGGC_CUDA(cudaMemcpyAsync(labels_out, F.log_y, sizeof(float) * k, kind, c.stream));
        c.sync();
        *count_out = rows;
        filter_free_log(c);
        F.mode = 0;
        c.sync();
    });
}

pggc_status pggc_filter_enable(pggc_context* ctx, const float* params, float threshold_logit) {
    return guarded([&] {
        need(ctx != nullptr, "NULL argument");
        Context& c = *ctx->ctx;
        auto& F = c.filt;
        need(F.mode != 1, "logging is active; stop it before enabling the filter");
        if (!params) {
            F.mode = 0;
            return;
        }
        if (!F.params) F.params = c.alloc<float>(MLP_PARAMS);
        if (!F.net) F.net = c.alloc<MlpDev>(1);
        if (!F.stats) {
            F.stats = c.alloc<unsigned long long>(2);
            PGGC_CUDA(cudaMemsetAsync(F.stats, 0, 2 * sizeof(unsigned long long), c.stream));
        }
        PGGC_CUDA(cudaMemcpyAsync(F.params, params, sizeof(float) * MLP_PARAMS, cudaMemcpyHostToDevice, c.stream));
        mlp_pack(c, F.params, F.net);
        F.threshold = threshold_logit;
        F.mode = 2;
        c.sync();
    });
}

pggc_status pggc_filter_log_label(pggc_context* ctx, int label) {
    return guarded([&] {
        need(ctx != nullptr, "NULL argument");
        need(label == 0 || label == 1, "label must be 0 (moved) or 1 (candidate)");
        ctx->ctx->filt.log_label = label;
    });
}

pggc_status pggc_filter_scope(pggc_context* ctx, int max_pass, int min_level) {
    return guarded([&] {
        need(ctx != nullptr, "NULL argument");
        need(min_level >= 0, "min_level must be >= 0");
        ctx->ctx->filt.max_pass = max_pass < 0 ? -1 : max_pass;
        ctx->ctx->filt.min_level = min_level;
    });
}

pggc_status pggc_filter_stats(pggc_context* ctx, int64_t* evaluated, int64_t* skipped, int reset) {
    return guarded([&] {
        need(ctx != nullptr, "NULL argument");
        Context& c = *ctx->ctx;
        auto& F = c.filt;
        unsigned long long h[2] = {0, 0};
        if (F.stats) {
            PGGC_CUDA(cudaMemcpyAsync(h, F.stats, sizeof(h), cudaMemcpyDeviceToHost, c.stream));
            c.sync();
            if (reset) PGGC_CUDA(cudaMemsetAsync(F.stats, 0, sizeof(h), c.stream));
        }
        if (evaluated) *evaluated = (int64_t)h[0];
        if (skipped) *skipped = (int64_t)h[1];
    });
}

}  // extern "C"
