// context.cuh -- the device-side counterpart of the reference's memory_store
// (interface/memory_store.hpp:12-91): one CUDA stream, stream-ordered
// allocations from the device memory pool, pinned host scalars for the few
// values the host must read, and a device error flag latched by bounded loops.
#pragma once
#include <chrono>
#include <map>
#include <mutex>
#include <vector>
#include <nvtx3/nvToolsExt.h>
#include "common.cuh"

namespace pggc {

struct MlpDev;

// workspace slots shared across kernel families (local_move uses 0..31)
enum WsSlot : int { WS_CONTRACT_GK = 40, WS_CONTRACT_GV = 41, WS_OWN_CLS = 42, WS_OWN_OFF = 43, WS_OWN_CNT = 44,
                    WS_MLP_SCRATCH = 45 };

// Per-kernel-family timing with CUDA events on the launching stream, plus the
// algorithmic bytes the kernels report (accumulated on the device per warp and
// flushed with one atomic per warp).  Off unless enabled.
struct ProfStat {
    i64 launches = 0;
    double ms = 0.0;
    double bytes = 0.0;
};

// Kernel-selection knobs of the local-move select step.  Results do not
// depend on them (every select kernel aggregates exact sums and applies the
// same argmax order); they only move work between kernels.  Set by
// pggc_tune_set or by the batch autotuner.
struct TuneParams {
    int thread_max_deg = 32;  // 0, 8, 16 or 32: one thread per vertex up to this degree
    int warp_max_deg = 127;   // 32 or 127: one warp per vertex up to this degree, a block above
    float load = 0.5f;        // load-factor bound of the warp / block hash tables: 0.5 or 0.7
    int streams = 4;          // batch width for batch calls that pass streams = 0
};

struct Context {
    int device = 0;
    TuneParams tune;
    cudaStream_t stream = nullptr;
    int* d_err = nullptr;          // DevErr latched by kernels
    void* h_pin = nullptr;         // pinned scratch for scalar readbacks
    size_t h_pin_bytes = 0;
    int num_sms = NUM_SMS;
    size_t max_smem_optin = 0;
    // fault injection: cap on hash-table probes (0 = only the table size bounds them)
    u32 probe_cap = 0;
    // profiling
    bool profiling = false;
    unsigned long long* d_prof = nullptr;  // [64] device byte counters
    std::map<std::string, int> prof_slot;
    std::map<std::string, ProfStat> prof;
    struct ProfPending {
        std::string family, level_key;
        cudaEvent_t a, b;
    };
    std::vector<ProfPending> prof_pending;
    // own-cluster weights of the last local move's best state (graph uid,
    // device array, vertex count); uid 0: none
    unsigned long long pv_uid = 0;
    const void* pv_ptr = nullptr;
    long long pv_n = 0;
    bool prof_by_level = false;  // also record "family@level[@tag]" (multilevel level index)
    const char* prof_tag = nullptr;  // e.g. which sweep of a local move
    std::vector<cudaEvent_t> ev_pool;
    // learned move filter (filter.cuh): mode 0 off, 1 log (features, label)
    // samples from plain sweeps, 2 skip the vertices the network rejects
    struct Filter {
        int mode = 0;
        MlpDev* net = nullptr;                  // BF16 inference copy (device)
        float* params = nullptr;                // FP32 master copy (device)
        float threshold = 0.f;                  // logit below which a vertex is skipped
        bool suspended = false;                 // set by the driver around exact sweeps
        // scope: the filter gates sweeps of passes below max_pass (< 0: every
        // pass) at levels at or above min_level; `pass` is set by the driver
        int max_pass = -1;
        int min_level = 0;
        int pass = 0;
        float* log_x = nullptr;                 // [log_cap][8]
        float* log_y = nullptr;                 // [log_cap]
        i32* log_v = nullptr;                   // [log_cap]
        unsigned long long* log_cnt = nullptr;  // [0] rows written, [1] first row of the current sweep
        i64 log_cap = 0;
        u32 log_rate = 0;                       // a row is sampled when its hash is below this
        int log_label = 0;                      // 0: moved, 1: candidate (select proposed a move)
        u64 log_seed = 0;
        unsigned long long* stats = nullptr;    // [0] vertices evaluated, [1] skipped
        int level = 0;                          // current level, set by the multilevel driver
        i32 stamp = 0;                          // sweep counter (moved-last-sweep feature)
    } filt;

    // The context's own stream-ordered memory pool.  One pool per context (not
    // the device's default pool) keeps contexts that run concurrently -- the
    // workers of a batch -- independent: memory freed on one stream is never
    // handed to another stream with a dependency on the first one's work.
    cudaMemPool_t pool = nullptr;

    explicit Context(int dev) : device(dev) {
        PGGC_CUDA(cudaSetDevice(dev));
        PGGC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.handleTypes = cudaMemHandleTypeNone;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        PGGC_CUDA(cudaMemPoolCreate(&pool, &props));
        u64 thr = ~0ull;
        PGGC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        PGGC_CUDA(dev_malloc((void**)&d_err, sizeof(int) * 8));
        PGGC_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int) * 8, stream));
        PGGC_CUDA(dev_malloc((void**)&d_prof, sizeof(unsigned long long) * 64));
        PGGC_CUDA(cudaMemsetAsync(d_prof, 0, sizeof(unsigned long long) * 64, stream));
        h_pin_bytes = 4096;
        PGGC_CUDA(cudaMallocHost(&h_pin, h_pin_bytes));
        cudaDeviceProp prop;
        PGGC_CUDA(cudaGetDeviceProperties(&prop, dev));
        num_sms = prop.multiProcessorCount;
        max_smem_optin = prop.sharedMemPerBlockOptin;
        PGGC_CUDA(cudaStreamSynchronize(stream));
    }
    // stream-ordered allocation from the context's pool
    cudaError_t dev_malloc(void** p, size_t bytes) { return cudaMallocFromPoolAsync(p, bytes, pool, stream); }
    // Stack arena for short-lived temporaries (scan tile sums, reduction
    // partials, sort histograms): LIFO reuse of one device buffer.  Work on the
    // context is ordered on one stream, so a region may be handed out again
    // as soon as the host has queued the kernels of its previous owner.
    unsigned char* arena = nullptr;
    size_t arena_cap = 0, arena_top = 0;
    // grow-only scratch slots reused across calls (one user at a time per slot)
    std::vector<std::pair<void*, size_t>> ws;
    template <class T>
    T* ws_get(int slot, i64 count) {
        size_t bytes = sizeof(T) * (size_t)(count > 0 ? count : 1);
        if (slot >= (int)ws.size()) ws.resize(slot + 1, {nullptr, 0});
        auto& e = ws[slot];
        if (e.second < bytes) {
            if (e.first) PGGC_CUDA(cudaFreeAsync(e.first, stream));
            size_t nb = bytes + bytes / 4;
            PGGC_CUDA(dev_malloc(&e.first, nb));
            e.second = nb;
        }
        return (T*)e.first;
    }

    ~Context() {
        if (stream) cudaStreamSynchronize(stream);
        for (auto& e : ws)
            if (e.first) cudaFreeAsync(e.first, stream);
        if (arena) cudaFreeAsync(arena, stream);
        for (auto& pe : prof_pending) {
            cudaEventDestroy(pe.a);
            cudaEventDestroy(pe.b);
        }
        for (auto e : ev_pool) cudaEventDestroy(e);
        for (void* q : {(void*)filt.net, (void*)filt.params, (void*)filt.log_x, (void*)filt.log_y, (void*)filt.log_v,
                        (void*)filt.log_cnt, (void*)filt.stats})
            if (q) cudaFreeAsync(q, stream);
        if (d_prof) cudaFreeAsync(d_prof, stream);
        if (d_err) cudaFreeAsync(d_err, stream);
        if (stream) cudaStreamSynchronize(stream);
        if (h_pin) cudaFreeHost(h_pin);
        if (stream) cudaStreamDestroy(stream);
        // blocks still held by other objects are released when they are freed
        if (pool) cudaMemPoolDestroy(pool);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;

    template <class T>
    T* alloc(i64 count) {
        if (count <= 0) count = 1;
        T* p = nullptr;
        if (profiling) {
            // host time spent in the stream-ordered allocator (pool growth shows here)
            auto t0 = std::chrono::steady_clock::now();
            PGGC_CUDA(dev_malloc((void**)&p, sizeof(T) * (size_t)count));
            auto& st = prof["host_alloc"];
            st.launches++;
            st.bytes += (double)(sizeof(T) * (size_t)count);
            st.ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        } else {
            PGGC_CUDA(dev_malloc((void**)&p, sizeof(T) * (size_t)count));
        }
        return p;
    }
    void release(void* p) {
        if (p) PGGC_CUDA(cudaFreeAsync(p, stream));
    }
    void sync() { PGGC_CUDA(cudaStreamSynchronize(stream)); }

    // Copy `bytes` from device to the pinned scratch and wait.
    void* readback(const void* d, size_t bytes) {
        if (bytes > h_pin_bytes) throw InvalidArg("readback larger than pinned scratch");
        PGGC_CUDA(cudaMemcpyAsync(h_pin, d, bytes, cudaMemcpyDeviceToHost, stream));
        sync();
        return h_pin;
    }
    template <class T>
    T read1(const T* d) {
        return *(T*)readback(d, sizeof(T));
    }
    // ---- profiling -----------------------------------------------------
    // device counter slot for a family (nullptr when profiling is off)
    unsigned long long* prof_counter(const char* family) {
        if (!profiling) return nullptr;
        auto it = prof_slot.find(family);
        int slot;
        if (it == prof_slot.end()) {
            slot = (int)prof_slot.size();
            if (slot >= 64) return nullptr;
            prof_slot[family] = slot;
        } else {
            slot = it->second;
        }
        return d_prof + slot;
    }
    cudaEvent_t take_event() {
        if (!ev_pool.empty()) {
            cudaEvent_t e = ev_pool.back();
            ev_pool.pop_back();
            return e;
        }
        cudaEvent_t e;
        PGGC_CUDA(cudaEventCreate(&e));
        return e;
    }
    // algorithmic bytes known on the host (sizes of the arrays a family streams)
    void prof_add_bytes(const std::string& family, double bytes) {
        if (profiling) prof[family].bytes += bytes;
    }
    void prof_record(const std::string& family, cudaEvent_t a, cudaEvent_t b) {
        std::string lk;
        if (prof_by_level) {
            lk = family + "@" + std::to_string(filt.level);
            if (prof_tag) lk += std::string("@") + prof_tag;
        }
        prof_pending.push_back({family, std::move(lk), a, b});
        if (prof_pending.size() >= 8192) prof_flush();
    }
    void prof_flush() {
        if (prof_pending.empty() && prof_slot.empty()) return;
        sync();
        for (auto& pe : prof_pending) {
            float ms = 0.f;
            PGGC_CUDA(cudaEventElapsedTime(&ms, pe.a, pe.b));
            auto& st = prof[pe.family];
            st.launches += 1;
            st.ms += ms;
            if (!pe.level_key.empty()) {
                auto& sl = prof[pe.level_key];
                sl.launches += 1;
                sl.ms += ms;
            }
            ev_pool.push_back(pe.a);
            ev_pool.push_back(pe.b);
        }
        prof_pending.clear();
        if (!prof_slot.empty()) {
            unsigned long long h[64];
            PGGC_CUDA(cudaMemcpy(h, d_prof, sizeof(h), cudaMemcpyDeviceToHost));
            for (auto& kv : prof_slot) prof[kv.first].bytes += (double)h[kv.second];
            PGGC_CUDA(cudaMemsetAsync(d_prof, 0, sizeof(h), stream));
            sync();
        }
    }
    void prof_reset() {
        prof_flush();
        prof.clear();
    }

    void check_device_error() { raise_device_error(read1(d_err)); }
    // for a caller that read the error word together with other results
    void raise_device_error(int e) {
        if (e != DEV_OK) {
            PGGC_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
            sync();
            throw DeviceFault("device-side bounded loop gave up (code " + std::to_string(e) + ")");
        }
    }
};

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) once per (kernel, device).
template <class K>
inline void set_dynamic_smem_once(K kernel, int bytes, int device) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    std::lock_guard<std::mutex> lk(mu);
    auto key = std::make_pair((const void*)kernel, device);
    auto it = done.find(key);
    if (it != done.end() && it->second >= bytes) return;
    PGGC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    done[key] = bytes;
}

// Brackets the launches of one kernel family with CUDA events when profiling,
// and always with an NVTX push/pop range of the family's name (free unless a
// tool such as ncu --nvtx is attached; lets a capture select one family).
struct ProfScope {
    Context& ctx;
    const char* family;
    cudaEvent_t a = nullptr, b = nullptr;
    ProfScope(Context& c, const char* f) : ctx(c), family(f) {
        nvtxRangePushA(f);
        if (ctx.profiling) {
            a = ctx.take_event();
            PGGC_CUDA(cudaEventRecord(a, ctx.stream));
        }
    }
    ~ProfScope() {
        if (a) {
            b = ctx.take_event();
            if (cudaEventRecord(b, ctx.stream) == cudaSuccess) ctx.prof_record(family, a, b);
        }
        nvtxRangePop();
    }
};

// A temporary of `count` T from the context's arena (released in LIFO order
// when this object goes out of scope), or from the stream-ordered pool when
// the arena has no room.  The arena is (re)sized to 64 MiB or the request,
// whichever is larger, when it is empty.
template <class T>
struct Tmp {
    Context& ctx;
    T* p = nullptr;
    size_t mark = 0;
    bool pooled = false;
    Tmp(Context& c, i64 count) : ctx(c) {
        const size_t bytes = ((sizeof(T) * (size_t)(count > 0 ? count : 1)) + 255) & ~(size_t)255;
        if (ctx.arena_top == 0 && ctx.arena_cap < bytes) {
            if (ctx.arena) PGGC_CUDA(cudaFreeAsync(ctx.arena, ctx.stream));
            ctx.arena_cap = std::max<size_t>(bytes, (size_t)64 << 20);
            PGGC_CUDA(ctx.dev_malloc((void**)&ctx.arena, ctx.arena_cap));
        }
        if (ctx.arena_top + bytes <= ctx.arena_cap) {
            mark = ctx.arena_top;
            p = (T*)(ctx.arena + ctx.arena_top);
            ctx.arena_top += bytes;
        } else {
            pooled = true;
            p = ctx.alloc<T>(count);
        }
    }
    ~Tmp() {
        if (pooled) cudaFreeAsync(p, ctx.stream);
        else ctx.arena_top = mark;
    }
    Tmp(const Tmp&) = delete;
    Tmp& operator=(const Tmp&) = delete;
};

// RAII device buffer allocated on the context stream.
template <class T>
struct DBuf {
    Context* ctx = nullptr;
    T* p = nullptr;
    i64 n = 0;
    DBuf() = default;
    DBuf(Context& c, i64 count) : ctx(&c), p(c.alloc<T>(count)), n(count) {}
    DBuf(DBuf&& o) noexcept : ctx(o.ctx), p(o.p), n(o.n) {
        o.p = nullptr;
        o.n = 0;
    }
    DBuf& operator=(DBuf&& o) noexcept {
        if (this != &o) {
            reset();
            ctx = o.ctx;
            p = o.p;
            n = o.n;
            o.p = nullptr;
            o.n = 0;
        }
        return *this;
    }
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    ~DBuf() { reset(); }
    void reset() {
        if (p && ctx) cudaFreeAsync(p, ctx->stream);
        p = nullptr;
        n = 0;
    }
    void ensure(Context& c, i64 count) {
        if (p && n >= count) return;
        reset();
        ctx = &c;
        p = c.alloc<T>(count);
        n = count;
    }
    T* get() const { return p; }
};

}  // namespace pggc
