// context.cuh -- the device-side counterpart of the reference's memory_store
// (interface/memory_store.hpp:12-91): one CUDA stream, stream-ordered
// allocations from the device memory pool, pinned host scalars for the few
// values the host must read, and a device error flag latched by bounded loops.
#pragma once
#include "common.cuh"

namespace pggc {

struct Context {
    int device = 0;
    cudaStream_t stream = nullptr;
    int* d_err = nullptr;          // DevErr latched by kernels
    void* h_pin = nullptr;         // pinned scratch for scalar readbacks
    size_t h_pin_bytes = 0;
    int num_sms = NUM_SMS;
    size_t max_smem_optin = 0;

    explicit Context(int dev) : device(dev) {
        PGGC_CUDA(cudaSetDevice(dev));
        PGGC_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        cudaMemPool_t pool;
        PGGC_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        u64 thr = ~0ull;
        PGGC_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        PGGC_CUDA(cudaMallocAsync((void**)&d_err, sizeof(int) * 8, stream));
        PGGC_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int) * 8, stream));
        h_pin_bytes = 4096;
        PGGC_CUDA(cudaMallocHost(&h_pin, h_pin_bytes));
        cudaDeviceProp prop;
        PGGC_CUDA(cudaGetDeviceProperties(&prop, dev));
        num_sms = prop.multiProcessorCount;
        max_smem_optin = prop.sharedMemPerBlockOptin;
        PGGC_CUDA(cudaStreamSynchronize(stream));
    }
    ~Context() {
        if (d_err) cudaFreeAsync(d_err, stream);
        if (stream) cudaStreamSynchronize(stream);
        if (h_pin) cudaFreeHost(h_pin);
        if (stream) cudaStreamDestroy(stream);
    }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;

    template <class T>
    T* alloc(i64 count) {
        if (count <= 0) count = 1;
        T* p = nullptr;
        PGGC_CUDA(cudaMallocAsync((void**)&p, sizeof(T) * (size_t)count, stream));
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
    void check_device_error() {
        int e = read1(d_err);
        if (e != DEV_OK) {
            PGGC_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), stream));
            sync();
            throw DeviceFault("device-side bounded loop gave up (code " + std::to_string(e) + ")");
        }
    }
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
