// ordering.cu -- generate_orderings (src/ordering.cpp:131-164).
//
// Two stable degree-bucketed permutations of the vertices:
//   order1: deg < 128 | 128 <= deg < 15000 | deg >= 15000
//   order2: deg <  64 |  64 <= deg < 15000 | deg >= 15000
// Within a bucket vertices keep ascending id order.  One counting pass writes
// per-block bucket counts, one scan turns them into positions, one scatter pass
// ranks vertices inside each block with warp ballots.  HBM traffic: two reads of
// the row offsets and one write of each permutation.
#include <mutex>
#include "kernels.cuh"
#include "pggc.h"

namespace pggc {

constexpr int ORD_THREADS = 1024;

// A negative "degree" (a decreasing row-offset pair, which only an invalid
// CSR has) falls in bucket 0 in both kernels, so the count and scatter passes
// agree and every write stays inside the two permutations.
__device__ __forceinline__ int bucket1(i64 d) { return d < LARGE_CUTOFF ? 0 : (d < MASSIVE_CUTOFF ? 1 : 2); }
__device__ __forceinline__ int bucket2(i64 d) { return d < MID_CUTOFF ? 0 : (d < MASSIVE_CUTOFF ? 1 : 2); }

__global__ void __launch_bounds__(ORD_THREADS) k_order_count(const i64* rowptr, i64 n, i64 nblocks, i64* cnt1,
                                                              i64* cnt2, unsigned long long* maxdeg) {
    __shared__ int c[6];
    if (threadIdx.x < 6) c[threadIdx.x] = 0;
    __syncthreads();
    i64 i = (i64)blockIdx.x * ORD_THREADS + threadIdx.x;
    i64 d = -1;
    if (i < n) d = rowptr[i + 1] - rowptr[i];
    int b1 = i < n ? bucket1(d) : -1, b2 = i < n ? bucket2(d) : -1;
    for (int b = 0; b < 3; b++) {
        unsigned m1 = __ballot_sync(FULL, b1 == b);
        unsigned m2 = __ballot_sync(FULL, b2 == b);
        if (lane_id() == 0) {
            atomicAdd(&c[b], __popc(m1));
            atomicAdd(&c[3 + b], __popc(m2));
        }
    }
    if (maxdeg) {
        i64 dm = d;
        for (int o = 16; o >= 1; o >>= 1) dm = max(dm, __shfl_xor_sync(FULL, dm, o));
        if (lane_id() == 0 && dm > 0) atomicMax(maxdeg, (unsigned long long)dm);
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        cnt1[(i64)threadIdx.x * nblocks + blockIdx.x] = c[threadIdx.x];
        cnt2[(i64)threadIdx.x * nblocks + blockIdx.x] = c[3 + threadIdx.x];
    }
}

__global__ void __launch_bounds__(ORD_THREADS) k_order_scatter(const i64* rowptr, i64 n, i64 nblocks, const i64* off1,
                                                                const i64* off2, i32* order1, i32* order2) {
    __shared__ int wc1[32][3], wc2[32][3];
    i64 i = (i64)blockIdx.x * ORD_THREADS + threadIdx.x;
    int w = threadIdx.x >> 5;
    i64 d = -1;
    if (i < n) d = rowptr[i + 1] - rowptr[i];
    int b1 = i < n ? bucket1(d) : -1, b2 = i < n ? bucket2(d) : -1;
    int r1 = 0, r2 = 0;
    for (int b = 0; b < 3; b++) {
        unsigned m1 = __ballot_sync(FULL, b1 == b);
        unsigned m2 = __ballot_sync(FULL, b2 == b);
        if (b1 == b) r1 = __popc(m1 & lanemask_lt());
        if (b2 == b) r2 = __popc(m2 & lanemask_lt());
        if (lane_id() == 0) {
            wc1[w][b] = __popc(m1);
            wc2[w][b] = __popc(m2);
        }
    }
    __syncthreads();
    if (i < n) {
        int p1 = 0, p2 = 0;
        for (int k = 0; k < w; k++) {
            p1 += wc1[k][b1];
            p2 += wc2[k][b2];
        }
        i64 pos1 = off1[(i64)b1 * nblocks + blockIdx.x] + p1 + r1;
        i64 pos2 = off2[(i64)b2 * nblocks + blockIdx.x] + p2 + r2;
        order1[pos1] = (i32)i;
        order2[pos2] = (i32)i;
    }
}

struct HugeFlag {
    const i64* rowptr;
    __device__ i64 operator()(i64 i) const { return (rowptr[i + 1] - rowptr[i]) > HUGE_DEG ? 1 : 0; }
};
struct HugeEpi {
    i32* out;
    __device__ void operator()(i64 i, i64 excl, i64 v) const {
        if (v) out[excl] = (i32)i;
    }
};

void generate_orderings(Context& ctx, const i64* rowptr, i64 n, Ordering& o) {
    o.n = n;
    o.order1.ensure(ctx, n);
    o.order2.ensure(ctx, n);
    o.huge.ensure(ctx, std::max<i64>(n, 1));
    if (n == 0) {
        o.off_large = o.off_large2 = o.off_mid = o.off_mid2 = o.max_deg = o.n_huge = 0;
        return;
    }
    ProfScope ps(ctx, "orderings");
    i64 nb = ceil_div(n, ORD_THREADS);
    DBuf<i64> cnt1(ctx, 3 * nb), cnt2(ctx, 3 * nb), scal(ctx, 8);
    PGGC_CUDA(cudaMemsetAsync(scal.p, 0, 8 * sizeof(i64), ctx.stream));
    k_order_count<<<(unsigned)nb, ORD_THREADS, 0, ctx.stream>>>(rowptr, n, nb, cnt1.p, cnt2.p,
                                                                (unsigned long long*)(scal.p + 4));
    PGGC_LAUNCH_CHECK();
    scan_apply(ctx, ArrIn{cnt1.p}, ArrOutExcl{cnt1.p}, 3 * nb, nullptr, nullptr);
    scan_apply(ctx, ArrIn{cnt2.p}, ArrOutExcl{cnt2.p}, 3 * nb, nullptr, nullptr);
    k_order_scatter<<<(unsigned)nb, ORD_THREADS, 0, ctx.stream>>>(rowptr, n, nb, cnt1.p, cnt2.p, o.order1.p,
                                                                  o.order2.p);
    PGGC_LAUNCH_CHECK();
    scan_apply(ctx, HugeFlag{rowptr}, HugeEpi{o.huge.p}, n, nullptr, scal.p + 5);
    // bucket starts: order1 bucket 1 / 2 begin at cnt1[nb] / cnt1[2nb]; order2 bucket 1 at cnt2[nb]
    PGGC_CUDA(cudaMemcpyAsync(scal.p + 0, cnt1.p + nb, sizeof(i64), cudaMemcpyDeviceToDevice, ctx.stream));
    PGGC_CUDA(cudaMemcpyAsync(scal.p + 1, cnt1.p + 2 * nb, sizeof(i64), cudaMemcpyDeviceToDevice, ctx.stream));
    PGGC_CUDA(cudaMemcpyAsync(scal.p + 2, cnt2.p + nb, sizeof(i64), cudaMemcpyDeviceToDevice, ctx.stream));
    const i64* h = (const i64*)ctx.readback(scal.p, 8 * sizeof(i64));
    o.off_large = h[0];
    o.off_large2 = h[1];
    o.off_mid = h[2];
    o.off_mid2 = h[1];
    o.max_deg = h[4];
    o.n_huge = h[5];
}

}  // namespace pggc

// ===========================================================================
// Allocation-free variant of generate_orderings.
//
// Some callers cannot allocate device memory at all: a host that hands this
// library a stream inside an allocator-controlled region (a framework that
// owns every byte of device memory through its own pool and budget), or a
// real-time loop that must not touch the driver's allocator.  This entry point serves them: the caller
// passes the inputs and outputs and a stream, and the only scratch (the
// per-block bucket counts) lives in a file-scope __device__ array of fixed
// size.  That array is part of the module image, so
// every GPU that loads the library holds it until process exit.
// ===========================================================================
namespace pggc {

// Up to NOALLOC_MAX_BLOCKS blocks of 1024 vertices: n <= 16,777,216.
constexpr i64 NOALLOC_MAX_BLOCKS = 16384;
constexpr i64 NOALLOC_MAX_N = NOALLOC_MAX_BLOCKS * ORD_THREADS;
// layout (int64 words): [0, 3B) order1 bucket counts, [3B, 6B) order2 bucket
// counts (B = NOALLOC_MAX_BLOCKS).  k_order_count rewrites the first 3 * nb
// words of each half on every call, so nothing needs clearing first.
constexpr i64 NOALLOC_WORDS = 6 * NOALLOC_MAX_BLOCKS;
static __device__ __align__(256) long long g_noalloc_scratch[NOALLOC_WORDS];

// In-place exclusive scan of k int64 values by one 1024-thread block; writes the
// three bucket starts the reference stores in memory_store::ordering.
__global__ void __launch_bounds__(1024) k_noalloc_scan(i64* cnt1, i64* cnt2, i64 nb, i64* offsets_out) {
    __shared__ i64 red[1024 / 32 + 1];
    for (int which = 0; which < 2; which++) {
        i64* a = which == 0 ? cnt1 : cnt2;
        const i64 k = 3 * nb;
        const i64 per = (k + 1023) / 1024;
        const i64 lo = (i64)threadIdx.x * per, hi = min(k, lo + per);
        i64 s = 0;
        for (i64 i = lo; i < hi; i++) s += a[i];
        i64 off = block_excl_scan_i64<1024>(s, red, nullptr);
        for (i64 i = lo; i < hi; i++) {
            i64 v = a[i];
            a[i] = off;
            off += v;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        offsets_out[0] = cnt1[nb];      // offset_large
        offsets_out[1] = cnt1[2 * nb];  // offset_large2
        offsets_out[2] = cnt2[nb];      // offset_mid
        offsets_out[3] = cnt1[2 * nb];  // offset_mid2
    }
}

}  // namespace pggc

namespace {
// device address of g_noalloc_scratch, looked up once per device
std::mutex g_noalloc_mu;
long long* g_noalloc_addr[64] = {nullptr};
}  // namespace

extern "C" pggc_status pggc_generate_orderings_noalloc(const int64_t* rowptr, int64_t n, int32_t* order1,
                                                       int32_t* order2, int64_t* offsets, void* stream) {
    using namespace pggc;
    try {
        if (n < 0 || n > NOALLOC_MAX_N) {
            pggc_set_last_error("n exceeds the allocation-free limit of 16,777,216 vertices");
            return PGGC_ERR_INVALID;
        }
        if (!rowptr || !offsets || (n > 0 && (!order1 || !order2))) {
            pggc_set_last_error("NULL argument");
            return PGGC_ERR_INVALID;
        }
        int dev = 0;
        PGGC_CUDA(cudaGetDevice(&dev));
        if (dev < 0 || dev >= 64) {
            pggc_set_last_error("device index out of range");
            return PGGC_ERR_INVALID;
        }
        long long* scratch = nullptr;
        {
            std::lock_guard<std::mutex> lk(g_noalloc_mu);
            if (!g_noalloc_addr[dev]) {
                void* p = nullptr;
                PGGC_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
                g_noalloc_addr[dev] = (long long*)p;
            }
            scratch = g_noalloc_addr[dev];
        }
        cudaStream_t s = (cudaStream_t)stream;
        i64* cnt1 = (i64*)scratch;
        i64* cnt2 = cnt1 + 3 * NOALLOC_MAX_BLOCKS;
        if (n == 0) {
            PGGC_CUDA(cudaMemsetAsync(offsets, 0, 4 * sizeof(int64_t), s));
            return PGGC_OK;
        }
        const i64 nb = ceil_div(n, ORD_THREADS);
        // the counts are fully rewritten by k_order_count; the layout uses the
        // first 3 * nb words of each half, so the bucket-major strides are nb.
        // No max-degree word: this entry point returns the orderings and the
        // four bucket offsets only.
        k_order_count<<<(unsigned)nb, ORD_THREADS, 0, s>>>(rowptr, n, nb, cnt1, cnt2, nullptr);
        PGGC_LAUNCH_CHECK();
        k_noalloc_scan<<<1, 1024, 0, s>>>(cnt1, cnt2, nb, offsets);
        PGGC_LAUNCH_CHECK();
        k_order_scatter<<<(unsigned)nb, ORD_THREADS, 0, s>>>(rowptr, n, nb, cnt1, cnt2, order1, order2);
        PGGC_LAUNCH_CHECK();
        return PGGC_OK;
    } catch (const std::exception& e) {
        pggc_set_last_error(e.what());
        return PGGC_ERR_CUDA;
    }
}
