// filter.cuh -- the learned move filter inside a local-move sweep.
//
// Before a sweep's select pass, one kernel visits the vertices the sweep would
// evaluate (dest == NULL_PART) and computes 8 features per vertex:
//   f0 log2(1 + degree) / 16
//   f1 own-cluster weight / vertex weight (clamped to [0, 1])
//   f2 best gain of the vertex's previous evaluation / vertex weight ([-4, 4])
//   f3 1 if the vertex moved in the previous sweep
//   f4 log2(1 + own-cluster size) / log2(2 + n)
//   f5 own-cluster volume / total volume
//   f6 level index / 16
//   f7 sweep index / 8
// In logging mode a hashed sample of those rows is appended to a log, and the
// rows are labelled after the afterburner (1 = the vertex moves in this
// sweep, or with the candidate label 1 = the select step proposed a move).  In filtering mode the network (mlp.cuh) scores all 32 vertices of a
// warp on the tensor cores and the vertices whose logit is below the threshold
// are not evaluated: their dest becomes NO_MOVE (as if evaluated without a
// move), so they return to the sweep when a neighbour moves.  Gains of the
// vertices that are evaluated stay exact.
#pragma once
#include "kernels.cuh"
#include "mlp.cuh"

namespace pggc {

template <class W>
struct FiltArgs {
    using V = typename Traits<W>::V;
    DGraph<W> g;
    const i32* part;
    const V* pvals;
    float* gain;
    const i32* moved_at;
    const i32* csize;
    const V* td;
    i32* dest;
    float inv_vol, inv_log_n, level_f, sweep_f;
    i32 prev_stamp;
    int mode;  // 1 log, 2 filter
    const MlpDev* net;
    float threshold;
    float* log_x;
    i32* log_v;
    float* log_y;
    unsigned long long* log_cnt;
    i64 log_cap;
    u32 rate, salt;
    unsigned long long* stats;  // [0] evaluated, [1] skipped
};

constexpr int FW_WARPS = 8;
constexpr int FW_XS = MLP_IN + 1;

template <class W>
__device__ __forceinline__ void filter_features(const FiltArgs<W>& a, i32 i, float (&f)[MLP_IN]) {
    const i64 deg = a.g.rowptr[i + 1] - a.g.rowptr[i];
    const float vw = (float)a.g.vtx_w[i];
    const i32 p = a.part[i];
    f[0] = log2f(1.f + (float)deg) * (1.f / 16.f);
    f[1] = vw > 0.f ? fminf(fmaxf((float)a.pvals[i] / vw, 0.f), 1.f) : 0.f;
    f[2] = vw > 0.f ? fminf(fmaxf(a.gain[i] / vw, -4.f), 4.f) : 0.f;
    f[3] = a.moved_at[i] == a.prev_stamp ? 1.f : 0.f;
    f[4] = log2f(1.f + (float)max(a.csize[p], 0)) * a.inv_log_n;
    f[5] = (float)a.td[p] * a.inv_vol;
    f[6] = a.level_f;
    f[7] = a.sweep_f;
}

template <class W>
__global__ void __launch_bounds__(FW_WARPS * 32) k_filter_sweep(FiltArgs<W> a) {
    __shared__ float xs[FW_WARPS][32 * FW_XS];
    __shared__ float sc[FW_WARPS][32];
    const int l = lane_id(), w = threadIdx.x >> 5;
    MlpRegs r;
    if (a.mode == 2) mlp_load(a.net, r);
    const i64 n = a.g.n;
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    unsigned long long n_eval = 0, n_skip = 0;
    for (i64 base = gw * 32; base < n; base += nw * 32) {
        const i64 x = base + l;
        const bool act = x < n && a.dest[x] == NULL_PART;
        const unsigned am = __ballot_sync(FULL, act);
        if (!am) continue;
        float f[MLP_IN];
#pragma unroll
        for (int k = 0; k < MLP_IN; k++) f[k] = 0.f;
        if (act) filter_features(a, (i32)x, f);
        if (a.mode == 1) {
            const bool smp = act && murmur3_32((u32)x ^ a.salt) < a.rate;
            const unsigned sm = __ballot_sync(FULL, smp);
            if (sm) {
                unsigned long long b0 = 0;
                if (l == 0) b0 = atomicAdd(&a.log_cnt[0], (unsigned long long)__popc(sm));
                b0 = __shfl_sync(FULL, b0, 0);
                const unsigned long long idx = b0 + __popc(sm & lanemask_lt());
                if (smp && idx < (unsigned long long)a.log_cap) {
#pragma unroll
                    for (int k = 0; k < MLP_IN; k++) a.log_x[idx * MLP_IN + k] = f[k];
                    a.log_v[idx] = (i32)x;
                    a.log_y[idx] = -1.f;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < MLP_IN; k++) xs[w][l * FW_XS + k] = f[k];
            __syncwarp();
            const float lg = mlp_warp32(r, xs[w], FW_XS, sc[w]);
            const bool skip = act && lg < a.threshold;
            if (skip) {
                a.dest[x] = NO_MOVE;
                a.gain[x] = OBJ_MIN;
            }
            const unsigned skm = __ballot_sync(FULL, skip);
            n_skip += __popc(skm);
            n_eval += __popc(am & ~skm);
        }
    }
    if (a.mode == 2 && l == 0 && a.stats) {
        if (n_eval) atomicAdd(&a.stats[0], n_eval);
        if (n_skip) atomicAdd(&a.stats[1], n_skip);
    }
}

// labels of this sweep's samples [log_cnt[1], log_cnt[0]): mode 0, 1 if the
// vertex was a candidate the afterburner kept (it moves); mode 1, 1 if the
// select step proposed a move for it (it is a candidate)
__global__ void k_filter_label(const i32* log_v, float* log_y, const unsigned long long* log_cnt, i64 log_cap,
                               const i32* dest, const unsigned char* keep, int mode) {
    const unsigned long long lo = log_cnt[1];
    unsigned long long hi = log_cnt[0];
    if (hi > (unsigned long long)log_cap) hi = (unsigned long long)log_cap;
    for (unsigned long long r = lo + blockIdx.x * (u64)blockDim.x + threadIdx.x; r < hi;
         r += (u64)gridDim.x * blockDim.x) {
        const i32 v = log_v[r];
        log_y[r] = (dest[v] != NO_MOVE && (mode == 1 || keep[v])) ? 1.f : 0.f;
    }
}

__global__ void k_cluster_sizes(const i32* part, i64 n, i32* csize) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < n; i += (i64)gridDim.x * blockDim.x)
        atomicAdd(&csize[part[i]], 1);
}

}  // namespace pggc
