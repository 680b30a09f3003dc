// mlp_train.cu -- the learned move filter's network: packing, batched
// inference from a feature matrix, and training (forward + backward + Adam) on
// the GPU with the project's own kernels.
//
// Training is deterministic: one thread per sample computes the forward pass
// and the per-sample deltas into a structure-of-arrays scratch, then one
// thread per parameter sums its gradient over the batch in sample order (no
// atomics), and Adam updates the FP32 master weights.  Gradients flow straight
// through the BF16 roundings of the forward pass.
#include "kernels.cuh"
#include "mlp.cuh"
#include "mlp_train.cuh"

namespace pggc {

// ---------------------------------------------------------------------------
// packing: FP32 master -> MlpDev (BF16 W1/W2, BF16-rounded W3, FP32 biases)
// ---------------------------------------------------------------------------
__global__ void k_mlp_pack(const float* p, MlpDev* m) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < MLP_PARAMS; i += gridDim.x * blockDim.x) {
        const float v = p[i];
        if (i < MLP_O_B1) m->w1[i - MLP_O_W1] = __float2bfloat16_rn(v);
        else if (i < MLP_O_W2) m->b1[i - MLP_O_B1] = v;
        else if (i < MLP_O_B2) m->w2[i - MLP_O_W2] = __float2bfloat16_rn(v);
        else if (i < MLP_O_W3) m->b2[i - MLP_O_B2] = v;
        else if (i < MLP_O_B3) m->w3[i - MLP_O_W3] = bf16_round(v);
        else m->b3 = v;
    }
}

void mlp_pack(Context& ctx, const float* params, MlpDev* out) {
    k_mlp_pack<<<ceil_div(MLP_PARAMS, 256), 256, 0, ctx.stream>>>(params, out);
    PGGC_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// inference over a feature matrix X[N][8] (tensor cores)
// ---------------------------------------------------------------------------
constexpr int MI_WARPS = 8;
constexpr int XS = MLP_IN + 1;  // padded row stride of the shared feature tile

__global__ void __launch_bounds__(MI_WARPS * 32) k_mlp_infer(const MlpDev* m, const float* X, i64 N, float* logits) {
    __shared__ float xs[MI_WARPS][32 * XS];
    __shared__ float sc[MI_WARPS][32];
    const int l = lane_id(), w = threadIdx.x >> 5;
    MlpRegs r;
    mlp_load(m, r);
    const i64 gw = (blockIdx.x * (i64)blockDim.x + threadIdx.x) >> 5;
    const i64 nw = ((i64)gridDim.x * blockDim.x) >> 5;
    for (i64 base = gw * 32; base < N; base += nw * 32) {
        const i64 x = base + l;
#pragma unroll
        for (int f = 0; f < MLP_IN; f++) xs[w][l * XS + f] = x < N ? X[x * MLP_IN + f] : 0.f;
        __syncwarp();
        float lg = mlp_warp32(r, xs[w], XS, sc[w]);
        if (x < N) logits[x] = lg;
        __syncwarp();
    }
}

void mlp_infer(Context& ctx, const MlpDev* m, const float* X, i64 N, float* logits) {
    if (N <= 0) return;
    int grid = (int)std::min<i64>(ceil_div(ceil_div(N, 32), MI_WARPS), (i64)ctx.num_sms * 8);
    k_mlp_infer<<<grid, MI_WARPS * 32, 0, ctx.stream>>>(m, X, N, logits);
    PGGC_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// training
// ---------------------------------------------------------------------------
// scratch rows (structure of arrays, B samples each)
constexpr int TS_XB = 0;                         // 8 rows
constexpr int TS_H1 = TS_XB + MLP_IN;            // 32 rows: BF16-rounded layer-1 activations
constexpr int TS_H2 = TS_H1 + MLP_H;             // 32 rows: layer-2 activations (FP32)
constexpr int TS_D2 = TS_H2 + MLP_H;             // 32 rows: dL/dz2
constexpr int TS_D1 = TS_D2 + MLP_H;             // 32 rows: dL/dz1
constexpr int TS_DL = TS_D1 + MLP_H;             // 1 row:  dL/dlogit
constexpr int TS_LOSS = TS_DL + 1;               // 1 row:  per-sample loss
constexpr int TS_ROWS = TS_LOSS + 1;

__device__ __forceinline__ float softplus(float x) { return fmaxf(x, 0.f) + log1pf(expf(-fabsf(x))); }

// One thread per sample of the batch (rows perm[off .. off + B) of X / y, or
// off .. off + B when perm is NULL).
__global__ void __launch_bounds__(128) k_mlp_sample(const float* p, const float* X, const float* y, const i32* perm,
                                                    i64 off, int B, float pos_w, float inv_b, float* S) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B) return;
    const i64 row = perm ? (i64)perm[off + s] : off + s;
    float xb[MLP_IN];
#pragma unroll
    for (int f = 0; f < MLP_IN; f++) {
        xb[f] = bf16_round(X[row * MLP_IN + f]);
        S[(i64)(TS_XB + f) * B + s] = xb[f];
    }
    float z1[MLP_H], h1[MLP_H];
#pragma unroll 4
    for (int k = 0; k < MLP_H; k++) {
        float acc = 0.f;
#pragma unroll
        for (int f = 0; f < MLP_IN; f++) acc = acc + bf16_round(p[MLP_O_W1 + k * MLP_IN + f]) * xb[f];
        z1[k] = acc + p[MLP_O_B1 + k];
        h1[k] = bf16_round(fmaxf(z1[k], 0.f));
        S[(i64)(TS_H1 + k) * B + s] = h1[k];
    }
    float z2[MLP_H];
    float logit = 0.f;
    for (int j = 0; j < MLP_H; j++) {
        float acc = 0.f;
#pragma unroll 8
        for (int k = 0; k < MLP_H; k++) acc = acc + bf16_round(p[MLP_O_W2 + j * MLP_H + k]) * h1[k];
        z2[j] = acc + p[MLP_O_B2 + j];
        const float h2 = fmaxf(z2[j], 0.f);
        S[(i64)(TS_H2 + j) * B + s] = h2;
        logit = logit + h2 * bf16_round(p[MLP_O_W3 + j]);
    }
    logit = logit + p[MLP_O_B3];
    const float yy = y[row];
    const float sg = 1.f / (1.f + expf(-logit));
    S[(i64)TS_LOSS * B + s] = pos_w * yy * softplus(-logit) + (1.f - yy) * softplus(logit);
    const float dl = (pos_w * yy * (sg - 1.f) + (1.f - yy) * sg) * inv_b;
    S[(i64)TS_DL * B + s] = dl;
    float d2[MLP_H];
    for (int j = 0; j < MLP_H; j++) {
        d2[j] = z2[j] > 0.f ? dl * bf16_round(p[MLP_O_W3 + j]) : 0.f;
        S[(i64)(TS_D2 + j) * B + s] = d2[j];
    }
    for (int k = 0; k < MLP_H; k++) {
        float acc = 0.f;
#pragma unroll 8
        for (int j = 0; j < MLP_H; j++) acc = acc + bf16_round(p[MLP_O_W2 + j * MLP_H + k]) * d2[j];
        S[(i64)(TS_D1 + k) * B + s] = z1[k] > 0.f ? acc : 0.f;
    }
}

// One thread per parameter (plus one for the loss): the batch sum in sample order.
__global__ void k_mlp_grad_reduce(const float* S, int B, float inv_b, float* grad, float* loss) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q > MLP_PARAMS) return;
    const float *u = nullptr, *v = nullptr;
    if (q == MLP_PARAMS) {
        u = S + (i64)TS_LOSS * B;
    } else if (q < MLP_O_B1) {
        u = S + (i64)(TS_D1 + q / MLP_IN) * B;
        v = S + (i64)(TS_XB + q % MLP_IN) * B;
    } else if (q < MLP_O_W2) {
        u = S + (i64)(TS_D1 + (q - MLP_O_B1)) * B;
    } else if (q < MLP_O_B2) {
        const int e = q - MLP_O_W2;
        u = S + (i64)(TS_D2 + e / MLP_H) * B;
        v = S + (i64)(TS_H1 + e % MLP_H) * B;
    } else if (q < MLP_O_W3) {
        u = S + (i64)(TS_D2 + (q - MLP_O_B2)) * B;
    } else if (q < MLP_O_B3) {
        u = S + (i64)TS_DL * B;
        v = S + (i64)(TS_H2 + (q - MLP_O_W3)) * B;
    } else {
        u = S + (i64)TS_DL * B;
    }
    float acc = 0.f;
    if (v) {
        for (int s = 0; s < B; s++) acc = acc + u[s] * v[s];
    } else {
        for (int s = 0; s < B; s++) acc = acc + u[s];
    }
    if (q == MLP_PARAMS) *loss = acc * inv_b;
    else grad[q] = acc;
}

__global__ void k_mlp_adam(float* p, float* m, float* v, const float* g, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= MLP_PARAMS) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    const float mh = mq / c1, vh = vq / c2;
    p[q] = p[q] - lr * mh / (sqrtf(vh) + eps);
}

__global__ void k_shuffle_keys(u64* keys, i32* vals, i64 N, u32 salt) {
    for (i64 i = blockIdx.x * (i64)blockDim.x + threadIdx.x; i < N; i += (i64)gridDim.x * blockDim.x) {
        keys[i] = ((u64)murmur3_32((u32)i ^ salt) << 32) | (u64)i;
        vals[i] = (i32)i;
    }
}

void mlp_loss_grad(Context& ctx, const float* params, const float* X, const float* y, const i32* perm, i64 off, int B,
                   float pos_w, float* grad, float* loss) {
    if (B <= 0) throw InvalidArg("empty batch");
    float* S = ctx.ws_get<float>(WS_MLP_SCRATCH, (i64)TS_ROWS * B);
    const float inv_b = 1.0f / (float)B;
    k_mlp_sample<<<ceil_div(B, 128), 128, 0, ctx.stream>>>(params, X, y, perm, off, B, pos_w, inv_b, S);
    PGGC_LAUNCH_CHECK();
    k_mlp_grad_reduce<<<ceil_div(MLP_PARAMS + 1, 128), 128, 0, ctx.stream>>>(S, B, inv_b, grad, loss);
    PGGC_LAUNCH_CHECK();
}

void mlp_train(Context& ctx, float* params, const float* X, const float* y, i64 N, int epochs, int batch, float lr,
               float pos_w, u64 seed, std::vector<float>* epoch_loss) {
    if (N <= 0 || batch <= 0 || epochs < 0) throw InvalidArg("training needs samples, a batch size and epochs");
    DBuf<float> m(ctx, MLP_PARAMS), v(ctx, MLP_PARAMS), g(ctx, MLP_PARAMS), lossv(ctx, 1);
    DBuf<float> losses(ctx, std::max<i64>(1, ceil_div(N, batch)));
    PGGC_CUDA(cudaMemsetAsync(m.p, 0, sizeof(float) * MLP_PARAMS, ctx.stream));
    PGGC_CUDA(cudaMemsetAsync(v.p, 0, sizeof(float) * MLP_PARAMS, ctx.stream));
    DBuf<u64> keys(ctx, N), keys2(ctx, N);
    DBuf<i32> perm(ctx, N), perm2(ctx, N);
    SplitMix64 sm(seed);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    i64 step = 0;
    for (int ep = 0; ep < epochs; ep++) {
        int grid = (int)std::min<i64>(ceil_div(N, 256), (i64)ctx.num_sms * 8);
        k_shuffle_keys<<<grid, 256, 0, ctx.stream>>>(keys.p, perm.p, N, (u32)sm.next());
        PGGC_LAUNCH_CHECK();
        radix_sort_pairs<i32>(ctx, keys.p, perm.p, N, 32, 64, keys2.p, perm2.p);
        // full batches only (one short batch when N < batch)
        const i64 nb = N >= batch ? N / batch : 1;
        for (i64 bi = 0; bi < nb; bi++) {
            const i64 off = bi * batch;
            const int B = (int)std::min<i64>(batch, N - off);
            step++;
            mlp_loss_grad(ctx, params, X, y, perm.p, off, B, pos_w, g.p, losses.p + bi);
            const float c1 = 1.f - (float)std::pow((double)b1, (double)step);
            const float c2 = 1.f - (float)std::pow((double)b2, (double)step);
            k_mlp_adam<<<ceil_div(MLP_PARAMS, 256), 256, 0, ctx.stream>>>(params, m.p, v.p, g.p, lr, b1, b2, eps, c1,
                                                                         c2);
            PGGC_LAUNCH_CHECK();
        }
        if (epoch_loss && nb > 0) {
            std::vector<float> h(nb);
            PGGC_CUDA(cudaMemcpyAsync(h.data(), losses.p, sizeof(float) * nb, cudaMemcpyDeviceToHost, ctx.stream));
            ctx.sync();
            double s = 0;
            for (float x : h) s += x;
            epoch_loss->push_back((float)(s / nb));
        }
    }
}

}  // namespace pggc
