// mlp_train.cuh -- host entry points of the learned move filter's network
// (packing, inference from features, loss/gradient, training).
#pragma once
#include <vector>
#include "context.cuh"
#include "mlp.cuh"

namespace pggc {

// FP32 master parameters (MLP_PARAMS) -> BF16 inference copy
void mlp_pack(Context& ctx, const float* params, MlpDev* out);
// logits of X[N][8] on the tensor cores
void mlp_infer(Context& ctx, const MlpDev* m, const float* X, i64 N, float* logits);
// mean positive-weighted BCE and its gradient over rows [off, off + B) of X / y
// (through perm when non-NULL); deterministic
void mlp_loss_grad(Context& ctx, const float* params, const float* X, const float* y, const i32* perm, i64 off, int B,
                   float pos_w, float* grad, float* loss);
// Adam on shuffled mini-batches; epoch_loss (optional) receives each epoch's mean batch loss
void mlp_train(Context& ctx, float* params, const float* X, const float* y, i64 N, int epochs, int batch, float lr,
               float pos_w, u64 seed, std::vector<float>* epoch_loss);

}  // namespace pggc
