// The learned initialiser's MLP (d -> 512 -> 512 -> dim), trained and applied on the GPU.
#pragma once
#include "engine.cuh"

namespace pacmap {
// Parameters in the flat host layout [W1 (512 x d), b1 (512), W2 (512 x 512), b2 (512), W3 (dim x 512), b3 (dim)].
uint64_t mlp_param_count(uint64_t d, uint64_t dim);
void mlp_init_params(uint64_t d, uint64_t dim, uint64_t seed, float* flat);
// out (n x dim, device) = MLP(x) for device x (n x d).
void mlp_apply_device(Ctx& c, const float* params, uint64_t d, uint64_t dim, const float* d_x, uint64_t n, float* d_out);
// One forward/backward of the mean-squared error on a batch of B rows (device x, t): flat gradients, loss.
void mlp_grad_device(Ctx& c, const float* params, uint64_t d, uint64_t dim, const float* d_x, const float* d_t,
                     uint64_t B, float* grads_flat, float* loss);
// AdamW training on (x, t) rows (device), params updated in place (host flat layout).
void mlp_train_device(Ctx& c, float* params, uint64_t d, uint64_t dim, const float* d_x, const float* d_t, uint64_t n,
                      uint64_t epochs, uint64_t batch, float lr, float wd, uint64_t seed, float* epoch_loss);

// ---- model.cu: the learned model on disk and the transform of new points ----
// Per-dimension mean and population std of an embedding (the standardisation of the MLP's targets).
void model_target_stats(const float* y, uint64_t n, uint64_t dim, float* mean, float* sd);
void model_save(const char* path, uint64_t d, uint64_t dim, const float* params, float pre_min, float pre_max,
                const float* pre_mean, const float* t_mean, const float* t_std);
// Any output pointer may be NULL (query the shape first, then read with buffers of that size).
void model_load(const char* path, uint64_t* d, uint64_t* dim, float* params, float* pre_min, float* pre_max,
                float* pre_mean, float* t_mean, float* t_std);
// out (n x dim, device) = MLP((x - min) / max - mean) * std + mean_t for device x (n x d); host constants.
// y = y * t_std + t_mean per dimension (host vectors of dim values), in place on the device.
void destandardise_device(Ctx& c, float* d_y, uint64_t n, uint64_t dim, const float* t_mean, const float* t_std);
void transform_device(Ctx& c, const float* d_x, uint64_t n, uint64_t d, uint64_t dim, const float* params,
                      float pre_min, float pre_max, const float* pre_mean, const float* t_mean, const float* t_std,
                      float* d_out);
}  // namespace pacmap
