// Internal entry points of the tensor-core GEMM and the warm-start MLP (csrc/mlp.cu).
#pragma once
#include "ctx.cuh"

namespace rumb {
struct Mlp;
int gemm_bf16_host(Ctx &c, int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C);
Mlp *mlp_create(Ctx &c, int n_layers, const int *dims, unsigned long long seed);
void mlp_destroy(Mlp *m);
ll mlp_num_params(const Mlp &m);
void mlp_get_params(Mlp &m, float *buf, bool grads);
void mlp_set_params(Mlp &m, const float *buf);
void mlp_forward(Mlp &m, const float *X, ll rows, float *Y);
double mlp_loss_grad(Mlp &m, const float *X, const float *T, ll rows, float *grad);
double mlp_train(Mlp &m, const float *X, const float *T, ll rows, int epochs, int batch, double lr,
                 unsigned long long seed);
}  // namespace rumb
