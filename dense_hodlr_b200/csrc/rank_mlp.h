// Rank predictor MLP launches (rank_mlp.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

int mlp_sample_floats();
int mlp_forward_launch(const float* p, const float* X, int B, float* y, cudaStream_t s);
int mlp_train_launch(float* p, float* m1, float* m2, const float* X, const float* T, int B,
                     float* S, float lr, int t, float* grad_out, float* loss_out,
                     cudaStream_t s);
int block_features_launch(const double* pts, int64_t ld, int dim, const int4* geom, int nb,
                          float log_l, float log_tol, float* F, cudaStream_t s);
