/* C ABI of the learned warm-start network: a ReLU multilayer perceptron whose
 * training and inference run on the B200's 5th-generation tensor cores
 * (tcgen05 MMA, BF16 operands, FP32 accumulation in tensor memory) through
 * this project's own forward, backward and Adam kernels.
 *
 * No counterpart in the reference: its parametric layer
 * (src/parametric/parametric.cpp:483-530, compareFamilyStrategies) warm-starts
 * nothing and has no learned model.  The network maps a parametric LP
 * family's parameters to coefficients of a PCA basis of PDHG primal-dual
 * solutions; the host side (pramana_b200/warmstart.py) turns them into the
 * starting points passed to b2p_engine_set_start / b2p_solve_pdhg_multi.
 *
 * Parameters: one FP32 master vector, per layer l = 0 .. L-1 the weight
 * W_l (widths[l+1] x widths[l], row-major) followed by the bias b_l
 * (widths[l+1]).  The GEMMs read a BF16 copy refreshed after every update.
 * Layer l computes h_{l+1} = relu(h_l W_l^T + b_l) (no ReLU on the last
 * layer); hidden activations are stored in BF16.  Loss on a batch of B:
 * (1 / B) * sum_b 0.5 * ||out_b - target_b||^2.
 *
 * Return codes and b2p_last_error() are those of b2p_pdhg.h. */
#ifndef B2P_MLP_H
#define B2P_MLP_H

#include <stdint.h>

#include "b2p_pdhg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct b2p_mlp b2p_mlp;

typedef struct b2p_mlp_train_options {
  int32_t epochs;       /* passes over the data */
  int32_t batch;        /* minibatch size (<= max_batch of the network) */
  float lr;             /* Adam step size at the start */
  float lr_final;       /* cosine decay reaches this at the last step */
  float beta1, beta2, eps;
  float weight_decay;   /* decoupled (AdamW) decay on the weights, 0 = off */
  uint64_t seed;        /* minibatch shuffling */
} b2p_mlp_train_options;

/* Defaults: 200 epochs, batch 512, lr 1e-3 -> 1e-5, betas 0.9 / 0.999,
 * eps 1e-8, no weight decay, seed 0. */
b2p_mlp_train_options b2p_mlp_default_train_options(void);

/* widths[0] = input size, widths[num_layers] = output size; every width a
 * multiple of 8.  Parameters start at zero (set them with b2p_mlp_set_params).
 * device < 0 picks as b2p_options.device does. */
int b2p_mlp_create(const int32_t* widths, int32_t num_layers, int32_t max_batch, int32_t device, b2p_mlp** out);
int b2p_mlp_destroy(b2p_mlp* net);
int b2p_mlp_num_params(const b2p_mlp* net, int64_t* count);
/* Host FP32 vectors of b2p_mlp_num_params entries in the layout above;
 * set_params also clears the Adam moments and step count. */
int b2p_mlp_set_params(b2p_mlp* net, const float* params);
int b2p_mlp_get_params(b2p_mlp* net, float* params);

/* Inference: x is batch x widths[0], y batch x widths[L] (host, row-major). */
int b2p_mlp_forward(b2p_mlp* net, const float* x, int64_t batch, float* y);
/* Same, on device pointers and a caller stream (cudaStream_t or NULL). */
int b2p_mlp_forward_device(b2p_mlp* net, const float* x, int64_t batch, float* y, void* stream);

/* Loss and its gradient with respect to every parameter on one batch
 * (batch <= max_batch), without updating the parameters.  grad may be NULL. */
int b2p_mlp_loss_grad(b2p_mlp* net, const float* x, const float* target, int32_t batch, double* loss, float* grad);

/* Adam training on count samples (x: count x widths[0], target:
 * count x widths[L], host).  epoch_loss (may be NULL) receives the mean
 * minibatch loss of each epoch.  Errors: B2P_ERR_CUDA when a tensor-core
 * wait times out (the network state is then undefined). */
int b2p_mlp_train(b2p_mlp* net, const float* x, const float* target, int64_t count,
                  const b2p_mlp_train_options* opts, float* epoch_loss);

/* Kernel-level entry, device pointers (BF16 as raw 16-bit words):
 * C(m, n) = epilogue(alpha * sum_k A(m, k) B(k, n)) with A(m, k) =
 * A[m * sam + k * sak], B(k, n) = B[k * sbk + n * sbn]; the epilogue adds
 * bias[n] (NULL = none), applies ReLU when relu != 0, zeroes C(m, n) where
 * mask[m * ldm + n] <= 0 (NULL = none), and stores FP32 to cf (ldcf) and/or
 * BF16 to cb (ldcb).  Synchronous on the given stream (NULL = default).
 * When both operands are K-contiguous (sak == 1, sbk == 1) with row strides
 * that are multiples of 8 elements and 16-byte aligned bases, the tiles are
 * brought in by TMA; otherwise by the threads' cp.async copies.  Both forms
 * issue the same tensor-core instructions in the same K order. */
int b2p_mlp_gemm_bf16(int32_t M, int32_t N, int32_t K, const uint16_t* A, int64_t sam, int64_t sak,
                      const uint16_t* B, int64_t sbk, int64_t sbn, float alpha, const float* bias, int32_t relu,
                      const uint16_t* mask, int64_t ldm, float* cf, int64_t ldcf, uint16_t* cb, int64_t ldcb,
                      void* stream);

/* Kernel timing: the tensor-core GEMM of b2p_mlp_gemm_bf16 (alpha 1, no
 * epilogue options, FP32 output) launched `reps` times back to back on a
 * private stream after one warm-up launch, bracketed by CUDA events;
 * *ms_per_launch = the events' elapsed time / reps.  Device pointers. */
int b2p_mlp_gemm_bf16_time(int32_t M, int32_t N, int32_t K, const uint16_t* A, int64_t sam, int64_t sak,
                           const uint16_t* B, int64_t sbk, int64_t sbn, float* cf, int64_t ldcf, int32_t reps,
                           double* ms_per_launch);

#ifdef __cplusplus
}
#endif

#endif
