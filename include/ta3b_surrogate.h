/* ta3b_surrogate.h -- C ABI of the surrogate fitness model (library
 * tetris_ai3_b200/_lib/libta3b.so). No counterpart in the reference: it is the
 * learned pre-screener of the island trainer (ta3b_trainer.h, ta3t_surrogate).
 *
 * Model: MLP 97 -> 128 -> 128 -> 2 (predicted mean score, log-variance), ReLU,
 * BF16 weights and activations on the sm_100a tensor cores (tcgen05.mma) with
 * FP32 accumulation; FP32 master parameters, Adam, Gaussian negative
 * log-likelihood 0.5 * (s + (y - mu)^2 exp(-s)) averaged over the batch.
 * Inputs and targets are standardised per column from the training set.
 *
 * Parameter vector (FP32, ta3s_num_params() = 31234 values):
 *   W1 [128][112] (row o, column i; columns 97..111 are zero padding),
 *   W2 [128][128], W3 [2][128], b1 [128], b2 [128], b3 [2].
 * Gradients use the same layout. A model is not thread-safe. */
#ifndef TA3B_SURROGATE_H
#define TA3B_SURROGATE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ta3s_model ta3s_model;

uint32_t ta3s_num_params(void);
/* He-uniform initialisation from mt19937(seed); NULL without an sm_100 device */
ta3s_model* ta3s_create(int device, uint32_t seed);
void ta3s_destroy(ta3s_model* m);
const char* ta3s_last_error(const ta3s_model* m);

int ta3s_set_params(ta3s_model* m, const float* params);   /* also resets the Adam moments */
int ta3s_get_params(ta3s_model* m, float* params_out);

/* training set: x row-major [n][97], y [n] (mean scores); computes the
 * standardisation used by later predictions */
int ta3s_set_data(ta3s_model* m, const float* x, const float* y, uint32_t n);
/* training set used as given (identity standardisation), for gradient checks */
int ta3s_set_data_standardized(ta3s_model* m, const float* x, const float* y, uint32_t n);
/* one forward + backward pass over the whole training set: gradient of the
 * mean loss (parameter layout) and the summed loss; no update */
int ta3s_gradients(ta3s_model* m, float* grad_out, float* loss_sum_out);
/* AdamW (beta 0.9 / 0.999, eps 1e-8, decoupled weight decay) over shuffled
 * minibatches from mt19937(seed); final_loss: mean loss of the last minibatch */
int ta3s_train(ta3s_model* m, uint32_t epochs, uint32_t batch, float lr, float weight_decay, uint32_t seed,
               float* final_loss);
/* predicted mean score (in target units) and log-variance for n rows [n][97].
 * Replaces the device copy of the training rows: call ta3s_set_data again
 * before the next ta3s_train. */
int ta3s_predict(ta3s_model* m, const float* x, uint32_t n, float* mean_out, float* logvar_out);

/* ---- the same scheme for any parameter-vector size (ta3w_*) ----
 * MLP in -> H -> H -> 2 for the widened evaluator's 4,929-parameter vectors
 * (H = 256) or any other size: in_dim >= 1, H a multiple of 128. Each matrix
 * product is one launch of a tcgen05 BF16 GEMM kernel (FP32 accumulation in
 * tensor memory, split-K for the first layer); bias, ReLU, output layer, loss and
 * bias gradients in FP32 on the CUDA cores. Rounding points (BF16, nearest
 * even): standardised inputs, W1, W2, relu(H1), dH2, dH1; everything else FP32.
 * Parameter vector (ta3w_num_params(in_dim, H) values), INP = in_dim rounded up
 * to a multiple of 128:
 *   W1 [H][INP] (columns in_dim.. are zero padding), W2 [H][H], W3 [2][H],
 *   b1 [H], b2 [H], b3 [2]. Gradients use the same layout.
 * Calls mirror the ta3s_* functions above; ta3w_gradients takes at most 65,536
 * rows and ta3w_train a minibatch of at most 65,536. A model is not thread-safe. */
typedef struct ta3w_model ta3w_model;

uint32_t ta3w_num_params(uint32_t in_dim, uint32_t hidden);   /* 0 for unsupported sizes */
ta3w_model* ta3w_create(int device, uint32_t in_dim, uint32_t hidden, uint32_t seed);
void ta3w_destroy(ta3w_model* m);
const char* ta3w_last_error(const ta3w_model* m);
uint32_t ta3w_model_params(const ta3w_model* m);
int ta3w_set_params(ta3w_model* m, const float* params);     /* also resets the Adam moments */
int ta3w_get_params(ta3w_model* m, float* params_out);
int ta3w_set_data(ta3w_model* m, const float* x, const float* y, uint32_t n);   /* x [n][in_dim] */
int ta3w_set_data_standardized(ta3w_model* m, const float* x, const float* y, uint32_t n);
int ta3w_gradients(ta3w_model* m, float* grad_out, float* loss_sum_out);
int ta3w_train(ta3w_model* m, uint32_t epochs, uint32_t batch, float lr, float weight_decay, uint32_t seed,
               float* final_loss);
int ta3w_predict(ta3w_model* m, const float* x, uint32_t n, float* mean_out, float* logvar_out);
/* Test hook: the GEMM kernel alone on host BF16 bit patterns. c [m][n] =
 * sum_k A(m, k) B(n, k) with A given as [m][k] (a_mn = 0) or [k][m] (a_mn = 1)
 * and B as [n][k] or [k][n]; m, n multiples of 128, k of 64; K split `splits` ways. */
int ta3w_gemm_test(int device, int a_mn, int b_mn, int m, int n, int k, int splits, const uint16_t* a,
                   const uint16_t* b, float* c);

#ifdef __cplusplus
}
#endif

#endif
