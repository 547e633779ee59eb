/* xyce_surrogate.h — C ABI of the learned surrogate's tensor-core kernels.
 *
 * No counterpart in the reference: the surrogate (a small MLP of the BSIM4 current/charge map,
 * used for Newton warm starts) is this project's addition. Its forward and backward passes are
 * sequences of one BF16 GEMM on the tcgen05 tensor cores with fused epilogues, plus loss, bias,
 * split-K and Adam kernels; the host sequences the calls. Buffers are caller-owned device
 * pointers (BF16 passed as void*); calls are stream-ordered. Status: >= 0 ok, < 0 error
 * (xd_last_error()). A kernel whose internal wait expires sets *err (device int) to 1.
 */
#ifndef XYCE_SURROGATE_H
#define XYCE_SURROGATE_H

#include "xyce_devload.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Epilogues of xd_gemm_bf16 (acc = (A B^T)[row][n], FP32):
 *   XD_EPI_F32        C32[split][row][n] = acc              (split-K partials; splits >= 1)
 *   XD_EPI_BIAS_F32   C32[row][n] = acc + bias[n]            (network output)
 *   XD_EPI_BIAS_SILU  z = acc + bias[n]; Z[row][n] = z, H[row][n] = silu(z), HT[n][row] = silu(z)
 *   XD_EPI_SILU_BACK  d = acc * silu'(Zin[row][n]); H[row][n] = d, HT[n][row] = d
 * Z, H, HT, Zin are BF16 (row stride ldc, HT row stride ldt); HT may be null. */
enum { XD_EPI_F32 = 0, XD_EPI_BIAS_F32 = 1, XD_EPI_BIAS_SILU = 2, XD_EPI_SILU_BACK = 3 };

typedef struct xd_gemm_args {
  const void *A; /* BF16 [M x K], row stride lda (K contiguous) */
  const void *B; /* BF16 [N x K], row stride ldb */
  int M, N, K, lda, ldb, ldc, ldt;
  int tile_n;    /* 16 or 128 */
  int epilogue;  /* XD_EPI_* */
  float *C32;
  const float *bias;
  void *Z, *H, *HT;
  const void *Zin;
  int *err;      /* device flag, set to 1 if an internal wait expired */
} xd_gemm_args;

/* C = A B^T with the chosen epilogue, K split into `splits` slices (partials for XD_EPI_F32).
 * Requires K % 16 == 0, lda % 8 == 0, ldb % 8 == 0, 16-byte aligned A and B. Returns the number of
 * K slices actually used (>= 1) or < 0. */
int xd_gemm_bf16(const xd_gemm_args *args, int splits, void *stream);

/* First layer in FP32 (CUDA cores), so that the inputs keep full precision: for each of the M
 * rows of x [M x ldx] (n_in <= 8 used columns) and each hidden unit u < n_hid (<= 1024),
 * z = w1[u] . x + b1[u] (w1 row stride ldw); Z, H = silu(z) BF16 [M x n_hid], HT [n_hid x ldt]. */
int xd_mlp_input_layer(int M, int n_in, int n_hid, const float *d_x, int ldx, const float *d_w1, int ldw,
                       const float *d_b1, void *d_z, void *d_h, void *d_ht, int ldt, void *stream);

/* Its weight gradient: gw[u][i] = sum_{r < M} dzt[u][r] x[r][i] (FP32, fixed tree). */
int xd_mlp_input_grad(int M, int n_in, int n_hid, const void *d_dzt, int ldt, const float *d_x, int ldx,
                      float *d_gw, int ldw, void *stream);

/* The whole surrogate network for inference in one persistent kernel: weights staged once per CTA
 * in shared memory, each 128-sample tile through the FP32 first layer (CUDA cores), three 128-wide
 * BF16 layers and the 16-wide output layer on the tcgen05 tensor cores (accumulator in tensor
 * memory, bias + SiLU epilogues writing the next operand back to shared memory). Reads x [n x ldx]
 * (n_in columns), writes y [n x ldy] (ldy >= 16; 16 outputs, padding included). max_ctas <= 0
 * means one CTA per SM. */
typedef struct xd_mlp_net {
  int n_in;            /* inputs, <= 8 */
  const float *w1;     /* FP32 [128 x ldw1] */
  int ldw1;
  const void *w[3];    /* BF16 [128 x 128], hidden layers 2..4, row-major [out][in] */
  const void *w5;      /* BF16 [16 x 128], output layer (rows past the outputs zero) */
  const float *b[5];   /* FP32 biases: 128, 128, 128, 128, 16 */
} xd_mlp_net;

int xd_mlp_forward(const xd_mlp_net *net, int n, const float *d_x, int ldx, float *d_y, int ldy, int *d_err,
                   int max_ctas, void *stream);

/* d = scale * (y - target) for the first n_out of ld columns (0 in the padding), as BF16 in
 * d_dz [M x ld] and transposed in d_dzt [ld x ldt]; per-sample squared error into d_sq (or null). */
int xd_mse_grad(int M, int n_out, int ld, const float *d_y, const float *d_target, float scale, void *d_dz,
                void *d_dzt, int ldt, float *d_sq, void *stream);

/* db[n] = sum_r dzt[n][r], r < M (BF16 input, FP32 sum in a fixed tree). */
int xd_bias_grad(int M, int N, const void *d_dzt, int ldt, float *d_db, void *stream);

/* out[i] = sum_{s < splits} part[s * n + i], in order. */
int xd_splitk_sum(int n, int splits, const float *d_part, float *d_out, void *stream);

/* out[c] = sum_{r < rows} in[r * ld + c] (FP32, fixed tree). */
int xd_column_sum(int rows, int cols, const float *d_in, int ld, float *d_out, void *stream);

/* Surrogate inputs of circuit instances idx[k] (k < n): from the solution d_sol and the
 * instances' terminal unknowns d_nodes4 [n_inst x 4] (D, G, S, B; -1 = ground), x[k] =
 * ((VG - VS) / vmax, (VD - VS) / vmax, (VB - VS) / vmax, geom2[2i], geom2[2i + 1]) (FP32, row
 * stride ldx >= 5); geom2 holds each instance's scaled log W and log L. */
int xd_surrogate_features(int n, const int *d_idx, const int *d_nodes4, const double *d_sol, const float *d_geom2,
                          float vmax, float *d_x, int ldx, void *stream);

/* Decodes outputs y[k] (row stride ldy; value = sinh(y) * out_scale[j] for j = Id, Qg, Qd, Qb)
 * of instances idx[k] and writes their terminal currents and charges into a staged array
 * [16 x n_inst] in the exact load's slot layout (F at D, G, S, B; Q at D, G, S, B; limiter slots
 * zero), ready for xd_load_vectors_staged. */
int xd_surrogate_stage(int n, const int *d_idx, const float *d_y, int ldy, const float *d_out_scale, int n_inst,
                       double *d_stage, void *stream);

typedef struct xd_adam_args {
  float lr, beta1, beta2, eps, bias_corr1, bias_corr2; /* bias_corr = 1 - beta^t */
} xd_adam_args;

/* One Adam step on FP32 parameters p [rows x cols] with gradient grad and moments m, v; refreshes
 * BF16 copies p16 [rows x ld16] and its transpose p16t [cols x ld16t] (either may be null). */
int xd_adam(int rows, int cols, float *d_p, const float *d_grad, float *d_m, float *d_v, const xd_adam_args *a,
            void *d_p16, void *d_p16t, int ld16, int ld16t, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* XYCE_SURROGATE_H */
