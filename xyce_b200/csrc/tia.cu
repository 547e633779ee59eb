// Time-integration combine step (include/xyce_tia.h): forms the Newton matrix and residual of one
// iterate from the device loads, in one pass over the CSR rows.
//
// Restates N_TIA_OneStep::obtainJacobian / obtainResidual
// (src/TimeIntegrationPKG/src/N_TIA_OneStep.C:272-312, 470-497) and the linear devices' loads
// (N_DEV_Resistor.C:1075-1161, N_DEV_Capacitor.C:1821-2002, N_DEV_Vsrc.C:941-1028), with the
// residual's operations in the reference's order: ((Q - Q_n) / h + f F) + g F_hist, negated, then
// the limiter corrections (1/h) dQdxdVp and f dFdxdVp added.
// One warp per row: lanes take the row's entries with a fixed stride, and the per-row sums of the
// linear devices' F and Q use a fixed shuffle tree, so the results do not vary between runs.
#include <cuda_runtime.h>

#include <string>

#include "../../include/xyce_tia.h"

int xd_internal_fail(int code, const std::string &msg);

struct xd_tia {
  int device = 0;
  int n_rows = 0;
  int nnz = 0;
  int *d_rowptr = nullptr;
  int *d_colind = nullptr;
};

namespace {

constexpr int kWarpsPerBlock = 8;

__global__ void __launch_bounds__(32 * kWarpsPerBlock) tia_combine_kernel(
    int n_rows, const int *__restrict__ rowptr, const int *__restrict__ colind, xd_tia_coef c,
    const double *__restrict__ x, const double *__restrict__ dfdx, const double *__restrict__ dqdx,
    const double *__restrict__ lin_f, const double *__restrict__ lin_q, const double *__restrict__ f,
    const double *__restrict__ q, const double *__restrict__ fx, const double *__restrict__ qx,
    const double *__restrict__ b, const double *__restrict__ qn0,
    const double *__restrict__ fhist, double *__restrict__ jac, double *__restrict__ rhs,
    double *__restrict__ q_tot, double *__restrict__ f_tot) {
  const int row = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n_rows) return;
  const int beg = rowptr[row], end = rowptr[row + 1];
  const bool tran = c.mode != 0;
  double af = 0.0, aq = 0.0;
  bool has_diag = false;
  for (int k = beg + lane; k < end; k += 32) {
    double jf = dfdx[k];
    if (lin_f) {
      const double g = lin_f[k];
      jf += g;
      af += g * x[colind[k]];
    }
    if (c.gshunt != 0.0 && colind[k] == row) {
      jf += c.gshunt;
      has_diag = true;
    }
    if (tran) {
      double jq = dqdx[k];
      if (lin_q) {
        const double cq = lin_q[k];
        jq += cq;
        aq += cq * x[colind[k]];
      }
      jac[k] = c.qscale * jq + c.fscale * jf;
    } else {
      jac[k] = jf;
    }
  }
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    af += __shfl_down_sync(0xffffffffu, af, w);
    aq += __shfl_down_sync(0xffffffffu, aq, w);
  }
  // The shunt goes on rows whose diagonal is in the pattern (the node rows): F and J together.
  has_diag = __any_sync(0xffffffffu, has_diag);
  if (lane == 0) {
    double F = f[row] + af;
    if (has_diag) F += c.gshunt * x[row];
    if (b) F -= b[row];
    if (f_tot) f_tot[row] = F;
    if (!tran) {
      double r = -F;
      if (fx) r = r + fx[row];
      rhs[row] = r;
      return;
    }
    const double Q = q[row] + aq;
    if (q_tot) q_tot[row] = Q;
    double r = (Q - qn0[row]) * c.inv_h + c.fscale * F;
    if (c.hist_scale != 0.0) r = r + c.hist_scale * fhist[row];
    r = -r;
    if (qx) r = r + c.qscale * qx[row];
    if (fx) r = r + c.fscale * fx[row];
    rhs[row] = r;
  }
}

// Small dense direct solve (n <= XD_DENSE_MAX_N). One CTA: all warps scatter the CSR values and
// the right-hand side into an augmented row-major matrix [A | b] in shared memory; warp 0 alone
// then runs Gaussian elimination with partial pivoting (pivot = first row of largest magnitude,
// as LAPACK's idamax picks it; whole rows swapped, so the stored multipliers follow the final
// row order; multipliers scaled by the pivot's reciprocal, as LAPACK's dgetf2 does) and back
// substitution, with __syncwarp between steps and no block barriers. The elimination is
// latency-bound, so each lane keeps its column slots and the pivot row in registers, and rows
// whose multiplier is zero are skipped (a warp ballot finds the others): the sparse matrices of
// circuits cost far less than n^3 / 3. The other warps write the factors out at the end.
constexpr int kDenseThreads = 256;

constexpr int kDenseChunks = (XD_DENSE_MAX_N + 1 + 31) / 32;  // lane-strided slots per row (rhs included)

__device__ __forceinline__ void dense_forward_backward(int n, int lda, double *A, int *spiv, double *sinv,
                                                       int *sinfo) {
  const int lane = threadIdx.x & 31;
  const unsigned full = 0xffffffffu;
  for (int k = 0; k < n; ++k) {
    // Pivot: the first row of largest magnitude in column k (rows k..n-1).
    double v[kDenseChunks];
#pragma unroll
    for (int c = 0; c < kDenseChunks; ++c) {
      const int i = k + lane + 32 * c;
      v[c] = (i < n) ? fabs(A[i * lda + k]) : -1.0;
    }
    double best = -1.0;
    int bi = n;
#pragma unroll
    for (int c = 0; c < kDenseChunks; ++c)
      if (v[c] > best) {
        best = v[c];
        bi = k + lane + 32 * c;
      }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ob = __shfl_xor_sync(full, best, off);
      const int oi = __shfl_xor_sync(full, bi, off);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    const int p = (bi < n) ? bi : k;  // a column of NaNs has no pivot: keep the row
    if (lane == 0) {
      spiv[k] = p;
      if (!(best > 0.0) && *sinfo == 0) *sinfo = k + 1;
    }
    if (p != k) {
      for (int j = lane; j <= n; j += 32) {
        const double t = A[k * lda + j];
        A[k * lda + j] = A[p * lda + j];
        A[p * lda + j] = t;
      }
      __syncwarp();
    }
    const double inv = 1.0 / A[k * lda + k];
    if (lane == 0) sinv[k] = inv;
    // The pivot row's entries right of the diagonal (rhs included), kept in registers.
    double u[kDenseChunks];
#pragma unroll
    for (int c = 0; c < kDenseChunks; ++c) {
      const int j = k + 1 + lane + 32 * c;
      u[c] = (j <= n) ? A[k * lda + j] : 0.0;
    }
#pragma unroll
    for (int c = 0; c < kDenseChunks; ++c) {
      const int base = k + 1 + 32 * c;
      if (base >= n) break;
      const int i = base + lane;
      double l = 0.0;
      if (i < n) {
        l = A[i * lda + k] * inv;
        A[i * lda + k] = l;
      }
      unsigned m = __ballot_sync(full, l != 0.0);
      while (m) {
        const int bit = __ffs(m) - 1;
        m &= m - 1;
        const double li = __shfl_sync(full, l, bit);
        double *row = A + (base + bit) * lda;
#pragma unroll
        for (int cc = 0; cc < kDenseChunks; ++cc) {
          const int j = k + 1 + lane + 32 * cc;
          if (j <= n) row[j] = row[j] - li * u[cc];
        }
      }
    }
    __syncwarp();
  }
  // Back substitution on U, column by column; y (column n) becomes x.
  for (int k = n - 1; k >= 0; --k) {
    const double xk = A[k * lda + n] * sinv[k];
#pragma unroll
    for (int c = 0; c < kDenseChunks; ++c) {
      const int i = lane + 32 * c;
      if (i < k) A[i * lda + n] = A[i * lda + n] - A[i * lda + k] * xk;
    }
    __syncwarp();
    if (lane == 0) A[k * lda + n] = xk;
    __syncwarp();
  }
}

__global__ void __launch_bounds__(kDenseThreads) dense_factor_solve_kernel(
    int n, const int *__restrict__ rowptr, const int *__restrict__ colind, const double *__restrict__ vals,
    const double *__restrict__ rhs, double *__restrict__ lu, int *__restrict__ piv, double *__restrict__ x,
    int *__restrict__ info) {
  extern __shared__ double A[];
  __shared__ int spiv[XD_DENSE_MAX_N];
  __shared__ double sinv[XD_DENSE_MAX_N];
  __shared__ int sinfo;
  const int lda = n + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int idx = tid; idx < n * lda; idx += kDenseThreads) A[idx] = 0.0;
  if (tid == 0) sinfo = 0;
  __syncthreads();
  for (int r = warp; r < n; r += kDenseThreads / 32) {
    for (int k = rowptr[r] + lane; k < rowptr[r + 1]; k += 32) A[r * lda + colind[k]] = vals[k];
    if (lane == 0) A[r * lda + n] = rhs[r];
  }
  __syncthreads();
  if (warp == 0) dense_forward_backward(n, lda, A, spiv, sinv, &sinfo);
  __syncthreads();
  for (int idx = tid; idx < n * n; idx += kDenseThreads) {
    const int r = idx / n, cc = idx - r * n;
    if (lu) lu[idx] = A[r * lda + cc];
  }
  for (int r = tid; r < n; r += kDenseThreads) {
    x[r] = A[r * lda + n];
    if (piv) piv[r] = spiv[r];
  }
  if (tid == 0 && info) *info = sinfo;
}

// Solve with kept factors: the row interchanges, then forward substitution with the unit lower
// factor and back substitution with the upper one, in the same order of operations as the
// elimination above applies them to its right-hand side.
__global__ void __launch_bounds__(32) dense_resolve_kernel(int n, const double *__restrict__ lu,
                                                            const int *__restrict__ piv,
                                                            const double *__restrict__ rhs, double *__restrict__ x) {
  __shared__ double y[XD_DENSE_MAX_N];
  const int lane = threadIdx.x;
  for (int i = lane; i < n; i += 32) y[i] = rhs[i];
  __syncwarp();
  if (lane == 0) {
    for (int k = 0; k < n; ++k) {
      const int p = piv[k];
      if (p != k) {
        const double t = y[k];
        y[k] = y[p];
        y[p] = t;
      }
    }
  }
  __syncwarp();
  for (int k = 0; k < n; ++k) {
    const double yk = y[k];
    for (int i = k + 1 + lane; i < n; i += 32) {
      const double l = lu[(size_t)i * n + k];
      if (l != 0.0) y[i] = y[i] - l * yk;
    }
    __syncwarp();
  }
  for (int k = n - 1; k >= 0; --k) {
    const double xk = y[k] * (1.0 / lu[(size_t)k * n + k]);
    for (int i = lane; i < k; i += 32) y[i] = y[i] - lu[(size_t)i * n + k] * xk;
    __syncwarp();
    if (lane == 0) y[k] = xk;
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) x[i] = y[i];
}

size_t dense_smem_bytes(int n) { return sizeof(double) * (size_t)n * (size_t)(n + 1); }

struct Guard {
  int prev = -1;
  explicit Guard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~Guard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int cuda_err(cudaError_t e, const char *where) {
  return xd_internal_fail(-3, std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int xd_tia_create(const xd_csr *pat, int cuda_device, xd_tia **out) {
  if (!pat || !out) return xd_internal_fail(-1, "null argument");
  *out = nullptr;
  if (pat->n_rows < 0 || !pat->rowptr) return xd_internal_fail(-1, "bad CSR pattern");
  const int nnz = pat->rowptr[pat->n_rows];
  if (nnz < 0 || (nnz > 0 && !pat->colind)) return xd_internal_fail(-1, "bad CSR pattern");
  for (int r = 0; r < pat->n_rows; ++r)
    if (pat->rowptr[r + 1] < pat->rowptr[r]) return xd_internal_fail(-1, "CSR rowptr is not monotone");
  for (int k = 0; k < nnz; ++k)
    if (pat->colind[k] < 0 || pat->colind[k] >= pat->n_rows)
      return xd_internal_fail(-1, "CSR column index out of range");
  cudaError_t e = cudaSetDevice(cuda_device);
  if (e != cudaSuccess) return cuda_err(e, "cudaSetDevice");
  xd_tia *t = new xd_tia();
  t->device = cuda_device;
  t->n_rows = pat->n_rows;
  t->nnz = nnz;
  if ((e = cudaMalloc(&t->d_rowptr, sizeof(int) * (size_t)(pat->n_rows + 1))) != cudaSuccess ||
      (e = cudaMalloc(&t->d_colind, sizeof(int) * (size_t)(nnz > 0 ? nnz : 1))) != cudaSuccess ||
      (e = cudaMemcpy(t->d_rowptr, pat->rowptr, sizeof(int) * (size_t)(pat->n_rows + 1),
                      cudaMemcpyHostToDevice)) != cudaSuccess ||
      (nnz > 0 && (e = cudaMemcpy(t->d_colind, pat->colind, sizeof(int) * (size_t)nnz, cudaMemcpyHostToDevice)) !=
                      cudaSuccess)) {
    cudaFree(t->d_rowptr);
    cudaFree(t->d_colind);
    delete t;
    return cuda_err(e, "xd_tia_create upload");
  }
  if (pat->n_rows <= XD_DENSE_MAX_N && dense_smem_bytes(pat->n_rows) > 48 * 1024) {
    e = cudaFuncSetAttribute(dense_factor_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dense_smem_bytes(pat->n_rows));
    if (e != cudaSuccess) {
      cudaFree(t->d_rowptr);
      cudaFree(t->d_colind);
      delete t;
      return cuda_err(e, "dense solve shared-memory attribute");
    }
  }
  *out = t;
  return 0;
}

int xd_tia_destroy(xd_tia *t) {
  if (!t) return 0;
  Guard g(t->device);
  cudaFree(t->d_rowptr);
  cudaFree(t->d_colind);
  delete t;
  return 0;
}

int xd_tia_combine(xd_tia *t, const xd_tia_coef *coef, const double *d_x, const double *d_dfdx,
                   const double *d_dqdx, const double *d_lin_dfdx, const double *d_lin_dqdx, const double *d_f,
                   const double *d_q, const double *d_dfdxdvp, const double *d_dqdxdvp, const double *d_b,
                   const double *d_qn0, const double *d_fhist, double *d_jac, double *d_rhs, double *d_q_tot,
                   double *d_f_tot, void *stream) {
  if (!t || !coef) return xd_internal_fail(-1, "null argument");
  if (t->n_rows == 0) return 0;
  if (!d_x || !d_dfdx || !d_f || !d_jac || !d_rhs) return xd_internal_fail(-1, "null device buffer");
  if (coef->mode != 0 && (!d_dqdx || !d_q || !d_qn0 || (coef->hist_scale != 0.0 && !d_fhist)))
    return xd_internal_fail(-1, "null device buffer for a time step");
  Guard g(t->device);
  const int blocks = (t->n_rows + kWarpsPerBlock - 1) / kWarpsPerBlock;
  tia_combine_kernel<<<blocks, 32 * kWarpsPerBlock, 0, (cudaStream_t)stream>>>(
      t->n_rows, t->d_rowptr, t->d_colind, *coef, d_x, d_dfdx, d_dqdx, d_lin_dfdx, d_lin_dqdx, d_f, d_q, d_dfdxdvp,
      d_dqdxdvp, d_b, d_qn0, d_fhist, d_jac, d_rhs, d_q_tot, d_f_tot);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "tia_combine_kernel launch");
  return 0;
}

int xd_tia_dense_solve(xd_tia *t, const double *d_jac, const double *d_rhs, double *d_lu, int *d_piv, double *d_x,
                       int *d_info, void *stream) {
  if (!t) return xd_internal_fail(-1, "null argument");
  if (t->n_rows == 0) return 0;
  if (t->n_rows > XD_DENSE_MAX_N)
    return xd_internal_fail(-1, "the dense solve takes at most " + std::to_string(XD_DENSE_MAX_N) + " unknowns");
  if (!d_jac || !d_rhs || !d_x) return xd_internal_fail(-1, "null device buffer");
  Guard g(t->device);
  dense_factor_solve_kernel<<<1, kDenseThreads, dense_smem_bytes(t->n_rows), (cudaStream_t)stream>>>(
      t->n_rows, t->d_rowptr, t->d_colind, d_jac, d_rhs, d_lu, d_piv, d_x, d_info);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "dense_factor_solve_kernel launch");
  return 0;
}

int xd_tia_dense_resolve(xd_tia *t, const double *d_lu, const int *d_piv, const double *d_rhs, double *d_x,
                         void *stream) {
  if (!t) return xd_internal_fail(-1, "null argument");
  if (t->n_rows == 0) return 0;
  if (t->n_rows > XD_DENSE_MAX_N)
    return xd_internal_fail(-1, "the dense solve takes at most " + std::to_string(XD_DENSE_MAX_N) + " unknowns");
  if (!d_lu || !d_piv || !d_rhs || !d_x) return xd_internal_fail(-1, "null device buffer");
  Guard g(t->device);
  dense_resolve_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(t->n_rows, d_lu, d_piv, d_rhs, d_x);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "dense_resolve_kernel launch");
  return 0;
}

}  // extern "C"
