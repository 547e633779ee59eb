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
  for (int k = beg + lane; k < end; k += 32) {
    double jf = dfdx[k];
    if (lin_f) {
      const double g = lin_f[k];
      jf += g;
      af += g * x[colind[k]];
    }
    if (c.gshunt != 0.0 && colind[k] == row) jf += c.gshunt;
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
  if (lane == 0) {
    double F = f[row] + af;
    if (c.gshunt != 0.0) F += c.gshunt * x[row];
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

}  // extern "C"
