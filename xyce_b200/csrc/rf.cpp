// GPU sparse LU refactorization for the Newton matrices of a transient (include/xyce_rf.h).
//
// Every Newton matrix of a circuit has the same sparsity pattern, so after one numeric
// factorization P A Q = L U on the host (its pivot order and fill pattern), every later matrix is
// refactored and solved on the GPU with that pattern, and the values never leave the device. The
// refactorization (lu.cu) and the triangular solves (sptrsv.cu) are the library's own kernels.
// cuSOLVER's refactorization library is kept only as a comparison (xd_rf_refactor_library,
// xd_rf_solve_library), set up on first use.
#include <cuda_runtime.h>
#include <cusolverRf.h>

#include <string>
#include <vector>

#include "../../include/xyce_rf.h"
#include "lu.h"
#include "sptrsv.h"

int xd_internal_fail(int code, const std::string &msg);

struct xd_rf {
  int device = 0;
  int n = 0, nnz_a = 0;
  int *d_rowptr = nullptr, *d_colind = nullptr, *d_p = nullptr, *d_q = nullptr;
  double *d_temp = nullptr;
  XdLu lu;        // the refactorization
  XdSptrsv tri;   // the triangular solves, over lu's bundled factors
  // The comparison library, created on first use from host copies of the set-up inputs.
  cusolverRfHandle_t h = nullptr;
  std::vector<int> ra, ca, rl, cl, ru, cu, hp, hq;
  std::vector<double> va, vl, vu;
};

namespace {

int rf_fail(cusolverStatus_t st, const char *where) {
  return xd_internal_fail(-4, std::string("cuSOLVER refactorization error ") + std::to_string((int)st) + " in " +
                                  where);
}

int cu_fail(cudaError_t e, const char *where) {
  return xd_internal_fail(-3, std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
}

void release(xd_rf *r) {
  if (!r) return;
  if (r->h) cusolverRfDestroy(r->h);
  xd_sptrsv_free(&r->tri);
  xd_lu_free(&r->lu);
  cudaFree(r->d_rowptr);
  cudaFree(r->d_colind);
  cudaFree(r->d_p);
  cudaFree(r->d_q);
  cudaFree(r->d_temp);
  delete r;
}

bool csr_ok(int n, int nnz, const int *rp, const int *ci) {
  if (!rp || (nnz > 0 && !ci) || rp[0] != 0 || rp[n] != nnz) return false;
  for (int r = 0; r < n; ++r)
    if (rp[r + 1] < rp[r]) return false;
  for (int k = 0; k < nnz; ++k)
    if (ci[k] < 0 || ci[k] >= n) return false;
  return true;
}

bool perm_ok(int n, const int *p) {
  if (!p) return false;
  std::vector<char> seen(n, 0);
  for (int i = 0; i < n; ++i) {
    if (p[i] < 0 || p[i] >= n || seen[p[i]]) return false;
    seen[p[i]] = 1;
  }
  return true;
}

}  // namespace

extern "C" {

int xd_rf_create(int n, int nnz_a, const int *rowptr_a, const int *colind_a, const double *vals_a, int nnz_l,
                 const int *rowptr_l, const int *colind_l, const double *vals_l, int nnz_u, const int *rowptr_u,
                 const int *colind_u, const double *vals_u, const int *p, const int *q, int cuda_device,
                 xd_rf **out) {
  if (!out || n <= 0 || !vals_a || !vals_l || !vals_u) return xd_internal_fail(-1, "bad refactorization arguments");
  *out = nullptr;
  if (!csr_ok(n, nnz_a, rowptr_a, colind_a) || !csr_ok(n, nnz_l, rowptr_l, colind_l) ||
      !csr_ok(n, nnz_u, rowptr_u, colind_u))
    return xd_internal_fail(-1, "bad CSR input to the refactorization set-up");
  if (!perm_ok(n, p) || !perm_ok(n, q)) return xd_internal_fail(-1, "P and Q must be permutations of 0..n-1");
  cudaError_t e = cudaSetDevice(cuda_device);
  if (e != cudaSuccess) return cu_fail(e, "cudaSetDevice");
  xd_rf *r = new xd_rf();
  r->device = cuda_device;
  r->n = n;
  r->nnz_a = nnz_a;
  if ((e = cudaMalloc(&r->d_rowptr, sizeof(int) * (n + 1))) != cudaSuccess ||
      (e = cudaMalloc(&r->d_colind, sizeof(int) * (nnz_a > 0 ? nnz_a : 1))) != cudaSuccess ||
      (e = cudaMalloc(&r->d_p, sizeof(int) * n)) != cudaSuccess ||
      (e = cudaMalloc(&r->d_q, sizeof(int) * n)) != cudaSuccess ||
      (e = cudaMalloc(&r->d_temp, sizeof(double) * n)) != cudaSuccess ||
      (e = cudaMemcpy(r->d_rowptr, rowptr_a, sizeof(int) * (n + 1), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(r->d_colind, colind_a, sizeof(int) * nnz_a, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(r->d_p, p, sizeof(int) * n, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(r->d_q, q, sizeof(int) * n, cudaMemcpyHostToDevice)) != cudaSuccess) {
    release(r);
    return cu_fail(e, "xd_rf_create upload");
  }
  // Host copies for the comparison library (created on first use).
  r->ra.assign(rowptr_a, rowptr_a + n + 1);
  r->ca.assign(colind_a, colind_a + nnz_a);
  r->va.assign(vals_a, vals_a + nnz_a);
  r->rl.assign(rowptr_l, rowptr_l + n + 1);
  r->cl.assign(colind_l, colind_l + nnz_l);
  r->vl.assign(vals_l, vals_l + nnz_l);
  r->ru.assign(rowptr_u, rowptr_u + n + 1);
  r->cu.assign(colind_u, colind_u + nnz_u);
  r->vu.assign(vals_u, vals_u + nnz_u);
  r->hp.assign(p, p + n);
  r->hq.assign(q, q + n);
  int rc = xd_lu_init(&r->lu, n, nnz_a, rowptr_a, colind_a, rowptr_l, colind_l, rowptr_u, colind_u, p, q);
  if (rc != 0) {
    release(r);
    return rc;
  }
  rc = xd_sptrsv_init(&r->tri, n, r->lu.nnz, r->lu.d_mp, r->lu.d_mi, p, q);
  if (rc != 0) {
    release(r);
    return rc;
  }
  // The set-up factors A's own values.
  double *d_a = nullptr;
  if ((e = cudaMalloc(&d_a, sizeof(double) * (nnz_a > 0 ? nnz_a : 1))) != cudaSuccess ||
      (e = cudaMemcpy(d_a, vals_a, sizeof(double) * nnz_a, cudaMemcpyHostToDevice)) != cudaSuccess) {
    cudaFree(d_a);
    release(r);
    return cu_fail(e, "xd_rf_create upload");
  }
  int info = 0;
  rc = xd_lu_refactor(&r->lu, d_a, 0);
  if (rc == 0) rc = xd_lu_info(&r->lu, 0, &info);
  cudaFree(d_a);
  if (rc == 0 && info != 0)
    rc = xd_internal_fail(-5, "zero pivot in row " + std::to_string(info - 1) + " of the refactorization");
  if (rc != 0) {
    release(r);
    return rc;
  }
  *out = r;
  return 0;
}

int xd_rf_refactor(xd_rf *r, const double *d_vals_a) {
  if (!r || !d_vals_a) return xd_internal_fail(-1, "null refactorization argument");
  cudaSetDevice(r->device);
  int rc = xd_lu_refactor(&r->lu, d_vals_a, 0);
  int info = 0;
  if (rc == 0) rc = xd_lu_info(&r->lu, 0, &info);
  if (rc == 0 && info != 0)
    return xd_internal_fail(-5, "zero pivot in row " + std::to_string(info - 1) + " of the refactorization");
  return rc;
}

int xd_rf_solve(xd_rf *r, double *d_x) {
  if (!r || !d_x) return xd_internal_fail(-1, "null refactorization argument");
  cudaSetDevice(r->device);
  return xd_sptrsv_solve(&r->tri, r->lu.d_mx, d_x, 0);
}

int xd_rf_levels(const xd_rf *r, int *levels_l, int *levels_u) {
  if (!r || !levels_l || !levels_u) return xd_internal_fail(-1, "null refactorization argument");
  *levels_l = r->tri.nlev[0];
  *levels_u = r->tri.nlev[1];
  return 0;
}

int xd_rf_stats(const xd_rf *r, int *nnz_factors, int *elimination_levels, long long *updates) {
  if (!r || !nnz_factors || !elimination_levels || !updates) return xd_internal_fail(-1, "null argument");
  *nnz_factors = r->lu.nnz;
  *elimination_levels = r->lu.nlev;
  *updates = r->lu.npairs;
  return 0;
}

int xd_rf_copy_factors(const xd_rf *r, double *h_vals) {
  if (!r || !h_vals) return xd_internal_fail(-1, "null argument");
  cudaSetDevice(r->device);
  cudaError_t e = cudaMemcpy(h_vals, r->lu.d_mx, sizeof(double) * r->lu.nnz, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cu_fail(e, "xd_rf_copy_factors");
  return 0;
}

}  // extern "C"

namespace {

// The comparison library's handle, set up on first use with the same inputs (algorithms 2 and 3:
// on the 200k-unknown placed netlist they were the fastest of its choices).
int library_handle(xd_rf *r) {
  if (r->h) return 0;
  cusolverStatus_t st;
  if ((st = cusolverRfCreate(&r->h)) != CUSOLVER_STATUS_SUCCESS) return rf_fail(st, "cusolverRfCreate");
  if ((st = cusolverRfSetMatrixFormat(r->h, CUSOLVERRF_MATRIX_FORMAT_CSR, CUSOLVERRF_UNIT_DIAGONAL_STORED_L)) !=
          CUSOLVER_STATUS_SUCCESS ||
      (st = cusolverRfSetResetValuesFastMode(r->h, CUSOLVERRF_RESET_VALUES_FAST_MODE_ON)) != CUSOLVER_STATUS_SUCCESS ||
      (st = cusolverRfSetAlgs(r->h, CUSOLVERRF_FACTORIZATION_ALG2, CUSOLVERRF_TRIANGULAR_SOLVE_ALG3)) !=
          CUSOLVER_STATUS_SUCCESS ||
      (st = cusolverRfSetupHost(r->n, r->nnz_a, r->ra.data(), r->ca.data(), r->va.data(), (int)r->cl.size(),
                                r->rl.data(), r->cl.data(), r->vl.data(), (int)r->cu.size(), r->ru.data(),
                                r->cu.data(), r->vu.data(), r->hp.data(), r->hq.data(), r->h)) !=
          CUSOLVER_STATUS_SUCCESS ||
      (st = cusolverRfAnalyze(r->h)) != CUSOLVER_STATUS_SUCCESS || (st = cusolverRfRefactor(r->h)) != CUSOLVER_STATUS_SUCCESS) {
    cusolverRfDestroy(r->h);
    r->h = nullptr;
    return rf_fail(st, "cusolverRf set-up");
  }
  return 0;
}

}  // namespace

extern "C" {

int xd_rf_refactor_library(xd_rf *r, const double *d_vals_a) {
  if (!r || !d_vals_a) return xd_internal_fail(-1, "null refactorization argument");
  cudaSetDevice(r->device);
  if (int rc = library_handle(r)) return rc;
  cusolverStatus_t st = cusolverRfResetValues(r->n, r->nnz_a, r->d_rowptr, r->d_colind, const_cast<double *>(d_vals_a),
                                              r->d_p, r->d_q, r->h);
  if (st != CUSOLVER_STATUS_SUCCESS) return rf_fail(st, "cusolverRfResetValues");
  st = cusolverRfRefactor(r->h);
  if (st != CUSOLVER_STATUS_SUCCESS) return rf_fail(st, "cusolverRfRefactor");
  return 0;
}

int xd_rf_solve_library(xd_rf *r, double *d_x) {
  if (!r || !d_x) return xd_internal_fail(-1, "null refactorization argument");
  cudaSetDevice(r->device);
  if (int rc = library_handle(r)) return rc;
  cusolverStatus_t st = cusolverRfSolve(r->h, r->d_p, r->d_q, 1, r->d_temp, r->n, d_x, r->n);
  if (st != CUSOLVER_STATUS_SUCCESS) return rf_fail(st, "cusolverRfSolve");
  return 0;
}

int xd_rf_destroy(xd_rf *r) {
  if (!r) return 0;
  cudaSetDevice(r->device);
  release(r);
  return 0;
}

}  // extern "C"
