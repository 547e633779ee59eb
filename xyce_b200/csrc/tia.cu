// Time-integration combine step (include/xyce_tia.h): forms the Newton matrix and residual of one
// iterate from the device loads, in one pass over the CSR rows.
//
// Restates N_TIA_OneStep::obtainJacobian / obtainResidual
// (src/TimeIntegrationPKG/src/N_TIA_OneStep.C:272-312, 470-497) and the linear devices' loads
// (N_DEV_Resistor.C:1075-1161, N_DEV_Capacitor.C:1821-2002, N_DEV_Vsrc.C:941-1028), with the
// residual's operations in the reference's order: ((Q - Q_n) / h + f F) + g F_hist, negated, then
// the limiter corrections (1/h) dQdxdVp and f dFdxdVp added.
// One warp per row: lanes take the row's entries with a fixed stride, and the per-row sums of the
// linear devices' F and Q use a fixed shuffle tree, so the results do not vary between runs. Rows
// of more than kLongRowEntries entries (the supply rail's) are cut into chunks first, a block per
// chunk, and their warp adds the chunk sums (tia_long.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <utility>
#include <vector>

#include "../../include/xyce_tia.h"
#include "tia_long.h"

int xd_internal_fail(int code, const std::string &msg);

struct xd_tia {
  int device = 0;
  int n_rows = 0;
  int nnz = 0;
  int *d_rowptr = nullptr;
  int *d_colind = nullptr;
  // Long rows (tia_long.h): the rows, each one's first chunk, the chunks' entry ranges and rows,
  // the chunk sums and diagonal flags.
  int n_lrows = 0, n_lchunks = 0;
  int *d_lrow = nullptr, *d_lfirst = nullptr, *d_lchunk_row = nullptr, *d_ldiag = nullptr;
  int2 *d_lchunk = nullptr;
  double *d_lpart = nullptr;
};

struct xd_slu {
  int device = 0;
  int n = 0;
  double tol = 1e-3;
  int *d_buf = nullptr;  // all index arrays, one allocation
  int off[12] = {};      // offsets in d_buf: rowptr, colind, pos, lptr, lidx, uptr, uidx, cptr, cidx, cpos, cperm
  int nsched = 0;        // entries of lptr .. cidx
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
    double *__restrict__ q_tot, double *__restrict__ f_tot, XdLongRows L) {
  const int row = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= n_rows) return;
  const int beg = rowptr[row], end = rowptr[row + 1];
  const bool tran = c.mode != 0;
  double af = 0.0, aq = 0.0;
  bool has_diag = false;
  // A long row's entries and chunk sums come from long_row_chunk_kernel.
  const bool long_row = end - beg > kLongRowEntries;
  if (long_row) long_row_sums(L, long_row_index(L, row), lane, af, aq, has_diag);
  for (int k = beg + lane; !long_row && k < end; k += 32) {
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
  if (!long_row) {
#pragma unroll
    for (int w = 16; w > 0; w >>= 1) {
      af += __shfl_down_sync(0xffffffffu, af, w);
      aq += __shfl_down_sync(0xffffffffu, aq, w);
    }
    // The shunt goes on rows whose diagonal is in the pattern (the node rows): F and J together.
    has_diag = __any_sync(0xffffffffu, has_diag);
  }
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

// gate (may be null): solve only when *gate is nonzero (a static-pivot solve before it failed).
__global__ void __launch_bounds__(kDenseThreads) dense_factor_solve_kernel(
    int n, const int *__restrict__ rowptr, const int *__restrict__ colind, const double *__restrict__ vals,
    const double *__restrict__ rhs, double *__restrict__ lu, int *__restrict__ piv, double *__restrict__ x,
    int *info, const int *gate) {
  if (gate && *gate == 0) return;
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

// Newton's bookkeeping between a solve and the next load, one block: x += dx; the update weights
// (when refreshed) rel * max(|x_ref|, |x|) + abs; norms[0] = sqrt(mean((dx / w)^2)), the weighted
// RMS norm of the update (N_NLS_DampedNewton.C's convergence test, :325-350, 1792-1830). Then,
// after the load, norms[1] = max |rhs| (not finite if any entry is not) and norms[2] = *flag.
// Sums and maxima use a fixed reduction tree: the same inputs give the same norms.
constexpr int kNormThreads = 1024;

__device__ __forceinline__ double block_sum(double v, double *red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
  if (warp == 0) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  }
  return v;
}

__global__ void __launch_bounds__(kNormThreads) newton_update_kernel(int n, double *__restrict__ x,
                                                                     const double *__restrict__ dx,
                                                                     const double *__restrict__ xref,
                                                                     double *__restrict__ w, double rel, double abs_,
                                                                     int update_w, double *__restrict__ norms) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += kNormThreads) {
    const double xi = x[i] + dx[i];
    x[i] = xi;
    double wi;
    if (update_w) {
      wi = rel * fmax(fabs(xref[i]), fabs(xi)) + abs_;
      w[i] = wi;
    } else {
      wi = w[i];
    }
    const double q = dx[i] / wi;
    s += q * q;
  }
  s = block_sum(s, red);
  if (threadIdx.x == 0) norms[0] = sqrt(s / (double)n);
}

__global__ void __launch_bounds__(kNormThreads) residual_norm_kernel(int n, const double *__restrict__ rhs,
                                                                     const int *__restrict__ flag,
                                                                     double *__restrict__ norms) {
  __shared__ double red[32];
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += kNormThreads) {
    const double a = fabs(rhs[i]);
    if (!isfinite(a)) bad = 1;
    m = fmax(m, a);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
  if (lane == 0) red[warp] = m;
  __syncthreads();
  if (warp == 0) {
    m = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
    if (lane == 0) {
      norms[1] = bad ? __longlong_as_double(0x7ff8000000000000LL) : m;
      norms[2] = flag ? (double)*flag : 0.0;
    }
  }
}

// Static-pivot refactorization of a small system (n <= XD_DENSE_MAX_N). The orders and the fill
// pattern come from one host factorization (xd_slu_create): a minimum-degree order of A + A^T
// applied to rows and columns (a supply node's dense row and column go last instead of filling the
// whole matrix: the ring oscillator's LU has 704 entries instead of 103^2), then row pivoting that
// keeps the diagonal unless it is below 0.1 of its column's largest entry; each
// Newton matrix is then eliminated in that order over the pattern alone: step k scales the
// multipliers of the rows that have an entry in column k and updates only the (row, column) pairs
// of the pattern, the right-hand side carried along as column n. A pivot smaller than tol times an
// entry below it (the threshold test of circuit solvers such as KLU) stops the solve with info =
// k + 1, and the pivoting kernel redoes it (xd_tia_dense_solve_fallback). One warp, shared memory,
// __syncwarp between steps: a few hundred cycles a step where the pivot search costs thousands.
struct SluArgs {
  int n;
  double tol;
  const int *rowptr, *colind;  // the system's CSR pattern
  const int *pos;              // [n] position of each row in the pivot order
  const int *lptr, *lidx;      // per step k: rows below k with an entry in column k
  const int *uptr, *uidx;      // per step k: columns right of k with an entry in row k
  const int *cptr, *cidx;      // per column k: rows above k with an entry in column k (back substitution)
  const int *cpos;             // [n] position of each column (unknown) in the elimination order
  const int *cperm;            // [n] the unknown at each column position
  int nsched;                  // entries of the six schedule arrays (lptr .. cidx) copied to shared memory
                               // (0: too many beside the matrix, read from global memory)
  const int *sched;            // lptr, lidx, uptr, uidx, cptr, cidx back to back
};

__global__ void __launch_bounds__(32) slu_kernel(SluArgs a, const double *__restrict__ vals,
                                                 const double *__restrict__ rhs, double *__restrict__ lu,
                                                 double *__restrict__ x, int *info) {
  extern __shared__ double M[];
  __shared__ double sinv[XD_DENSE_MAX_N];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x, n = a.n, lda = n + 1;
  // The schedule moves to shared memory first (each launch starts with cold caches; read from
  // global memory, every step would wait on a chain of dependent loads).
  int *ss = reinterpret_cast<int *>(M + (size_t)n * lda);
  for (int idx = lane; idx < a.nsched; idx += 32) ss[idx] = a.sched[idx];
  for (int idx = lane; idx < n * lda; idx += 32) M[idx] = 0.0;
  __syncwarp();
  if (a.nsched > 0) {
    a.lidx = ss + (a.lidx - a.sched);
    a.uptr = ss + (a.uptr - a.sched);
    a.uidx = ss + (a.uidx - a.sched);
    a.cptr = ss + (a.cptr - a.sched);
    a.cidx = ss + (a.cidx - a.sched);
    a.lptr = ss;
  }
  for (int r = lane; r < n; r += 32) {
    double *row = M + a.pos[r] * lda;
    for (int k = a.rowptr[r]; k < a.rowptr[r + 1]; ++k) row[a.cpos[a.colind[k]]] = vals[k];
    row[n] = rhs[r];
  }
  __syncwarp();
  for (int k = 0; k < n; ++k) {
    const double pv = M[k * lda + k];
    const int lb = a.lptr[k], le = a.lptr[k + 1], ub = a.uptr[k], nu = a.uptr[k + 1] - ub + 1;
    bool ok = fabs(pv) > 0.0;
    for (int t = lb + lane; t < le; t += 32) ok = ok && (fabs(M[a.lidx[t] * lda + k]) * a.tol <= fabs(pv));
    if (!__all_sync(full, ok)) {
      if (lane == 0) *info = k + 1;
      return;
    }
    const double inv = 1.0 / pv;
    if (lane == 0) sinv[k] = inv;
    for (int t = lb + lane; t < le; t += 32) M[a.lidx[t] * lda + k] *= inv;
    __syncwarp();
    const int tot = (le - lb) * nu;
    for (int t = lane; t < tot; t += 32) {
      const int q = t / nu, c = t - q * nu;
      const int i = a.lidx[lb + q], j = c < nu - 1 ? a.uidx[ub + c] : n;
      M[i * lda + j] = M[i * lda + j] - M[i * lda + k] * M[k * lda + j];
    }
    __syncwarp();
  }
  // Back substitution on U, column by column; column n becomes x.
  for (int k = n - 1; k >= 0; --k) {
    if (lane == 0) M[k * lda + n] = M[k * lda + n] * sinv[k];
    __syncwarp();
    const double xk = M[k * lda + n];
    for (int t = a.cptr[k] + lane; t < a.cptr[k + 1]; t += 32) {
      const int i = a.cidx[t];
      M[i * lda + n] = M[i * lda + n] - M[i * lda + k] * xk;
    }
    __syncwarp();
  }
  for (int j = lane; j < n; j += 32) x[a.cperm[j]] = M[j * lda + n];
  if (lu) {
    for (int idx = lane; idx < n * n; idx += 32) {
      const int r = idx / n, c = idx - r * n;
      lu[idx] = M[r * lda + c];
    }
  }
  if (lane == 0) *info = 0;
}

// Solve with factors kept from slu_kernel (in its row and column orders): forward substitution
// over the unit lower factor's pattern, back substitution over the upper one's, then the
// unknowns back to their own order. One warp.
__global__ void __launch_bounds__(32) slu_resolve_kernel(SluArgs a, const double *__restrict__ lu,
                                                         const double *__restrict__ rhs, double *__restrict__ x) {
  __shared__ double y[XD_DENSE_MAX_N];
  const int lane = threadIdx.x, n = a.n;
  for (int r = lane; r < n; r += 32) y[a.pos[r]] = rhs[r];
  __syncwarp();
  for (int k = 0; k < n; ++k) {
    const double yk = y[k];
    for (int t = a.lptr[k] + lane; t < a.lptr[k + 1]; t += 32) {
      const int i = a.lidx[t];
      y[i] = y[i] - lu[(size_t)i * n + k] * yk;
    }
    __syncwarp();
  }
  for (int k = n - 1; k >= 0; --k) {
    if (lane == 0) y[k] = y[k] * (1.0 / lu[(size_t)k * n + k]);
    __syncwarp();
    const double xk = y[k];
    for (int t = a.cptr[k] + lane; t < a.cptr[k + 1]; t += 32) {
      const int i = a.cidx[t];
      y[i] = y[i] - lu[(size_t)i * n + k] * xk;
    }
    __syncwarp();
  }
  for (int j = lane; j < n; j += 32) x[a.cperm[j]] = y[j];
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

// Independent voltage sources' values at an analysis time, on the device (PWLinData::updateSource,
// src/DeviceModelPKG/Core/src/N_DEV_SourceData.C:1371-1490, restated with its own arithmetic, so the
// values equal the reference's bit for bit; Vsrc::Master::updateState picks the transient value in a
// transient or its operating point and the DC value otherwise, N_DEV_Vsrc.C:941-960).
struct xd_pwl {
  int device = 0, n = 0;
  int *d_row = nullptr;     // b-vector row of each source
  int *d_first = nullptr;   // [n + 1] first (t, v) pair of each source; no pairs = DC only
  double *d_tv = nullptr;   // concatenated (t, v) pairs
  double *d_par = nullptr;  // per source: DC value, delay TD, repeat time (negative: no repeat)
};

namespace {

__global__ void pwl_eval_kernel(int n, const int *__restrict__ row, const int *__restrict__ first,
                                const double *__restrict__ tv, const double *__restrict__ par, double t, int transient,
                                double *__restrict__ b) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int f = first[k], num = first[k + 1] - f;
  const double *T = tv + 2 * (size_t)f;  // T[2 i] = time i, T[2 i + 1] = value i
  const double dc = par[3 * k], td = par[3 * k + 1], rep = par[3 * k + 2];
  if (!transient || num == 0) {
    b[row[k]] = dc;
    return;
  }
  double time = t, time1, time2, v1, v2, value;
  if (time >= td) {
    time -= td;
    const double tlast = T[2 * (num - 1)];
    if (time <= tlast) {
      int loc = num - 1;  // time == the last time: the segment that ends there
      for (int i = 0; i < num; ++i)
        if (time < T[2 * i]) {
          loc = i;
          break;
        }
      if (loc == 0) {
        time1 = 0.0;
        v1 = 0.0;
      } else {
        time1 = T[2 * (loc - 1)];
        v1 = T[2 * (loc - 1) + 1];
      }
      time2 = T[2 * loc];
      v2 = T[2 * loc + 1];
    } else if (rep < 0.0) {
      time1 = 0.0;
      time2 = 1.0;
      v1 = v2 = T[2 * (num - 1) + 1];
    } else {
      const double looptime = tlast - rep;
      time -= tlast;
      time -= looptime * floor(time / looptime);
      time += rep;
      int loc = num - 1;
      for (int i = 0; i < num; ++i)
        if (time < T[2 * i]) {
          loc = i;
          break;
        }
      if (time == rep) {
        time1 = 0.0;
        time2 = 1.0;
        v1 = v2 = T[2 * (num - 1) + 1];
      } else {
        if (loc == 0) {
          time1 = rep;
          v1 = T[2 * (num - 1) + 1];
        } else {
          time1 = T[2 * (loc - 1)];
          v1 = T[2 * (loc - 1) + 1];
        }
        time2 = T[2 * loc];
        v2 = T[2 * loc + 1];
      }
    }
    if (time1 == time2) {
      value = v2;
    } else {
      const double length = time2 - time1;
      value = (time2 - time) * v1 / length;
      value += (-time1 + time) * v2 / length;
    }
  } else {
    value = 0.0;
  }
  b[row[k]] = value;
}

// One chunk of a long row (tia_long.h) per block: with JAC, the chunk's Newton matrix entries as
// tia_combine_kernel forms them; always the chunk's linear-device F and Q sums (threads take
// entries with a fixed stride, then a fixed tree) and whether it holds the row's diagonal (with a
// gmin shunt on).
template <bool JAC>
__global__ void __launch_bounds__(kLongBlock) long_row_chunk_kernel(
    int n_chunks, const int2 *__restrict__ chunk, const int *__restrict__ chunk_row, const int *__restrict__ colind,
    xd_tia_coef c, const double *__restrict__ x, const double *__restrict__ dfdx, const double *__restrict__ dqdx,
    const double *__restrict__ lin_f, const double *__restrict__ lin_q, double *__restrict__ jac,
    double *__restrict__ part, int *__restrict__ diag) {
  __shared__ double red[2][kLongBlock];
  __shared__ int hd;
  const int ch = blockIdx.x, tid = threadIdx.x;
  const int2 rg = chunk[ch];
  const int row = chunk_row[ch];
  const bool tran = c.mode != 0;
  if (tid == 0) hd = 0;
  __syncthreads();
  double af = 0.0, aq = 0.0;
  bool has = false;
  for (int k = rg.x + tid; k < rg.y; k += kLongBlock) {
    const int col = colind[k];
    double jf = JAC ? dfdx[k] : 0.0;
    if (lin_f) {
      const double g = lin_f[k];
      if (JAC) jf += g;
      af += g * x[col];
    }
    if (c.gshunt != 0.0 && col == row) {
      if (JAC) jf += c.gshunt;
      has = true;
    }
    if (tran) {
      double jq = JAC ? dqdx[k] : 0.0;
      if (lin_q) {
        const double cq = lin_q[k];
        if (JAC) jq += cq;
        aq += cq * x[col];
      }
      if (JAC) jac[k] = c.qscale * jq + c.fscale * jf;
    } else if (JAC) {
      jac[k] = jf;
    }
  }
  if (has) hd = 1;
  red[0][tid] = af;
  red[1][tid] = aq;
  __syncthreads();
  for (int w = kLongBlock / 2; w > 0; w >>= 1) {
    if (tid < w) {
      red[0][tid] += red[0][tid + w];
      red[1][tid] += red[1][tid + w];
    }
    __syncthreads();
  }
  if (tid == 0) {
    part[ch] = red[0][0];
    part[n_chunks + ch] = red[1][0];
    diag[ch] = hd;
  }
}

void free_long_rows(xd_tia *t) {
  cudaFree(t->d_lrow);
  cudaFree(t->d_lfirst);
  cudaFree(t->d_lchunk_row);
  cudaFree(t->d_ldiag);
  cudaFree(t->d_lchunk);
  cudaFree(t->d_lpart);
  t->d_lrow = t->d_lfirst = t->d_lchunk_row = t->d_ldiag = nullptr;
  t->d_lchunk = nullptr;
  t->d_lpart = nullptr;
  t->n_lrows = t->n_lchunks = 0;
}

// The long rows of the pattern and their chunks (kLongChunk consecutive entries, the last one of a
// row shorter), uploaded.
cudaError_t setup_long_rows(xd_tia *t, const int *rowptr) {
  std::vector<int> lrow, lfirst(1, 0), crow;
  std::vector<int2> chunk;
  for (int r = 0; r < t->n_rows; ++r) {
    const int b = rowptr[r], e = rowptr[r + 1];
    if (e - b <= kLongRowEntries) continue;
    lrow.push_back(r);
    for (int k = b; k < e; k += kLongChunk) {
      chunk.push_back(make_int2(k, std::min(e, k + kLongChunk)));
      crow.push_back(r);
    }
    lfirst.push_back((int)chunk.size());
  }
  if (lrow.empty()) return cudaSuccess;
  const size_t nr = lrow.size(), nc = chunk.size();
  cudaError_t e;
  if ((e = cudaMalloc(&t->d_lrow, nr * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&t->d_lfirst, (nr + 1) * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&t->d_lchunk_row, nc * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&t->d_ldiag, nc * sizeof(int))) != cudaSuccess ||
      (e = cudaMalloc(&t->d_lchunk, nc * sizeof(int2))) != cudaSuccess ||
      (e = cudaMalloc(&t->d_lpart, 2 * nc * sizeof(double))) != cudaSuccess ||
      (e = cudaMemcpy(t->d_lrow, lrow.data(), nr * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(t->d_lfirst, lfirst.data(), (nr + 1) * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(t->d_lchunk_row, crow.data(), nc * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(t->d_lchunk, chunk.data(), nc * sizeof(int2), cudaMemcpyHostToDevice)) != cudaSuccess)
    return e;
  t->n_lrows = (int)nr;
  t->n_lchunks = (int)nc;
  return cudaSuccess;
}

}  // namespace

int xd_tia_internal_long_rows(const xd_tia *t, XdLongRows *out) {
  if (!t || !out) return xd_internal_fail(-1, "null combine object");
  out->n_rows = t->n_lrows;
  out->n_chunks = t->n_lchunks;
  out->row = t->d_lrow;
  out->first = t->d_lfirst;
  out->part = t->d_lpart;
  out->diag = t->d_ldiag;
  return 0;
}

int xd_tia_internal_long_chunks(xd_tia *t, const xd_tia_coef *c, const double *x, const double *dfdx,
                                const double *dqdx, const double *lin_f, const double *lin_q, double *jac,
                                cudaStream_t st) {
  if (!t || !c) return xd_internal_fail(-1, "null argument");
  if (t->n_lchunks == 0) return 0;
  if (jac)
    long_row_chunk_kernel<true><<<t->n_lchunks, kLongBlock, 0, st>>>(t->n_lchunks, t->d_lchunk, t->d_lchunk_row,
                                                                     t->d_colind, *c, x, dfdx, dqdx, lin_f, lin_q,
                                                                     jac, t->d_lpart, t->d_ldiag);
  else
    long_row_chunk_kernel<false><<<t->n_lchunks, kLongBlock, 0, st>>>(t->n_lchunks, t->d_lchunk, t->d_lchunk_row,
                                                                      t->d_colind, *c, x, dfdx, dqdx, lin_f, lin_q,
                                                                      jac, t->d_lpart, t->d_ldiag);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "long_row_chunk_kernel launch");
  return 0;
}

// The pattern a combine object was created on (for the fused load-and-combine in devload.cu).
int xd_tia_internal_pattern(const xd_tia *t, int *device, int *n_rows, int *nnz, const int **rowptr,
                            const int **colind) {
  if (!t) return xd_internal_fail(-1, "null combine object");
  *device = t->device;
  *n_rows = t->n_rows;
  *nnz = t->nnz;
  *rowptr = t->d_rowptr;
  *colind = t->d_colind;
  return 0;
}

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
  if ((e = setup_long_rows(t, pat->rowptr)) != cudaSuccess) {
    free_long_rows(t);
    cudaFree(t->d_rowptr);
    cudaFree(t->d_colind);
    delete t;
    return cuda_err(e, "xd_tia_create long rows");
  }
  if (pat->n_rows <= XD_DENSE_MAX_N && dense_smem_bytes(pat->n_rows) > 48 * 1024) {
    e = cudaFuncSetAttribute(dense_factor_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)dense_smem_bytes(pat->n_rows));
    if (e != cudaSuccess) {
      free_long_rows(t);
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
  free_long_rows(t);
  cudaFree(t->d_rowptr);
  cudaFree(t->d_colind);
  delete t;
  return 0;
}

int xd_pwl_create(int n_src, const int *row, const int *n_pairs, const double *tv, const double *dc, const double *td,
                  const double *repeat, int cuda_device, xd_pwl **out) {
  if (!out || n_src < 0 || (n_src > 0 && (!row || !n_pairs || !dc))) return xd_internal_fail(-1, "null argument");
  *out = nullptr;
  std::vector<int> first(n_src + 1, 0);
  std::vector<double> par(3 * (size_t)std::max(1, n_src), 0.0);
  for (int k = 0; k < n_src; ++k) {
    if (n_pairs[k] < 0) return xd_internal_fail(-1, "negative PWL pair count");
    first[k + 1] = first[k] + n_pairs[k];
    par[3 * k] = dc[k];
    par[3 * k + 1] = td ? td[k] : 0.0;
    par[3 * k + 2] = repeat ? repeat[k] : -1.0;
  }
  const size_t npairs = (size_t)first[n_src];
  if (npairs > 0 && !tv) return xd_internal_fail(-1, "null PWL pairs");
  for (int k = 0; k < n_src; ++k) {
    // The reference's checks (PWLinData, N_DEV_SourceData.C:1314-1317).
    if (n_pairs[k] > 0 && par[3 * k + 2] >= 0.0 && par[3 * k + 2] >= tv[2 * (size_t)(first[k + 1] - 1)])
      return xd_internal_fail(-1, "PWL source's repeat value (R) must be >= 0 and < last value in Time-Voltage list");
  }
  cudaError_t ce = cudaSetDevice(cuda_device);
  if (ce != cudaSuccess) return cuda_err(ce, "cudaSetDevice");
  xd_pwl *p = new xd_pwl();
  p->device = cuda_device;
  p->n = n_src;
  if ((ce = cudaMalloc(&p->d_row, std::max(1, n_src) * sizeof(int))) != cudaSuccess ||
      (ce = cudaMalloc(&p->d_first, (n_src + 1) * sizeof(int))) != cudaSuccess ||
      (ce = cudaMalloc(&p->d_tv, std::max<size_t>(1, 2 * npairs) * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&p->d_par, par.size() * sizeof(double))) != cudaSuccess ||
      (n_src > 0 && (ce = cudaMemcpy(p->d_row, row, n_src * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (ce = cudaMemcpy(p->d_first, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (npairs > 0 && (ce = cudaMemcpy(p->d_tv, tv, 2 * npairs * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess) ||
      (ce = cudaMemcpy(p->d_par, par.data(), par.size() * sizeof(double), cudaMemcpyHostToDevice)) != cudaSuccess) {
    xd_pwl_destroy(p);
    return cuda_err(ce, "xd_pwl_create");
  }
  *out = p;
  return 0;
}

int xd_pwl_destroy(xd_pwl *p) {
  if (!p) return 0;
  Guard g(p->device);
  cudaFree(p->d_row);
  cudaFree(p->d_first);
  cudaFree(p->d_tv);
  cudaFree(p->d_par);
  delete p;
  return 0;
}

int xd_pwl_eval(xd_pwl *p, double t, int transient, double *d_b, void *stream) {
  if (!p || !d_b) return xd_internal_fail(-1, "null argument");
  if (p->n == 0) return 0;
  Guard g(p->device);
  pwl_eval_kernel<<<(p->n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(p->n, p->d_row, p->d_first, p->d_tv, p->d_par,
                                                                       t, transient, d_b);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "pwl_eval_kernel launch");
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
  int rc = xd_tia_internal_long_chunks(t, coef, d_x, d_dfdx, d_dqdx, d_lin_dfdx, d_lin_dqdx, d_jac,
                                       (cudaStream_t)stream);
  if (rc) return rc;
  XdLongRows L;
  xd_tia_internal_long_rows(t, &L);
  const int blocks = (t->n_rows + kWarpsPerBlock - 1) / kWarpsPerBlock;
  tia_combine_kernel<<<blocks, 32 * kWarpsPerBlock, 0, (cudaStream_t)stream>>>(
      t->n_rows, t->d_rowptr, t->d_colind, *coef, d_x, d_dfdx, d_dqdx, d_lin_dfdx, d_lin_dqdx, d_f, d_q, d_dfdxdvp,
      d_dqdxdvp, d_b, d_qn0, d_fhist, d_jac, d_rhs, d_q_tot, d_f_tot, L);
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
      t->n_rows, t->d_rowptr, t->d_colind, d_jac, d_rhs, d_lu, d_piv, d_x, d_info, nullptr);
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

int xd_tia_dense_solve_fallback(xd_tia *t, const double *d_jac, const double *d_rhs, double *d_lu, int *d_piv,
                                double *d_x, int *d_info, void *stream) {
  if (!t || !d_info) return xd_internal_fail(-1, "null argument");
  if (t->n_rows == 0) return 0;
  if (t->n_rows > XD_DENSE_MAX_N)
    return xd_internal_fail(-1, "the dense solve takes at most " + std::to_string(XD_DENSE_MAX_N) + " unknowns");
  if (!d_jac || !d_rhs || !d_x) return xd_internal_fail(-1, "null device buffer");
  Guard g(t->device);
  dense_factor_solve_kernel<<<1, kDenseThreads, dense_smem_bytes(t->n_rows), (cudaStream_t)stream>>>(
      t->n_rows, t->d_rowptr, t->d_colind, d_jac, d_rhs, d_lu, d_piv, d_x, d_info, d_info);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "dense_factor_solve_kernel launch");
  return 0;
}

int xd_tia_newton_update(xd_tia *t, double *d_x, const double *d_dx, const double *d_xref, double *d_w, double rel_tol,
                         double abs_tol, int update_weights, double *d_norms, void *stream) {
  if (!t || !d_x || !d_dx || !d_w || !d_norms || (update_weights && !d_xref)) return xd_internal_fail(-1, "null argument");
  if (t->n_rows == 0) return 0;
  Guard g(t->device);
  newton_update_kernel<<<1, kNormThreads, 0, (cudaStream_t)stream>>>(t->n_rows, d_x, d_dx, d_xref, d_w, rel_tol, abs_tol,
                                                                     update_weights, d_norms);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "newton_update_kernel launch");
  return 0;
}

int xd_tia_residual_norm(xd_tia *t, const double *d_rhs, const int *d_flag, double *d_norms, void *stream) {
  if (!t || !d_rhs || !d_norms) return xd_internal_fail(-1, "null argument");
  if (t->n_rows == 0) return 0;
  Guard g(t->device);
  residual_norm_kernel<<<1, kNormThreads, 0, (cudaStream_t)stream>>>(t->n_rows, d_rhs, d_flag, d_norms);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "residual_norm_kernel launch");
  return 0;
}

int xd_slu_create(int n, const int *rowptr, const int *colind, const double *vals, double tol, int cuda_device,
                  xd_slu **out) {
  if (!out || !rowptr || n <= 0 || n > XD_DENSE_MAX_N || !(tol > 0.0 && tol <= 1.0))
    return xd_internal_fail(-1, "bad static-pivot solve arguments (n must be 1.." + std::to_string(XD_DENSE_MAX_N) +
                                    ", 0 < tol <= 1)");
  *out = nullptr;
  const int nnz = rowptr[n];
  if (rowptr[0] != 0 || nnz < 0 || (nnz > 0 && (!colind || !vals))) return xd_internal_fail(-1, "bad CSR pattern");
  for (int r = 0; r < n; ++r)
    if (rowptr[r + 1] < rowptr[r]) return xd_internal_fail(-1, "bad CSR pattern");
  for (int k = 0; k < nnz; ++k)
    if (colind[k] < 0 || colind[k] >= n) return xd_internal_fail(-1, "bad CSR pattern");
  // Minimum-degree order of A + A^T (greedy; ties to the lowest index), applied to rows and
  // columns: cperm[j] = the unknown eliminated j-th.
  std::vector<char> G((size_t)n * n, 0), alive(n, 1);
  for (int r = 0; r < n; ++r)
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k)
      if (colind[k] != r) G[(size_t)r * n + colind[k]] = G[(size_t)colind[k] * n + r] = 1;
  std::vector<int> cperm(n), cpos(n);
  for (int step = 0; step < n; ++step) {
    int v = -1, best = n + 1;
    for (int i = 0; i < n; ++i) {
      if (!alive[i]) continue;
      int d = 0;
      for (int j = 0; j < n; ++j) d += (alive[j] && G[(size_t)i * n + j]) ? 1 : 0;
      if (d < best) {
        best = d;
        v = i;
      }
    }
    cperm[step] = v;
    alive[v] = 0;
    std::vector<int> nb;
    for (int j = 0; j < n; ++j)
      if (alive[j] && G[(size_t)v * n + j]) nb.push_back(j);
    for (int p : nb)
      for (int q : nb)
        if (p != q) G[(size_t)p * n + q] = 1;
  }
  for (int j = 0; j < n; ++j) cpos[cperm[j]] = j;
  // Host factorization in that order, tracking the pattern: row pivoting that keeps the diagonal
  // unless it is below 0.1 of the column's largest entry (then the first largest), as circuit
  // solvers pivot; the row order and the fill of every later matrix with this pattern.
  std::vector<double> A((size_t)n * n, 0.0);
  std::vector<char> S((size_t)n * n, 0);
  for (int r = 0; r < n; ++r)
    for (int k = rowptr[r]; k < rowptr[r + 1]; ++k) {
      const size_t at = (size_t)cpos[r] * n + cpos[colind[k]];
      A[at] = vals[k];
      S[at] = 1;
    }
  std::vector<int> rowof(n);  // original row at each row position
  for (int i = 0; i < n; ++i) rowof[i] = cperm[i];
  for (int k = 0; k < n; ++k) {
    int p = k;
    double best = std::fabs(A[(size_t)k * n + k]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[(size_t)i * n + k]) > best) {
        best = std::fabs(A[(size_t)i * n + k]);
        p = i;
      }
    if (!(best > 0.0)) return xd_internal_fail(-2, "the matrix for the static pivot order is singular");
    if (std::fabs(A[(size_t)k * n + k]) >= 0.1 * best) p = k;
    if (p != k) {
      for (int j = 0; j < n; ++j) {
        std::swap(A[(size_t)k * n + j], A[(size_t)p * n + j]);
        std::swap(S[(size_t)k * n + j], S[(size_t)p * n + j]);
      }
      std::swap(rowof[k], rowof[p]);
    }
    for (int i = k + 1; i < n; ++i) {
      if (!S[(size_t)i * n + k]) continue;
      const double l = A[(size_t)i * n + k] / A[(size_t)k * n + k];
      for (int j = k + 1; j < n; ++j)
        if (S[(size_t)k * n + j]) {
          A[(size_t)i * n + j] -= l * A[(size_t)k * n + j];
          S[(size_t)i * n + j] = 1;
        }
    }
  }
  std::vector<int> pos(n), lptr(n + 1, 0), lidx, uptr(n + 1, 0), uidx, cptr(n + 1, 0), cidx;
  for (int i = 0; i < n; ++i) pos[rowof[i]] = i;
  for (int k = 0; k < n; ++k) {
    for (int i = k + 1; i < n; ++i)
      if (S[(size_t)i * n + k]) lidx.push_back(i);
    lptr[k + 1] = (int)lidx.size();
    for (int j = k + 1; j < n; ++j)
      if (S[(size_t)k * n + j]) uidx.push_back(j);
    uptr[k + 1] = (int)uidx.size();
    for (int i = 0; i < k; ++i)
      if (S[(size_t)i * n + k]) cidx.push_back(i);
    cptr[k + 1] = (int)cidx.size();
  }
  const std::vector<int> *parts[11] = {nullptr, nullptr, &pos, &lptr, &lidx, &uptr, &uidx, &cptr, &cidx, &cpos, &cperm};
  std::vector<int> rp(rowptr, rowptr + n + 1), ci(colind, colind + nnz);
  parts[0] = &rp;
  parts[1] = &ci;
  // Parts 3..8 (the schedule) are contiguous in that order; the kernel copies them to shared
  // memory behind the matrix when they fit there.
  size_t nsched = 0;
  for (int q = 3; q <= 8; ++q) nsched += parts[q]->size();
  if (dense_smem_bytes(n) + sizeof(int) * nsched + sizeof(double) * XD_DENSE_MAX_N > 227 * 1024) nsched = 0;
  xd_slu *h = new xd_slu();
  h->device = cuda_device;
  h->n = n;
  h->tol = tol;
  h->nsched = (int)nsched;
  std::vector<int> all;
  for (int q = 0; q < 11; ++q) {
    h->off[q] = (int)all.size();
    all.insert(all.end(), parts[q]->begin(), parts[q]->end());
  }
  Guard g(cuda_device);
  cudaError_t e;
  if ((e = cudaMalloc(&h->d_buf, sizeof(int) * std::max<size_t>(1, all.size()))) != cudaSuccess ||
      (e = cudaMemcpy(h->d_buf, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice)) != cudaSuccess ||
      (dense_smem_bytes(n) + sizeof(int) * nsched > 48 * 1024 &&
       (e = cudaFuncSetAttribute(slu_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(dense_smem_bytes(n) + sizeof(int) * nsched))) != cudaSuccess)) {
    cudaFree(h->d_buf);
    delete h;
    return cuda_err(e, "xd_slu_create");
  }
  *out = h;
  return 0;
}

static SluArgs slu_args(const xd_slu *s) {
  const int *b = s->d_buf;
  return SluArgs{s->n,           s->tol,           b + s->off[0], b + s->off[1], b + s->off[2], b + s->off[3],
                 b + s->off[4], b + s->off[5],    b + s->off[6], b + s->off[7], b + s->off[8], b + s->off[9],
                 b + s->off[10], s->nsched,        b + s->off[3]};
}

int xd_slu_solve(xd_slu *s, const double *d_vals, const double *d_rhs, double *d_lu, double *d_x, int *d_info,
                 void *stream) {
  if (!s || !d_vals || !d_rhs || !d_x || !d_info) return xd_internal_fail(-1, "null argument");
  Guard g(s->device);
  slu_kernel<<<1, 32, dense_smem_bytes(s->n) + sizeof(int) * s->nsched, (cudaStream_t)stream>>>(
      slu_args(s), d_vals, d_rhs, d_lu, d_x, d_info);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "slu_kernel launch");
  return 0;
}

int xd_slu_resolve(xd_slu *s, const double *d_lu, const double *d_rhs, double *d_x, void *stream) {
  if (!s || !d_lu || !d_rhs || !d_x) return xd_internal_fail(-1, "null argument");
  Guard g(s->device);
  slu_resolve_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(slu_args(s), d_lu, d_rhs, d_x);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_err(e, "slu_resolve_kernel launch");
  return 0;
}

int xd_slu_destroy(xd_slu *s) {
  if (!s) return 0;
  Guard g(s->device);
  cudaFree(s->d_buf);
  delete s;
  return 0;
}

}  // extern "C"
