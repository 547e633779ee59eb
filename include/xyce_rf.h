/* xyce_rf.h — GPU sparse LU refactorization for the transient driver's Newton matrices.
 *
 * Stands in for the reference's direct solve (KLU through Amesos, src/LinearAlgebraServicesPKG/
 * src/N_LAS_AmesosSolver.C:160, 305) where the matrix values are already on the GPU: one host
 * factorization P A Q = L U fixes the pivot order and the fill pattern, every later matrix with
 * A's pattern is refactored and solved on the device. Calls run on the CUDA legacy default stream
 * (the refactorization library has no stream argument); order them after the producer of the
 * values on that stream. Status: 0 ok, < 0 error (xd_last_error()).
 */
#ifndef XYCE_RF_H
#define XYCE_RF_H

#include "xyce_devload.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xd_rf xd_rf;

/* Host inputs, all CSR 0-based, n x n: A's pattern and values, the factors L (unit lower, the
 * unit diagonal stored) and U (upper) of P A Q = L U, and P, Q as arrays: (P A Q)[i][j] =
 * A[P[i]][Q[j]]. The patterns of L and U must cover every position of P A Q's pattern and its
 * fill, including positions whose value is zero in this A (a host factorization that drops
 * numerical zeros must be given placeholders there), because later values may fill them. */
int xd_rf_create(int n, int nnz_a, const int *rowptr_a, const int *colind_a, const double *vals_a, int nnz_l,
                 const int *rowptr_l, const int *colind_l, const double *vals_l, int nnz_u, const int *rowptr_u,
                 const int *colind_u, const double *vals_u, const int *p, const int *q, int cuda_device,
                 xd_rf **out);

/* Refactors with new values of A (device, in A's pattern), keeping the pivot order: the library's
 * own elimination (one thread block over the factors' dependency levels, a warp per row, each
 * entry updated in a fixed order, so the factors do not depend on timing). A zero pivot in that
 * order is an error (< 0, which synchronises the legacy default stream to read); a small one is
 * not detected here, so a caller that cannot bound the growth checks the solution's residual
 * (the transient driver refines and, failing that, makes a new host factorization). */
int xd_rf_refactor(xd_rf *rf, const double *d_vals_a);

/* The same refactorization through cuSOLVER's refactorization library (cusolverRfRefactor), for
 * comparison; it is set up on the first call of this or xd_rf_solve_library, and its factors are
 * separate from xd_rf_refactor's. */
int xd_rf_refactor_library(xd_rf *rf, const double *d_vals_a);

/* Size of the refactorization: entries of the bundled factors L - I + U, dependency levels of
 * the elimination, and multiply-subtract updates per refactorization. */
int xd_rf_stats(const xd_rf *rf, int *nnz_factors, int *elimination_levels, long long *updates);

/* Copies the bundled factors' values (nnz_factors doubles, CSR over P A Q's indices, columns
 * ascending in each row) to host memory. */
int xd_rf_copy_factors(const xd_rf *rf, double *h_vals);

/* Solves A x = b in place: d_x holds b on entry and x on return (device, length n). The forward
 * and back substitutions are the library's own kernels (one thread block walking the factors'
 * dependency levels, deterministic sums), ordered on the legacy default stream. */
int xd_rf_solve(xd_rf *rf, double *d_x);

/* The solve through the refactorization library's own triangular solve, with its factors from
 * xd_rf_refactor_library (for comparison). */
int xd_rf_solve_library(xd_rf *rf, double *d_x);

/* Dependency levels of the lower and upper factors: the number of sequential steps of each
 * substitution, which bounds the solve's latency. */
int xd_rf_levels(const xd_rf *rf, int *levels_l, int *levels_u);

int xd_rf_destroy(xd_rf *rf);

#ifdef __cplusplus
}
#endif

#endif /* XYCE_RF_H */
