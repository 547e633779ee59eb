// Numeric sparse LU refactorization with a fixed pivot order (internal to the library; used by
// the transient driver's refactorization, include/xyce_rf.h).
#pragma once

#include <cuda_runtime.h>

#include <vector>

// P A Q = L U with the pivot order and the fill pattern of one host factorization. The factors
// are kept bundled as one CSR matrix M = L - I + U over P A Q's indices (columns sorted; L's unit
// diagonal implicit, U's diagonal stored), the layout the triangular solves read.
constexpr int kLuNoZeroPivot = 0x7f7f7f7f;  // the zero-pivot report's reset value (every byte 0x7f)

struct XdLu {
  int n = 0, nnz = 0, nnz_a = 0;
  int *d_mp = nullptr, *d_mi = nullptr;  // M's pattern
  double *d_mx = nullptr;                // M's values
  int *d_a2m = nullptr;                  // [nnz_a] position in M of each entry of A
  int *d_diag = nullptr;                 // [n] position of each pivot U(k, k)
  // Pivot levels: pivot k is applied once the pivots that change its row (L(k, k') != 0) or its
  // column (U(k', k) != 0) have been. Per level, the divisions l = M[i][k] / U(k, k) of its pivots'
  // columns, then the updates, grouped by destination (each destination's updates of the level in
  // increasing k, applied by one thread).
  int nlev = 0;
  std::vector<int> lev_div, lev_dst;     // [nlev + 1] ranges of divisions / destinations (host)
  int *d_lev_div = nullptr, *d_lev_dst = nullptr;
  int2 *d_div = nullptr;                 // [ndiv] (position of L(i, k), position of U(k, k))
  // [ndst] with one update (destination M[i][j], position of L(i, k), of U(k, j), of U(k, k)); with
  // more, (destination, first pair in d_pairs, count, -1).
  int4 *d_dst = nullptr;
  int4 *d_pairs = nullptr;               // [npairs - inline ones] (L(i, k), U(k, j), U(k, k), 0) positions
  long long npairs = 0;
  // Launch plan: consecutive light levels run in one single-block launch; a level with more work
  // than one block turns over quickly runs as its own grid-wide launches.
  std::vector<int2> segments;            // (first level, end level); end = first + 1 and heavy: grid-wide
  std::vector<char> segment_grid;
  int *d_info = nullptr;                 // 1 + the first zero pivot's row, or kLuNoZeroPivot
};

// Builds the bundled pattern (L and U of the host factorization, A's permuted pattern, and the
// fill they imply, closed under elimination), the pivot levels and the division and update lists.
// Host CSR inputs; p, q as in (P A Q)[i][j] = A[P[i]][Q[j]]. Returns 0 or < 0 (xd_last_error()).
int xd_lu_init(XdLu *lu, int n, int nnz_a, const int *rowptr_a, const int *colind_a, const int *rowptr_l,
               const int *colind_l, const int *rowptr_u, const int *colind_u, const int *p, const int *q);
void xd_lu_free(XdLu *lu);
// Refactors with A's values d_vals_a (device, A's CSR order): M = P A Q scattered, then
// eliminated in place. Stream-ordered; the zero-pivot report is left in d_info.
int xd_lu_refactor(XdLu *lu, const double *d_vals_a, cudaStream_t st);
// Reads the zero-pivot report (synchronises the stream): 0, or 1 + the first row found.
int xd_lu_info(XdLu *lu, cudaStream_t st, int *info);
