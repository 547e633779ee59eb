// Long rows of the combine step's Newton matrix: rows with more than kLongRowEntries entries (the
// supply rail's row couples to every transistor that the rail feeds: ~0.9 entries per MOSFET).
// One warp walking such a row with a chain of dependent loads took ~13 ms per combine at 1M
// MOSFETs, so their entries are cut into chunks of kLongChunk consecutive entries, one block per
// chunk (tia.cu, long_row_chunk_kernel): the block forms the chunk's Newton matrix entries (the
// separate combine only) and sums the chunk's linear-device currents and charges with a fixed
// strided split and a fixed tree. The row's warp then adds the chunk sums in a fixed lane-strided
// order and shuffle tree (long_row_sums below). The separate combine (tia_combine_kernel) and the
// fused load-and-combine (fused_row_kernel) both take long rows this way, so the two stay bitwise
// equal, and every sum is reduced in an order fixed by the pattern.
#pragma once

#include <cuda_runtime.h>

#include "../../include/xyce_tia.h"

constexpr int kLongRowEntries = 1024;  // rows with more entries take the chunked path
constexpr int kLongChunk = 1024;       // entries per chunk
constexpr int kLongBlock = 256;        // threads of a chunk's block

struct XdLongRows {
  int n_rows = 0;                 // long rows
  int n_chunks = 0;
  const int *row = nullptr;       // [n_rows] the long rows, ascending
  const int *first = nullptr;     // [n_rows + 1] first chunk of each long row
  const double *part = nullptr;   // [2][n_chunks] the chunks' linear F and Q sums
  const int *diag = nullptr;      // [n_chunks] 1 where the chunk holds its row's diagonal (separate combine)
};

// The long-row index of row r (a row with more than kLongRowEntries entries), by bisection.
__device__ __forceinline__ int long_row_index(const XdLongRows &L, int r) {
  int lo = 0, hi = L.n_rows - 1;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (L.row[mid] < r)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Warp-wide: the long row j's linear F and Q sums from its chunks' sums (every lane gets lane 0's
// partial result only after the tree; lane 0 holds the row's totals), and whether any chunk held
// the row's diagonal.
__device__ __forceinline__ void long_row_sums(const XdLongRows &L, int j, int lane, double &af, double &aq,
                                              bool &has_diag) {
  af = 0.0;
  aq = 0.0;
  bool hd = false;
  for (int c = L.first[j] + lane; c < L.first[j + 1]; c += 32) {
    af += L.part[c];
    aq += L.part[L.n_chunks + c];
    if (L.diag[c]) hd = true;
  }
#pragma unroll
  for (int w = 16; w > 0; w >>= 1) {
    af += __shfl_down_sync(0xffffffffu, af, w);
    aq += __shfl_down_sync(0xffffffffu, aq, w);
  }
  has_diag = __any_sync(0xffffffffu, hd);
}

// The combine object's long rows (tia.cu).
int xd_tia_internal_long_rows(const xd_tia *t, XdLongRows *out);
// Launches the chunk kernel on stream st: the long rows' chunk sums of the linear devices' F and
// Q (lin_f, lin_q may be null) and, with jac non-null, the long rows' Newton matrix entries from
// the family's dfdx / dqdx as tia_combine_kernel forms them.
int xd_tia_internal_long_chunks(xd_tia *t, const xd_tia_coef *c, const double *x, const double *dfdx,
                                const double *dqdx, const double *lin_f, const double *lin_q, double *jac,
                                cudaStream_t st);
