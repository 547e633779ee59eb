// Numeric sparse LU refactorization with a fixed pivot order (lu.h).
//
// The transient driver's Newton matrices all share one pattern, and one host factorization fixes
// the pivot order and the fill. Every later matrix is refactored here, on the device, by
// right-looking elimination of P A Q over "pivot levels": pivot k is applied once every pivot that
// changes its row (k' with L(k, k') != 0) or its column (k' with U(k', k) != 0) has been, so all
// pivots of one level apply together. Applying a level is two steps (in the single-block runs the
// updates come first and form their L factors on the spot, the divisions follow in the next
// level's step; see lu_levels_block_kernel):
//   1. divisions: for each pivot k of the level and each row i below it with L(i, k) != 0,
//      L(i, k) = M[i][k] / U(k, k) (final: every pivot that changes M[i][k] is in an earlier level);
//   2. updates: M[i][j] -= L(i, k) * U(k, j) for every such i and every U(k, j) != 0, j > k,
//      grouped by destination: one thread applies all of a destination's updates of the level, in
//      increasing k, so no two threads write one entry and the factors do not depend on timing.
// (A destination written in a level is never read in it: M[i][k] being divided would need a pivot
// of the same level to change column k, and U(k, j) being read would need one to change row k.)
//
// Circuit factors are deep and narrow: at 200k unknowns ~2,900 levels of a few pivots each, with a
// few dozen levels holding half of the ~13M updates. The light levels are latency-bound, so runs of
// them execute in ONE thread block with a block barrier after each step (the values written are
// then visible to the whole block); a level with more work than one block turns over quickly runs
// as two grid-wide launches. The set-up closes the host factorization's L and U patterns under
// elimination, so every update has its destination.
#include "lu.h"

#include <algorithm>
#include <climits>
#include <queue>
#include <string>
#include <vector>

int xd_internal_fail(int code, const std::string &msg);

namespace {

constexpr int kLuThreads = 1024;
// A level whose divisions plus updates exceed this runs grid-wide instead of in the single block.
constexpr long long kGridWork = 24 * 1024;
// Levels of one single-block launch (their division / destination ranges are staged in shared
// memory, 2 x 4 bytes per level).
constexpr int kSegmentLevels = 4096;

__global__ void lu_scatter_kernel(int nnz_a, const int *__restrict__ a2m, const double *__restrict__ a,
                                  double *__restrict__ mx) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz_a) mx[a2m[k]] = a[k];
}

__device__ __forceinline__ void lu_divide(int2 dv, double *mx) { mx[dv.x] = mx[dv.x] / mx[dv.y]; }

// A destination's updates with the level's L factors already stored (after its division step).
// ds = (destination, L(i, k), U(k, j), U(k, k)) for one update; (destination, first pair, count,
// -1) for more, pairs (L(i, k), U(k, j), U(k, k), 0) in increasing k.
__device__ __forceinline__ void lu_update(int4 ds, const int4 *__restrict__ pairs, double *mx) {
  double acc = mx[ds.x];
  if (ds.w >= 0) {
    acc = acc - mx[ds.y] * mx[ds.z];
  } else {
    for (int p = ds.y; p < ds.y + ds.z; ++p) {
      const int4 lu = pairs[p];
      acc = acc - mx[lu.x] * mx[lu.y];
    }
  }
  mx[ds.x] = acc;
}

// The same updates before the level's divisions: each L factor formed on the spot from the
// undivided column entry and the pivot, the division the division step makes, so the same value.
__device__ __forceinline__ void lu_update_divide(int4 ds, const int4 *__restrict__ pairs, double *mx) {
  double acc = mx[ds.x];
  if (ds.w >= 0) {
    acc = acc - (mx[ds.y] / mx[ds.w]) * mx[ds.z];
  } else {
    for (int p = ds.y; p < ds.y + ds.z; ++p) {
      const int4 lu = pairs[p];
      acc = acc - (mx[lu.x] / mx[lu.z]) * mx[lu.y];
    }
  }
  mx[ds.x] = acc;
}

// Levels [l0, l1) in one block, one barrier per level: step l applies level l's updates, forming
// their L factors on the spot (lu_update_divide), together with level l - 1's divisions, which
// store those factors. The two never touch one entry: level l's updates read column entries and
// pivots of level l's pivots and U rows of them and write entries of later pivots' columns, while
// level l - 1's divisions write its own columns' L entries (a level-l update reading one of those
// as U(k, j), or writing one, would make a pivot of level l - 1 depend on one of level l). After
// the last step the run's last level is divided. Each thread loads the index entries of its first
// items of the next step before the barrier that precedes it, so the barrier's wait covers them.
__global__ void __launch_bounds__(kLuThreads, 1) lu_levels_block_kernel(
    int l0, int l1, const int *__restrict__ lev_div, const int *__restrict__ lev_dst, const int2 *__restrict__ div,
    const int4 *__restrict__ dst, const int4 *__restrict__ pairs, double *mx) {
  __shared__ int s_div[kSegmentLevels + 1], s_dst[kSegmentLevels + 1];
  const int nl = l1 - l0;
  for (int l = threadIdx.x; l <= nl; l += kLuThreads) {
    s_div[l] = lev_div[l0 + l];
    s_dst[l] = lev_dst[l0 + l];
  }
  __syncthreads();
  const int tid = threadIdx.x;
  int4 ds_next = make_int4(0, 0, 0, 0);
  if (s_dst[0] + tid < s_dst[1]) ds_next = dst[s_dst[0] + tid];
  int2 dv_next = make_int2(0, 0);  // the first division of the level before the current one
  for (int l = 0; l < nl; ++l) {
    const int ub = s_dst[l], ue = s_dst[l + 1];
    const int4 ds = ds_next;
    const int2 dv = dv_next;
    // The next step's first items: level l + 1's update, level l's division.
    if (l + 1 < nl && s_dst[l + 1] + tid < s_dst[l + 2]) ds_next = dst[s_dst[l + 1] + tid];
    if (s_div[l] + tid < s_div[l + 1]) dv_next = div[s_div[l] + tid];
    if (ub + tid < ue) {
      lu_update_divide(ds, pairs, mx);
      for (int d = ub + tid + kLuThreads; d < ue; d += kLuThreads) lu_update_divide(dst[d], pairs, mx);
    }
    if (l > 0) {
      const int db = s_div[l - 1], de = s_div[l];
      if (db + tid < de) {
        lu_divide(dv, mx);
        for (int t = db + tid + kLuThreads; t < de; t += kLuThreads) lu_divide(div[t], mx);
      }
    }
    __syncthreads();
  }
  // The last level's divisions.
  const int db = s_div[nl - 1], de = s_div[nl];
  if (db + tid < de) {
    lu_divide(dv_next, mx);
    for (int t = db + tid + kLuThreads; t < de; t += kLuThreads) lu_divide(div[t], mx);
  }
}

// One heavy level's divisions, then (a second launch) its updates, grid-wide.
__global__ void lu_divide_grid_kernel(int b, int e, const int2 *__restrict__ div, double *mx) {
  const int t = b + blockIdx.x * blockDim.x + threadIdx.x;
  if (t < e) lu_divide(div[t], mx);
}
__global__ void lu_update_grid_kernel(int b, int e, const int4 *__restrict__ dst, const int4 *__restrict__ pairs,
                                      double *mx) {
  const int d = b + blockIdx.x * blockDim.x + threadIdx.x;
  if (d < e) lu_update(dst[d], pairs, mx);
}

// Zero pivots after the elimination: 1 + the smallest row whose U(k, k) is zero.
__global__ void lu_pivot_check_kernel(int n, const int *__restrict__ diag, const double *__restrict__ mx, int *info) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n && mx[diag[k]] == 0.0) atomicMin(info, k + 1);
}

template <class T>
cudaError_t upload(T **d, const std::vector<T> &h) {
  cudaError_t e = cudaMalloc(d, std::max<size_t>(1, h.size()) * sizeof(T));
  if (e != cudaSuccess || h.empty()) return e;
  return cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

}  // namespace

int xd_lu_init(XdLu *lu, int n, int nnz_a, const int *rowptr_a, const int *colind_a, const int *rowptr_l,
               const int *colind_l, const int *rowptr_u, const int *colind_u, const int *p, const int *q) {
  xd_lu_free(lu);
  std::vector<int> pinv(n), qinv(n);
  for (int i = 0; i < n; ++i) {
    pinv[p[i]] = i;
    qinv[q[i]] = i;
  }
  // Symbolic elimination, row by row: row i starts with L's and U's entries and P A Q's, then
  // takes row k's U columns for each of its L columns k in increasing order (a column added below
  // i is itself eliminated later in the same pass).
  std::vector<int> mp(1, 0), mi, diag(n, -1);
  std::vector<int> mark(n, -1);
  std::vector<int> cols;
  for (int i = 0; i < n; ++i) {
    cols.clear();
    std::priority_queue<int, std::vector<int>, std::greater<int>> lower;
    auto add = [&](int j) {
      if (mark[j] == i) return;
      mark[j] = i;
      cols.push_back(j);
      if (j < i) lower.push(j);
    };
    for (int t = rowptr_l[i]; t < rowptr_l[i + 1]; ++t)
      if (colind_l[t] < i) add(colind_l[t]);
    for (int t = rowptr_u[i]; t < rowptr_u[i + 1]; ++t)
      if (colind_u[t] >= i) add(colind_u[t]);
    const int r = p[i];
    for (int t = rowptr_a[r]; t < rowptr_a[r + 1]; ++t) add(qinv[colind_a[t]]);
    add(i);
    while (!lower.empty()) {
      const int k = lower.top();
      lower.pop();
      for (int t = diag[k] + 1; t < mp[k + 1]; ++t) add(mi[t]);
    }
    std::sort(cols.begin(), cols.end());
    for (int j : cols) {
      if (j == i) diag[i] = (int)mi.size();
      mi.push_back(j);
    }
    if (mi.size() > (size_t)INT_MAX) return xd_internal_fail(-1, "the factors exceed 2^31 entries");
    mp.push_back((int)mi.size());
  }
  const int nnz = mp[n];
  // A's entries in M.
  std::vector<int> a2m(nnz_a);
  for (int r = 0; r < n; ++r)
    for (int t = rowptr_a[r]; t < rowptr_a[r + 1]; ++t) {
      const int i = pinv[r], j = qinv[colind_a[t]];
      const int *b = mi.data() + mp[i], *e = mi.data() + mp[i + 1];
      a2m[t] = (int)(std::lower_bound(b, e, j) - mi.data());
    }
  // Columns of the strict lower part (rows i > k with L(i, k)) and of the strict upper part (rows
  // k' < k with U(k', k)), both with their positions, in increasing row order.
  std::vector<int> lcp(n + 1, 0), ucp(n + 1, 0);
  for (int i = 0; i < n; ++i)
    for (int t = mp[i]; t < mp[i + 1]; ++t) {
      if (mi[t] < i) ++lcp[mi[t] + 1];
      if (mi[t] > i) ++ucp[mi[t] + 1];
    }
  for (int k = 0; k < n; ++k) {
    lcp[k + 1] += lcp[k];
    ucp[k + 1] += ucp[k];
  }
  std::vector<int> lci(lcp[n]), lcpos(lcp[n]), uci(ucp[n]);
  {
    std::vector<int> fl(lcp.begin(), lcp.end() - 1), fu(ucp.begin(), ucp.end() - 1);
    for (int i = 0; i < n; ++i)
      for (int t = mp[i]; t < mp[i + 1]; ++t) {
        const int j = mi[t];
        if (j < i) {
          lci[fl[j]] = i;
          lcpos[fl[j]++] = t;
        }
        if (j > i) uci[fu[j]++] = i;
      }
  }
  // Pivot levels.
  std::vector<int> lev(n, 0);
  int nlev = 0;
  for (int k = 0; k < n; ++k) {
    int l = 0;
    for (int t = mp[k]; t < diag[k]; ++t) l = std::max(l, lev[mi[t]] + 1);
    for (int t = ucp[k]; t < ucp[k + 1]; ++t) l = std::max(l, lev[uci[t]] + 1);
    lev[k] = l;
    nlev = std::max(nlev, l + 1);
  }
  std::vector<int> piv_start(nlev + 1, 0);
  for (int k = 0; k < n; ++k) ++piv_start[lev[k] + 1];
  for (int l = 0; l < nlev; ++l) piv_start[l + 1] += piv_start[l];
  std::vector<int> pivots(n);
  {
    std::vector<int> fp(piv_start.begin(), piv_start.end() - 1);
    for (int k = 0; k < n; ++k) pivots[fp[lev[k]]++] = k;
  }
  // Per level: divisions, then destinations with their pairs ordered by k. A destination's
  // updates are collected in a map from its position to its pairs, in the level's pivot order
  // (increasing k within the level).
  std::vector<int> lev_div(1, 0), lev_dst(1, 0);
  std::vector<int2> div;
  std::vector<int4> dst, pairs;
  std::vector<long long> lev_work(1, 0);  // divisions plus updates up to each level
  std::vector<int> slot(nnz, -1);   // destination position -> index in this level's list
  std::vector<int> touched;
  std::vector<std::vector<int4>> lists;
  for (int l = 0; l < nlev; ++l) {
    touched.clear();
    lists.clear();
    for (int s = piv_start[l]; s < piv_start[l + 1]; ++s) {
      const int k = pivots[s];
      for (int t = lcp[k]; t < lcp[k + 1]; ++t) {
        const int i = lci[t], lpos = lcpos[t];
        div.push_back(make_int2(lpos, diag[k]));
        const int *rb = mi.data() + mp[i], *re = mi.data() + mp[i + 1];
        for (int u = diag[k] + 1; u < mp[k + 1]; ++u) {
          const int j = mi[u];
          const int *f = std::lower_bound(rb, re, j);
          if (f == re || *f != j) return xd_internal_fail(-1, "LU set-up: the symbolic pattern is not closed under fill");
          const int dpos = (int)(f - mi.data());
          if (slot[dpos] < 0) {
            slot[dpos] = (int)lists.size();
            touched.push_back(dpos);
            lists.emplace_back();
          }
          lists[slot[dpos]].push_back(make_int4(lpos, u, diag[k], 0));
        }
      }
    }
    // Pivots of a level are visited in increasing k (pivots[] keeps k order within a level), so
    // each destination's pairs are already in increasing k.
    long long work = 0;
    for (size_t d = 0; d < touched.size(); ++d) {
      const std::vector<int4> &ls = lists[d];
      if (ls.size() == 1) {
        dst.push_back(make_int4(touched[d], ls[0].x, ls[0].y, ls[0].z));
      } else {
        dst.push_back(make_int4(touched[d], (int)pairs.size(), (int)ls.size(), -1));
        pairs.insert(pairs.end(), ls.begin(), ls.end());
      }
      work += (long long)ls.size();
      slot[touched[d]] = -1;
    }
    if (pairs.size() > (size_t)INT_MAX || div.size() > (size_t)INT_MAX || dst.size() > (size_t)INT_MAX)
      return xd_internal_fail(-1, "LU set-up: more than 2^31 updates");
    work += (long long)div.size() - lev_div.back();
    lev_div.push_back((int)div.size());
    lev_dst.push_back((int)dst.size());
    lev_work.push_back(lev_work.back() + work);
  }
  // Launch plan.
  std::vector<int2> segments;
  std::vector<char> grid;
  auto heavy = [&](int l) { return lev_work[l + 1] - lev_work[l] > kGridWork; };
  for (int l = 0; l < nlev;) {
    if (heavy(l)) {
      segments.push_back(make_int2(l, l + 1));
      grid.push_back(1);
      ++l;
      continue;
    }
    int e = l + 1;
    while (e < nlev && e - l < kSegmentLevels && !heavy(e)) ++e;
    segments.push_back(make_int2(l, e));
    grid.push_back(0);
    l = e;
  }
  long long npairs = (long long)pairs.size();
  for (const int4 &d : dst)
    if (d.w >= 0) ++npairs;
  lu->n = n;
  lu->nnz = nnz;
  lu->nnz_a = nnz_a;
  lu->nlev = nlev;
  lu->lev_div = lev_div;
  lu->lev_dst = lev_dst;
  lu->npairs = npairs;
  lu->segments = segments;
  lu->segment_grid = grid;
  cudaError_t e;
  if ((e = upload(&lu->d_mp, mp)) != cudaSuccess || (e = upload(&lu->d_mi, mi)) != cudaSuccess ||
      (e = cudaMalloc(&lu->d_mx, std::max(1, nnz) * sizeof(double))) != cudaSuccess ||
      (e = upload(&lu->d_a2m, a2m)) != cudaSuccess || (e = upload(&lu->d_diag, diag)) != cudaSuccess ||
      (e = upload(&lu->d_lev_div, lev_div)) != cudaSuccess || (e = upload(&lu->d_lev_dst, lev_dst)) != cudaSuccess ||
      (e = upload(&lu->d_div, div)) != cudaSuccess || (e = upload(&lu->d_dst, dst)) != cudaSuccess ||
      (e = upload(&lu->d_pairs, pairs)) != cudaSuccess || (e = cudaMalloc(&lu->d_info, sizeof(int))) != cudaSuccess) {
    xd_lu_free(lu);
    return xd_internal_fail(-3, std::string("LU set-up upload: ") + cudaGetErrorString(e));
  }
  return 0;
}

void xd_lu_free(XdLu *lu) {
  cudaFree(lu->d_mp);
  cudaFree(lu->d_mi);
  cudaFree(lu->d_mx);
  cudaFree(lu->d_a2m);
  cudaFree(lu->d_diag);
  cudaFree(lu->d_lev_div);
  cudaFree(lu->d_lev_dst);
  cudaFree(lu->d_div);
  cudaFree(lu->d_dst);
  cudaFree(lu->d_pairs);
  cudaFree(lu->d_info);
  *lu = XdLu();
}

int xd_lu_refactor(XdLu *lu, const double *d_vals_a, cudaStream_t st) {
  cudaError_t e;
  if ((e = cudaMemsetAsync(lu->d_mx, 0, std::max(1, lu->nnz) * sizeof(double), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(lu->d_info, 0x7f, sizeof(int), st)) != cudaSuccess)
    return xd_internal_fail(-3, std::string("LU refactorization: ") + cudaGetErrorString(e));
  if (lu->nnz_a > 0)
    lu_scatter_kernel<<<(lu->nnz_a + 255) / 256, 256, 0, st>>>(lu->nnz_a, lu->d_a2m, d_vals_a, lu->d_mx);
  for (size_t s = 0; s < lu->segments.size(); ++s) {
    const int l0 = lu->segments[s].x, l1 = lu->segments[s].y;
    if (lu->segment_grid[s]) {
      const int db = lu->lev_div[l0], de = lu->lev_div[l1];
      const int ub = lu->lev_dst[l0], ue = lu->lev_dst[l1];
      if (de > db) lu_divide_grid_kernel<<<(de - db + 255) / 256, 256, 0, st>>>(db, de, lu->d_div, lu->d_mx);
      if (ue > ub)
        lu_update_grid_kernel<<<(ue - ub + 255) / 256, 256, 0, st>>>(ub, ue, lu->d_dst, lu->d_pairs, lu->d_mx);
    } else {
      lu_levels_block_kernel<<<1, kLuThreads, 0, st>>>(l0, l1, lu->d_lev_div, lu->d_lev_dst, lu->d_div, lu->d_dst,
                                                        lu->d_pairs, lu->d_mx);
    }
  }
  if (lu->n > 0) lu_pivot_check_kernel<<<(lu->n + 255) / 256, 256, 0, st>>>(lu->n, lu->d_diag, lu->d_mx, lu->d_info);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return xd_internal_fail(-3, std::string("LU refactorization launch: ") + cudaGetErrorString(e));
  return 0;
}

int xd_lu_info(XdLu *lu, cudaStream_t st, int *info) {
  int v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, lu->d_info, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return xd_internal_fail(-3, std::string("LU pivot report: ") + cudaGetErrorString(e));
  *info = v == kLuNoZeroPivot ? 0 : v;
  return 0;
}
