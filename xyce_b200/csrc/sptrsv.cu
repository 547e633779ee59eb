// Forward and back substitution with the refactorization's factors (P A Q = L U, bundled by the
// refactorization library as one CSR matrix M = L - I + U in the permuted index space).
//
// Circuit factors are deep and narrow: the 200k-unknown placed netlist's L and U have 2,300-4,100
// dependency levels each, a few dozen rows per level (plus one level of ~85k independent rows in
// L), 2M entries in all. The solve is bound by the latency of a level, not by its arithmetic (4M
// flops) or bytes (24 MB), so each triangle runs in ONE thread block that walks the levels with a
// block barrier between them (level-by-level launches, or grid-wide waits on per-row flags, cost
// microseconds a level). What keeps a level short is that its rows read shared memory only:
//   * the set-up renumbers each triangle's rows in level order and lays out, per level, the rows'
//     entry ranges, the entries (column as a level-order position, value) and the right-hand side
//     contiguously; a gather kernel refreshes the values and the right-hand side before each solve;
//   * the block streams the next kAhead levels into shared memory with asynchronous copies
//     (cp.async, one commit group per level) while it computes the current one, together with the
//     solved values their entries read that are already final (positions before the current level);
//   * the last kWindow solved values stay in shared memory (slot = position mod kWindow; a value
//     read during level l comes from there when its position is within kWindow of the level's
//     end, so no row of level l can have reused the slot), others are read from global memory.
// Levels of short rows are solved a thread per row, others a warp per row; levels with more rows
// or entries than a staging slot holds are read from global memory directly. Every sum is reduced
// in a fixed order, so results do not depend on the timing. In a staged level the short rows (at
// most kShortRow entries, ordered first by the set-up) are solved a thread each while the warps the
// short rows leave free solve the longer rows a warp each.
// Thin levels (at most kChainShort short and kChainLong longer rows) are most of the lower
// triangle's levels (median two rows), and a block step (staging, barrier) costs far more than
// their rows. Runs of consecutive thin levels that fit one staging slot are staged as one step,
// which the first kChainLong warps solve level by level (short rows a thread each, longer rows a
// warp each) with a barrier of those warps alone between levels; each row is summed as in any
// other staged level, so the results are the same bits.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>
#include <vector>

#include "sptrsv.h"

int xd_internal_fail(int code, const std::string &msg);

namespace {

#ifndef XD_SPTRSV_THREADS
#define XD_SPTRSV_THREADS 1024
#endif
// Threads of the solve block. Every warp runs the per-level bookkeeping (staging, barrier), so a
// level costs about (warps x that) issue slots on the one SM: few warps keep levels short, and
// levels of short rows are solved a thread per row, so they do not need many.
constexpr int kThreads = XD_SPTRSV_THREADS;
constexpr int kWarps = kThreads / 32;
constexpr int kAhead = 2;               // levels staged ahead of the one being solved
constexpr int kSlots = kAhead + 1;      // staging slots (a level uses slot level % kSlots)
constexpr int kSlotRows = 384;          // rows per staged level
constexpr int kSlotEnts = 3072;         // entries per staged level
constexpr int kWindow = 1 << 11;        // solved values kept in shared memory
constexpr int kBlockRow = 2048;         // in unstaged levels, longer rows are summed by the whole block
constexpr int kThreadRowEnts = 4;       // unstaged levels averaging at most this many entries a row: a thread a row
constexpr int kShortRow = 8;            // staged levels: rows of at most this many entries a thread each, longer a warp
constexpr int kChainShort = 128;        // a thin level: at most this many short rows ...
constexpr int kChainLong = 16;          // ... and this many longer ones (a warp each)
constexpr int kChainThreads = 32 * kChainLong;
constexpr int kMaxSub = 32;             // thin levels per run
constexpr int kSubInts = 2 * kMaxSub + 2;  // a run's record: count, (first row, first long row) per level, end

constexpr int kEntsPerThread = kSlotEnts / kThreads;
static_assert(kSlotEnts % kThreads == 0, "a staged level's entries split evenly over the threads");

struct Smem {
  double win[kWindow];
  double val[kSlots][kSlotEnts];
  double xv[kSlots][kSlotEnts];  // solved values of the entries' columns that were final when staged
  int pos[kSlots][kSlotEnts];
  int cut[kSlots];               // columns at positions below cut[s] have their value in xv
  int nshort[kSlots];            // the level's short rows (they come first)
  int chain[kSlots];             // 1: the step is a run of thin levels, described by sub
  int sub[kSlots][kSubInts];
  double rhs[kSlots][kSlotRows];
  double diag[kSlots][kSlotRows];
  int dst[kSlots][kSlotRows];
  int eptr[kSlots][kSlotRows + 1];
  double red[2][kWarps];
};
static_assert(sizeof(Smem) <= 227 * 1024, "the staging fits one block's shared memory");

__device__ __forceinline__ void cp_async4(void *s, const void *g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async8(void *s, const void *g) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(s);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_ahead() {
  asm volatile("cp.async.wait_group %0;" ::"n"(kAhead - 1) : "memory");
}

// One triangle in level order. meta[l] = (first position, end position, first entry, end entry);
// lstart[2l] = the first of level l's rows longer than kBlockRow entries (they come last);
// lstart[2l + 1] = the first of its rows longer than kShortRow entries (the short ones come first).
struct Tri {
  const int4 *meta;
  const int *lstart;
  const int *eptr;   // [n+1] entry range of each position
  const int *epos;   // [nnz] column of each entry as a level-order position
  const double *val; // [nnz]
  const double *rhs; // [n]
  const double *diag;// [n] (upper)
  const int *dst;    // [n] lower: position in the upper order; upper: solution index
  double *out;       // [n] solved values by position
  double *next_rhs;  // lower: the upper triangle's right-hand side (by its positions)
  double *x;         // upper: the solution
  int nlev;          // steps
  const int *chain;  // [nlev] offset of the step's run record in sub, or -1
  const int *sub;    // run records (rows relative to the step's first position), padded by kSubInts
};

__device__ __forceinline__ double solved(int p, int lo, const Smem &sm, const double *out) {
  return p >= lo ? sm.win[p & (kWindow - 1)] : out[p];
}

template <bool UPPER>
__device__ __forceinline__ void publish(int p, double v, int dst, Smem &sm, const Tri &t) {
  sm.win[p & (kWindow - 1)] = v;
  t.out[p] = v;
  if (UPPER)
    t.x[dst] = v;
  else
    t.next_rhs[dst] = v;
}

__device__ __forceinline__ bool staged(const int4 &m) { return m.y - m.x <= kSlotRows && m.w - m.z <= kSlotEnts; }

// The column positions of a staged level's entries this thread copies (entries tid, tid + kThreads,
// ...), loaded one iteration before they are staged, so that the staging issues its copies without
// waiting for a load.
struct PosAhead {
  int p[kEntsPerThread];
  int ls;  // thread 0: the level's first row longer than kShortRow entries
  int ch;  // the step's run record offset, or -1
};

__device__ __forceinline__ PosAhead load_pos(int l, const int4 &m, const Tri &t, int tid) {
  PosAhead a;
  const bool st = l < t.nlev && staged(m);
#pragma unroll
  for (int q = 0; q < kEntsPerThread; ++q) {
    const int k = tid + q * kThreads;
    a.p[q] = (st && k < m.w - m.z) ? t.epos[m.z + k] : -1;
  }
  a.ls = (st && tid == 0) ? t.lstart[2 * l + 1] : 0;
  a.ch = st ? t.chain[l] : -1;
  return a;
}

// Stages level l (metadata m, column positions pa) into slot l % kSlots: its rows' entry ranges,
// right-hand sides, diagonals and destinations, its entries' values and column positions, and the
// solved values of columns at positions below cut (final and visible when this is called).
__device__ __forceinline__ void stage_level(int l, const int4 &m, const PosAhead &pa, int cut, Smem &sm,
                                            const Tri &t, int tid) {
  if (l < t.nlev && staged(m)) {
    const int s = l % kSlots, nr = m.y - m.x, ne = m.w - m.z;
    for (int k = tid; k < nr; k += kThreads) {
      cp_async8(&sm.rhs[s][k], t.rhs + m.x + k);
      if (t.diag) cp_async8(&sm.diag[s][k], t.diag + m.x + k);
      cp_async4(&sm.dst[s][k], t.dst + m.x + k);
    }
    for (int k = tid; k <= nr; k += kThreads) cp_async4(&sm.eptr[s][k], t.eptr + m.x + k);
#pragma unroll
    for (int q = 0; q < kEntsPerThread; ++q) {
      const int k = tid + q * kThreads;
      if (k < ne) {
        cp_async8(&sm.val[s][k], t.val + m.z + k);
        sm.pos[s][k] = pa.p[q];
        if (pa.p[q] < cut) cp_async8(&sm.xv[s][k], t.out + pa.p[q]);
      }
    }
    if (pa.ch >= 0)
      for (int k = tid; k < kSubInts; k += kThreads) cp_async4(&sm.sub[s][k], t.sub + pa.ch + k);
    if (tid == 0) {
      sm.cut[s] = cut;
      sm.nshort[s] = pa.ls - m.x;
      sm.chain[s] = pa.ch >= 0;
    }
  }
  cp_async_commit();
}

// A staged entry's column value: staged, in the window, or from global memory.
__device__ __forceinline__ double staged_solved(const Smem &sm, int s, int k, int lo, const double *out) {
  const int p = sm.pos[s][k];
  return p < sm.cut[s] ? sm.xv[s][k] : (p >= lo ? sm.win[p & (kWindow - 1)] : out[p]);
}

template <bool UPPER>
__global__ void __launch_bounds__(kThreads) level_solve_kernel(Tri t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Smem &sm = *reinterpret_cast<Smem *>(smem_raw);
  const unsigned full = 0xffffffffu;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int l = 0; l < kAhead; ++l) {
    const int4 m = l < t.nlev ? t.meta[l] : make_int4(0, 0, 0, 0);
    stage_level(l, m, load_pos(l, m, t, tid), 0, sm, t, tid);
  }
  // Loads run ahead of their use so that no level waits for one: the metadata of level l + 2 (to
  // solve), of levels l + kAhead + 2 and + 4 (to stage), the column positions of level
  // l + kAhead + 2. Each parity of l has its own registers, reloaded only after their last use:
  // copying a register whose load is still in flight would wait for it.
  auto meta_at = [&](int l) { return l < t.nlev ? t.meta[l] : make_int4(0, 0, 0, 0); };
  // cur: meta[l]; ahp: meta[l + kAhead]; ahq: meta[l + kAhead + 2]; pa: positions of l + kAhead.
  auto step = [&](int l, int4 &cur, int4 &ahp, int4 &ahq, PosAhead &pa) {
    const int b = cur.x, e = cur.y, lo = e - kWindow;
    const bool by_thread = cur.w - cur.z <= kThreadRowEnts * (e - b);
    if (staged(cur)) {
      const int s = l % kSlots, eb = cur.z;
      auto short_row = [&](int r) {
        const int kb = sm.eptr[s][r] - eb, ke = sm.eptr[s][r + 1] - eb;
        double acc = 0.0;
        for (int k = kb; k < ke; ++k) acc += sm.val[s][k] * staged_solved(sm, s, k, lo, t.out);
        const double v = UPPER ? (sm.rhs[s][r] - acc) / sm.diag[s][r] : sm.rhs[s][r] - acc;
        publish<UPPER>(b + r, v, sm.dst[s][r], sm, t);
      };
      auto warp_row = [&](int r) {
        const int kb = sm.eptr[s][r] - eb, ke = sm.eptr[s][r + 1] - eb;
        double acc = 0.0;
        for (int k = kb + lane; k < ke; k += 32) acc += sm.val[s][k] * staged_solved(sm, s, k, lo, t.out);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(full, acc, off);
        if (lane == 0) {
          const double v = UPPER ? (sm.rhs[s][r] - acc) / sm.diag[s][r] : sm.rhs[s][r] - acc;
          publish<UPPER>(b + r, v, sm.dst[s][r], sm, t);
        }
      };
      if (sm.chain[s]) {
        // A run of thin levels: the first kChainLong warps solve them in order, named barrier 1
        // (theirs alone) between levels.
        if (warp < kChainLong) {
          const int *sb = sm.sub[s];
          const int nsub = sb[0];
          for (int j = 0; j < nsub; ++j) {
            const int rb = sb[1 + 2 * j], rs = sb[2 + 2 * j], re = sb[3 + 2 * j];
            for (int r = rb + tid; r < rs; r += kChainThreads) short_row(r);
            for (int r = rs + warp; r < re; r += kChainLong) warp_row(r);
            asm volatile("bar.sync 1, %0;" ::"n"(kChainThreads) : "memory");
          }
        }
      } else {
        // Short rows (the first ns) a thread each; longer ones a warp each, on the warps after
        // those the short rows occupy, at the same time.
        const int ns = sm.nshort[s];
        for (int r = tid; r < ns; r += kThreads) short_row(r);
        const int w0 = min(kWarps - 1, (ns + 31) >> 5);
        for (int r = ns + warp - w0; warp >= w0 && r < e - b; r += kWarps - w0) warp_row(r);
      }
    } else {
      // Unstaged level: rows from global memory, one thread or one warp each; very long rows by
      // the block.
      const int m = t.lstart[2 * l];
      if (by_thread) {
        for (int r = b + tid; r < m; r += kThreads) {
          const int kb = t.eptr[r], ke = t.eptr[r + 1];
          double acc = 0.0;
          for (int k = kb; k < ke; ++k) acc += t.val[k] * solved(t.epos[k], lo, sm, t.out);
          const double v = UPPER ? (t.rhs[r] - acc) / t.diag[r] : t.rhs[r] - acc;
          publish<UPPER>(r, v, t.dst[r], sm, t);
        }
      }
      for (int r = b + warp; r < (by_thread ? b : m); r += kWarps) {
        const int kb = t.eptr[r], ke = t.eptr[r + 1];
        double acc = 0.0;
        for (int k = kb + lane; k < ke; k += 32) acc += t.val[k] * solved(t.epos[k], lo, sm, t.out);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(full, acc, off);
        if (lane == 0) {
          const double v = UPPER ? (t.rhs[r] - acc) / t.diag[r] : t.rhs[r] - acc;
          publish<UPPER>(r, v, t.dst[r], sm, t);
        }
      }
      for (int r = m; r < e; ++r) {
        const int kb = t.eptr[r], ke = t.eptr[r + 1];
        double acc = 0.0;
        for (int k = kb + tid; k < ke; k += kThreads) acc += t.val[k] * solved(t.epos[k], lo, sm, t.out);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(full, acc, off);
        __syncthreads();  // red free (a previous long row may still be reading it)
        if (lane == 0) sm.red[0][warp] = acc;
        __syncthreads();
        if (warp == 0) {
          acc = lane < kWarps ? sm.red[0][lane] : 0.0;
#pragma unroll
          for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(full, acc, off);
          if (lane == 0) {
            const double v = UPPER ? (t.rhs[r] - acc) / t.diag[r] : t.rhs[r] - acc;
            publish<UPPER>(r, v, t.dst[r], sm, t);
          }
        }
      }
    }
    // Stage level l + kAhead into the slot level l - 1 used, then make level l + 1's copies (and
    // this level's results) visible to the block.
    stage_level(l + kAhead, ahp, pa, b, sm, t, tid);
    pa = load_pos(l + kAhead + 2, ahq, t, tid);
    ahp = ahq;
    ahq = meta_at(l + kAhead + 4);
    cur = meta_at(l + 2);
    cp_async_wait_ahead();
    __syncthreads();
  };
  int4 cur0 = meta_at(0), cur1 = meta_at(1);
  int4 ahp0 = meta_at(kAhead), ahp1 = meta_at(kAhead + 1), ahq0 = meta_at(kAhead + 2), ahq1 = meta_at(kAhead + 3);
  PosAhead pa0 = load_pos(kAhead, ahp0, t, tid), pa1 = load_pos(kAhead + 1, ahp1, t, tid);
  cp_async_wait_ahead();
  __syncthreads();
  for (int l = 0; l < t.nlev; l += 2) {
    step(l, cur0, ahp0, ahq0, pa0);
    if (l + 1 < t.nlev) step(l + 1, cur1, ahp1, ahq1, pa1);
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// Before a solve: the triangles' values from the bundled factors, and the lower triangle's
// right-hand side b[P[row]] in its level order.
__global__ void gather_kernel(int nl, const int *__restrict__ src_l, double *__restrict__ val_l, int nu,
                              const int *__restrict__ src_u, double *__restrict__ val_u, int n,
                              const int *__restrict__ dsrc, double *__restrict__ diag, const int *__restrict__ bsrc,
                              const double *__restrict__ b, double *__restrict__ rhs_l,
                              const double *__restrict__ mx) {
  const int stride = gridDim.x * blockDim.x;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nl; k += stride) val_l[k] = mx[src_l[k]];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < nu; k += stride) val_u[k] = mx[src_u[k]];
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += stride) {
    diag[k] = mx[dsrc[k]];
    rhs_l[k] = b[bsrc[k]];
  }
}

int cu_err(cudaError_t e, const char *where) {
  return xd_internal_fail(-3, std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
}

// One triangle's level order: rows by dependency depth (ascending row index within a level),
// each row's entries of this triangle, the level metadata.
struct HostTri {
  std::vector<int> rows, pos, eptr, epos, src, lstart, chain, sub;
  std::vector<int4> meta;  // per step
  int nlev = 0;            // dependency levels
};

void build_tri(int n, const std::vector<int> &mp, const std::vector<int> &mi, bool upper, HostTri &h) {
  std::vector<int> lev(n, 0);
  int nlev = 0;
  for (int t = 0; t < n; ++t) {
    const int r = upper ? n - 1 - t : t;
    int d = 0;
    for (int k = mp[r]; k < mp[r + 1]; ++k) {
      const int j = mi[k];
      if (upper ? (j > r) : (j < r)) d = std::max(d, lev[j] + 1);
    }
    lev[r] = d;
    nlev = std::max(nlev, d + 1);
  }
  // Buckets (level, length class): within a level the rows of at most kShortRow entries first, then
  // the longer ones, the rows longer than kBlockRow entries last.
  auto len = [&](int r) {
    int c = 0;
    for (int k = mp[r]; k < mp[r + 1]; ++k) c += (upper ? (mi[k] > r) : (mi[k] < r)) ? 1 : 0;
    return c;
  };
  std::vector<int> bucket(n);
  for (int r = 0; r < n; ++r) {
    const int c = len(r);
    bucket[r] = 3 * lev[r] + (c > kBlockRow ? 2 : c > kShortRow ? 1 : 0);
  }
  std::vector<int> start(3 * (size_t)nlev + 1, 0);
  for (int r = 0; r < n; ++r) ++start[bucket[r] + 1];
  for (size_t k = 1; k < start.size(); ++k) start[k] += start[k - 1];
  h.rows.assign(n, 0);
  h.pos.assign(n, 0);
  std::vector<int> fill(start.begin(), start.end() - 1);
  for (int r = 0; r < n; ++r) {
    h.pos[r] = fill[bucket[r]]++;
    h.rows[h.pos[r]] = r;
  }
  h.eptr.assign(n + 1, 0);
  h.epos.clear();
  h.src.clear();
  for (int p = 0; p < n; ++p) {
    const int r = h.rows[p];
    for (int k = mp[r]; k < mp[r + 1]; ++k) {
      const int j = mi[k];
      if (upper ? (j > r) : (j < r)) h.src.push_back(k);
    }
    h.eptr[p + 1] = (int)h.src.size();
  }
  h.epos.resize(h.src.size());
  for (size_t k = 0; k < h.src.size(); ++k) h.epos[k] = h.pos[mi[h.src[k]]];
  // Steps: a level, or a run of 2..kMaxSub consecutive thin levels that fits one staging slot. A
  // run's record in sub: the level count, then per level its first row and first long row
  // (relative to the run's first position), then the run's row count.
  h.nlev = nlev;
  h.meta.clear();
  h.lstart.clear();
  h.chain.clear();
  h.sub.clear();
  auto thin = [&](int l) {
    return start[3 * l + 1] - start[3 * l] <= kChainShort && start[3 * l + 3] - start[3 * l + 1] <= kChainLong;
  };
  for (int l = 0; l < nlev;) {
    int l2 = l, rows = 0, ents = 0;
    while (l2 < nlev && l2 - l < kMaxSub && thin(l2)) {
      const int b = start[3 * l2], e = start[3 * l2 + 3];
      const int r2 = rows + (e - b), e2 = ents + (h.eptr[e] - h.eptr[b]);
      if (r2 > kSlotRows || e2 > kSlotEnts) break;
      rows = r2;
      ents = e2;
      ++l2;
    }
    if (l2 - l >= 2) {
      const int b = start[3 * l], e = start[3 * l2];
      h.meta.push_back(make_int4(b, e, h.eptr[b], h.eptr[e]));
      h.lstart.push_back(e);
      h.lstart.push_back(b);
      h.chain.push_back((int)h.sub.size());
      h.sub.push_back(l2 - l);
      for (int k = l; k < l2; ++k) {
        h.sub.push_back(start[3 * k] - b);
        h.sub.push_back(start[3 * k + 1] - b);
      }
      h.sub.push_back(e - b);
      l = l2;
    } else {
      const int b = start[3 * l], e = start[3 * l + 3];
      h.meta.push_back(make_int4(b, e, h.eptr[b], h.eptr[e]));
      h.lstart.push_back(start[3 * l + 2]);
      h.lstart.push_back(start[3 * l + 1]);
      h.chain.push_back(-1);
      ++l;
    }
  }
  h.sub.resize(h.sub.size() + kSubInts, 0);  // the staging copies kSubInts ints from a record's offset
}

template <class T>
int upload(T **d, const std::vector<T> &h) {
  cudaError_t e = cudaMalloc(d, sizeof(T) * std::max<size_t>(1, h.size()));
  if (e == cudaSuccess && !h.empty()) e = cudaMemcpy(*d, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice);
  return e == cudaSuccess ? 0 : cu_err(e, "triangular-solve set-up");
}

}  // namespace

int xd_sptrsv_init(XdSptrsv *s, int n, int nnz_m, const int *d_mp, const int *d_mi, const int *p, const int *q) {
  std::vector<int> mp(n + 1), mi(std::max(1, nnz_m));
  cudaError_t e;
  if ((e = cudaMemcpy(mp.data(), d_mp, sizeof(int) * (n + 1), cudaMemcpyDeviceToHost)) != cudaSuccess ||
      (e = cudaMemcpy(mi.data(), d_mi, sizeof(int) * (size_t)nnz_m, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cu_err(e, "triangular-solve set-up (factor pattern)");
  if (mp[0] != 0 || mp[n] != nnz_m) return xd_internal_fail(-4, "unexpected bundled factor pattern");
  for (int r = 0; r < n; ++r)
    if (mp[r + 1] < mp[r]) return xd_internal_fail(-4, "unexpected bundled factor pattern");
  for (int k = 0; k < nnz_m; ++k)
    if (mi[k] < 0 || mi[k] >= n) return xd_internal_fail(-4, "unexpected bundled factor pattern");
  HostTri lo, up;
  build_tri(n, mp, mi, false, lo);
  build_tri(n, mp, mi, true, up);
  // Upper diagonal entries, the lower triangle's right-hand side sources and destinations.
  std::vector<int> dsrc(n, -1), bsrc(n), ldst(n), udst(n);
  for (int pu = 0; pu < n; ++pu) {
    const int r = up.rows[pu];
    for (int k = mp[r]; k < mp[r + 1]; ++k)
      if (mi[k] == r) dsrc[pu] = k;
    if (dsrc[pu] < 0) return xd_internal_fail(-4, "a factor row has no diagonal entry");
    udst[pu] = q[r];
  }
  for (int pl = 0; pl < n; ++pl) {
    bsrc[pl] = p[lo.rows[pl]];
    ldst[pl] = up.pos[lo.rows[pl]];
  }
  s->n = n;
  s->nnz[0] = (int)lo.src.size();
  s->nnz[1] = (int)up.src.size();
  s->nlev[0] = lo.nlev;
  s->nlev[1] = up.nlev;
  s->nstep[0] = (int)lo.meta.size();
  s->nstep[1] = (int)up.meta.size();
  int rc;
  if ((rc = upload(&s->d_meta[0], lo.meta)) || (rc = upload(&s->d_meta[1], up.meta)) ||
      (rc = upload(&s->d_eptr[0], lo.eptr)) || (rc = upload(&s->d_eptr[1], up.eptr)) ||
      (rc = upload(&s->d_lstart[0], lo.lstart)) || (rc = upload(&s->d_lstart[1], up.lstart)) ||
      (rc = upload(&s->d_chain[0], lo.chain)) || (rc = upload(&s->d_chain[1], up.chain)) ||
      (rc = upload(&s->d_sub[0], lo.sub)) || (rc = upload(&s->d_sub[1], up.sub)) ||
      (rc = upload(&s->d_epos[0], lo.epos)) || (rc = upload(&s->d_epos[1], up.epos)) ||
      (rc = upload(&s->d_src[0], lo.src)) || (rc = upload(&s->d_src[1], up.src)) ||
      (rc = upload(&s->d_dst[0], ldst)) || (rc = upload(&s->d_dst[1], udst)) || (rc = upload(&s->d_dsrc, dsrc)) ||
      (rc = upload(&s->d_bsrc, bsrc)))
    return rc;
  if ((e = cudaMalloc(&s->d_val[0], sizeof(double) * std::max<size_t>(1, lo.src.size()))) != cudaSuccess ||
      (e = cudaMalloc(&s->d_val[1], sizeof(double) * std::max<size_t>(1, up.src.size()))) != cudaSuccess ||
      (e = cudaMalloc(&s->d_vec, sizeof(double) * 5 * (size_t)n)) != cudaSuccess ||
      (e = cudaFuncSetAttribute(level_solve_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(Smem))) != cudaSuccess ||
      (e = cudaFuncSetAttribute(level_solve_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sizeof(Smem))) != cudaSuccess)
    return cu_err(e, "triangular-solve set-up");
  return 0;
}

void xd_sptrsv_free(XdSptrsv *s) {
  for (int u = 0; u < 2; ++u) {
    cudaFree(s->d_meta[u]);
    cudaFree(s->d_eptr[u]);
    cudaFree(s->d_lstart[u]);
    s->d_lstart[u] = nullptr;
    cudaFree(s->d_chain[u]);
    cudaFree(s->d_sub[u]);
    s->d_chain[u] = s->d_sub[u] = nullptr;
    cudaFree(s->d_epos[u]);
    cudaFree(s->d_src[u]);
    cudaFree(s->d_dst[u]);
    cudaFree(s->d_val[u]);
    s->d_meta[u] = nullptr;
    s->d_eptr[u] = s->d_epos[u] = s->d_src[u] = s->d_dst[u] = nullptr;
    s->d_val[u] = nullptr;
  }
  cudaFree(s->d_dsrc);
  cudaFree(s->d_bsrc);
  cudaFree(s->d_vec);
  s->d_dsrc = s->d_bsrc = nullptr;
  s->d_vec = nullptr;
}

int xd_sptrsv_solve(XdSptrsv *s, const double *d_mx, double *d_x, cudaStream_t st) {
  const int n = s->n;
  // d_vec: lower rhs, lower out, upper rhs, upper out, upper diagonal (each n, by position).
  double *rhs_l = s->d_vec, *out_l = rhs_l + n, *rhs_u = out_l + n, *out_u = rhs_u + n, *diag = out_u + n;
  const int work = std::max(std::max(s->nnz[0], s->nnz[1]), n);
  const int blocks = std::max(1, std::min((work + 255) / 256, 148 * 8));
  gather_kernel<<<blocks, 256, 0, st>>>(s->nnz[0], s->d_src[0], s->d_val[0], s->nnz[1], s->d_src[1], s->d_val[1], n,
                                        s->d_dsrc, diag, s->d_bsrc, d_x, rhs_l, d_mx);
  Tri lo{s->d_meta[0], s->d_lstart[0], s->d_eptr[0], s->d_epos[0], s->d_val[0], rhs_l, nullptr,
         s->d_dst[0], out_l, rhs_u, nullptr, s->nstep[0], s->d_chain[0], s->d_sub[0]};
  Tri up{s->d_meta[1], s->d_lstart[1], s->d_eptr[1], s->d_epos[1], s->d_val[1], rhs_u, diag,
         s->d_dst[1], out_u, nullptr, d_x, s->nstep[1], s->d_chain[1], s->d_sub[1]};
  level_solve_kernel<false><<<1, kThreads, sizeof(Smem), st>>>(lo);
  level_solve_kernel<true><<<1, kThreads, sizeof(Smem), st>>>(up);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cu_err(e, "triangular solve launch");
  return 0;
}
