// Triangular solves with bundled LU factors (internal to the library; used by the GPU
// refactorization's solve).
#pragma once

#include <cuda_runtime.h>

// Both triangles of P A Q = L U renumbered in dependency-level order ([0] lower, [1] upper).
struct XdSptrsv {
  int n = 0;
  int nlev[2] = {0, 0};                   // dependency levels of each triangle
  int nstep[2] = {0, 0};                  // the kernel's steps: levels, with runs of thin levels as one
  int nnz[2] = {0, 0};                    // strictly lower / strictly upper entries
  int4 *d_meta[2] = {nullptr, nullptr};   // per level: first and end position, first and end entry
  int *d_lstart[2] = {nullptr, nullptr};  // per level: first row summed by the whole block
  int *d_chain[2] = {nullptr, nullptr};   // per step: offset of its thin-level run in d_sub, or -1
  int *d_sub[2] = {nullptr, nullptr};     // the runs' level boundaries (see sptrsv.cu)
  int *d_eptr[2] = {nullptr, nullptr};    // [n+1] entry range of each position
  int *d_epos[2] = {nullptr, nullptr};    // [nnz] each entry's column as a position
  int *d_src[2] = {nullptr, nullptr};     // [nnz] each entry's index in the bundled factors
  int *d_dst[2] = {nullptr, nullptr};     // [n] lower: position in the upper order; upper: solution index
  double *d_val[2] = {nullptr, nullptr};  // [nnz] entry values (regathered before each solve)
  int *d_dsrc = nullptr;                  // [n] upper diagonal's index in the bundled factors
  int *d_bsrc = nullptr;                  // [n] right-hand side index of each lower position
  double *d_vec = nullptr;                // [5n] right-hand sides, solved values, upper diagonal
};

// Level order from the pattern of M = L - I + U (device CSR, read once to the host); p, q (host)
// as in the refactorization: (P A Q)[i][j] = A[P[i]][Q[j]].
int xd_sptrsv_init(XdSptrsv *s, int n, int nnz_m, const int *d_mp, const int *d_mi, const int *p, const int *q);
void xd_sptrsv_free(XdSptrsv *s);
// Solves A x = b in place in d_x with the current values d_mx of M (the pattern given to
// xd_sptrsv_init). Stream-ordered.
int xd_sptrsv_solve(XdSptrsv *s, const double *d_mx, double *d_x, cudaStream_t st);
