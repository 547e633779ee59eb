/* xyce_tia.h — C ABI of the B200 time-integration combine step.
 *
 * Replaces, for one Newton iterate, the caller-side passes the reference makes after the device
 * loads:
 *   N_TIA_OneStep::obtainJacobian  (src/TimeIntegrationPKG/src/N_TIA_OneStep.C:470-497)
 *       J = -(alpha/h) dQ/dx + f dF/dx, via N_LAS_Matrix::linearCombo (N_LAS_Matrix.C:835-853)
 *   N_TIA_OneStep::obtainResidual  (N_TIA_OneStep.C:272-312)
 *       rhs = -((Q - Q_n) / h + f F + g F_hist)
 * fused into one pass over the CSR rows, together with the loads of the linear devices whose
 * stamps do not depend on the solution (resistors N_DEV_Resistor.C:1075-1161, capacitors
 * N_DEV_Capacitor.C:1821-2002, independent voltage sources N_DEV_Vsrc.C:941-1028): their dF/dx and
 * dQ/dx are constant CSR value arrays, their F and Q are those matrices times x, and the source
 * values enter through a vector b(t) (F = ... - b). An optional shunt conductance on every node row
 * supports gmin stepping, the operating-point continuation of the reference's nonlinear solver
 * (N_NLS_NOX_AugmentLinSys_GStepping.C:142-197 augments the voltage nodes).
 *
 * Buffers are caller-owned device pointers; calls are stream-ordered and capturable. Status: 0 =
 * ok, < 0 = error (xd_last_error()).
 */
#ifndef XYCE_TIA_H
#define XYCE_TIA_H

#include "xyce_devload.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct xd_tia xd_tia;

/* mode 0: DC operating point  — J = dF/dx,                           rhs = -F + dFdxdVp
 * mode 1: time step           — J = qscale dQ/dx + fscale dF/dx,
 *                               rhs = -((Q - qn0) inv_h + fscale F + hist_scale fhist) + qscale dQdxdVp + fscale dFdxdVp
 * The dFdxdVp / dQdxdVp terms are the devices' voltage-limiter corrections, added when limiting is
 * on (N_TIA_OneStep.C:322-336, N_TIA_NoTimeIntegration.C:152-157); pass null pointers without it.
 * Backward Euler (the one-step method's first order): qscale = inv_h = 1/h, fscale = 1, hist_scale = 0.
 * Trapezoid (second order): qscale = inv_h = 1/h, fscale = hist_scale = 1/2, fhist = F at t_n. */
typedef struct xd_tia_coef {
  int mode;
  double qscale, fscale, inv_h, hist_scale;
  double gshunt; /* conductance to ground on every row whose diagonal is in the pattern, i.e. the
                   node rows, not a voltage source's branch row (gmin stepping); 0 for none */
} xd_tia_coef;

/* Uploads the CSR pattern (rows = unknowns). */
int xd_tia_create(const xd_csr *pattern, int cuda_device, xd_tia **out);
int xd_tia_destroy(xd_tia *t);

/* Per row i, in one pass over the row's entries k:
 *   jac[k]   = qscale (dqdx[k] + lin_dqdx[k]) + fscale (dfdx[k] + lin_dfdx[k] + gshunt [k diagonal])
 *   F_i      = f[i] + sum_k lin_dfdx[k] x[col k] + gshunt x[i] [row i has its diagonal] - b[i]
 *   Q_i      = q[i] + sum_k lin_dqdx[k] x[col k]
 *   rhs[i]   as above (limiter corrections dfdxdvp / dqdxdvp, when non-null, added last);
 *   f_tot[i] = F_i and q_tot[i] = Q_i when those pointers are non-null.
 * dfdx / dqdx / f / q hold the nonlinear devices' loads (for instance from xd_load_assign);
 * lin_* may be null (no linear devices), b may be null (no sources); in mode 0 dqdx, lin_dqdx,
 * qn0 and fhist are not read. Row sums use a fixed lane split and a fixed reduction tree (rows of
 * more than 1,024 entries, such as a supply rail's: fixed 1,024-entry chunks, a block each, then a
 * fixed tree over the chunks), so the results are bit-identical from run to run. */
int xd_tia_combine(xd_tia *t, const xd_tia_coef *coef, const double *d_x, const double *d_dfdx,
                   const double *d_dqdx, const double *d_lin_dfdx, const double *d_lin_dqdx,
                   const double *d_f, const double *d_q, const double *d_dfdxdvp, const double *d_dqdxdvp,
                   const double *d_b, const double *d_qn0, const double *d_fhist, double *d_jac,
                   double *d_rhs, double *d_q_tot, double *d_f_tot, void *stream);

/* Independent voltage sources' values at an analysis time, evaluated on the device: stands in for
 * the device manager's source update (DeviceMaster::updateSources -> PWLinData::updateSource,
 * src/DeviceModelPKG/Core/src/N_DEV_SourceData.C:1371-1490) and the value the sources load into
 * the branch rows (Vsrc::Master::updateState, N_DEV_Vsrc.C:941-960). Source k writes b[row[k]]:
 * with transient != 0 (a transient step or its operating point) its piecewise-linear value at
 * time t — n_pairs[k] (t, v) pairs in tv, all sources' pairs concatenated, delay td[k], repeat
 * from time repeat[k] (negative or a null array: no repeat), computed with the reference's own
 * arithmetic, so the values are bit-identical to its — and otherwise, or when it has no pairs,
 * its DC value dc[k]. No other entry of d_b is written. xd_pwl_create copies the table to the
 * device (set-up only); xd_pwl_eval is one kernel launch. */
typedef struct xd_pwl xd_pwl;
int xd_pwl_create(int n_src, const int *row, const int *n_pairs, const double *tv, const double *dc, const double *td,
                  const double *repeat, int cuda_device, xd_pwl **out);
int xd_pwl_destroy(xd_pwl *p);
int xd_pwl_eval(xd_pwl *p, double t, int transient, double *d_b, void *stream);

/* Fused device load and combine (no counterpart in the reference, where the device manager's loads
 * and the integrator's combine are separate passes over memory: N_DEV_DeviceMgr.C:2117-2123,
 * 2452-2461, 2256-2261, then N_TIA_OneStep.C:272-312, 470-497).
 *
 * xd_tia_fused_create binds a combine object and a MOSFET family built on the same pattern and
 * device, and precomputes, per CSR entry and per row, where the family's contributions sit in its
 * gather maps (set-up only; it allocates). xd_tia_load_combine then does, in one call, what
 * xd_load_assign (into the family buffers d_fam_*) followed by xd_tia_combine (with those buffers
 * as dfdx / dqdx / f / q and, when limiter != 0, fx / qx) does, with bit-identical jac, rhs, q_tot
 * and f_tot: the evaluation kernel stages the stamps, and one pass over the rows forms every Newton
 * matrix entry and residual straight from them, so the family's dF/dx and dQ/dx never go through
 * memory (only the few entries with very many contributions, such as supply rails, are summed
 * into d_fam_dfdx / d_fam_dqdx first). The family's F, Q and limiter vectors are stored into
 * d_fam_f / d_fam_q / d_fam_fx / d_fam_qx as by xd_load_assign (by the same vector gather, before
 * the row pass reads them); d_fam_dfdx / d_fam_dqdx hold
 * the family's sums only at those long entries afterwards. Buffers as for the two calls it
 * replaces (d_fam_* zeroed once when allocated). */
typedef struct xd_tia_fused xd_tia_fused;
int xd_tia_fused_create(xd_tia *t, xd_ctx *family, xd_tia_fused **out);
int xd_tia_fused_destroy(xd_tia_fused *f);
int xd_tia_load_combine(xd_tia_fused *f, const xd_flags *flags, const xd_tia_coef *coef, const double *d_x,
                        double *d_next_sta, double *d_curr_sta, double *d_next_sto, const double *d_curr_sto,
                        double *d_fam_f, double *d_fam_q, double *d_fam_fx, double *d_fam_qx, double *d_fam_dfdx,
                        double *d_fam_dqdx, const double *d_lin_dfdx, const double *d_lin_dqdx, int limiter,
                        const double *d_b, const double *d_qn0, const double *d_fhist, double *d_jac,
                        double *d_rhs, double *d_q_tot, double *d_f_tot, void *stream);

/* Small dense direct solve of the Newton system J x = rhs (J in the pattern's CSR values), for
 * circuits of at most XD_DENSE_MAX_N unknowns; stands in for the reference's direct solve (KLU
 * through Amesos, src/LinearAlgebraServicesPKG/src/N_LAS_AmesosSolver.C:160, 305) where the
 * system is small enough for one SM's shared memory. Gaussian elimination with partial pivoting
 * (the first row of largest magnitude in the column; rows swapped whole, LAPACK's convention),
 * then back substitution. d_lu (n * n doubles, row-major: U on and above the diagonal, the unit
 * lower factor's multipliers below) and d_piv (n ints: row k was swapped with row piv[k] at step
 * k) receive the factors when non-null; d_info (may be null) receives 0, or k + 1 for the first
 * column k without a nonzero pivot (the solution is then not finite). One kernel launch. */
#define XD_DENSE_MAX_N 160
int xd_tia_dense_solve(xd_tia *t, const double *d_jac, const double *d_rhs, double *d_lu, int *d_piv, double *d_x,
                       int *d_info, void *stream);
/* Solves with factors kept from xd_tia_dense_solve (a chord step). */
int xd_tia_dense_resolve(xd_tia *t, const double *d_lu, const int *d_piv, const double *d_rhs, double *d_x,
                         void *stream);
/* The same solve, run only when *d_info is nonzero on entry (a static-pivot solve before it
 * stopped, below); it then overwrites d_x, the factors and *d_info. */
int xd_tia_dense_solve_fallback(xd_tia *t, const double *d_jac, const double *d_rhs, double *d_lu, int *d_piv,
                                double *d_x, int *d_info, void *stream);

/* Newton's bookkeeping on the device (N_NLS_DampedNewton.C:325-350, 1792-1830), one block each:
 * xd_tia_newton_update adds the update d_dx to d_x, refreshes the weights d_w = rel_tol *
 * max(|d_xref|, |d_x|) + abs_tol when update_weights is set, and writes the update's weighted RMS
 * norm sqrt(mean((dx / w)^2)) to d_norms[0]; xd_tia_residual_norm writes max |d_rhs| to d_norms[1]
 * (NaN when an entry is not finite) and *d_flag (0 when d_flag is null) to d_norms[2]. Fixed
 * reduction order: the same inputs give the same norms. */
int xd_tia_newton_update(xd_tia *t, double *d_x, const double *d_dx, const double *d_xref, double *d_w,
                         double rel_tol, double abs_tol, int update_weights, double *d_norms, void *stream);
int xd_tia_residual_norm(xd_tia *t, const double *d_rhs, const int *d_flag, double *d_norms, void *stream);

/* Static-pivot solve of small systems (n <= XD_DENSE_MAX_N) whose matrices share one pattern, as
 * the Newton matrices of a transient do: xd_slu_create orders the unknowns by minimum degree of
 * A + A^T (rows and columns alike), factors one matrix on the host in that order with row pivoting
 * that keeps the diagonal unless it is below 0.1 of its column's largest entry, and keeps the
 * orders and the fill pattern; xd_slu_solve eliminates each later matrix in those orders over the
 * pattern alone (no pivot search), on one warp. A pivot smaller than tol times an entry below it
 * (the threshold test of circuit solvers; 1e-3 as KLU's default) stops the solve with *d_info =
 * k + 1 for step k and leaves d_x unwritten; xd_tia_dense_solve_fallback queued after it then
 * solves that system with partial pivoting, so the pair is one stream-ordered, capturable solve.
 * On success *d_info = 0, d_x holds the solution and, when d_lu is given (n * n doubles), the
 * factors in the static orders, for xd_slu_resolve (a chord step). */
typedef struct xd_slu xd_slu;
int xd_slu_create(int n, const int *rowptr, const int *colind, const double *vals, double tol, int cuda_device,
                  xd_slu **out);
int xd_slu_solve(xd_slu *s, const double *d_vals, const double *d_rhs, double *d_lu, double *d_x, int *d_info,
                 void *stream);
int xd_slu_resolve(xd_slu *s, const double *d_lu, const double *d_rhs, double *d_x, void *stream);
int xd_slu_destroy(xd_slu *s);

#ifdef __cplusplus
}
#endif

#endif /* XYCE_TIA_H */
