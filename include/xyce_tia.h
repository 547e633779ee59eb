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
 * values enter through a vector b(t) (F = ... - b). An optional shunt conductance on every unknown
 * supports gmin stepping, the operating-point continuation of the reference's nonlinear solver.
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
  double gshunt; /* conductance from every unknown to ground (gmin stepping); 0 for none */
} xd_tia_coef;

/* Uploads the CSR pattern (rows = unknowns). */
int xd_tia_create(const xd_csr *pattern, int cuda_device, xd_tia **out);
int xd_tia_destroy(xd_tia *t);

/* Per row i, in one pass over the row's entries k:
 *   jac[k]   = qscale (dqdx[k] + lin_dqdx[k]) + fscale (dfdx[k] + lin_dfdx[k] + gshunt [k diagonal])
 *   F_i      = f[i] + sum_k lin_dfdx[k] x[col k] + gshunt x[i] - b[i]
 *   Q_i      = q[i] + sum_k lin_dqdx[k] x[col k]
 *   rhs[i]   as above (limiter corrections dfdxdvp / dqdxdvp, when non-null, added last);
 *   f_tot[i] = F_i and q_tot[i] = Q_i when those pointers are non-null.
 * dfdx / dqdx / f / q hold the nonlinear devices' loads (for instance from xd_load_assign);
 * lin_* may be null (no linear devices), b may be null (no sources); in mode 0 dqdx, lin_dqdx,
 * qn0 and fhist are not read. Row sums use a fixed lane split and a fixed reduction tree, so the
 * results are bit-identical from run to run. */
int xd_tia_combine(xd_tia *t, const xd_tia_coef *coef, const double *d_x, const double *d_dfdx,
                   const double *d_dqdx, const double *d_lin_dfdx, const double *d_lin_dqdx,
                   const double *d_f, const double *d_q, const double *d_dfdxdvp, const double *d_dqdxdvp,
                   const double *d_b, const double *d_qn0, const double *d_fhist, double *d_jac,
                   double *d_rhs, double *d_q_tot, double *d_f_tot, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* XYCE_TIA_H */
