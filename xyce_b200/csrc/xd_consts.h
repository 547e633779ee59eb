// Physical constants, clamped exponentials and Newton voltage limiters shared by the host set-up
// and the device kernels. Values are the ones the reference device layer uses
// (src/DeviceModelPKG/Core/include/N_DEV_Const.h:50-114; the BSIM4-local definitions in
// src/DeviceModelPKG/OpenModels/src/N_DEV_MOSFET_B4.C:86-137); the limiters restate
// DeviceSupport::limvds / pnjlim / fetlim (src/DeviceModelPKG/Core/src/N_DEV_DeviceSupport.C:186-420).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define XD_HD __host__ __device__ __forceinline__
#else
#define XD_HD inline
#endif

namespace xdc {

constexpr double CONSTQ = 1.6021918e-19;
constexpr double CONSTCtoK = 273.15;
constexpr double CONSTboltz = 1.3806226e-23;
constexpr double CONSTREFTEMP = 300.15;
constexpr double CONSTKoverQ = CONSTboltz / CONSTQ;
constexpr double CONSTvt0 = CONSTboltz * (27.0 + CONSTCtoK) / CONSTQ;
constexpr double CONSTroot2 = 1.4142135623730951;  // sqrt(2.0), correctly rounded
constexpr int CONSTNMOS = 1;
constexpr int CONSTPMOS = -1;
constexpr double CONSTEPSOX = 3.453133e-11;
constexpr double CONSTEPSSI = 1.03594e-10;
constexpr double CONSTEXP_THRESHOLD = 34.0;
constexpr double CONSTMAX_EXP = 5.834617425e14;
constexpr double CONSTMIN_EXP = 1.713908431e-15;
constexpr double CONSTMAX_EXP_ARG = 100.0;
constexpr double CONSTDELTA_1 = 0.02;
constexpr double CONSTDELTA_3 = 0.02;
constexpr double CONSTDELTA_4 = 0.02;
// BSIM4-local constants.
constexpr double CONSTEPS0 = 8.85418e-12;
constexpr double Charge_q = 1.60219e-19;
constexpr double CONSTKboQ = 8.617087e-5;
constexpr double CONSTMM = 3.0;
constexpr double DELTA = 1.0E-9;
// 2 * 10^-digits10(double): the limiter's "did limiting change anything" threshold.
constexpr double kMachPrec = 2.0e-15;

// Exponential clamped above and below, with its derivative (B4.C DEXP).
XD_HD void dexp(double A, double &B, double &C) {
  if (A > CONSTEXP_THRESHOLD) {
    B = CONSTMAX_EXP * (1.0 + (A)-CONSTEXP_THRESHOLD);
    C = CONSTMAX_EXP;
  } else if (A < -CONSTEXP_THRESHOLD) {
    B = CONSTMIN_EXP;
    C = 0;
  } else {
    B = exp(A);
    C = B;
  }
}

XD_HD void dexp2(double A, double &B) {
  if (A > CONSTEXP_THRESHOLD) {
    B = CONSTMAX_EXP * (1.0 + (A)-CONSTEXP_THRESHOLD);
  } else if (A < -CONSTEXP_THRESHOLD) {
    B = CONSTMIN_EXP;
  } else {
    B = exp(A);
  }
}

XD_HD double dmin(double a, double b) { return a < b ? a : b; }
XD_HD double dmax(double a, double b) { return a > b ? a : b; }

// Drain-source voltage step limiter.
XD_HD double limvds(double vnew, double vold) {
  if (vold >= 3.5) {
    if (vnew > vold)
      vnew = dmin(vnew, (3.0 * vold) + 2.0);
    else if (vnew < 3.5)
      vnew = dmax(vnew, 2.0);
  } else {
    if (vnew > vold)
      vnew = dmin(vnew, 4.0);
    else
      vnew = dmax(vnew, -0.5);
  }
  return vnew;
}

// pn-junction voltage step limiter; *icheck = 1 when it limited.
XD_HD double pnjlim(double vnew, double vold, double vt, double vcrit, int *icheck) {
  if ((vnew > vcrit) && (fabs(vnew - vold) > (vt + vt))) {
    if (vold > 0) {
      double arg = 1 + (vnew - vold) / vt;
      if (arg > 0)
        vnew = vold + vt * log(arg);
      else
        vnew = vcrit;
    } else {
      vnew = vt * log(vnew / vt);
    }
    *icheck = 1;
  } else {
    *icheck = 0;
  }
  return vnew;
}

// Gate-source voltage step limiter around the threshold vto.
XD_HD double fetlim(double vnew, double vold, double vto) {
  const double vtsthi = fabs(2 * (vold - vto)) + 2;
  const double vtstlo = vtsthi / 2 + 2;
  const double vtox = vto + 3.5;
  const double delv = vnew - vold;
  if (vold >= vto) {
    if (vold >= vtox) {
      if (delv <= 0) {
        if (vnew >= vtox) {
          if (-delv > vtstlo) vnew = vold - vtstlo;
        } else {
          vnew = dmax(vnew, vto + 2.0);
        }
      } else {
        if (delv >= vtsthi) vnew = vold + vtsthi;
      }
    } else {
      if (delv <= 0)
        vnew = dmax(vnew, vto - 0.5);
      else
        vnew = dmin(vnew, vto + 4.0);
    }
  } else {
    if (delv <= 0) {
      if (-delv > vtsthi) vnew = vold - vtsthi;
    } else {
      const double vtemp = vto + 0.5;
      if (vnew <= vtemp) {
        if (delv > vtstlo) vnew = vold + vtstlo;
      } else {
        vnew = vtemp;
      }
    }
  }
  return vnew;
}

}  // namespace xdc
