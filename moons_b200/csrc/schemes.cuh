// schemes.cuh -- point arithmetic of the time schemes' predictor RHS.
//
// The reference builds each scheme's right-hand side as a chain of
// whole-array passes (time_marching_methods.f90, time_marching_methods_SF.f90);
// k_ab2_rhs does the same operations in the same order per point in one
// pass.  The arithmetic is split at the wall mask (assign_wall_Dirichlet
// zeroes the increment on wall-located points before X is added):
//   inc = scheme_increment(form, ...) ; inc = 0 on walls ;
//   t   = scheme_rhs(form, inc, X, Xnm1)
// Forms:
//  4 AB2:        inc = (F*1.5 + Fnm1*(-0.5)) * dts             t = inc + X
//  5 Euler:      inc = F * dts                                  t = inc + X
//  6 AB2 + L:    inc = (F*1.5 + Fnm1*(-0.5) + L) * dts          t = inc + X
//  7 BDF2:       inc = (F*1.5 + Fnm1*(-0.5)) * dts (dts = 2/3 dt)
//                t = inc + X*(4/3) + Xnm1*(-1/3)  (added left to right)
//  8 RK stage:   inc = F*a0 + Fnm1*a1 + L*a2                    t = inc + X
#pragma once
#include "core.cuh"

namespace mg {

enum { kFormAB2 = 4, kFormEuler = 5, kFormAB2L = 6, kFormBDF2 = 7, kFormRK = 8 };

MG_HD double scheme_increment(int form, double F, double Fm, double L, double dts, double a0, double a1,
                              double a2) {
  double v;
  if (form == kFormRK) {
    v = F * a0;
    v = v + Fm * a1;
    v = v + L * a2;
    return v;
  }
  if (form == kFormEuler) {
    v = F;
  } else {
    v = F * 1.5;
    v = v + Fm * (-0.5);
    if (form == kFormAB2L) v = v + L;
  }
  return v * dts;
}

MG_HD double scheme_rhs(int form, double inc, double X, double Xnm1) {
  double v = inc;
  if (form == kFormBDF2) {
    v = v + X * (4.0 / 3.0);
    v = v + Xnm1 * (-1.0 / 3.0);
  } else {
    v = v + X;
  }
  return v;
}

}  // namespace mg
