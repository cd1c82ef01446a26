// coeffs.hpp -- host-side 1-D stencil coefficients of one axis
// (HW/grid/coordinates_extend.f90:78-173 init_c, :506-523 init_stencils_c;
// HW/grid/derivative_stencils.f90:31-217; HW/grid/interpolation_stencils.f90:12-35).
// Arrays are 1-based: a[0] unused.  Built once per mesh and copied to HBM.
#pragma once
#include <algorithm>
#include <vector>

namespace mg {
namespace host {
struct HostCoord {
  int sn, sc;
  std::vector<double> hn, hc, dhn, dhc, cc2nD, cc2nU, n2ccD, n2ccU, thD, thU, diagC, diagN;
  std::vector<double> colCC_L[2], colCC_D[2], colCC_U[2], colN_L[2], colN_D[2], colN_U[2];
};

inline void build_col(std::vector<double>& L, std::vector<double>& D, std::vector<double>& U,
               const std::vector<double>& dh, int s, bool cc, int order) {
  int n = std::max(s - 2, 1);
  L.assign(n + 1, 0.0);
  D.assign(n + 1, 0.0);
  U.assign(n + 1, 0.0);
  if (cc ? s <= 2 : s <= 3) return;
  auto h = [&](int i) { return dh[i]; };
  if (order == 2) {
    if (cc) {
      double a = 0.5 * h(1);
      L[1] = 2.0 / (a * (a + h(2)));
      D[1] = -2.0 / (a * h(2));
      U[1] = 2.0 / (h(2) * (a + h(2)));
    } else {
      L[1] = 2.0 / (h(2) * (h(3) + h(2)));
      D[1] = -2.0 / (h(3) * h(2));
      U[1] = 2.0 / (h(3) * (h(3) + h(2)));
    }
    for (int i = 3; i <= s - 2; i++) {
      L[i - 1] = 2.0 / (h(i - 1) * (h(i - 1) + h(i)));
      D[i - 1] = cc ? -(2.0 / (h(i - 1) * h(i))) : -2.0 / (h(i - 1) * h(i));
      U[i - 1] = 2.0 / (h(i) * (h(i - 1) + h(i)));
    }
    int i = s - 1;
    if (cc) {
      double b = 0.5 * h(i);
      L[s - 2] = 2.0 / (h(i - 1) * (h(i - 1) + b));
      D[s - 2] = -2.0 / (h(i - 1) * b);
      U[s - 2] = 2.0 / (b * (h(i - 1) + b));
    } else {
      L[s - 2] = 2.0 / (h(i - 2) * (h(i - 1) + h(i - 2)));
      D[s - 2] = -2.0 / (h(i - 1) * h(i - 2));
      U[s - 2] = 2.0 / (h(i - 1) * (h(i - 1) + h(i - 2)));
    }
  } else {
    if (cc) {
      double a = 0.5 * h(1);
      L[1] = (-(h(2)) / (a * (a + h(2))));
      D[1] = ((-a + h(2)) / (a * h(2)));
      U[1] = (a / (h(2) * (a + h(2))));
    } else {
      L[1] = -(h(3) + 2.0 * h(2)) / (h(2) * (h(3) + h(2)));
      D[1] = (h(3) + h(2)) / (h(3) * h(2));
      U[1] = -h(2) / (h(3) * (h(3) + h(2)));
    }
    for (int i = 3; i <= s - 2; i++) {
      L[i - 1] = cc ? (-h(i) / (h(i - 1) * (h(i - 1) + h(i)))) : -((h(i) / (h(i - 1) * (h(i - 1) + h(i)))));
      D[i - 1] = ((-h(i - 1) + h(i)) / (h(i - 1) * h(i)));
      U[i - 1] = (h(i - 1) / (h(i) * (h(i - 1) + h(i))));
    }
    int i = s - 1;
    if (cc) {
      double b = 0.5 * h(i);
      L[s - 2] = (-b / (h(i - 1) * (h(i - 1) + b)));
      D[s - 2] = ((-h(i - 1) + b) / (h(i - 1) * b));
      U[s - 2] = (h(i - 1) / (b * (h(i - 1) + b)));
    } else {
      L[s - 2] = h(i - 1) / (h(i - 2) * (h(i - 1) + h(i - 2)));
      D[s - 2] = -(h(i - 1) + h(i - 2)) / (h(i - 1) * h(i - 2));
      U[s - 2] = (2.0 * h(i - 1) + h(i - 2)) / (h(i - 1) * (h(i - 1) + h(i - 2)));
    }
  }
}

inline HostCoord build_coord(const double* h, int sn) {
  HostCoord c;
  c.sn = sn;
  c.sc = sn - 1;
  c.hn.assign(sn + 1, 0.0);
  for (int i = 1; i <= sn; i++) c.hn[i] = h[i - 1];
  c.dhn.assign(sn, 0.0);
  for (int i = 1; i <= sn - 1; i++) c.dhn[i] = c.hn[i + 1] - c.hn[i];
  c.hc.assign(c.sc + 1, 0.0);
  for (int i = 1; i <= sn - 1; i++) c.hc[i] = (c.hn[i + 1] + c.hn[i]) / 2.0;
  c.dhc.assign(c.sc, 0.0);
  for (int i = 1; i <= c.sc - 1; i++) c.dhc[i] = c.hc[i + 1] - c.hc[i];
  c.cc2nD.assign(c.sc, 0.0);
  c.cc2nU.assign(c.sc, 0.0);
  for (int i = 1; i <= c.sc - 1; i++) {
    c.cc2nD[i] = -(1.0 / c.dhc[i]);
    c.cc2nU[i] = 1.0 / c.dhc[i];
  }
  c.n2ccD.assign(sn, 0.0);
  c.n2ccU.assign(sn, 0.0);
  for (int i = 1; i <= sn - 1; i++) {
    c.n2ccD[i] = -(1.0 / c.dhn[i]);
    c.n2ccU[i] = 1.0 / c.dhn[i];
  }
  c.thD.assign(c.sc, 0.0);
  c.thU.assign(c.sc, 0.0);
  for (int i = 1; i <= c.sc - 1; i++) {
    c.thD[i] = (c.hn[i + 1] - c.hc[i]) / (c.hc[i + 1] - c.hc[i]);
    c.thU[i] = 1.0 - c.thD[i];
  }
  for (int o = 1; o <= 2; o++) {
    build_col(c.colCC_L[o - 1], c.colCC_D[o - 1], c.colCC_U[o - 1], c.dhc, c.sc, true, o);
    build_col(c.colN_L[o - 1], c.colN_D[o - 1], c.colN_U[o - 1], c.dhn, c.sn, false, o);
  }
  // per-axis share of laplacian_diagonal (GF_diagonals.f90:15-35)
  c.diagC.assign(c.sc + 1, 0.0);
  for (int i = 2; i <= c.sc - 1; i++) c.diagC[i] = c.n2ccD[i] * c.cc2nU[i - 1] + c.n2ccU[i] * c.cc2nD[i];
  c.diagN.assign(c.sn + 1, 0.0);
  for (int i = 2; i <= c.sn - 1; i++) c.diagN[i] = c.n2ccD[i] * c.cc2nU[i - 1] + c.n2ccU[i - 1] * c.cc2nD[i - 1];
  return c;
}
}  // namespace host
}  // namespace mg
