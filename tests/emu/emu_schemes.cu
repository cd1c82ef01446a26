// emu_schemes.cu -- CPU check of the time schemes' point arithmetic.
//
// Compiled by nvcc as a host program: scheme_increment and scheme_rhs of
// moons_b200/csrc/schemes.cuh, with the wall mask between them (as k_ab2_rhs
// runs them), are compared bit for bit with the reference's whole-array
// sequences restated with the oracle's primitives
// (time_marching_methods.f90:70-73, :104-108, :137-142, :217-222, :289-292;
// time_marching_methods_SF.f90:61-65, :91-94, :121-125) on face fields with
// Dirichlet walls (so assign_wall_Dirichlet zeroes boundary points) and on a
// cell-centred field, for every form.  Prints one line per case and exits
// non-zero on a mismatch.
#include <cstdio>
#include <random>
#include <vector>

#include "../../moons_b200/csrc/schemes.cuh"
#include "../../oracle/moons_oracle.hpp"

static std::vector<double> nodes(int n, double a, double b) {
  std::vector<double> h;
  const double dh = (b - a) / n;
  for (int i = -1; i <= n + 1; i++) h.push_back(a + i * dh * (1.0 + 0.01 * (i % 3)));
  return h;
}

int main() {
  mo::Grid g;
  const int n[3] = {5, 6, 7};
  std::vector<double> hs[3];
  for (int d = 0; d < 3; d++) {
    hs[d] = nodes(n[d], 0.0, 1.0 + d);
    g.c[d].init(hs[d].data(), (int)hs[d].size());
  }
  std::mt19937_64 rng(7);
  std::normal_distribution<double> nd(0.0, 1.0);
  const double dt = 1.3e-3, gam = 5.0 / 12.0, zeta = -17.0 / 60.0, alpha = 1.0 / 15.0;
  const double two_thirds = 2.0 / 3.0, four_thirds = 4.0 / 3.0, neg_one_third = -1.0 / 3.0;
  const int type[6] = {1, 1, 1, 1, 1, 1}, pres[6] = {0, 0, 0, 0, 0, 0}, order[6] = {1, 2, 3, 4, 5, 6};
  const double val[6] = {0, 0, 0, 0, 0, 0}, cw[6] = {0, 0, 0, 0, 0, 0};
  int fails = 0;
  for (int dl : {0, 1, 2, 3}) {  // CC, faces x/y/z
    mo::SF F, Fm, L, X, Xnm1, t, ones;
    for (mo::SF* f : {&F, &Fm, &L, &X, &Xnm1, &t, &ones}) f->init(g, dl);
    mo::set_bcs(X, g, type, pres, val, cw, order);
    for (mo::SF* f : {&F, &Fm, &L, &X, &Xnm1})
      for (size_t i = 0; i < f->n(); i++) f->f[i] = nd(rng);
    mo::assign(ones, 1.0);
    mo::assign_wall_Dirichlet(ones, 0.0, &X);
    size_t walls = 0;
    for (size_t i = 0; i < ones.n(); i++) walls += ones.f[i] == 0.0;
    // (form, a0, a1, a2, name): form 8 twice, with the VF (2 alpha) and SF (alpha) weights
    struct Case {
      int form;
      double a2;
      const char* name;
    };
    const Case cases[] = {{mg::kFormAB2, 0, "AB2"},       {mg::kFormEuler, 0, "Euler"},
                          {mg::kFormAB2L, 0, "AB2+L"},    {mg::kFormBDF2, 0, "BDF2"},
                          {mg::kFormRK, dt * 2.0 * alpha, "RK (VF)"}, {mg::kFormRK, dt * alpha, "RK (SF)"}};
    for (const Case& c : cases) {
      // the reference's sequence with the oracle's primitives
      switch (c.form) {
        case mg::kFormEuler:
          mo::assign(t, F);
          mo::multiply(t, dt);
          break;
        case mg::kFormRK:
          for (size_t i = 0; i < t.n(); i++) t.f[i] = F.f[i] * (dt * gam);
          mo::add_product(t, Fm, dt * zeta);
          mo::add_product(t, L, c.a2);
          break;
        default:  // AB2 (AB2.f90:53-64), then + L, then the time factor
          for (size_t i = 0; i < t.n(); i++) t.f[i] = F.f[i] * 1.5;
          mo::add_product(t, Fm, -0.5);
          if (c.form == mg::kFormAB2L) mo::add(t, L);
          mo::multiply(t, c.form == mg::kFormBDF2 ? two_thirds * dt : dt);
      }
      mo::assign_wall_Dirichlet(t, 0.0, &X);
      if (c.form == mg::kFormBDF2) {
        mo::add_product(t, X, four_thirds);
        mo::add_product(t, Xnm1, neg_one_third);
      } else {
        mo::add(t, X);
      }
      // the point functions with the wall mask between them
      const double dts = c.form == mg::kFormBDF2 ? (2.0 / 3.0) * dt : dt;
      size_t bad = 0;
      for (size_t i = 0; i < t.n(); i++) {
        double v = mg::scheme_increment(c.form, F.f[i], Fm.f[i], L.f[i], dts, dt * gam, dt * zeta, c.a2);
        if (ones.f[i] == 0.0) v = 0.0;
        v = mg::scheme_rhs(c.form, v, X.f[i], Xnm1.f[i]);
        bad += !(v == t.f[i]);
      }
      std::printf("dl %d %-8s points %zu walls %zu mismatches %zu\n", dl, c.name, t.n(), walls, bad);
      fails += bad != 0;
      if (dl != 0 && walls == 0) {
        std::printf("dl %d: no wall points to mask\n", dl);
        fails++;
      }
    }
  }
  if (!fails) std::printf("ALL OK\n");
  return fails ? 1 : 0;
}
