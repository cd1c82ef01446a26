// emu_fused.cu -- CPU check of the fused PCG kernels' point math.
//
// Compiled by nvcc as a host program: the __host__ __device__ point functions
// of moons_b200/csrc/fused.cuh run on the CPU and are compared, point by
// point, with the oracle's sequence apply_BCs_implicit -> operator ->
// wall masks -> *vol (PCG_solver_algorithm.f90:70-76) on small stretched
// meshes, for every operator and many BC combinations.  Prints one line per
// case and exits non-zero on the first mismatch.
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

#include "../../moons_b200/csrc/coeffs.hpp"
#include "../../moons_b200/csrc/fused.cuh"
#include "../../oracle/moons_oracle.hpp"

using namespace mg;

struct HGrid {
  host::HostCoord hc[3];
  DGrid dg;
  mo::Grid og;
  int sn[3];
};

static std::vector<double> roberts(double a, double b, int n, double beta) {
  double al = 0.5, g = (beta + 1) / (beta - 1);
  std::vector<double> h(n + 1);
  for (int i = 0; i <= n; i++) {
    double x = double(i) / n, e = std::pow(g, (x - al) / (1 - al));
    h[i] = a + (b - a) * (((beta + 2 * al) * e - beta + 2 * al) / ((2 * al + 1) * (1 + e)));
  }
  std::vector<double> o;
  o.push_back(h[0] - (h[1] - h[0]));
  for (double v : h) o.push_back(v);
  o.push_back(h[n] + (h[n] - h[n - 1]));
  return o;
}

static void make_grid(HGrid& G, int nx, int ny, int nz) {
  std::vector<double> hs[3] = {roberts(0, 1, nx, 1.05), roberts(0, 2, ny, 1.2), roberts(-1, 1, nz, 1.1)};
  for (int d = 0; d < 3; d++) {
    G.sn[d] = (int)hs[d].size();
    G.hc[d] = host::build_coord(hs[d].data(), G.sn[d]);
    G.og.c[d].init(hs[d].data(), G.sn[d]);
    host::HostCoord& c = G.hc[d];
    DCoord& dc = G.dg.c[d];
    dc.sn = c.sn;
    dc.sc = c.sc;
    dc.hn = c.hn.data(); dc.hc = c.hc.data(); dc.dhn = c.dhn.data(); dc.dhc = c.dhc.data();
    dc.cc2nD = c.cc2nD.data(); dc.cc2nU = c.cc2nU.data(); dc.n2ccD = c.n2ccD.data(); dc.n2ccU = c.n2ccU.data();
    dc.thD = c.thD.data(); dc.thU = c.thU.data();
    dc.diagC = c.diagC.data(); dc.diagN = c.diagN.data();
    for (int o = 0; o < 2; o++) {
      dc.colCC_L[o] = c.colCC_L[o].data(); dc.colCC_D[o] = c.colCC_D[o].data(); dc.colCC_U[o] = c.colCC_U[o].data();
      dc.colN_L[o] = c.colN_L[o].data(); dc.colN_D[o] = c.colN_D[o].data(); dc.colN_U[o] = c.colN_U[o].data();
    }
  }
}

static DBC dbc_of(const mo::SF& f) {
  DBC b{};
  b.defined = 1;
  for (int face = 1; face <= 6; face++) {
    b.type[face] = f.bc->type[face];
    b.prescribed[face] = f.bc->prescribed[face];
    b.value[face] = f.bc->value[face];
    b.c_w[face] = f.bc->c_w[face];
    b.dh[face] = f.bc->dh[face];
    b.nhat[face] = f.bc->nhat[face];
    b.order[face] = f.bc->order[face];
  }
  return b;
}
static DF df_of(mo::SF& f) {
  DF d{};
  d.f = f.f.data();
  d.s0 = f.s[1];
  d.s1 = f.s[2];
  d.s2 = f.s[3];
  d.dl = f.dl;
  return d;
}

static int fails = 0;
static double compare(const char* name, mo::SF& ref, std::vector<double>& got, double dot_ref, double dot_got) {
  double mx = 1e-300, err = 0;
  for (size_t i = 0; i < ref.n(); i++) mx = std::max(mx, std::fabs(ref.f[i]));
  size_t worst = 0;
  for (size_t i = 0; i < ref.n(); i++) {
    double e = std::fabs(ref.f[i] - got[i]);
    if (e > err) {
      err = e;
      worst = i;
    }
  }
  double rel = err / mx;
  double drel = std::fabs(dot_ref - dot_got) / std::max(std::fabs(dot_ref), 1e-300);
  bool ok = rel < 1e-12 && drel < 1e-11;
  int i = (int)(worst % ref.s[1]) + 1, j = (int)((worst / ref.s[1]) % ref.s[2]) + 1,
      k = (int)(worst / ((size_t)ref.s[1] * ref.s[2])) + 1;
  printf("%-52s rel %.2e dot %.2e %s (worst at %d,%d,%d of %dx%dx%d: ref %.6e got %.6e)\n", name, rel, drel,
         ok ? "ok" : "MISMATCH", i, j, k, ref.s[1], ref.s[2], ref.s[3], ref.f[worst], got[worst]);
  if (!ok) fails++;
  return rel;
}

// oracle: apply_BCs_implicit, op, masks, vol ; dot(p~, Ap) with Dirichlet walls of x dropped
static double oracle_dot(const std::vector<mo::SF*>& p, const std::vector<mo::SF*>& A) {
  double d = 0;
  for (size_t c = 0; c < p.size(); c++) {
    mo::SF t = *A[c];
    mo::multiply(t, *p[c]);
    mo::assign_wall_Dirichlet(t, 0.0, p[c]);
    d += mo::sum_pad(t, 1);
  }
  return d;
}
static void oracle_mask_vol(mo::SF& A, const mo::SF& x, const mo::Grid& g) {
  mo::multiply_wall_Neumann(A, 0.5, &x);
  mo::assign_wall_Dirichlet(A, 0.0, &x);
  mo::assign_wall_Periodic_single(A, 0.0, &x);
  mo::SF v;
  v.init(g, A.dl);
  mo::volume(v, g);
  mo::multiply(A, v);
}

int main() {
  HGrid G;
  make_grid(G, 9, 7, 8);
  std::mt19937_64 rng(7);
  std::normal_distribution<double> nd(0.0, 1.0);
  const int D = mo::BC_DIRICHLET, N = mo::BC_NEUMANN, P = mo::BC_PERIODIC, R = mo::BC_ROBIN;
  std::vector<std::array<int, 6>> sets = {{N, N, N, N, N, N}, {D, D, D, D, D, D}, {N, N, N, N, P, P},
                                          {D, D, D, D, P, P}, {P, P, D, N, N, D}, {R, R, N, D, P, P},
                                          {D, N, R, R, D, N}};
  int order[6] = {5, 6, 1, 2, 3, 4};
  double cw[6] = {0.7, 1.3, 0.4, 2.0, 0.9, 1.1};
  char name[128];
  for (auto& st : sets) {
    int types[6];
    for (int f = 0; f < 6; f++) types[f] = st[f];
    // ---- scalar CC: LAP_UNIFORM (0) and LAP_PROPS (1)
    for (int mode = 0; mode <= 1; mode++) {
      mo::SF p, A, kf[3];
      p.init(G.og, 0);
      A.init(G.og, 0);
      mo::set_bcs(p, G.og, types, nullptr, nullptr, cw, order);
      for (auto& v : p.f) v = nd(rng);
      for (int d = 0; d < 3; d++) {
        kf[d].init(G.og, 1 + d);
        for (auto& v : kf[d].f) v = std::exp(nd(rng));
      }
      mo::SF praw = p;
      mo::apply_BCs_implicit(p);
      if (mode == 0) mo::lap_centered(A, p, G.og);
      else mo::lap_var(A, p, kf[0], kf[1], kf[2], G.og);
      oracle_mask_vol(A, p, G.og);
      double dref = oracle_dot({&p}, {&A});
      DBC b = dbc_of(p);
      int ext[4] = {0, p.s[1], p.s[2], p.s[3]};
      FBC fb = make_fbc(b, b, 0, ext);
      DF pd = df_of(praw), Ad{}, kx = df_of(kf[0]), ky = df_of(kf[1]), kz = df_of(kf[2]);
      Ad.s0 = A.s[1]; Ad.s1 = A.s[2]; Ad.s2 = A.s[3]; Ad.dl = 0;
      std::vector<double> got(A.n());
      double dgot = 0;
      for (int k = 1; k <= A.s[3]; k++)
        for (int j = 1; j <= A.s[2]; j++)
          for (int i = 1; i <= A.s[1]; i++) {
            double v, acc;
            if (mode == 0) lap_ap_point<0>(Ad, pd, fb, G.dg, kx, ky, kz, 0.0, i, j, k, v, acc);
            else lap_ap_point<1>(Ad, pd, fb, G.dg, kx, ky, kz, 0.0, i, j, k, v, acc);
            got[Ad.at(i, j, k)] = v;
            dgot += acc;
          }
      snprintf(name, sizeof name, "CC %s bc %d%d%d%d%d%d", mode ? "lap_props" : "lap_uniform", types[0], types[1],
               types[2], types[3], types[4], types[5]);
      compare(name, A, got, dref, dgot);
    }
    // ---- faces: MOM_DIFFUSION (per component) and IND_DIFFUSION (all three)
    mo::SF U[3], Ur[3], Am[3];
    for (int c = 0; c < 3; c++) {
      U[c].init(G.og, 1 + c);
      Am[c].init(G.og, 1 + c);
      // pseudo-vacuum style: the component normal to a face pair gets Neumann
      // there when the set is Dirichlet on that pair (different BCs per component)
      int tc[6];
      for (int f = 0; f < 6; f++) tc[f] = types[f];
      if (types[2 * c] == D && types[2 * c + 1] == D) tc[2 * c] = tc[2 * c + 1] = N;
      mo::set_bcs(U[c], G.og, tc, nullptr, nullptr, cw, order);
      for (auto& v : U[c].f) v = nd(rng);
      Ur[c] = U[c];
    }
    double coeff = -0.37;
    for (int c = 0; c < 3; c++) {
      mo::SF p = Ur[c];
      mo::apply_BCs_implicit(p);
      mo::lap_centered(Am[c], p, G.og);
      mo::multiply(Am[c], coeff);
      mo::add(Am[c], p);
      oracle_mask_vol(Am[c], p, G.og);
      double dref = oracle_dot({&p}, {&Am[c]});
      DBC b = dbc_of(p);
      int ext[4] = {0, p.s[1], p.s[2], p.s[3]};
      FBC fb = make_fbc(b, b, p.dl, ext);
      DF pd = df_of(Ur[c]), Ad{}, z{};
      Ad.s0 = Am[c].s[1]; Ad.s1 = Am[c].s[2]; Ad.s2 = Am[c].s[3]; Ad.dl = p.dl;
      std::vector<double> got(Am[c].n());
      double dgot = 0;
      for (int k = 1; k <= Ad.s2; k++)
        for (int j = 1; j <= Ad.s1; j++)
          for (int i = 1; i <= Ad.s0; i++) {
            double v, acc;
            lap_ap_point<2>(Ad, pd, fb, G.dg, z, z, z, coeff, i, j, k, v, acc);
            got[Ad.at(i, j, k)] = v;
            dgot += acc;
          }
      snprintf(name, sizeof name, "face%d mom_diffusion bc %d%d%d%d%d%d", c, types[0], types[1], types[2], types[3],
               types[4], types[5]);
      compare(name, Am[c], got, dref, dgot);
    }
    {
      mo::SF p[3], sig[3], t[3], A[3];
      for (int c = 0; c < 3; c++) {
        p[c] = Ur[c];
        mo::apply_BCs_implicit(p[c]);
        sig[c].init(G.og, 4 + c);
        for (auto& v : sig[c].f) v = std::exp(nd(rng));
        t[c].init(G.og, 4 + c);
        A[c].init(G.og, 1 + c);
      }
      mo::curl(t[0], t[1], t[2], p[0], p[1], p[2], G.og);
      for (int c = 0; c < 3; c++) mo::multiply(t[c], sig[c]);
      mo::curl(A[0], A[1], A[2], t[0], t[1], t[2], G.og);
      for (int c = 0; c < 3; c++) {
        mo::multiply(A[c], coeff);
        mo::add(A[c], p[c]);
        oracle_mask_vol(A[c], p[c], G.og);
      }
      // fused: E on edges then Ap
      FBC fb[3];
      DF pd[3], E[3], S[3];
      std::vector<double> Eh[3];
      for (int c = 0; c < 3; c++) {
        DBC b = dbc_of(p[c]);
        int ext[4] = {0, p[c].s[1], p[c].s[2], p[c].s[3]};
        fb[c] = make_fbc(b, b, p[c].dl, ext);
        pd[c] = df_of(Ur[c]);
        Eh[c].assign(t[c].n(), 0.0);
        E[c] = df_of(t[c]);
        E[c].f = Eh[c].data();
        S[c] = df_of(sig[c]);
      }
      for (int l = 0; l < 3; l++)
        for (int k = 1; k <= E[l].s2; k++)
          for (int j = 1; j <= E[l].s1; j++)
            for (int i = 1; i <= E[l].s0; i++) {
              double v;
              if (l == 0) v = curl_sig_point<0>(E[0], pd[2], fb[2], pd[1], fb[1], S[0], G.dg, i, j, k);
              else if (l == 1) v = curl_sig_point<1>(E[1], pd[0], fb[0], pd[2], fb[2], S[1], G.dg, i, j, k);
              else v = curl_sig_point<2>(E[2], pd[1], fb[1], pd[0], fb[0], S[2], G.dg, i, j, k);
              E[l](i, j, k) = v;
            }
      double dref = oracle_dot({&p[0], &p[1], &p[2]}, {&A[0], &A[1], &A[2]});
      double dgot = 0;
      std::vector<double> got[3];
      for (int c = 0; c < 3; c++) {
        DF Ad{};
        Ad.s0 = A[c].s[1]; Ad.s1 = A[c].s[2]; Ad.s2 = A[c].s[3]; Ad.dl = A[c].dl;
        got[c].assign(A[c].n(), 0.0);
        for (int k = 1; k <= Ad.s2; k++)
          for (int j = 1; j <= Ad.s1; j++)
            for (int i = 1; i <= Ad.s0; i++) {
              double v, acc;
              if (c == 0) curl_ap_point<0>(Ad, pd[0], fb[0], E[2], E[1], G.dg, coeff, i, j, k, v, acc);
              else if (c == 1) curl_ap_point<1>(Ad, pd[1], fb[1], E[0], E[2], G.dg, coeff, i, j, k, v, acc);
              else curl_ap_point<2>(Ad, pd[2], fb[2], E[1], E[0], G.dg, coeff, i, j, k, v, acc);
              got[c][Ad.at(i, j, k)] = v;
              dgot += acc;
            }
      }
      for (int c = 0; c < 3; c++) {
        snprintf(name, sizeof name, "face%d ind_diffusion bc %d%d%d%d%d%d", c, types[0], types[1], types[2],
                 types[3], types[4], types[5]);
        compare(name, A[c], got[c], c == 2 ? dref : 0.0, c == 2 ? dgot : 0.0);
      }
    }
  }
  printf("%s\n", fails ? "FAILED" : "ALL OK");
  return fails ? 1 : 0;
}
