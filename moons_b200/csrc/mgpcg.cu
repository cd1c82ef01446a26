// mgpcg.cu -- multigrid-preconditioned CG for cell-centred Poisson problems
// (MOONS_PREC_MG: FP64 V-cycle inside CG; MOONS_PREC_MG_MIXED: FP32 V-cycle
// inside an FP64 flexible CG).
//
// The outer iteration is the reference's PCG (PCG_solver_algorithm.f90:69-96)
// with z = Minv r replaced by z = V(r): the residual, the CG inner products,
// alpha/beta and the exit tests stay FP64 in both variants.  The mixed
// variant uses the flexible (Polak-Ribiere) beta = z.(r - r_prev) / rho, so
// the FP32 rounding inside the V-cycle cannot stall the recurrence.
// Supported: one CC unknown (pressure, potential) with LAP_UNIFORM or
// LAP_PROPS and Dirichlet / Neumann / periodic BCs.  Each level halves every
// axis with at least 4 interior cells (periodic axes: an even count) and
// keeps the others (semi-coarsening), until no axis can be halved: fine
// cells are merged in pairs from the low end; an odd count leaves its last
// fine cell as a coarse cell of its own.  An odd count on a periodic axis of
// the finest mesh works but weakens the smoother (same-colour neighbours
// across the seam).
#include <array>

#include "eig.hpp"
#include "mgrid.cuh"
#include "runtime.cuh"

using namespace mg;

// ---------------------------------------------------------------------------
// the hierarchy
// ---------------------------------------------------------------------------
struct MGHier {
  bool mixed = false;
  int nl = 0;
  int sweeps_coarse = 24;  // coarsest level without a dense inverse
  int nu = 2;              // red-black sweeps before and after the coarse correction
  double omega = 1.15;     // over-relaxation of the sweeps
  int nsm = 148;
  int occ[4] = {1, 1, 1, 1};  // resident blocks per SM: smooth, resid, restrict, prolong
  std::vector<std::array<int, 3>> s;  // CC extents per level
  std::vector<MGLev<double>> Ld;
  std::vector<MGLev<float>> Lf;
  std::vector<std::array<MGProl<double>, 3>> Pd;  // [l]: fine level l-1 from coarse level l
  std::vector<std::array<MGProl<float>, 3>> Pf;
  std::vector<std::array<MGRest<double>, 3>> Rd;
  std::vector<std::array<MGRest<float>, 3>> Rf;
  double* rprev = nullptr;  // flexible CG: previous residual
  std::vector<void*> rt1, rt2;  // separable restriction temporaries per coarse level (compact, level type)
  double* ts_part = nullptr;   // two-stage scaling: block partials of N.t, N.A N
  double* ts_gamma = nullptr;  // and the resulting multiple of N
  // coarsest level: dense inverse (direct solve) when small enough
  int ncoarse = 0;
  double* cinv_d = nullptr;  // coarsest-level inverse (FP64 for both variants)
  // MOONS_PREC_FD: fast diagonalization of the separable operator instead of
  // a V-cycle (interior extents, per-axis transforms and eigenvalues, two
  // interior-sized work arrays)
  bool fd = false;
  int fn[3] = {0, 0, 0};
  double *fwd[3] = {nullptr, nullptr, nullptr}, *bwd[3] = {nullptr, nullptr, nullptr};
  double* lam[3] = {nullptr, nullptr, nullptr};
  int zmode[3] = {-1, -1, -1};  // the constant mode's index per axis, all -1 if the operator is regular
  double *w0 = nullptr, *w1 = nullptr;
  std::vector<void*> allocs;
  ~MGHier() {
    for (void* p : allocs) cudaFree(p);
  }
};

namespace {

template <typename T>
T* dev_copy(MGHier* h, const std::vector<T>& v, cudaStream_t st) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(1, v.size()) * sizeof(T)) != cudaSuccess) return nullptr;
  h->allocs.push_back(p);
  if (!v.empty()) cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st);
  return (T*)p;
}
template <typename T>
T* dev_zeros(MGHier* h, size_t n, cudaStream_t st) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)) != cudaSuccess) return nullptr;
  h->allocs.push_back(p);
  cudaMemsetAsync(p, 0, std::max<size_t>(1, n) * sizeof(T), st);
  return (T*)p;
}
template <typename T>
std::vector<T> conv(const std::vector<double>& v) {
  return std::vector<T>(v.begin(), v.end());
}

// coarse node coordinates (with ghost nodes) keeping every other fine node
// from the first physical one, and the last physical node (an odd cell
// count leaves its last fine cell unpaired).  Ghost cells mirror the end
// cells, or on a periodic axis take the size of the periodic partner (the
// cell at the other end), so that both sides of the seam see the same
// centre distance and the coarse operator stays symmetric.
std::vector<double> coarsen_nodes(const std::vector<double>& hn, bool periodic) {
  const int sn = (int)hn.size();
  std::vector<double> c;
  c.push_back(0.0);
  int last = 0;
  for (int i = 1; i <= sn - 2; i += 2) {
    c.push_back(hn[i]);
    last = i;
  }
  if (last != sn - 2) c.push_back(hn[sn - 2]);
  c.push_back(0.0);
  const int m = (int)c.size();
  const double h_first = c[2] - c[1], h_last = c[m - 2] - c[m - 3];
  c[0] = c[1] - (periodic ? h_last : h_first);
  c[m - 1] = c[m - 2] + (periodic ? h_first : h_last);
  return c;
}

struct Axis1D {
  // prolongation of one axis (fine f = 1..scf, only 2..scf-1 used)
  std::vector<int> i0, i1;
  std::vector<double> w0, w1;
  // restriction = transpose, CSR over coarse I = 1..scc
  std::vector<int> off, fi;
  std::vector<double> fw;
};

// coarse index -> (interior index, sign) through the homogeneous BC of the face
void resolve(int& I, double& w, int scc, int tlo, int thi) {
  if (I == 1) {
    if (tlo == MOONS_BC_PERIODIC) I = scc - 1;
    else {
      I = 2;
      if (tlo == MOONS_BC_DIRICHLET) w = -w;
    }
  } else if (I == scc) {
    if (thi == MOONS_BC_PERIODIC) I = 2;
    else {
      I = scc - 1;
      if (thi == MOONS_BC_DIRICHLET) w = -w;
    }
  }
}

Axis1D build_axis(const host::HostCoord& cc, int scf, int tlo, int thi, bool coarsened) {
  Axis1D a;
  const int scc = cc.sc;
  a.i0.assign(scf + 1, 2);
  a.i1.assign(scf + 1, 2);
  a.w0.assign(scf + 1, 0.0);
  a.w1.assign(scf + 1, 0.0);
  std::vector<std::vector<std::pair<int, double>>> cols(scc + 1);
  for (int f = 2; f <= scf - 1 && !coarsened; f++) {  // axis kept: identity
    a.i0[f] = a.i1[f] = f;
    a.w0[f] = 1.0;
    cols[f].push_back({f, 1.0});
  }
  const bool odd = ((scf - 2) & 1) != 0;
  for (int f = 2; f <= scf - 1 && coarsened; f++) {
    const int I = (f + 2) / 2;
    if (odd && f == scf - 1) {  // unpaired last cell: same centre as its coarse cell
      a.i0[f] = a.i1[f] = I;
      a.w0[f] = 1.0;
      cols[I].push_back({f, 1.0});
      continue;
    }
    int nb;
    double wp, wn;
    if ((f & 1) == 0) {  // left child: face I-1|I
      wp = 0.5 + 0.5 * cc.thD[I - 1];
      wn = 0.5 * cc.thU[I - 1];
      nb = I - 1;
    } else {  // right child: face I|I+1
      wp = 0.5 + 0.5 * cc.thU[I];
      wn = 0.5 * cc.thD[I];
      nb = I + 1;
    }
    resolve(nb, wn, scc, tlo, thi);
    a.i0[f] = I;
    a.w0[f] = wp;
    a.i1[f] = nb;
    a.w1[f] = wn;
    cols[I].push_back({f, wp});
    cols[nb].push_back({f, wn});
  }
  a.off.assign(scc + 2, 0);
  for (int I = 1; I <= scc; I++) {
    a.off[I + 1] = a.off[I] + (int)cols[I].size();
    for (auto& e : cols[I]) {
      a.fi.push_back(e.first);
      a.fw.push_back(e.second);
    }
  }
  a.off[0] = 0;
  return a;
}

template <typename T>
MGAxis<T> axis_tables(MGHier* h, const host::HostCoord& c, cudaStream_t st) {
  MGAxis<T> a{};
  a.cD = dev_copy(h, conv<T>(c.cc2nD), st);
  a.cU = dev_copy(h, conv<T>(c.cc2nU), st);
  a.nD = dev_copy(h, conv<T>(c.n2ccD), st);
  a.nU = dev_copy(h, conv<T>(c.n2ccU), st);
  a.dg = dev_copy(h, conv<T>(c.diagC), st);
  a.hv = dev_copy(h, conv<T>(c.dhn), st);
  return a;
}

// face weights of axis d on a level (face array, x fastest): the volume-
// weighted operator's coupling across the face, W = vol * cc2nD[t-1] * k *
// n2ccD[t] for the low face of cell t, and vol * cc2nU[t] * k * n2ccU[t] of
// the last cell for the top boundary face; (A e)(c) = sum_f W_f (e_nb - e_c)
std::vector<double> face_weights(const host::HostCoord* c, const std::array<int, 3>& s, int d,
                                 const std::vector<double>* K) {
  std::array<int, 3> e = s;
  e[d] += 1;
  std::vector<double> w((size_t)e[0] * e[1] * e[2], 0.0);
  auto fid = [&](int a, int b, int cc) { return (size_t)(a - 1) + (size_t)e[0] * ((b - 1) + (size_t)e[1] * (cc - 1)); };
  for (int k = 2; k <= s[2] - 1; k++)
    for (int j = 2; j <= s[1] - 1; j++)
      for (int i = 2; i <= s[0] - 1; i++) {
        const int ii[3] = {i, j, k};
        const int t = ii[d];
        const double vol = (c[0].dhn[i] * c[1].dhn[j]) * c[2].dhn[k];
        const size_t flo = fid(i, j, k);
        const double kl = K ? (*K)[flo] : 1.0;
        w[flo] = c[d].cc2nD[t - 1] * kl * c[d].n2ccD[t] * vol;
        if (t == s[d] - 1) {
          const size_t fhi = fid(i + (d == 0), j + (d == 1), k + (d == 2));
          const double kr = K ? (*K)[fhi] : 1.0;
          w[fhi] = c[d].cc2nU[t] * kr * c[d].n2ccU[t] * vol;
        }
      }
  return w;
}

// area-weighted mean of the fine faces covering each coarse face of axis d
std::vector<double> coarsen_faces(const std::vector<double>& kf, int d, const std::array<int, 3>& sf,
                                  const std::array<int, 3>& sc, const host::HostCoord* cf, const bool* cz) {
  std::array<int, 3> ef = sf, ec = sc;
  ef[d] += 1;
  ec[d] += 1;
  std::vector<double> kc((size_t)ec[0] * ec[1] * ec[2], 1.0);
  auto fid = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)ef[0] * ((j - 1) + (size_t)ef[1] * (k - 1)); };
  auto cid = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)ec[0] * ((j - 1) + (size_t)ec[1] * (k - 1)); };
  const int a = d == 0 ? 1 : 0, b = d == 2 ? 1 : 2;  // transverse axes
  for (int K = 1; K <= ec[2]; K++)
    for (int J = 1; J <= ec[1]; J++)
      for (int I = 1; I <= ec[0]; I++) {
        int C[3] = {I, J, K};
        // interior coarse cells along the transverse axes, physical nodes along d
        bool inner = true;
        for (int q = 0; q < 3; q++) {
          const int lo = 2, hi = q == d ? ec[q] - 1 : ec[q] - 1;
          if (C[q] < lo || C[q] > hi) inner = false;
        }
        if (!inner) continue;
        int F[3];
        // coincident fine node (the last physical node closes an unpaired cell)
        F[d] = cz[d] ? std::min(2 * C[d] - 2, ef[d] - 1) : C[d];
        double num = 0.0, den = 0.0;
        for (int u = 0; u < (cz[a] ? 2 : 1); u++)
          for (int v = 0; v < (cz[b] ? 2 : 1); v++) {
            F[a] = cz[a] ? 2 * C[a] - 2 + u : C[a];
            F[b] = cz[b] ? 2 * C[b] - 2 + v : C[b];
            if (F[a] > sf[a] - 1 || F[b] > sf[b] - 1) continue;  // no second child
            const double w = cf[a].dhn[F[a]] * cf[b].dhn[F[b]];
            num += w * kf[fid(F[0], F[1], F[2])];
            den += w;
          }
        kc[cid(I, J, K)] = num / den;
      }
  return kc;
}

// dense operator of one level over its interior cells (the same arithmetic
// as apply_A, with ghost neighbours resolved through the homogeneous BCs)
std::vector<double> dense_operator(const host::HostCoord* c, const std::array<int, 3>& s, const int* bt,
                                   const std::array<std::vector<double>, 3>* K) {
  const int nx = s[0] - 2, ny = s[1] - 2, nz = s[2] - 2;
  const int n = nx * ny * nz;
  std::vector<double> A((size_t)n * n, 0.0);
  auto row_of = [&](int i, int j, int k) { return (i - 2) + nx * ((j - 2) + ny * (k - 2)); };
  for (int k = 2; k <= s[2] - 1; k++)
    for (int j = 2; j <= s[1] - 1; j++)
      for (int i = 2; i <= s[0] - 1; i++) {
        const int row = row_of(i, j, k);
        const int ii[3] = {i, j, k};
        const double vol = (c[0].dhn[i] * c[1].dhn[j]) * c[2].dhn[k];
        for (int d = 0; d < 3; d++) {
          const int t = ii[d];
          double kl = 1.0, kr = 1.0;
          if (K) {
            std::array<int, 3> e = s;
            e[d] += 1;
            auto fid = [&](int a, int b, int cc) { return (size_t)(a - 1) + (size_t)e[0] * ((b - 1) + (size_t)e[1] * (cc - 1)); };
            int lo[3] = {i, j, k}, hi[3] = {i, j, k};
            hi[d] += 1;
            kl = (*K)[d][fid(lo[0], lo[1], lo[2])];
            kr = (*K)[d][fid(hi[0], hi[1], hi[2])];
          }
          const double cm = c[d].cc2nD[t - 1] * kl * c[d].n2ccD[t];
          const double c0 = c[d].cc2nU[t - 1] * kl * c[d].n2ccD[t] + c[d].cc2nD[t] * kr * c[d].n2ccU[t];
          const double cp = c[d].cc2nU[t] * kr * c[d].n2ccU[t];
          A[(size_t)row * n + row] += c0 * vol;
          for (int side = 0; side < 2; side++) {
            int nb[3] = {i, j, k};
            nb[d] += side == 0 ? -1 : 1;
            double w = (side == 0 ? cm : cp) * vol;
            if (nb[d] == 1) {
              if (bt[2 * d + 1] == MOONS_BC_PERIODIC) nb[d] = s[d] - 1;
              else {
                nb[d] = 2;
                if (bt[2 * d + 1] == MOONS_BC_DIRICHLET) w = -w;
              }
            } else if (nb[d] == s[d]) {
              if (bt[2 * d + 2] == MOONS_BC_PERIODIC) nb[d] = 2;
              else {
                nb[d] = s[d] - 1;
                if (bt[2 * d + 2] == MOONS_BC_DIRICHLET) w = -w;
              }
            }
            A[(size_t)row * n + row_of(nb[0], nb[1], nb[2])] += w;
          }
        }
      }
  return A;
}

// inverse by Gauss-Jordan with partial pivoting; false if singular
bool invert(std::vector<double> A, int n, std::vector<double>& inv) {
  inv.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) inv[(size_t)i * n + i] = 1.0;
  for (int col = 0; col < n; col++) {
    int piv = col;
    for (int r = col + 1; r < n; r++)
      if (std::fabs(A[(size_t)r * n + col]) > std::fabs(A[(size_t)piv * n + col])) piv = r;
    if (A[(size_t)piv * n + col] == 0.0) return false;
    if (piv != col)
      for (int c = 0; c < n; c++) {
        std::swap(A[(size_t)piv * n + c], A[(size_t)col * n + c]);
        std::swap(inv[(size_t)piv * n + c], inv[(size_t)col * n + c]);
      }
    const double d = 1.0 / A[(size_t)col * n + col];
    for (int c = 0; c < n; c++) {
      A[(size_t)col * n + c] *= d;
      inv[(size_t)col * n + c] *= d;
    }
    for (int r = 0; r < n; r++) {
      if (r == col) continue;
      const double f = A[(size_t)r * n + col];
      if (f == 0.0) continue;
      for (int c = 0; c < n; c++) {
        A[(size_t)r * n + c] -= f * A[(size_t)col * n + c];
        inv[(size_t)r * n + c] -= f * inv[(size_t)col * n + c];
      }
    }
  }
  return true;
}

}  // namespace

// build the hierarchy for a PCG object (CC, one component)
int mg_build(moons_pcg* s, moons_mesh* m, int mixed, const DBC& bc, const DF* kf, MGHier** out) {
  *out = nullptr;
  auto h = std::make_unique<MGHier>();
  h->mixed = mixed != 0;
  cudaStream_t st = m->stream;
  std::vector<host::HostCoord> C[3];
  std::array<int, 3> s0 = {m->sn[0] - 1, m->sn[1] - 1, m->sn[2] - 1};
  for (int d = 0; d < 3; d++) C[d].push_back(host::build_coord(m->hn[d].data(), m->sn[d]));
  h->s.push_back(s0);
  int bt[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int f = 1; f <= 6; f++) bt[f] = bc.defined ? bc.type[f] : MOONS_BC_NEUMANN;
  // each level halves every axis with at least 4 interior cells (the others
  // are kept), until no axis can be halved.  A periodic axis is halved only
  // while its count is even: on an odd periodic ring the red-black colouring
  // gives the two seam cells the same colour, so the sweeps would update
  // neighbours together there
  bool per[3];
  for (int d = 0; d < 3; d++) per[d] = bt[2 * d + 1] == MOONS_BC_PERIODIC || bt[2 * d + 2] == MOONS_BC_PERIODIC;
  std::vector<std::array<bool, 3>> coarsened(1, std::array<bool, 3>{false, false, false});
  for (;;) {
    const auto& sl = h->s.back();
    std::array<bool, 3> cz{};
    bool any = false;
    for (int d = 0; d < 3; d++) {
      const int N = sl[d] - 2;
      cz[d] = N >= 4 && (!per[d] || (N & 1) == 0);
      any = any || cz[d];
    }
    // small enough for the dense direct solve: stop
    if ((long)(sl[0] - 2) * (sl[1] - 2) * (sl[2] - 2) <= 512) any = false;
    if (!any || h->s.size() >= 16) break;
    std::array<int, 3> sc{};
    for (int d = 0; d < 3; d++) {
      const std::vector<double>& hf = C[d].back().hn;  // 1-based
      std::vector<double> h0(hf.begin() + 1, hf.end());
      std::vector<double> hc = cz[d] ? coarsen_nodes(h0, per[d]) : h0;
      C[d].push_back(host::build_coord(hc.data(), (int)hc.size()));
      sc[d] = (int)hc.size() - 1;
    }
    h->s.push_back(sc);
    coarsened.push_back(cz);
  }
  h->nl = (int)h->s.size();
  // face coefficients per level (LAP_PROPS)
  std::vector<std::array<std::vector<double>, 3>> K(h->nl);
  if (kf) {
    for (int d = 0; d < 3; d++) {
      K[0][d].resize(kf[d].n());
      cudaMemcpy(K[0][d].data(), kf[d].f, kf[d].n() * sizeof(double), cudaMemcpyDeviceToHost);
    }
    for (int l = 1; l < h->nl; l++)
      for (int d = 0; d < 3; d++) {
        const host::HostCoord cf[3] = {C[0][l - 1], C[1][l - 1], C[2][l - 1]};
        K[l][d] = coarsen_faces(K[l - 1][d], d, h->s[l - 1], h->s[l], cf, coarsened[l].data());
      }
  }
  for (int l = 0; l < h->nl; l++) {
    const size_t n = (size_t)h->s[l][0] * h->s[l][1] * h->s[l][2];
    MGLev<double> Ld{};
    MGLev<float> Lf{};
    for (int f = 0; f < 7; f++) Ld.bt[f] = Lf.bt[f] = bt[f];
    Ld.s0 = Lf.s0 = h->s[l][0];
    Ld.s1 = Lf.s1 = h->s[l][1];
    Ld.s2 = Lf.s2 = h->s[l][2];
    const host::HostCoord cl[3] = {C[0][l], C[1][l], C[2][l]};
    for (int d = 0; d < 3; d++) {
      const std::vector<double> W = face_weights(cl, h->s[l], d, kf ? &K[l][d] : nullptr);
      if (!h->mixed) Ld.w[d] = dev_copy(h.get(), W, st);
      else Lf.w[d] = dev_copy(h.get(), conv<float>(W), st);
      if (!(h->mixed ? (const void*)Lf.w[d] : (const void*)Ld.w[d])) return MOONS_ERR_NOMEM;
    }
    if (!h->mixed) {
      for (int d = 0; d < 3; d++) Ld.ax[d] = axis_tables<double>(h.get(), C[d][l], st);
      Ld.e = l == 0 ? s->z[0].f : dev_zeros<double>(h.get(), n, st);
      Ld.r = l == 0 ? s->r[0].f : dev_zeros<double>(h.get(), n, st);
      Ld.t = dev_zeros<double>(h.get(), n, st);
      if (kf) {
        Ld.kx = dev_copy(h.get(), K[l][0], st);
        Ld.ky = dev_copy(h.get(), K[l][1], st);
        Ld.kz = dev_copy(h.get(), K[l][2], st);
      }
      if (!Ld.t || !Ld.e || !Ld.r) return MOONS_ERR_NOMEM;
    } else {
      for (int d = 0; d < 3; d++) Lf.ax[d] = axis_tables<float>(h.get(), C[d][l], st);
      Lf.e = dev_zeros<float>(h.get(), n, st);
      Lf.r = dev_zeros<float>(h.get(), n, st);
      Lf.t = dev_zeros<float>(h.get(), n, st);
      if (kf) {
        Lf.kx = dev_copy(h.get(), conv<float>(K[l][0]), st);
        Lf.ky = dev_copy(h.get(), conv<float>(K[l][1]), st);
        Lf.kz = dev_copy(h.get(), conv<float>(K[l][2]), st);
      }
      if (!Lf.t || !Lf.e || !Lf.r) return MOONS_ERR_NOMEM;
    }
    h->Ld.push_back(Ld);
    h->Lf.push_back(Lf);
    std::array<MGProl<double>, 3> Pd{};
    std::array<MGProl<float>, 3> Pf{};
    std::array<MGRest<double>, 3> Rd{};
    std::array<MGRest<float>, 3> Rf{};
    if (l > 0) {
      for (int d = 0; d < 3; d++) {
        Axis1D A = build_axis(C[d][l], h->s[l - 1][d], bt[2 * d + 1], bt[2 * d + 2], coarsened[l][d]);
        const int* i0 = dev_copy(h.get(), A.i0, st);
        const int* i1 = dev_copy(h.get(), A.i1, st);
        const int* off = dev_copy(h.get(), A.off, st);
        const int* fi = dev_copy(h.get(), A.fi, st);
        if (!h->mixed) {
          Pd[d] = MGProl<double>{i0, i1, dev_copy(h.get(), A.w0, st), dev_copy(h.get(), A.w1, st)};
          Rd[d] = MGRest<double>{off, fi, dev_copy(h.get(), A.fw, st)};
        } else {
          Pf[d] = MGProl<float>{i0, i1, dev_copy(h.get(), conv<float>(A.w0), st),
                                dev_copy(h.get(), conv<float>(A.w1), st)};
          Rf[d] = MGRest<float>{off, fi, dev_copy(h.get(), conv<float>(A.fw), st)};
        }
      }
    }
    h->Pd.push_back(Pd);
    h->Pf.push_back(Pf);
    h->Rd.push_back(Rd);
    h->Rf.push_back(Rf);
  }
  if (h->mixed) {
    h->rprev = dev_zeros<double>(h.get(), (size_t)s0[0] * s0[1] * s0[2], st);
    h->ts_part = dev_zeros<double>(h.get(), 2 * kTsBlocks, st);
    h->ts_gamma = dev_zeros<double>(h.get(), 1, st);
    if (!h->rprev || !h->ts_part || !h->ts_gamma) return MOONS_ERR_NOMEM;
  }
  // separable restriction temporaries (x pass: cx*fy*fz, y pass: cx*cy*fz)
  h->rt1.assign(h->nl, nullptr);
  h->rt2.assign(h->nl, nullptr);
  for (int l = 1; l < h->nl; l++) {
    const size_t cx = h->s[l][0] - 2, cy = h->s[l][1] - 2, fy = h->s[l - 1][1] - 2, fz = h->s[l - 1][2] - 2;
    const size_t es = h->mixed ? sizeof(float) : sizeof(double);
    for (int q = 0; q < 2; q++) {
      void* ptr = nullptr;
      if (cudaMalloc(&ptr, es * std::max<size_t>(1, q == 0 ? cx * fy * fz : cx * cy * fz)) != cudaSuccess)
        return MOONS_ERR_NOMEM;
      h->allocs.push_back(ptr);
      (q == 0 ? h->rt1 : h->rt2)[l] = ptr;
    }
  }
  {  // coarsest level: dense inverse, regularised on the constants when singular
    const int l = h->nl - 1;
    const auto& sc = h->s[l];
    const int n = (sc[0] - 2) * (sc[1] - 2) * (sc[2] - 2);
    if (n <= kDirectMax) {
      const host::HostCoord cc[3] = {C[0][l], C[1][l], C[2][l]};
      std::vector<double> A = dense_operator(cc, sc, bt, kf ? &K[l] : nullptr);
      bool dir = false;
      for (int f = 1; f <= 6; f++) dir = dir || bt[f] == MOONS_BC_DIRICHLET;
      if (!dir) {
        double avg = 0.0;
        for (int i = 0; i < n; i++) avg += A[(size_t)i * n + i];
        avg /= n;
        for (size_t q = 0; q < A.size(); q++) A[q] += avg / n;
      }
      std::vector<double> inv;
      if (invert(A, n, inv)) {
        h->ncoarse = n;
        // row-major: a warp of the direct-solve kernel reads one row
        h->cinv_d = dev_copy(h.get(), inv, st);
      }
    }
  }
  {
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    h->nsm = std::max(nsm, 1);
    const void* ks[2][4] = {{(const void*)k_mg_smooth<double>, (const void*)k_mg_resid<double>,
                             (const void*)k_mg_restrict<double>, (const void*)k_mg_prolong<double>},
                            {(const void*)k_mg_smooth<float>, (const void*)k_mg_resid<float>,
                             (const void*)k_mg_restrict<float>, (const void*)k_mg_prolong<float>}};
    for (int q = 0; q < 4; q++) {
      int occ = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ks[h->mixed ? 1 : 0][q], 256, 0);
      h->occ[q] = std::max(occ, 1);
    }
  }
  MG_CUDA(cudaStreamSynchronize(st));
  *out = h.release();
  return MOONS_OK;
}

void mg_free(MGHier* h) { delete h; }

namespace mg {
// out = (volume-weighted operator) in, on the finest FP32 level (interior;
// ghost values of `in` are implied by the BCs, never read)
__global__ void __launch_bounds__(256) k_mg_apply_f32(MGLev<float> L, const float* in, float* out) {
  const int nx = L.s0 - 2, ny = L.s1 - 2, nz = L.s2 - 2;
  const unsigned n = (unsigned)nx * (unsigned)ny * (unsigned)nz;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const unsigned q = t / (unsigned)nx;
    const int i = (int)(t - q * (unsigned)nx) + 2;
    const unsigned kk = q / (unsigned)ny;
    const int j = (int)(q - kk * (unsigned)ny) + 2, k = (int)kk + 2;
    float D;
    out[lidx(L, i, j, k)] = apply_A<float>(L, in, i, j, k, D);
  }
}

int mg_apply_fine_f32(MGHier* h, const float* in, float* out, cudaStream_t st) {
  if (!h || !h->mixed || h->Lf.empty()) {
    set_error("multigrid: no FP32 finest level");
    return MOONS_ERR_STATE;
  }
  const MGLev<float>& L = h->Lf[0];
  const size_t n = (size_t)(L.s0 - 2) * (L.s1 - 2) * (L.s2 - 2);
  MG_LAUNCH(k_mg_apply_f32, (unsigned)std::min<size_t>((n + 255) / 256, (size_t)h->nsm * 8), 256, st, L, in, out);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// block partials of y.(A y) over the interior, the operator evaluated and
// summed in FP64 from the FP32 level (the sum cancels heavily where the
// coefficients are large, which FP32 accumulation cannot carry)
__global__ void __launch_bounds__(256) k_mg_energy_f64(MGLev<float> L, const float* y, double* partial) {
  const int nx = L.s0 - 2, ny = L.s1 - 2, nz = L.s2 - 2;
  const unsigned n = (unsigned)nx * (unsigned)ny * (unsigned)nz;
  double acc = 0.0;
  for (unsigned t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const unsigned q = t / (unsigned)nx;
    const int i = (int)(t - q * (unsigned)nx) + 2;
    const unsigned kk = q / (unsigned)ny;
    const int j = (int)(q - kk * (unsigned)ny) + 2, k = (int)kk + 2;
    const size_t id = lidx(L, i, j, k);
    const double e0 = y[id];
    const int ii[3] = {i, j, k};
    const size_t st[3] = {1, (size_t)L.s0, (size_t)L.s0 * L.s1};
    const bool inner = i > 2 && i < L.s0 - 1 && j > 2 && j < L.s1 - 1 && k > 2 && k < L.s2 - 1;
    double v = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const MGAxis<float>& A = L.ax[d];
      const int tt = ii[d];
      const int di = d == 0, dj = d == 1, dk = d == 2;
      const double em = inner ? y[id - st[d]] : ev(L, y, i - di, j - dj, k - dk);
      const double ep = inner ? y[id + st[d]] : ev(L, y, i + di, j + dj, k + dk);
      double gl = em * (double)A.cD[tt - 1] + e0 * (double)A.cU[tt - 1];
      double gr = e0 * (double)A.cD[tt] + ep * (double)A.cU[tt];
      const float* kf = d == 0 ? L.kx : (d == 1 ? L.ky : L.kz);
      if (kf) {
        gl *= (double)kf[fidx(L, d, i, j, k)];
        gr *= (double)kf[fidx(L, d, i + di, j + dj, k + dk)];
      }
      v += gl * (double)A.nD[tt] + gr * (double)A.nU[tt];
    }
    const double vol = ((double)L.ax[0].hv[i] * (double)L.ax[1].hv[j]) * (double)L.ax[2].hv[k];
    acc += e0 * v * vol;
  }
  __shared__ double sh[8];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += sh[w];
    partial[blockIdx.x] = s;
  }
}

int mg_energy_fine_f64(MGHier* h, const float* y, double* partial, int nblocks, cudaStream_t st) {
  if (!h || !h->mixed || h->Lf.empty()) {
    set_error("multigrid: no FP32 finest level");
    return MOONS_ERR_STATE;
  }
  MG_LAUNCH(k_mg_energy_f64, (unsigned)nblocks, 256, st, h->Lf[0], y, partial);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

bool mg_is_mixed(const MGHier* h) { return h && h->mixed; }
}  // namespace mg
double* mg_rprev(MGHier* h) { return h->rprev; }

namespace {
// coarsest levels up to this many cells are swept by one block
constexpr size_t kCoarseOneBlock = 8192;

// grid-stride kernels: at most one resident wave
unsigned vgrid(size_t n, int occ = 8, int nsm = 148) {
  return (unsigned)std::max<size_t>(1, std::min<size_t>((n + 255) / 256, (size_t)occ * nsm));
}


// coarse r = R (fine t) from level l to l + 1: three separable passes
// (large levels) or one gather per coarse cell; pdl: dependent launches
template <typename T>
int restrict_level(MGHier* h, const std::vector<MGLev<T>>& L, const std::vector<std::array<MGRest<T>, 3>>& R,
                   int l, bool sep, bool pdl, cudaStream_t st, const PcgScalars* S) {
  const MGLev<T>& F = L[l];
  const MGLev<T>& C = L[l + 1];
  const int cx = C.s0 - 2, cy = C.s1 - 2, fy = F.s1 - 2, fz = F.s2 - 2;
  const size_t nc = (size_t)cx * (C.s1 - 2) * (C.s2 - 2);
  if (!sep) {
    if (pdl) MG_LAUNCH_PDL(k_mg_restrict<T>, vgrid(nc, h->occ[2], h->nsm), 256, st, F, C, R[l + 1][0], R[l + 1][1],
                           R[l + 1][2], S);
    else MG_LAUNCH(k_mg_restrict<T>, vgrid(nc, h->occ[2], h->nsm), 256, st, F, C, R[l + 1][0], R[l + 1][1],
                   R[l + 1][2], S);
    return MOONS_OK;
  }
  T* t1 = (T*)h->rt1[l + 1];
  T* t2 = (T*)h->rt2[l + 1];
  const size_t n1 = (size_t)cx * fy * fz, n2 = (size_t)cx * cy * fz;
  if (pdl) {
    MG_LAUNCH_PDL(k_mg_rx<T>, vgrid(n1, 8, h->nsm), 256, st, F, R[l + 1][0], t1, cx, S);
    MG_LAUNCH_PDL(k_mg_ry<T>, vgrid(n2, 8, h->nsm), 256, st, (const T*)t1, cx, fy, cy, fz, R[l + 1][1], t2, S);
    MG_LAUNCH_PDL(k_mg_rz<T>, vgrid(nc, 8, h->nsm), 256, st, (const T*)t2, C, R[l + 1][2], S);
  } else {
    MG_LAUNCH(k_mg_rx<T>, vgrid(n1, 8, h->nsm), 256, st, F, R[l + 1][0], t1, cx, S);
    MG_LAUNCH(k_mg_ry<T>, vgrid(n2, 8, h->nsm), 256, st, (const T*)t1, cx, fy, cy, fz, R[l + 1][1], t2, S);
    MG_LAUNCH(k_mg_rz<T>, vgrid(nc, 8, h->nsm), 256, st, (const T*)t2, C, R[l + 1][2], S);
  }
  return MOONS_OK;
}

template <typename T>
int vcycle_t(MGHier* h, const std::vector<MGLev<T>>& L, const std::vector<std::array<MGProl<T>, 3>>& P,
             const std::vector<std::array<MGRest<T>, 3>>& R, cudaStream_t st, const PcgScalars* S) {
  const int nl = h->nl;
  auto npts = [&](int l) { return (size_t)(L[l].s0 - 2) * (L[l].s1 - 2) * (L[l].s2 - 2); };
  const T om = (T)h->omega;
  for (int l = 0; l < nl - 1; l++) {  // down: pre-smooth, residual, restrict
    const unsigned g = vgrid(npts(l) / 2 + 1, h->occ[0], h->nsm);
    for (int q = 0; q < h->nu; q++) {
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[l], 0, q == 0 ? 1 : 0, om, S);
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[l], 1, 0, om, S);
    }
    MG_LAUNCH_PDL(k_mg_resid<T>, vgrid(npts(l), h->occ[1], h->nsm), 256, st, L[l], S);
    const int rc = restrict_level<T>(h, L, R, l, npts(l) >= kRsepMin, true, st, S);
    if (rc) return rc;
  }
  if (h->ncoarse > 0) {
    MG_LAUNCH_PDL(k_mg_direct<T>, (unsigned)((h->ncoarse + kDirectRowsPerBlock - 1) / kDirectRowsPerBlock), 256, st,
              L[nl - 1], (const double*)h->cinv_d, h->ncoarse, S);
  } else if (npts(nl - 1) <= kCoarseOneBlock) {
    MG_LAUNCH_PDL(k_mg_coarse<T>, 1, 256, st, L[nl - 1], h->sweeps_coarse, S);
  } else {  // large coarsest level (the level cap): the same sweeps, grid-wide
    const unsigned g = vgrid(npts(nl - 1) / 2 + 1, h->occ[0], h->nsm);
    for (int q = 0; q < h->sweeps_coarse; q++) {
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[nl - 1], 0, q == 0 ? 1 : 0, (T)1, S);
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[nl - 1], 1, 0, (T)1, S);
    }
    for (int q = 0; q < h->sweeps_coarse; q++) {
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[nl - 1], 1, 0, (T)1, S);
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[nl - 1], 0, 0, (T)1, S);
    }
  }
  for (int l = nl - 2; l >= 0; l--) {  // up: prolong + correct, post-smooth (reverse colours)
    const unsigned g = vgrid(npts(l) / 2 + 1, h->occ[0], h->nsm);
    MG_LAUNCH_PDL(k_mg_prolong<T>, vgrid(npts(l), h->occ[3], h->nsm), 256, st, L[l], L[l + 1], P[l + 1][0], P[l + 1][1],
              P[l + 1][2], S);
    for (int q = 0; q < h->nu; q++) {
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[l], 1, 0, om, S);
      MG_LAUNCH_PDL(k_mg_smooth<T>, g, 256, st, L[l], 0, 0, om, S);
    }
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
}  // namespace

int fd_apply(MGHier* h, DF z, DF r, cudaStream_t st, const PcgScalars* S);

// z = V(r) on the PCG's fine level (z, r: FP64 PCG arrays)
int mg_vcycle(MGHier* h, DF z, DF r, cudaStream_t st, const PcgScalars* S) {
  if (h->fd) return fd_apply(h, z, r, st, S);
  if (!h->mixed) return vcycle_t<double>(h, h->Ld, h->Pd, h->Rd, st, S);
  const size_t n = r.n();
  MG_LAUNCH_PDL((k_mg_cast<float, double>), vgrid(n), 256, st, h->Lf[0].r, (const double*)r.f, n, S);
  int rc = vcycle_t<float>(h, h->Lf, h->Pf, h->Rf, st, S);
  if (rc) return rc;
  MG_LAUNCH_PDL((k_mg_cast<double, float>), vgrid(n), 256, st, z.f, (const float*)h->Lf[0].e, n, S);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// after a mixed (FP32) V-cycle: t = r - A e on its finest level, in FP64
int mg_vcycle_resid_f64(MGHier* h, DF t, cudaStream_t st, const PcgScalars* S) {
  if (!h->mixed || h->fd) {
    set_error("two-stage preconditioner: needs the FP32 V-cycle");
    return MOONS_ERR_STATE;
  }
  const MGLev<float>& L = h->Lf[0];
  const size_t npts = (size_t)(L.s0 - 2) * (L.s1 - 2) * (L.s2 - 2);
  MG_LAUNCH_PDL(k_mg_resid<float>, vgrid(npts, h->occ[1], h->nsm), 256, st, L, S);
  const size_t n = t.n();
  MG_LAUNCH_PDL((k_mg_cast<double, float>), vgrid(n), 256, st, t.f, (const float*)L.t, n, S);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// z += gamma N, gamma = (N.t) / (N.A N) on the FP32 finest level (N, t: FP64
// arrays of the PCG's layout; N's copy overwrites the level's e, which the
// next V-cycle's first sweep rewrites)
int mg_two_stage_combine(MGHier* h, DF z, const double* N, const double* t, cudaStream_t st, const PcgScalars* S) {
  if (!h->mixed || h->fd || !h->ts_part) {
    set_error("two-stage preconditioner: needs the FP32 V-cycle");
    return MOONS_ERR_STATE;
  }
  const MGLev<float>& L = h->Lf[0];
  const size_t n = z.n();
  MG_LAUNCH_PDL((k_mg_cast<float, double>), vgrid(n), 256, st, L.e, N, n, S);
  MG_LAUNCH_PDL(k_ts_dots<float>, kTsBlocks, 256, st, L, t, h->ts_part, S);
  MG_LAUNCH_PDL(k_ts_gamma, 1, 32, st, (const double*)h->ts_part, kTsBlocks, h->ts_gamma, S);
  MG_LAUNCH_PDL(k_ts_axpy, vgrid(n), 256, st, z.f, N, (const double*)h->ts_gamma, n, S);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// ---------------------------------------------------------------------------
// MOONS_PREC_FD: direct solve of the separable constant-coefficient operator
// by fast diagonalization (Lynch, Rice & Thomas, Numer. Math. 6, 1964).
//
// The PCG's LAP_UNIFORM operator on a CC field is A = V (Lx (+) Ly (+) Lz):
// V = vx (x) vy (x) vz the cell volumes, L_d the 1-D two-gradient second
// difference of axis d with its homogeneous BC folded in (Neumann: ghost =
// first cell, Dirichlet: minus it, periodic: the opposite cell).  v_d L_d is
// symmetric, so M_d = v_d^{1/2} L_d v_d^{-1/2} = W_d Lam_d W_d^T with W_d
// orthogonal, and
//   A^{-1} b = (B_x (x) B_y (x) B_z) diag(1 / (lx_a + ly_b + lz_c)) (F_x (x) F_y (x) F_z) b,
//   F_d = W_d^T v_d^{-1/2},  B_d = v_d^{-1/2} W_d,
// with the constant (zero) mode of an operator without a Dirichlet face
// dropped.  The
// eigen-decomposition (implicit QL on the tridiagonal M_d; on a periodic
// axis, whose M_d has corner entries, after a Householder reduction to
// tridiagonal form) runs once on the host at create time; each application is six dense 1-D
// transforms (mode products) and one diagonal scaling on the device.  As
// the preconditioner of the reference's CG recurrence it makes the solve
// converge in one or two iterations, to the same tolerance and solution.
// ---------------------------------------------------------------------------
namespace {

// the 1-D operator L of one CC axis over its interior cells (row a = cell
// a + 2), homogeneous BCs folded in; vol = the cells' widths
bool axis_operator(const host::HostCoord& c, int s, int tlo, int thi, std::vector<double>& L, std::vector<double>& vol) {
  const int n = s - 2;
  L.assign((size_t)n * n, 0.0);
  vol.assign(n, 0.0);
  for (int t = 2; t <= s - 1; t++) {
    const int a = t - 2;
    vol[a] = c.dhn[t];
    const double cm = c.cc2nD[t - 1] * c.n2ccD[t];
    const double c0 = c.cc2nU[t - 1] * c.n2ccD[t] + c.cc2nD[t] * c.n2ccU[t];
    const double cp = c.cc2nU[t] * c.n2ccU[t];
    L[(size_t)a * n + a] += c0;
    for (int side = 0; side < 2; side++) {
      int nb = side == 0 ? t - 1 : t + 1;
      double w = side == 0 ? cm : cp;
      if (nb == 1 || nb == s) {
        const int ty = nb == 1 ? tlo : thi;
        if (ty == MOONS_BC_PERIODIC) nb = nb == 1 ? s - 1 : 2;
        else if (ty == MOONS_BC_NEUMANN) nb = t;
        else if (ty == MOONS_BC_DIRICHLET) { nb = t; w = -w; }
        else return false;
      }
      L[(size_t)a * n + (nb - 2)] += w;
    }
  }
  return true;
}

__global__ void __launch_bounds__(256) k_fd_gather(const double* __restrict__ r, int s0, int s1, double* __restrict__ T,
                                                   int nx, int ny, int nz, const PcgScalars* S) {
  if (S && S->done) return;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const size_t q = t / nx;
    const int j = (int)(q % ny), k = (int)(q / ny);
    T[t] = r[(size_t)(i + 1) + (size_t)s0 * ((size_t)(j + 1) + (size_t)s1 * (size_t)(k + 1))];
  }
}
__global__ void __launch_bounds__(256) k_fd_scatter(double* __restrict__ z, int s0, int s1, const double* __restrict__ T,
                                                    int nx, int ny, int nz, const PcgScalars* S) {
  if (S && S->done) return;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const size_t q = t / nx;
    const int j = (int)(q % ny), k = (int)(q / ny);
    z[(size_t)(i + 1) + (size_t)s0 * ((size_t)(j + 1) + (size_t)s1 * (size_t)(k + 1))] = T[t];
  }
}
// One axis transform of the interior tensor (x fastest) as a tiled FP64 GEMM,
// C (R x Cn, column-major) = X (R x K) Y (K x Cn), 64 x 64 outputs per block,
// 4 x 4 per thread, K in steps of 16 through shared memory:
//  LEFT  (axis 0):    X = F (row-major K x K), Y = the tensor as K x (ny nz)
//  RIGHT (axes 1, 2): X = the tensor slice as R x K (leading dim R, batch
//                     blockIdx.z at stride R K), Y = F^T (F row-major)
constexpr int kFT = 64, kFK = 16;
template <bool LEFT>
__global__ void __launch_bounds__(256) k_fd_gemm(const double* __restrict__ T, const double* __restrict__ F,
                                                 double* __restrict__ C, int R, int Cn, int K, const PcgScalars* S) {
  if (S && S->done) return;
  __shared__ double Xs[kFK][kFT + 1];
  __shared__ double Ys[kFK][kFT + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int r0 = blockIdx.x * kFT, c0 = blockIdx.y * kFT;
  const size_t boff = (size_t)blockIdx.z * (size_t)R * (size_t)K;  // RIGHT: batch of slices
  double acc[4][4] = {};
  for (int m0 = 0; m0 < K; m0 += kFK) {
    for (int e = threadIdx.x; e < kFK * kFT; e += 256) {
      // X tile: element (kk, r)
      if (LEFT) {  // F row-major: kk fastest across threads
        const int kk = e % kFK, r = e / kFK;
        const int gr = r0 + r, gk = m0 + kk;
        Xs[kk][r] = (gr < R && gk < K) ? F[(size_t)gr * K + gk] : 0.0;
      } else {  // tensor slice, column-major: r fastest
        const int r = e % kFT, kk = e / kFT;
        const int gr = r0 + r, gk = m0 + kk;
        Xs[kk][r] = (gr < R && gk < K) ? T[boff + (size_t)gr + (size_t)R * gk] : 0.0;
      }
      // Y tile: element (kk, c)
      {
        const int kk = e % kFK, c = e / kFK;
        const int gc = c0 + c, gk = m0 + kk;
        double v = 0.0;
        if (gc < Cn && gk < K) v = LEFT ? T[(size_t)gk + (size_t)K * gc] : F[(size_t)gc * K + gk];
        Ys[kk][c] = v;
      }
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kFK; kk++) {
      double xv[4], yv[4];
#pragma unroll
      for (int u = 0; u < 4; u++) xv[u] = Xs[kk][tx + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; v++) yv[v] = Ys[kk][ty + 16 * v];
#pragma unroll
      for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v] += xv[u] * yv[v];
    }
    __syncthreads();
  }
  const size_t coff = LEFT ? 0 : boff / (size_t)K * (size_t)Cn;  // RIGHT: batch of R x Cn slices
#pragma unroll
  for (int u = 0; u < 4; u++)
#pragma unroll
    for (int v = 0; v < 4; v++) {
      const int gr = r0 + tx + 16 * u, gc = c0 + ty + 16 * v;
      if (gr < R && gc < Cn) C[coff + (size_t)gr + (size_t)R * gc] = acc[u][v];
    }
}
// divide by the 3-D eigenvalue; (zi, zj, zk): the constant mode of an
// operator without a Dirichlet face (dropped), or -1
__global__ void __launch_bounds__(256) k_fd_scale(double* __restrict__ T, const double* __restrict__ lx,
                                                  const double* __restrict__ ly, const double* __restrict__ lz, int nx,
                                                  int ny, int nz, int zi, int zj, int zk, const PcgScalars* S) {
  if (S && S->done) return;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(t % nx);
    const size_t q = t / nx;
    const int j = (int)(q % ny), k = (int)(q / ny);
    T[t] = (i == zi && j == zj && k == zk) ? 0.0 : T[t] / (lx[i] + ly[j] + lz[k]);
  }
}

}  // namespace

int fd_build(moons_pcg* s, moons_mesh* m, const DBC& bc, MGHier** out) {
  (void)s;
  *out = nullptr;
  auto h = std::make_unique<MGHier>();
  h->fd = true;
  cudaStream_t st = m->stream;
  int bt[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int f = 1; f <= 6; f++) bt[f] = bc.defined ? bc.type[f] : MOONS_BC_NEUMANN;
  for (int d = 0; d < 3; d++) {
    const host::HostCoord c = host::build_coord(m->hn[d].data(), m->sn[d]);
    const int sc = m->sn[d] - 1, n = sc - 2;
    h->fn[d] = n;
    std::vector<double> L, vol;
    if (n < 1 || !axis_operator(c, sc, bt[2 * d + 1], bt[2 * d + 2], L, vol)) {
      set_error("fast diagonalization: each axis needs interior cells and Dirichlet/Neumann/periodic BCs");
      return MOONS_ERR_ARG;
    }
    // symmetric form M = v^{1/2} L v^{-1/2}; the operator must be symmetric
    // in the volume-weighted sense (true for any node distribution, and for
    // periodic axes whose two end cells have the same width)
    std::vector<double> M((size_t)n * n);
    double mmax = 0.0, asym = 0.0;
    for (int a = 0; a < n; a++)
      for (int b = 0; b < n; b++) {
        M[(size_t)a * n + b] = std::sqrt(vol[a]) * L[(size_t)a * n + b] / std::sqrt(vol[b]);
        mmax = std::max(mmax, std::fabs(M[(size_t)a * n + b]));
      }
    for (int a = 0; a < n; a++)
      for (int b = a + 1; b < n; b++) {
        const double x = M[(size_t)a * n + b], y = M[(size_t)b * n + a];
        asym = std::max(asym, std::fabs(x - y));
        M[(size_t)a * n + b] = M[(size_t)b * n + a] = 0.5 * (x + y);
      }
    if (asym > 1e-10 * mmax) {
      set_error("fast diagonalization: the axis operator is not symmetric (periodic axis with unequal end cells)");
      return MOONS_ERR_ARG;
    }
    std::vector<double> w, W;
    if (bt[2 * d + 1] == MOONS_BC_PERIODIC || bt[2 * d + 2] == MOONS_BC_PERIODIC) {
      eig::symmetric_eigen(M, n, w, W);  // cyclic: corner entries
    } else {
      std::vector<double> dg(n), od(n, 0.0);
      for (int a = 0; a < n; a++) dg[a] = M[(size_t)a * n + a];
      for (int a = 0; a + 1 < n; a++) od[a] = M[(size_t)a * n + a + 1];
      if (!eig::tridiag_ql(dg, od, n, w, W)) {
        set_error("fast diagonalization: the tridiagonal eigen-iteration did not converge");
        return MOONS_ERR_ARG;
      }
    }
    std::vector<double> F((size_t)n * n), B((size_t)n * n);
    for (int a = 0; a < n; a++)
      for (int b = 0; b < n; b++) {
        F[(size_t)a * n + b] = W[(size_t)b * n + a] / std::sqrt(vol[b]);  // W^T v^{-1/2}
        B[(size_t)a * n + b] = W[(size_t)a * n + b] / std::sqrt(vol[a]);  // v^{-1/2} W
      }
    // an axis without a Dirichlet face has the constant as its zero mode:
    // the eigenvalue of smallest magnitude
    if (bt[2 * d + 1] != MOONS_BC_DIRICHLET && bt[2 * d + 2] != MOONS_BC_DIRICHLET) {
      int z = 0;
      for (int a = 1; a < n; a++)
        if (std::fabs(w[a]) < std::fabs(w[z])) z = a;
      h->zmode[d] = z;
    }
    h->lam[d] = dev_copy(h.get(), w, st);
    h->fwd[d] = dev_copy(h.get(), F, st);
    h->bwd[d] = dev_copy(h.get(), B, st);
    if (!h->lam[d] || !h->fwd[d] || !h->bwd[d]) return MOONS_ERR_NOMEM;
  }
  if (h->zmode[0] < 0 || h->zmode[1] < 0 || h->zmode[2] < 0) h->zmode[0] = h->zmode[1] = h->zmode[2] = -1;
  const size_t nint = (size_t)h->fn[0] * h->fn[1] * h->fn[2];
  h->w0 = dev_zeros<double>(h.get(), nint, st);
  h->w1 = dev_zeros<double>(h.get(), nint, st);
  if (!h->w0 || !h->w1) return MOONS_ERR_NOMEM;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
  h->nsm = std::max(nsm, 1);
  MG_CUDA(cudaStreamSynchronize(st));
  *out = h.release();
  return MOONS_OK;
}

int fd_apply(MGHier* h, DF z, DF r, cudaStream_t st, const PcgScalars* S) {
  const int nx = h->fn[0], ny = h->fn[1], nz = h->fn[2];
  const size_t n = (size_t)nx * ny * nz;
  const unsigned g = vgrid(n, 8, h->nsm);
  double *a = h->w0, *b = h->w1;
  const unsigned tiles = (unsigned)kFT;
  // axis 0: (nx x nx) F times the tensor as nx x (ny nz)
  const dim3 g0((nx + tiles - 1) / tiles, (unsigned)(((size_t)ny * nz + tiles - 1) / tiles), 1);
  // axis 1: each z slice (nx x ny) times F^T
  const dim3 g1((nx + tiles - 1) / tiles, (ny + tiles - 1) / tiles, (unsigned)nz);
  // axis 2: the tensor as (nx ny) x nz times F^T
  const dim3 g2((unsigned)(((size_t)nx * ny + tiles - 1) / tiles), (nz + tiles - 1) / tiles, 1);
  const int nxy = nx * ny;
  MG_LAUNCH(k_fd_gather, g, 256, st, (const double*)r.f, r.s0, r.s1, a, nx, ny, nz, S);
  MG_LAUNCH(k_fd_gemm<true>, g0, 256, st, (const double*)a, (const double*)h->fwd[0], b, nx, ny * nz, nx, S);
  MG_LAUNCH(k_fd_gemm<false>, g1, 256, st, (const double*)b, (const double*)h->fwd[1], a, nx, ny, ny, S);
  MG_LAUNCH(k_fd_gemm<false>, g2, 256, st, (const double*)a, (const double*)h->fwd[2], b, nxy, nz, nz, S);
  MG_LAUNCH(k_fd_scale, g, 256, st, b, (const double*)h->lam[0], (const double*)h->lam[1], (const double*)h->lam[2], nx,
            ny, nz, h->zmode[0], h->zmode[1], h->zmode[2], S);
  MG_LAUNCH(k_fd_gemm<true>, g0, 256, st, (const double*)b, (const double*)h->bwd[0], a, nx, ny * nz, nx, S);
  MG_LAUNCH(k_fd_gemm<false>, g1, 256, st, (const double*)a, (const double*)h->bwd[1], b, nx, ny, ny, S);
  MG_LAUNCH(k_fd_gemm<false>, g2, 256, st, (const double*)b, (const double*)h->bwd[2], a, nxy, nz, nz, S);
  MG_LAUNCH(k_fd_scatter, g, 256, st, z.f, z.s0, z.s1, (const double*)a, nx, ny, nz, S);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// ---------------------------------------------------------------------------
// Diagnostics (no reference counterpart): the multigrid building blocks of an
// MOONS_PREC_MG solver's FP64 hierarchy, one launch each, on host arrays, so
// that each can be checked against a CPU restatement of the reference's
// prolongate_C (GF_prolongate.f90:22-56), its transpose and the point update
// of redBlack (SOR.f90:234-268).  Level arrays are the level's cell-centred
// arrays with ghosts, Fortran order; the level's ghost entries are not read
// (homogeneous BCs imply them) and are returned as zeros.
// ---------------------------------------------------------------------------
extern "C" {

int moons_mg_level_shape(moons_pcg* s, int level, int* shape3, int* nlevels) {
  if (!s || !shape3) {
    set_error("moons_mg_level_shape: null pointer");
    return MOONS_ERR_ARG;
  }
  MGHier* h = s->mgh;
  if (!h || h->fd || h->mixed) {
    set_error("moons_mg_level_shape: the solver has no FP64 multigrid hierarchy (MOONS_PREC_MG)");
    return MOONS_ERR_STATE;
  }
  if (nlevels) *nlevels = h->nl;
  if (level < 0 || level >= h->nl) {
    set_error("moons_mg_level_shape: level out of range");
    return MOONS_ERR_ARG;
  }
  for (int d = 0; d < 3; d++) shape3[d] = h->s[level][d];
  return MOONS_OK;
}

/* op 0: out (level) = P a, a the coarse correction on level+1;
 * op 1: out (level+1) = R a = P^T a, a the residual on level;
 * op 2: out (level) = e after one red and one black SOR sweep (omega of the
 *       V-cycle) from e = a with right-hand side b;
 * op 3: out (level) = b - A a (the level's volume-weighted operator). */
int moons_mg_debug(moons_pcg* s, int op, int level, const double* a, const double* b, double* out) {
  int sh[3], nl = 0;
  int r = moons_mg_level_shape(s, level, sh, &nl);
  if (r) return r;
  if (!a || !out || ((op == 2 || op == 3) && !b) || op < 0 || op > 3 || ((op == 0 || op == 1) && level + 1 >= nl)) {
    set_error("moons_mg_debug: bad op, level or array");
    return MOONS_ERR_ARG;
  }
  MGHier* h = s->mgh;
  cudaStream_t st = s->m->stream;
  cudaSetDevice(s->m->device);
  const MGLev<double>& L = h->Ld[level];
  auto bytes = [&](int l) { return (size_t)h->s[l][0] * h->s[l][1] * h->s[l][2] * sizeof(double); };
  auto npts = [&](int l) { return (size_t)(h->s[l][0] - 2) * (h->s[l][1] - 2) * (h->s[l][2] - 2); };
  if (op == 0) {
    const MGLev<double>& C = h->Ld[level + 1];
    MG_CUDA(cudaMemcpyAsync(C.e, a, bytes(level + 1), cudaMemcpyHostToDevice, st));
    MG_CUDA(cudaMemsetAsync(L.e, 0, bytes(level), st));
    MG_LAUNCH(k_mg_prolong<double>, vgrid(npts(level), h->occ[3], h->nsm), 256, st, L, C, h->Pd[level + 1][0],
              h->Pd[level + 1][1], h->Pd[level + 1][2], (const PcgScalars*)nullptr);
    MG_CUDA(cudaMemcpyAsync(out, L.e, bytes(level), cudaMemcpyDeviceToHost, st));
  } else if (op == 1) {
    const MGLev<double>& C = h->Ld[level + 1];
    MG_CUDA(cudaMemcpyAsync(L.t, a, bytes(level), cudaMemcpyHostToDevice, st));
    MG_CUDA(cudaMemsetAsync(C.r, 0, bytes(level + 1), st));
    // the separable passes, the V-cycle's restriction of its large levels
    const int rc = restrict_level<double>(h, h->Ld, h->Rd, level, true, false, st, nullptr);
    if (rc) return rc;
    MG_CUDA(cudaMemcpyAsync(out, C.r, bytes(level + 1), cudaMemcpyDeviceToHost, st));
  } else {
    MG_CUDA(cudaMemcpyAsync(L.e, a, bytes(level), cudaMemcpyHostToDevice, st));
    MG_CUDA(cudaMemcpyAsync(L.r, b, bytes(level), cudaMemcpyHostToDevice, st));
    if (op == 2) {
      const unsigned g = vgrid(npts(level) / 2 + 1, h->occ[0], h->nsm);
      MG_LAUNCH(k_mg_smooth<double>, g, 256, st, L, 0, 0, h->omega, (const PcgScalars*)nullptr);
      MG_LAUNCH(k_mg_smooth<double>, g, 256, st, L, 1, 0, h->omega, (const PcgScalars*)nullptr);
      MG_CUDA(cudaMemcpyAsync(out, L.e, bytes(level), cudaMemcpyDeviceToHost, st));
    } else {
      MG_CUDA(cudaMemsetAsync(L.t, 0, bytes(level), st));
      MG_LAUNCH(k_mg_resid<double>, vgrid(npts(level), h->occ[1], h->nsm), 256, st, L, (const PcgScalars*)nullptr);
      MG_CUDA(cudaMemcpyAsync(out, L.t, bytes(level), cudaMemcpyDeviceToHost, st));
    }
  }
  MG_CUDA(cudaStreamSynchronize(st));
  // ghost entries of the result: zero (the host arrays may carry any ghosts)
  const int l = op == 1 ? level + 1 : level;
  const int s0 = h->s[l][0], s1 = h->s[l][1], s2 = h->s[l][2];
  for (int k = 1; k <= s2; k++)
    for (int j = 1; j <= s1; j++)
      for (int i = 1; i <= s0; i++)
        if (i == 1 || i == s0 || j == 1 || j == s1 || k == 1 || k == s2)
          out[(size_t)(i - 1) + (size_t)s0 * ((size_t)(j - 1) + (size_t)s1 * (size_t)(k - 1))] = 0.0;
  return MOONS_OK;
}

}  // extern "C"
