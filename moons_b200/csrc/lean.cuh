// lean.cuh -- the PCG iteration as lean, bandwidth-bound kernels.
//
// Same three steps as fused.cuh (K1 op+mask+vol+p.Ap -> alpha, K2 x/r update
// + r.r, z.r -> exit test and beta, K3 p = beta p + Minv r), organised for
// the memory system instead of for brevity:
//  * a block is a 32x4 tile of (i,j) columns marching KC planes in k; every
//    per-column quantity (stencil coefficients, volumes, wall masks, index
//    arithmetic) is formed once per column, the centre column rolls its z
//    neighbours in registers, and x/y neighbours come from L1/L2;
//  * K3 also writes p's homogeneous (implicit) BC values -- ghost planes,
//    Dirichlet boundary nodes (0), periodic boundary nodes (copy of node 2)
//    -- computing the new value of each source point on the fly, so K1 and
//    K2 read p raw, exactly as the reference's operator reads p after
//    apply_BCs_implicit (which only ever writes these points, and only from
//    one interior point each; edge and corner ghosts, which no interior
//    stencil reads, are filled in a fixed order);
//  * Minv of prec_Lap/prec_mom is rebuilt from per-axis tables
//    (diag = (dx+dy)+dz, vol = (hx*hy)*hz) instead of being read.
#pragma once
#include "fused.cuh"

namespace mg {

constexpr int kTX = 32, kTY = 4, kKC = 16;

struct Col {  // per-column (fixed i,j) data of one component
  int i, j;
  bool ok, gij;  // inside the field; ghost in x or y
};

__device__ __forceinline__ Col col_of(const DF& a) {
  Col c;
  c.i = blockIdx.x * kTX + threadIdx.x + 1;
  c.j = blockIdx.y * kTY + threadIdx.y + 1;
  c.ok = c.i <= a.s0 && c.j <= a.s1;
  c.gij = c.i == 1 || c.i == a.s0 || c.j == 1 || c.j == a.s1;
  return c;
}

// Minv on the fly (per-axis tables, same formula as k_prec's)
MG_HD double diag_axis(const DCoord& c, bool N, int t) { return N ? c.diagN[t] : c.diagC[t]; }
MG_HD double vol_axis(const DCoord& c, bool N, int t) { return N ? c.dhc[t - 1] : c.dhn[t]; }

// ---- K1: LAP_UNIFORM (MODE 0), LAP_PROPS (1), MOM_DIFFUSION (2) ---------------
template <int MODE>
__device__ __forceinline__ double lap_column(const DF& A, const DF& p, const FBC& b, const DGrid& g, const DF& kx,
                                             const DF& ky, const DF& kz, double coeff, int k0, int k1) {
  Col cl = col_of(A);
  if (!cl.ok || k0 > k1) return 0.0;  // k chunks past this component's last plane
  const int i = cl.i, j = cl.j;
  const bool Nx = n_along(A.dl, 1), Ny = n_along(A.dl, 2), Nz = n_along(A.dl, 3);
  const DCoord &cx = g.c[0], &cy = g.c[1], &cz = g.c[2];
  const size_t sx = 1, sy = (size_t)A.s0, sz = (size_t)A.s0 * A.s1;
  double acc = 0.0;
  if (cl.gij) {  // ghost columns: Ap = vol*... = 0
    for (int k = k0; k <= k1; k++) A(i, j, k) = 0.0;
    return 0.0;
  }
  // per-column coefficients (x, y): part = a*pm + b*p0 + c*pp form kept as
  // the reference's two-gradient composition
  double xa1, xa2, xb1, xb2, xo1, xo2, ya1, ya2, yb1, yb2, yo1, yo2;
  if (!Nx) { xa1 = cx.cc2nD[i - 1]; xa2 = cx.cc2nU[i - 1]; xb1 = cx.cc2nD[i]; xb2 = cx.cc2nU[i]; xo1 = cx.n2ccD[i]; xo2 = cx.n2ccU[i]; }
  else { xa1 = cx.n2ccD[i - 1]; xa2 = cx.n2ccU[i - 1]; xb1 = cx.n2ccD[i]; xb2 = cx.n2ccU[i]; xo1 = cx.cc2nD[i - 1]; xo2 = cx.cc2nU[i - 1]; }
  if (!Ny) { ya1 = cy.cc2nD[j - 1]; ya2 = cy.cc2nU[j - 1]; yb1 = cy.cc2nD[j]; yb2 = cy.cc2nU[j]; yo1 = cy.n2ccD[j]; yo2 = cy.n2ccU[j]; }
  else { ya1 = cy.n2ccD[j - 1]; ya2 = cy.n2ccU[j - 1]; yb1 = cy.n2ccD[j]; yb2 = cy.n2ccU[j]; yo1 = cy.cc2nD[j - 1]; yo2 = cy.cc2nU[j - 1]; }
  const double vxy = vol_axis(cx, Nx, i) * vol_axis(cy, Ny, j);
  // wall masks along x and y (only node directions have wall planes)
  double fxy = 1.0;
  bool zxy = false;
  {
    int t[3] = {i, j, 0};
    int s[3] = {A.s0, A.s1, 0};
    for (int d = 0; d < 2; d++) {
      if (((b.wall_neu >> (2 * d)) & 1) && t[d] == 2) fxy *= 0.5;
      if (((b.wall_neu >> (2 * d + 1)) & 1) && t[d] == s[d] - 1) fxy *= 0.5;
      if (((b.wall_dir >> (2 * d)) & 1) && t[d] == 2) zxy = true;
      if (((b.wall_dir >> (2 * d + 1)) & 1) && t[d] == s[d] - 1) zxy = true;
      if (((b.wall_per >> d) & 1) && t[d] == s[d] - 1) zxy = true;
    }
  }
  const bool dot_xy = !(((b.dot_wall & 1) && i == 2) || ((b.dot_wall & 2) && i == A.s0 - 1) ||
                        ((b.dot_wall & 4) && j == 2) || ((b.dot_wall & 8) && j == A.s1 - 1));
  size_t idx = A.at(i, j, k0);
  // coefficient fields have their own (face) extents
  size_t ix = 0, iy = 0, iz = 0, szx = 0, szy = 0, szz = 0;
  if (MODE == 1) {
    ix = kx.at(i, j, k0);
    iy = ky.at(i, j, k0);
    iz = kz.at(i, j, k0);
    szx = (size_t)kx.s0 * kx.s1;
    szy = (size_t)ky.s0 * ky.s1;
    szz = (size_t)kz.s0 * kz.s1;
  }
  double pm = k0 > 1 ? p.f[idx - sz] : 0.0;
  double p0 = p.f[idx];
  for (int k = k0; k <= k1; k++, idx += sz, ix += szx, iy += szy, iz += szz) {
    double pp = k < A.s2 ? p.f[idx + sz] : 0.0;
    if (k == 1 || k == A.s2) {
      A.f[idx] = 0.0;
    } else {
      double pxm = p.f[idx - sx], pxp = p.f[idx + sx], pym = p.f[idx - sy], pyp = p.f[idx + sy];
      double za1, za2, zb1, zb2, zo1, zo2;
      if (!Nz) { za1 = cz.cc2nD[k - 1]; za2 = cz.cc2nU[k - 1]; zb1 = cz.cc2nD[k]; zb2 = cz.cc2nU[k]; zo1 = cz.n2ccD[k]; zo2 = cz.n2ccU[k]; }
      else { za1 = cz.n2ccD[k - 1]; za2 = cz.n2ccU[k - 1]; zb1 = cz.n2ccD[k]; zb2 = cz.n2ccU[k]; zo1 = cz.cc2nD[k - 1]; zo2 = cz.cc2nU[k - 1]; }
      double gl = pxm * xa1 + p0 * xa2, gr = p0 * xb1 + pxp * xb2;
      if (MODE == 1 && !Nx) { gl = gl * kx.f[ix]; gr = gr * kx.f[ix + 1]; }
      double v = gl * xo1 + gr * xo2;
      gl = pym * ya1 + p0 * ya2;
      gr = p0 * yb1 + pyp * yb2;
      if (MODE == 1 && !Ny) { gl = gl * ky.f[iy]; gr = gr * ky.f[iy + ky.s0]; }
      v = v + (gl * yo1 + gr * yo2);
      gl = pm * za1 + p0 * za2;
      gr = p0 * zb1 + pp * zb2;
      if (MODE == 1 && !Nz) { gl = gl * kz.f[iz]; gr = gr * kz.f[iz + szz]; }
      v = v + (gl * zo1 + gr * zo2);
      if (MODE == 2) {
        v = v * coeff;
        v = v + p0;
      }
      double f = fxy;
      bool zero = zxy;
      if (Nz) {
        if (((b.wall_neu >> 4) & 1) && k == 2) f *= 0.5;
        if (((b.wall_neu >> 5) & 1) && k == A.s2 - 1) f *= 0.5;
        if ((((b.wall_dir >> 4) & 1) && k == 2) || (((b.wall_dir >> 5) & 1) && k == A.s2 - 1) ||
            (((b.wall_per >> 2) & 1) && k == A.s2 - 1))
          zero = true;
      }
      if (f != 1.0) v = v * f;
      if (zero) v = 0.0;
      v = v * (vxy * vol_axis(cz, Nz, k));
      A.f[idx] = v;
      bool in = dot_xy && !(((b.dot_wall & 16) && k == 2) || ((b.dot_wall & 32) && k == A.s2 - 1));
      if (in) acc += p0 * v;
    }
    pm = p0;
    p0 = pp;
  }
  return acc;
}

template <int MODE>
__global__ void __launch_bounds__(kTX* kTY) k_l_lap(FComp Ap, FComp P, DGrid g, FBC b0, FBC b1, FBC b2, DF kx, DF ky,
                                                     DF kz, double coeff, int nkc, PcgScalars* S, double* partial,
                                                     unsigned* ticket) {
  if (S->done) return;
  int c = blockIdx.z / nkc;
  int k0 = (blockIdx.z - c * nkc) * kKC + 1;
  double acc = 0.0;
  if (c == 0) acc = lap_column<MODE>(Ap.f[0], P.f[0], b0, g, kx, ky, kz, coeff, k0, min(k0 + kKC - 1, Ap.f[0].s2));
  else if (c == 1) acc = lap_column<MODE>(Ap.f[1], P.f[1], b1, g, kx, ky, kz, coeff, k0, min(k0 + kKC - 1, Ap.f[1].s2));
  else acc = lap_column<MODE>(Ap.f[2], P.f[2], b2, g, kx, ky, kz, coeff, k0, min(k0 + kKC - 1, Ap.f[2].s2));
  finish_alpha(acc, S, partial, ticket);
}

// ---- K1 curl-curl: E_l = sig_l * curl_l(p) on edges (raw p) --------------------
// l=0: d/dy(pz) - d/dz(py) ; l=1: d/dz(px) - d/dx(pz) ; l=2: d/dx(py) - d/dy(px)
// (curl_SF with del assign/subtract: the CC->N passes are 0 at their end nodes)
template <int L>
__device__ __forceinline__ void curl_sig_column(const DF& E, const DF& pa, const DF& pb, const DF& sg, const DGrid& g,
                                                int k0, int k1) {
  constexpr int da = L == 0 ? 2 : (L == 1 ? 3 : 1);
  constexpr int db = L == 0 ? 3 : (L == 1 ? 1 : 2);
  Col cl = col_of(E);
  if (!cl.ok) return;
  const int i = cl.i, j = cl.j;
  const DCoord& ca = g.c[da - 1];
  const DCoord& cb = g.c[db - 1];
  const size_t stride_a = da == 1 ? 1 : (da == 2 ? (size_t)pa.s0 : (size_t)pa.s0 * pa.s1);
  const size_t stride_b = db == 1 ? 1 : (db == 2 ? (size_t)pb.s0 : (size_t)pb.s0 * pb.s1);
  for (int k = k0; k <= k1; k++) {
    int ta = da == 1 ? i : (da == 2 ? j : k);
    int tb = db == 1 ? i : (db == 2 ? j : k);
    double v = 0.0;
    if (!(ta == 1 || ta == E.s(da))) {
      size_t ia = pa.at(i, j, k);
      v = pa.f[ia - stride_a] * ca.cc2nD[ta - 1] + pa.f[ia] * ca.cc2nU[ta - 1];
    }
    if (tb == 1 || tb == E.s(db)) v = 0.0;
    else {
      size_t ib = pb.at(i, j, k);
      v = v - (pb.f[ib - stride_b] * cb.cc2nD[tb - 1] + pb.f[ib] * cb.cc2nU[tb - 1]);
    }
    E(i, j, k) = v * sg(i, j, k);
  }
}
__global__ void __launch_bounds__(kTX* kTY) k_l_curl_sig(DF E0, DF E1, DF E2, FComp P, DF s0, DF s1, DF s2, DGrid g,
                                                          int nkc, PcgScalars* S) {
  if (S->done) return;
  int l = blockIdx.z / nkc;
  int k0 = (blockIdx.z - l * nkc) * kKC + 1;
  if (l == 0) curl_sig_column<0>(E0, P.f[2], P.f[1], s0, g, k0, min(k0 + kKC - 1, E0.s2));
  else if (l == 1) curl_sig_column<1>(E1, P.f[0], P.f[2], s1, g, k0, min(k0 + kKC - 1, E1.s2));
  else curl_sig_column<2>(E2, P.f[1], P.f[0], s2, g, k0, min(k0 + kKC - 1, E2.s2));
}
// Ap_c = vol*mask(coeff*curl_c(E) + p) and p.Ap (edges -> faces: N->CC passes)
template <int C>
__device__ __forceinline__ double curl_ap_column(const DF& A, const DF& p, const FBC& b, const DF& Ea, const DF& Eb,
                                                 const DGrid& g, double coeff, int k0, int k1) {
  constexpr int da = C == 0 ? 2 : (C == 1 ? 3 : 1);
  constexpr int db = C == 0 ? 3 : (C == 1 ? 1 : 2);
  Col cl = col_of(A);
  if (!cl.ok) return 0.0;
  const int i = cl.i, j = cl.j;
  double acc = 0.0;
  const DCoord& ca = g.c[da - 1];
  const DCoord& cb = g.c[db - 1];
  const size_t stride_a = da == 1 ? 1 : (da == 2 ? (size_t)Ea.s0 : (size_t)Ea.s0 * Ea.s1);
  const size_t stride_b = db == 1 ? 1 : (db == 2 ? (size_t)Eb.s0 : (size_t)Eb.s0 * Eb.s1);
  const bool Nx = n_along(A.dl, 1), Ny = n_along(A.dl, 2), Nz = n_along(A.dl, 3);
  for (int k = k0; k <= k1; k++) {
    bool ghost = cl.gij || k == 1 || k == A.s2;
    double v = 0.0;
    if (!ghost) {
      int ta = da == 1 ? i : (da == 2 ? j : k);
      int tb = db == 1 ? i : (db == 2 ? j : k);
      size_t ia = Ea.at(i, j, k), ib = Eb.at(i, j, k);
      double w = Ea.f[ia] * ca.n2ccD[ta] + Ea.f[ia + stride_a] * ca.n2ccU[ta];
      w = w - (Eb.f[ib] * cb.n2ccD[tb] + Eb.f[ib + stride_b] * cb.n2ccU[tb]);
      w = w * coeff;
      double p0 = p(i, j, k);
      w = w + p0;
      bool zero;
      double f = wall_fac(A, b, i, j, k, zero);
      if (f != 1.0) w = w * f;
      if (zero) w = 0.0;
      v = w * ((vol_axis(g.c[0], Nx, i) * vol_axis(g.c[1], Ny, j)) * vol_axis(g.c[2], Nz, k));
      if (in_dot(A, i, j, k, b.dot_wall)) acc += p0 * v;
    }
    A(i, j, k) = v;
  }
  return acc;
}
__global__ void __launch_bounds__(kTX* kTY) k_l_curl_ap(FComp Ap, FComp P, DF E0, DF E1, DF E2, DGrid g, FBC b0,
                                                         FBC b1, FBC b2, double coeff, int nkc, PcgScalars* S,
                                                         double* partial, unsigned* ticket) {
  if (S->done) return;
  int c = blockIdx.z / nkc;
  int k0 = (blockIdx.z - c * nkc) * kKC + 1;
  double acc;
  if (c == 0) acc = curl_ap_column<0>(Ap.f[0], P.f[0], b0, E2, E1, g, coeff, k0, min(k0 + kKC - 1, Ap.f[0].s2));
  else if (c == 1) acc = curl_ap_column<1>(Ap.f[1], P.f[1], b1, E0, E2, g, coeff, k0, min(k0 + kKC - 1, Ap.f[1].s2));
  else acc = curl_ap_column<2>(Ap.f[2], P.f[2], b2, E1, E0, g, coeff, k0, min(k0 + kKC - 1, Ap.f[2].s2));
  finish_alpha(acc, S, partial, ticket);
}

// ---- K2: x += alpha p ; r -= alpha Ap ; r.r, z.r ; exit test ; beta --------------
__device__ __forceinline__ void update_column(const DF& x, const DF& p, const DF& r, const DF& Ap, const DF& M,
                                              const FBC& b, const DGrid& g, int mm, double coeff, double alpha,
                                              int k0, int k1, double& arr, double& azr) {
  Col cl = col_of(x);
  if (!cl.ok) return;
  const int i = cl.i, j = cl.j;
  const bool Nx = n_along(x.dl, 1), Ny = n_along(x.dl, 2), Nz = n_along(x.dl, 3);
  const bool inxy = !cl.gij && !(((b.dot_wall & 1) && i == 2) || ((b.dot_wall & 2) && i == x.s0 - 1) ||
                                 ((b.dot_wall & 4) && j == 2) || ((b.dot_wall & 8) && j == x.s1 - 1));
  double dxy = 0.0, vxy = 0.0;
  if (mm != 0 && !cl.gij) {
    dxy = diag_axis(g.c[0], Nx, i) + diag_axis(g.c[1], Ny, j);
    vxy = vol_axis(g.c[0], Nx, i) * vol_axis(g.c[1], Ny, j);
  }
  const size_t sz = (size_t)x.s0 * x.s1;
  size_t idx = x.at(i, j, k0);
  for (int k = k0; k <= k1; k++, idx += sz) {
    x.f[idx] = x.f[idx] + p.f[idx] * alpha;
    double rv = r.f[idx] + Ap.f[idx] * (-alpha);
    r.f[idx] = rv;
    bool in = inxy && k != 1 && k != x.s2 && !(((b.dot_wall & 16) && k == 2) || ((b.dot_wall & 32) && k == x.s2 - 1));
    if (in) {
      double mv;
      if (mm == 0) mv = M.f[idx];
      else {
        double d = dxy + diag_axis(g.c[2], Nz, k);
        if (mm == 2) {
          d = d * coeff;
          d = d + 1.0;
        }
        mv = 1.0 / (d * (vxy * vol_axis(g.c[2], Nz, k)));
      }
      double zv = mv * rv;
      arr += rv * rv;
      azr += zv * rv;
    }
  }
}
__global__ void __launch_bounds__(kTX* kTY) k_l_update(FComp X, FComp P, FComp R, FComp Ap, FComp M, DGrid g, int mm,
                                                        double coeff, FBC b0, FBC b1, FBC b2, int nkc, PcgScalars* S,
                                                        double* partial, unsigned* ticket) {
  if (S->done) return;
  int c = blockIdx.z / nkc;
  int k0 = (blockIdx.z - c * nkc) * kKC + 1;
  double arr = 0.0, azr = 0.0;
  double alpha = S->alpha;
  if (c == 0)
    update_column(X.f[0], P.f[0], R.f[0], Ap.f[0], M.f[0], b0, g, mm, coeff, alpha, k0, min(k0 + kKC - 1, X.f[0].s2), arr, azr);
  else if (c == 1)
    update_column(X.f[1], P.f[1], R.f[1], Ap.f[1], M.f[1], b1, g, mm, coeff, alpha, k0, min(k0 + kKC - 1, X.f[1].s2), arr, azr);
  else
    update_column(X.f[2], P.f[2], R.f[2], Ap.f[2], M.f[2], b2, g, mm, coeff, alpha, k0, min(k0 + kKC - 1, X.f[2].s2), arr, azr);
  double s_rr = block_sum(arr);
  double s_zr = block_sum(azr);
  unsigned fb = flat_block(), nb = n_blocks();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    partial[fb] = s_rr;
    partial[nb + fb] = s_zr;
  }
  if (last_block_any(ticket)) {
    double rr = sum_partials(partial, nb);
    double zr = sum_partials(partial + nb, nb);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
      *ticket = 0;
      S->rr = rr;
      S->zr = zr;
      S->iter += 1;
      S->iter_total += 1;
      bool stop = false;
      if (S->iter % S->nskip == 0) {
        double res = sqrt(fabs(rr));
        S->res = res;
        bool e1 = res / S->res0 < S->tol_rel;
        bool e2 = res < S->tol_abs;
        bool e3 = S->iter >= S->iter_max;
        if (e1 || e2 || e3) {
          stop = true;
          S->exit_reason = e1 ? 1 : (e2 ? 2 : 3);
        }
        if (isnan(res)) {
          S->nan = 1;
          S->nan_any = 1;
          stop = true;
        }
      }
      if (!stop) {
        S->beta = zr / S->rhok;
        S->rhok = zr;
        if (S->iter >= S->iter_max) {
          stop = true;
          S->exit_reason = 3;
        }
      }
      S->done = stop ? 1 : 0;
    }
  }
}

// ---- K3: p = p*beta + Minv r, plus p's implicit BC values ------------------------
// where p~ at (i,j,k) comes from: source point, factor, and an optional second
// (Robin_N) term; interior points map to themselves.  Resolves every ghost
// direction in turn (edge/corner ghosts, which no stencil reads, get the
// composition).
struct Src {
  int I, J, K;
  double fac;
  bool zero;
  int rI, rJ, rK;  // Robin_N boundary-node term (rc != 0)
  double rc;
};
MG_HD Src src_of(const DF& p, const FBC& b, int i, int j, int k) {
  Src s;
  int I[4] = {0, i, j, k};
  s.fac = 1.0;
  s.zero = false;
  s.rc = 0.0;
  int rd = 0, rb = 0;
  if (b.defined) {
    for (int d = 1; d <= 3; d++) {
      int t = I[d], n = p.s(d);
      bool N = n_along(p.dl, d);
      int fmin = 2 * d - 1, fmax = 2 * d;
      if (!N) {
        if (t == 1 || t == n) {
          int ty = b.type[t == 1 ? fmin : fmax];
          int in = t == 1 ? 2 : n - 1;
          if (ty == MOONS_BC_DIRICHLET) { I[d] = in; s.fac = -s.fac; }
          else if (ty == MOONS_BC_NEUMANN) I[d] = in;
          else if (ty == MOONS_BC_PERIODIC) I[d] = t == 1 ? n - 1 : 2;
          else if (ty == MOONS_BC_ROBIN) { I[d] = in; s.fac *= b.rc[t == 1 ? fmin : fmax]; }
        }
      } else {
        bool many = n > 4;
        bool per = b.type[fmin] == MOONS_BC_PERIODIC && b.type[fmax] == MOONS_BC_PERIODIC;
        if (t == 1) {
          int ty = b.type[fmin];
          if (ty == MOONS_BC_DIRICHLET) { I[d] = 3; s.fac = -s.fac; }
          else if (ty == MOONS_BC_NEUMANN) I[d] = 3;
          else if (ty == MOONS_BC_PERIODIC) I[d] = n - 2;
          else if (ty == MOONS_BC_ROBIN) { I[d] = 3; rd = d; rb = 2; s.rc = b.rc[fmin]; }
        } else if (t == n) {
          int ty = b.type[fmax];
          if (ty == MOONS_BC_DIRICHLET) { I[d] = n - 2; s.fac = -s.fac; }
          else if (ty == MOONS_BC_NEUMANN) I[d] = n - 2;
          else if (ty == MOONS_BC_PERIODIC) { if (!many) I[d] = 3; }
          else if (ty == MOONS_BC_ROBIN) { I[d] = n - 2; rd = d; rb = n - 1; s.rc = b.rc[fmax]; }
        } else if ((t == 2 && b.type[fmin] == MOONS_BC_DIRICHLET) || (t == n - 1 && b.type[fmax] == MOONS_BC_DIRICHLET)) {
          s.zero = true;
        } else if (t == n - 1 && many && per) {
          I[d] = 2;
        }
      }
    }
    for (int d = 1; d <= 3; d++) {  // a source on a Dirichlet boundary plane is 0
      if (!n_along(p.dl, d)) continue;
      int n = p.s(d);
      if ((I[d] == 2 && b.type[2 * d - 1] == MOONS_BC_DIRICHLET) || (I[d] == n - 1 && b.type[2 * d] == MOONS_BC_DIRICHLET))
        s.zero = true;
    }
  }
  s.I = I[1];
  s.J = I[2];
  s.K = I[3];
  int R[4] = {0, I[1], I[2], I[3]};
  if (rd) R[rd] = rb;
  s.rI = R[1];
  s.rJ = R[2];
  s.rK = R[3];
  return s;
}

__device__ __forceinline__ double pnew_at(const DF& p, const DF& r, const DF& M, const DGrid& g, int mm, double coeff,
                                          double beta, int i, int j, int k) {
  double mv;
  bool ghost = i == 1 || i == p.s0 || j == 1 || j == p.s1 || k == 1 || k == p.s2;
  if (mm == 0) mv = M(i, j, k);
  else if (ghost) mv = 0.0;
  else {
    const bool Nx = n_along(p.dl, 1), Ny = n_along(p.dl, 2), Nz = n_along(p.dl, 3);
    double d = (diag_axis(g.c[0], Nx, i) + diag_axis(g.c[1], Ny, j)) + diag_axis(g.c[2], Nz, k);
    if (mm == 2) {
      d = d * coeff;
      d = d + 1.0;
    }
    mv = 1.0 / (d * ((vol_axis(g.c[0], Nx, i) * vol_axis(g.c[1], Ny, j)) * vol_axis(g.c[2], Nz, k)));
  }
  return p(i, j, k) * beta + mv * r(i, j, k);
}

// The new p of a source point is needed by the BC points that copy it, while
// that source's own thread overwrites p: the kernel therefore reads p_old
// from `p` and writes `pn` (the two buffers swap every iteration).
__device__ __forceinline__ void pupd_column(const DF& p, const DF& pn, const DF& r, const DF& M, const FBC& b,
                                            const DGrid& g, int mm, double coeff, double beta, int k0, int k1) {
  Col cl = col_of(p);
  if (!cl.ok) return;
  const int i = cl.i, j = cl.j;
  const bool Nx = n_along(p.dl, 1), Ny = n_along(p.dl, 2), Nz = n_along(p.dl, 3);
  // columns next to a boundary (or with special boundary nodes) take the general path
  bool edge_xy = cl.gij || (Nx && (i == 2 || i == p.s0 - 1)) || (Ny && (j == 2 || j == p.s1 - 1));
  double dxy = 0.0, vxy = 0.0;
  if (mm != 0 && !cl.gij) {
    dxy = diag_axis(g.c[0], Nx, i) + diag_axis(g.c[1], Ny, j);
    vxy = vol_axis(g.c[0], Nx, i) * vol_axis(g.c[1], Ny, j);
  }
  const size_t sz = (size_t)p.s0 * p.s1;
  size_t idx = p.at(i, j, k0);
  for (int k = k0; k <= k1; k++, idx += sz) {
    bool special = edge_xy || k == 1 || k == p.s2 || (Nz && (k == 2 || k == p.s2 - 1));
    if (!special || !b.defined) {
      double mv;
      if (mm == 0) mv = M.f[idx];
      else if (cl.gij || k == 1 || k == p.s2) mv = 0.0;
      else {
        double d = dxy + diag_axis(g.c[2], Nz, k);
        if (mm == 2) {
          d = d * coeff;
          d = d + 1.0;
        }
        mv = 1.0 / (d * (vxy * vol_axis(g.c[2], Nz, k)));
      }
      pn.f[idx] = p.f[idx] * beta + mv * r.f[idx];
    } else {
      Src s = src_of(p, b, i, j, k);
      double v = 0.0;
      if (!s.zero) {
        v = pnew_at(p, r, M, g, mm, coeff, beta, s.I, s.J, s.K);
        if (s.rc != 0.0) v = v + pnew_at(p, r, M, g, mm, coeff, beta, s.rI, s.rJ, s.rK) * s.rc;
        v = s.fac * v;
      }
      pn.f[idx] = v;
    }
  }
}
__global__ void __launch_bounds__(kTX* kTY) k_l_pupd(FComp P, FComp Pn, FComp R, FComp M, DGrid g, int mm,
                                                      double coeff, FBC b0, FBC b1, FBC b2, int nkc, PcgScalars* S) {
  if (S->done) return;
  int c = blockIdx.z / nkc;
  int k0 = (blockIdx.z - c * nkc) * kKC + 1;
  double beta = S->beta;
  if (c == 0) pupd_column(P.f[0], Pn.f[0], R.f[0], M.f[0], b0, g, mm, coeff, beta, k0, min(k0 + kKC - 1, P.f[0].s2));
  else if (c == 1) pupd_column(P.f[1], Pn.f[1], R.f[1], M.f[1], b1, g, mm, coeff, beta, k0, min(k0 + kKC - 1, P.f[1].s2));
  else pupd_column(P.f[2], Pn.f[2], R.f[2], M.f[2], b2, g, mm, coeff, beta, k0, min(k0 + kKC - 1, P.f[2].s2));
}

}  // namespace mg
