// fused.cuh -- fused PCG iteration kernels.
//
// One PCG iteration of the reference (PCG_solver_algorithm.f90:69-96) is
//   apply_BCs_implicit(p); Ap = op(p); wall masks; Ap *= vol; alpha = rho/(p.Ap)
//   x += alpha p; r -= alpha Ap; z = Minv r; rho' = z.r; p = z + (rho'/rho) p
// Here that is three kernels:
//   K1 (op_ap):  Ap = vol * mask(op(p~)) and the block partials of p.Ap; the
//                last block forms alpha.  p~ is p with its homogeneous
//                (implicit) BCs applied -- computed on the fly, never stored:
//                every ghost value an interior stencil reads depends on one
//                interior value only, and implicit BCs are linear and
//                homogeneous, so the order in which the reference applies
//                the six faces cannot change the values read.  Ap at ghost
//                points is vol*... = 0 (vol is 0 on ghosts).
//   K2 (update): x += alpha p; r -= alpha Ap; partials of r.r and z.r with
//                z = Minv r (not stored); last block runs update_exit_loop
//                and forms beta.
//   K3 (pupd):   p = p beta + Minv r.
// Minv of prec_Lap / prec_mom is a product of 1-D terms, so it is recomputed
// instead of read.  Grids are (plane chunk, k, component): no 64-bit index
// division anywhere.
#pragma once
#include "kernels.cuh"

namespace mg {

struct PcgScalars {
  double rhok, alpha, res, res0, beta, pap, rr, zr, mean;
  int iter, done, exit_reason, nan;
  int iter_max, nskip;
  double tol_rel, tol_abs;
  int body_runs;  // executions of the loop body (second bound on the loop)
  // accumulated over solves until the host clears them
  int iter_total, runs_total, nan_any;
  // stagnation test of flexible CG with a learned preconditioner: every
  // stag_window iterations, stop (exit_reason 4) unless the residual fell
  // below stag_factor times its value stag_window iterations before
  int stag_window;
  double stag_factor, stag_ref;
  // nonzero: a bounded wait in a loop kernel ran out (the code names the site)
  int wait_err;
  // fused CC iteration: the x update x += alpha p of an iteration is applied
  // by the next iteration's operator kernel; last_half names the p buffer of
  // the iteration that ended the loop (0: p2, 1: p; -1: none ran), whose
  // update a kernel after the loop applies
  int last_half;
};

// implicit BCs + masks of one unknown component, as the fused kernels see them
struct FBC {
  int type[7];     // per face (x_BC's / p's BCs; MOONS_BC_*), 0 when undefined
  double rc[7];    // Robin implicit coefficient per face
  int defined;
  int wall_neu;    // face bits: Ap *= 0.5 on the wall plane (multiply_wall_Neumann)
  int wall_dir;    // face bits: Ap = 0 on the wall plane (assign_wall_Dirichlet)
  int wall_per;    // dir bits: Ap = 0 on plane s-1 (assign_wall_Periodic_single)
  int dot_wall;    // face bits: wall planes dropped from dot products (Dirichlet of x)
};

struct FComp {
  DF f[3];
  int nc;
};

// host: the fused kernels' view of one component's BCs.  xb: BCs of x (copied
// to p: implicit BCs, dot-product walls); xbcb: BCs of x_BC (masks of Ap,
// PCG_solver_algorithm.f90:72-75); ext: extents of the field (1-based).
inline FBC make_fbc(const DBC& xb, const DBC& xbcb, int dl, const int ext[4]) {
  FBC f{};
  f.defined = xb.defined;
  for (int face = 1; face <= 6; face++) {
    f.type[face] = xb.defined ? xb.type[face] : 0;
    double dh = xb.dh[face], nhat = xb.nhat[face], cw = xb.c_w[face];
    int d = (face + 1) / 2;
    if (f.type[face] == MOONS_BC_ROBIN)
      f.rc[face] = n_along(dl, d) ? -2.0 * dh * nhat / cw : (2.0 * cw * nhat / dh - 1.0) / (2.0 * cw * nhat / dh + 1.0);
  }
  for (int face = 1; face <= 6; face++) {
    int d = (face + 1) / 2;
    if (!n_along(dl, d)) continue;
    bool def = xbcb.defined != 0;
    if (def ? xbcb.type[face] == MOONS_BC_NEUMANN : true) f.wall_neu |= 1 << (face - 1);
    if (def ? xbcb.type[face] == MOONS_BC_DIRICHLET : true) f.wall_dir |= 1 << (face - 1);
    if (xb.defined ? xb.type[face] == MOONS_BC_DIRICHLET : true) f.dot_wall |= 1 << (face - 1);
  }
  if (xbcb.defined)
    for (int d = 1; d <= 3; d++)
      if (n_along(dl, d) && xbcb.type[2 * d - 1] == MOONS_BC_PERIODIC && xbcb.type[2 * d] == MOONS_BC_PERIODIC &&
          ext[d] > 4)
        f.wall_per |= 1 << (d - 1);
  return f;
}

MG_HD int tget(int d, int i, int j, int k) { return d == 1 ? i : (d == 2 ? j : k); }

// value of p~ (p after apply_BCs_implicit) at (i,j,k) for points an interior
// output reads: at most one index is a ghost index.
MG_HD double pt(const DF& p, const FBC& b, int i, int j, int k) {
  // points two or more away from every boundary are neither ghosts nor
  // boundary nodes: p~ = p there
  if (i >= 3 && i <= p.s0 - 2 && j >= 3 && j <= p.s1 - 2 && k >= 3 && k <= p.s2 - 2) return p(i, j, k);
  int I[4] = {0, i, j, k};
  double fac = 1.0;
  bool robin_n = false;
  int rn_d = 0, rn_b = 0;
  double rn_c = 0.0;
#pragma unroll
  for (int d = 1; d <= 3; d++) {
    int t = I[d], s = p.s(d);
    bool N = n_along(p.dl, d);
    int fmin = 2 * d - 1, fmax = 2 * d;
    if (!b.defined) continue;
    if (!N) {
      if (t == 1) {
        int ty = b.type[fmin];
        if (ty == MOONS_BC_DIRICHLET) { I[d] = 2; fac = -fac; }
        else if (ty == MOONS_BC_NEUMANN) { I[d] = 2; }
        else if (ty == MOONS_BC_PERIODIC) { I[d] = s - 1; }
        else if (ty == MOONS_BC_ROBIN) { I[d] = 2; fac *= b.rc[fmin]; }
      } else if (t == s) {
        int ty = b.type[fmax];
        if (ty == MOONS_BC_DIRICHLET) { I[d] = s - 1; fac = -fac; }
        else if (ty == MOONS_BC_NEUMANN) { I[d] = s - 1; }
        else if (ty == MOONS_BC_PERIODIC) { I[d] = 2; }
        else if (ty == MOONS_BC_ROBIN) { I[d] = s - 1; fac *= b.rc[fmax]; }
      }
    } else {
      bool many = s > 4;
      if (t == 1) {
        int ty = b.type[fmin];
        if (ty == MOONS_BC_DIRICHLET) { I[d] = 3; fac = -fac; }
        else if (ty == MOONS_BC_NEUMANN) { I[d] = 3; }
        else if (ty == MOONS_BC_PERIODIC) { I[d] = s - 2; }
        else if (ty == MOONS_BC_ROBIN) { I[d] = 3; robin_n = true; rn_d = d; rn_b = 2; rn_c = b.rc[fmin]; }
      } else if (t == s) {
        int ty = b.type[fmax];
        if (ty == MOONS_BC_DIRICHLET) { I[d] = s - 2; fac = -fac; }
        else if (ty == MOONS_BC_NEUMANN) { I[d] = s - 2; }
        else if (ty == MOONS_BC_PERIODIC) { if (!many) I[d] = 3; }  // many-cell: ghost node s untouched
        else if (ty == MOONS_BC_ROBIN) { I[d] = s - 2; robin_n = true; rn_d = d; rn_b = s - 1; rn_c = b.rc[fmax]; }
      } else if (t == 2 && b.type[fmin] == MOONS_BC_DIRICHLET) {
        return 0.0;  // Dirichlet_N_implicit: ub = 0
      } else if (t == s - 1 && b.type[fmax] == MOONS_BC_DIRICHLET) {
        return 0.0;
      } else if (t == s - 1 && many && b.type[fmin] == MOONS_BC_PERIODIC && b.type[fmax] == MOONS_BC_PERIODIC) {
        I[d] = 2;  // Periodic_N_implicit: boundary node s-1 := node 2
      }
    }
  }
  // a source point on a Dirichlet boundary plane of an N direction is 0
  if (b.defined) {
#pragma unroll
    for (int d = 1; d <= 3; d++) {
      if (!n_along(p.dl, d)) continue;
      int s = p.s(d);
      if ((I[d] == 2 && b.type[2 * d - 1] == MOONS_BC_DIRICHLET) || (I[d] == s - 1 && b.type[2 * d] == MOONS_BC_DIRICHLET))
        return 0.0;
    }
  }
  double v = p(I[1], I[2], I[3]);
  if (robin_n) {  // Robin_N_implicit: ug = ui + ub*coeff
    int J[4] = {0, I[1], I[2], I[3]};
    J[rn_d] = rn_b;
    v = v + p(J[1], J[2], J[3]) * rn_c;
  }
  return fac * v;
}

// laplacian_diagonal (GF_diagonals.f90:15-35) and the cell volume of a point,
// formed per axis: diag = (dx + dy) + dz with each axis' two terms from the
// mesh tables (diagC/diagN), vol = (hx*hy)*hz
MG_HD double lap_diag_at(const DGrid& g, int dl, int i, int j, int k) {
  const DCoord &c1 = g.c[0], &c2 = g.c[1], &c3 = g.c[2];
  double dx = n_along(dl, 1) ? c1.diagN[i] : c1.diagC[i];
  double dy = n_along(dl, 2) ? c2.diagN[j] : c2.diagC[j];
  double dz = n_along(dl, 3) ? c3.diagN[k] : c3.diagC[k];
  return (dx + dy) + dz;
}
MG_HD double vol_at(const DGrid& g, int dl, int i, int j, int k) {
  int ex = n_along(dl, 1), ey = n_along(dl, 2), ez = n_along(dl, 3);
  return ((ex ? g.c[0].dhc[i - 1] : g.c[0].dhn[i]) * (ey ? g.c[1].dhc[j - 1] : g.c[1].dhn[j])) *
         (ez ? g.c[2].dhc[k - 1] : g.c[2].dhn[k]);
}
// Minv at a point: mode 1 prec_Lap, 2 prec_mom (coeff), 0 stored
MG_HD double minv_at(int mode, const DGrid& g, const DF& M, int dl, int i, int j, int k, bool ghost, double coeff) {
  if (mode == 0) return M(i, j, k);
  if (ghost) return 0.0;
  double d = lap_diag_at(g, dl, i, j, k);
  if (mode == 2) {
    d = d * coeff;
    d = d + 1.0;
  }
  return 1.0 / (d * vol_at(g, dl, i, j, k));
}

MG_HD bool in_dot(const DF& a, int i, int j, int k, int wall) { return dot_keep(a, i, j, k, wall); }

MG_HD double wall_fac(const DF& a, const FBC& b, int i, int j, int k, bool& zero) {
  double f = 1.0;
  zero = false;
  int t[4] = {0, i, j, k};
#pragma unroll
  for (int d = 1; d <= 3; d++) {
    int s = a.s(d);
    if (((b.wall_neu >> (2 * d - 2)) & 1) && t[d] == 2) f *= 0.5;
    if (((b.wall_neu >> (2 * d - 1)) & 1) && t[d] == s - 1) f *= 0.5;
    if (((b.wall_dir >> (2 * d - 2)) & 1) && t[d] == 2) zero = true;
    if (((b.wall_dir >> (2 * d - 1)) & 1) && t[d] == s - 1) zero = true;
    if (((b.wall_per >> (d - 1)) & 1) && t[d] == s - 1) zero = true;
  }
  return f;
}

// ---- block bookkeeping for (plane chunk, k, component) grids -----------------
__device__ __forceinline__ bool point_of(const DF& a, int& i, int& j, int& k) {
  unsigned p = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned s0 = (unsigned)a.s0;
  k = (int)blockIdx.y + 1;
  if (k > a.s2) return false;
  unsigned jj = p / s0;
  if (jj >= (unsigned)a.s1) return false;
  i = (int)(p - jj * s0) + 1;
  j = (int)jj + 1;
  return true;
}
__device__ __forceinline__ unsigned flat_block() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ __forceinline__ unsigned n_blocks() { return gridDim.x * gridDim.y * gridDim.z; }

__device__ __forceinline__ bool last_block_any(unsigned* ticket) {
  __shared__ bool amlast;
  if (lin_tid() == 0) {
    __threadfence();  // this block's partial (written by thread 0) before its ticket
    unsigned t = atomicAdd(ticket, 1u);
    amlast = (t == n_blocks() - 1);
  }
  __syncthreads();
  return amlast;
}

// ---- K1 variants ---------------------------------------------------------------
// centred Laplacian of p~ at a non-ghost point (lap_centered_SF_new /
// lap_centered_SF_given_both composed per point; ghost-point rules are not
// needed because ghost outputs are multiplied by vol = 0).
// k_faces: optional face coefficients (Lap_nonuniform_props: grad, *k, div).
template <bool KF>
MG_HD double lap_pt(const DF& p, const FBC& b, const DGrid& g, const DF& kx, const DF& ky,
                                         const DF& kz, int i, int j, int k) {
  double v = 0.0;
#pragma unroll
  for (int d = 1; d <= 3; d++) {
    const DCoord& c = g.c[d - 1];
    int t = tget(d, i, j, k);
    int di = d == 1, dj = d == 2, dk = d == 3;
    double part;
    double pm = pt(p, b, i - di, j - dj, k - dk), p0 = pt(p, b, i, j, k), pp = pt(p, b, i + di, j + dj, k + dk);
    if (!n_along(p.dl, d)) {
      // g(t) = p(t-1)*D(t-1) + p(t)*U(t-1) (stag CC->N), part = g(t)*D(t) + g(t+1)*U(t)
      double gl = pm * c.cc2nD[t - 1] + p0 * c.cc2nU[t - 1];
      double gr = p0 * c.cc2nD[t] + pp * c.cc2nU[t];
      if (KF) {
        const DF& kf = d == 1 ? kx : (d == 2 ? ky : kz);
        gl = gl * kf(i, j, k);
        gr = gr * kf(i + di, j + dj, k + dk);
      }
      part = gl * c.n2ccD[t] + gr * c.n2ccU[t];
    } else {
      // tx(t) = p(t)*D(t) + p(t+1)*U(t) (stag N->CC), part = tx(t-1)*D(t-1) + tx(t)*U(t-1) (CC->N)
      double tl = pm * c.n2ccD[t - 1] + p0 * c.n2ccU[t - 1];
      double tr = p0 * c.n2ccD[t] + pp * c.n2ccU[t];
      part = tl * c.cc2nD[t - 1] + tr * c.cc2nU[t - 1];
    }
    v = (d == 1) ? part : v + part;
  }
  return v;
}

// reduce `acc` over the grid; the last block stores alpha = rhok/sum
__device__ __forceinline__ void finish_alpha(double acc, PcgScalars* S, double* partial, unsigned* ticket) {
  double bs = block_sum(acc);
  unsigned fb = flat_block();
  if (lin_tid() == 0) partial[fb] = bs;
  if (last_block_any(ticket)) {
    double tot = sum_partials(partial, n_blocks());
    if (lin_tid() == 0) {
      S->pap = tot;
      S->alpha = S->rhok / tot;
      *ticket = 0;
    }
  }
}

// K1 body of one component: LAP_UNIFORM (MODE 0), LAP_PROPS (1), MOM_DIFFUSION (2)
// value of Ap at one point and its share of p.Ap (host-callable, for checks)
template <int MODE>
MG_HD void lap_ap_point(const DF& A, const DF& p, const FBC& b, const DGrid& g, const DF& kx, const DF& ky,
                        const DF& kz, double coeff, int i, int j, int k, double& v, double& acc) {
  bool ghost = (i == 1 || i == A.s0 || j == 1 || j == A.s1 || k == 1 || k == A.s2);
  acc = 0.0;
  v = 0.0;
  if (!ghost) {
    double lap = lap_pt<MODE == 1>(p, b, g, kx, ky, kz, i, j, k);
    if (MODE == 2) {
      lap = lap * coeff;
      lap = lap + pt(p, b, i, j, k);
    }
    bool zero;
    double f = wall_fac(A, b, i, j, k, zero);
    if (f != 1.0) lap = lap * f;
    if (zero) lap = 0.0;
    v = lap * vol_at(g, A.dl, i, j, k);
    if (in_dot(A, i, j, k, b.dot_wall)) acc = p(i, j, k) * v;
  }
}
template <int MODE>
__device__ __forceinline__ double lap_ap_body(const DF& A, const DF& p, const FBC& b, const DGrid& g, const DF& kx,
                                              const DF& ky, const DF& kz, double coeff) {
  int i, j, k;
  if (!point_of(A, i, j, k)) return 0.0;
  double v, acc;
  lap_ap_point<MODE>(A, p, b, g, kx, ky, kz, coeff, i, j, k, v, acc);
  A(i, j, k) = v;
  return acc;
}

template <int MODE>
__global__ void k_f_lap_ap(FComp Ap, FComp P, DGrid g, FBC b0, FBC b1, FBC b2, DF kx, DF ky, DF kz, double coeff,
                           PcgScalars* S, double* partial, unsigned* ticket) {
  if (S->done) return;
  double acc = 0.0;
  if (blockIdx.z == 0) acc = lap_ap_body<MODE>(Ap.f[0], P.f[0], b0, g, kx, ky, kz, coeff);
  else if (blockIdx.z == 1) acc = lap_ap_body<MODE>(Ap.f[1], P.f[1], b1, g, kx, ky, kz, coeff);
  else acc = lap_ap_body<MODE>(Ap.f[2], P.f[2], b2, g, kx, ky, kz, coeff);
  finish_alpha(acc, S, partial, ticket);
}

// ---- curl-curl (ind_diffusion) -----------------------------------------------
// K1a: E_l = sig_l * curl_l(p~) on edges l (curl_SF with del assign/subtract,
// ops_discrete.f90:184-202; ends of CC->N passes are 0)
MG_HD double dstag_cc2n(const DF& u, const FBC& b, const DCoord& c, int d, int i, int j, int k,
                                             int sout) {
  int t = tget(d, i, j, k);
  if (t == 1 || t == sout) return 0.0;
  int di = d == 1, dj = d == 2, dk = d == 3;
  return pt(u, b, i - di, j - dj, k - dk) * c.cc2nD[t - 1] + pt(u, b, i, j, k) * c.cc2nU[t - 1];
}
// l=0: d/dy(pz) - d/dz(py) ; l=1: d/dz(px) - d/dx(pz) ; l=2: d/dx(py) - d/dy(px)
template <int L>
MG_HD double curl_sig_point(const DF& E, const DF& pa, const FBC& ba, const DF& pb, const FBC& bb, const DF& sg,
                            const DGrid& g, int i, int j, int k) {
  constexpr int da = L == 0 ? 2 : (L == 1 ? 3 : 1);  // derivative dir of the first term
  constexpr int db = L == 0 ? 3 : (L == 1 ? 1 : 2);  // derivative dir of the subtracted term
  double v = dstag_cc2n(pa, ba, g.c[da - 1], da, i, j, k, E.s(da));
  int tb = tget(db, i, j, k);
  v = (tb == 1 || tb == E.s(db)) ? 0.0 : v - dstag_cc2n(pb, bb, g.c[db - 1], db, i, j, k, E.s(db));
  return v * sg(i, j, k);
}
template <int L>
__device__ __forceinline__ void curl_sig_body(const DF& E, const DF& pa, const FBC& ba, const DF& pb, const FBC& bb,
                                              const DF& sg, const DGrid& g) {
  int i, j, k;
  if (!point_of(E, i, j, k)) return;
  E(i, j, k) = curl_sig_point<L>(E, pa, ba, pb, bb, sg, g, i, j, k);
}
__global__ void k_f_curl_sig(DF E0, DF E1, DF E2, FComp P, DGrid g, FBC b0, FBC b1, FBC b2, DF s0, DF s1, DF s2,
                             PcgScalars* S) {
  if (S->done) return;
  if (blockIdx.z == 0) curl_sig_body<0>(E0, P.f[2], b2, P.f[1], b1, s0, g);
  else if (blockIdx.z == 1) curl_sig_body<1>(E1, P.f[0], b0, P.f[2], b2, s1, g);
  else curl_sig_body<2>(E2, P.f[1], b1, P.f[0], b0, s2, g);
}
// K1b: Ap_c = vol*mask(coeff*curl_c(E) + p~) and p.Ap (edges -> faces: N->CC passes)
template <int C>
MG_HD void curl_ap_point(const DF& A, const DF& p, const FBC& b, const DF& Ea, const DF& Eb, const DGrid& g,
                         double coeff, int i, int j, int k, double& v, double& acc) {
  // C=0: d/dy(Ez) - d/dz(Ey) ; C=1: d/dz(Ex) - d/dx(Ez) ; C=2: d/dx(Ey) - d/dy(Ex)
  constexpr int da = C == 0 ? 2 : (C == 1 ? 3 : 1);
  constexpr int db = C == 0 ? 3 : (C == 1 ? 1 : 2);
  bool ghost = (i == 1 || i == A.s0 || j == 1 || j == A.s1 || k == 1 || k == A.s2);
  acc = 0.0;
  v = 0.0;
  if (!ghost) {
    const DCoord& ca = g.c[da - 1];
    const DCoord& cb = g.c[db - 1];
    int ta = tget(da, i, j, k), tb = tget(db, i, j, k);
    double w = Ea(i, j, k) * ca.n2ccD[ta] + Ea(i + (da == 1), j + (da == 2), k + (da == 3)) * ca.n2ccU[ta];
    w = w - (Eb(i, j, k) * cb.n2ccD[tb] + Eb(i + (db == 1), j + (db == 2), k + (db == 3)) * cb.n2ccU[tb]);
    w = w * coeff;
    w = w + pt(p, b, i, j, k);
    bool zero;
    double f = wall_fac(A, b, i, j, k, zero);
    if (f != 1.0) w = w * f;
    if (zero) w = 0.0;
    v = w * vol_at(g, A.dl, i, j, k);
    if (in_dot(A, i, j, k, b.dot_wall)) acc = p(i, j, k) * v;
  }
}
template <int C>
__device__ __forceinline__ double curl_ap_body(const DF& A, const DF& p, const FBC& b, const DF& Ea, const DF& Eb,
                                               const DGrid& g, double coeff) {
  int i, j, k;
  if (!point_of(A, i, j, k)) return 0.0;
  double v, acc;
  curl_ap_point<C>(A, p, b, Ea, Eb, g, coeff, i, j, k, v, acc);
  A(i, j, k) = v;
  return acc;
}
__global__ void k_f_curl_ap(FComp Ap, FComp P, DF E0, DF E1, DF E2, DGrid g, FBC b0, FBC b1, FBC b2, double coeff,
                            PcgScalars* S, double* partial, unsigned* ticket) {
  if (S->done) return;
  double acc;
  if (blockIdx.z == 0) acc = curl_ap_body<0>(Ap.f[0], P.f[0], b0, E2, E1, g, coeff);
  else if (blockIdx.z == 1) acc = curl_ap_body<1>(Ap.f[1], P.f[1], b1, E0, E2, g, coeff);
  else acc = curl_ap_body<2>(Ap.f[2], P.f[2], b2, E1, E0, g, coeff);
  finish_alpha(acc, S, partial, ticket);
}

// ---- K2: x += alpha p ; r -= alpha Ap ; rr, zr ; exit test ; beta -----------
// p~ where it differs from p at a point x is updated on: the periodic
// boundary node s-1 of a node direction (Periodic_N_implicit copies node 2
// there).  x keeps that value when its own periodic BCs are prescribed, so
// the update must add alpha*p~ as the reference does.  (Dirichlet boundary
// nodes of p are 0 in both; ghost entries of x are rewritten by apply_BCs.)
MG_HD double p_for_x(const DF& p, const FBC& b, int i, int j, int k, size_t idx) {
  int t[4] = {0, i, j, k};
#pragma unroll
  for (int d = 1; d <= 3; d++) {
    int s = p.s(d);
    if (n_along(p.dl, d) && t[d] == s - 1 && s > 4 && b.type[2 * d - 1] == MOONS_BC_PERIODIC &&
        b.type[2 * d] == MOONS_BC_PERIODIC) {
      int u[4] = {0, i, j, k};
      u[d] = 2;
      return p(u[1], u[2], u[3]);
    }
  }
  return p.f[idx];
}
__device__ __forceinline__ void update_body(const DF& x, const DF& p, const FBC& b, const DF& r, const DF& Ap,
                                            const DF& M, const DGrid& g, int minv_mode, double coeff, int dw,
                                            double alpha, double& arr, double& azr) {
  int i, j, k;
  if (!point_of(x, i, j, k)) return;
  size_t idx = x.at(i, j, k);
  x.f[idx] = x.f[idx] + p_for_x(p, b, i, j, k, idx) * alpha;
  double rv = r.f[idx] + Ap.f[idx] * (-alpha);
  r.f[idx] = rv;
  if (in_dot(x, i, j, k, dw)) {
    double zv = minv_at(minv_mode, g, M, x.dl, i, j, k, false, coeff) * rv;
    arr = rv * rv;
    azr = zv * rv;
  }
}
__global__ void k_f_update(FComp X, FComp P, FComp R, FComp Ap, FComp M, DGrid g, int minv_mode, double coeff,
                           FBC b0, FBC b1, FBC b2, PcgScalars* S, double* partial, unsigned* ticket) {
  if (S->done) return;
  double arr = 0.0, azr = 0.0;
  double alpha = S->alpha;
  if (blockIdx.z == 0)
    update_body(X.f[0], P.f[0], b0, R.f[0], Ap.f[0], M.f[0], g, minv_mode, coeff, b0.dot_wall, alpha, arr, azr);
  else if (blockIdx.z == 1)
    update_body(X.f[1], P.f[1], b1, R.f[1], Ap.f[1], M.f[1], g, minv_mode, coeff, b1.dot_wall, alpha, arr, azr);
  else update_body(X.f[2], P.f[2], b2, R.f[2], Ap.f[2], M.f[2], g, minv_mode, coeff, b2.dot_wall, alpha, arr, azr);
  double s_rr = block_sum(arr);
  double s_zr = block_sum(azr);
  unsigned fb = flat_block(), nb = n_blocks();
  if (threadIdx.x == 0) {
    partial[fb] = s_rr;
    partial[nb + fb] = s_zr;
  }
  if (last_block_any(ticket)) {
    double rr = sum_partials(partial, nb);
    double zr = sum_partials(partial + nb, nb);
    if (threadIdx.x == 0) {
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

// ---- K3: p = p*beta + Minv r ----------------------------------------------------
__device__ __forceinline__ void pupd_body(const DF& p, const DF& r, const DF& M, const DGrid& g, int minv_mode,
                                          double coeff, double beta) {
  int i, j, k;
  if (!point_of(p, i, j, k)) return;
  size_t idx = p.at(i, j, k);
  bool ghost = (i == 1 || i == p.s0 || j == 1 || j == p.s1 || k == 1 || k == p.s2);
  double z = minv_at(minv_mode, g, M, p.dl, i, j, k, ghost, coeff) * r.f[idx];
  p.f[idx] = p.f[idx] * beta + z;
}
__global__ void k_f_pupd(FComp P, FComp R, FComp M, DGrid g, int minv_mode, double coeff, PcgScalars* S) {
  if (S->done) return;
  double beta = S->beta;
  if (blockIdx.z == 0) pupd_body(P.f[0], R.f[0], M.f[0], g, minv_mode, coeff, beta);
  else if (blockIdx.z == 1) pupd_body(P.f[1], R.f[1], M.f[1], g, minv_mode, coeff, beta);
  else pupd_body(P.f[2], R.f[2], M.f[2], g, minv_mode, coeff, beta);
}

}  // namespace mg
