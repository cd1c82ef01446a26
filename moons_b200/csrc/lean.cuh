// lean.cuh -- the PCG iteration as lean, bandwidth-bound kernels.
//
// Same three steps as fused.cuh (K1 op+mask+vol+p.Ap -> alpha, K2 x/r update
// + r.r, z.r -> exit test and beta, K3 p = beta p + Minv r), organised for
// the memory system instead of for brevity:
//  * a block owns 256 consecutive columns of the plane's inner set or of its
//    perimeter ring (coalesced, no tile waste, no BC divergence among inner
//    columns) and strides over the k chunks of kKC planes: grid = (plane
//    blocks, k stride, component), sized to one resident wave.  Per-column
//    quantities (index, stencil coefficients, volumes, wall masks) are
//    formed once per thread; every load of a chunk is issued before its
//    first result is formed, so each thread keeps several loads in flight;
//  * p carries its homogeneous (implicit) BC values: K3 forms the new p at
//    every point and k_l_bcfill rewrites the BC points -- ghost planes,
//    Dirichlet boundary nodes (0), periodic boundary nodes (copy of node 2)
//    -- from their source points, so K1 and K2 read p raw, exactly as the
//    reference's operator reads p after apply_BCs_implicit (which only ever
//    writes these points, and only from one interior point each; edge and
//    corner ghosts, which no interior stencil reads, are composed in a fixed
//    order);
//  * Minv of prec_Lap / prec_mom is formed per point from the per-axis tables
//    (the same expression k_prec stores, so bit-identical); prec_ind and the
//    identity read the stored PCG%Minv.
#pragma once
#include "fused.cuh"

namespace mg {

// Programmatic dependent launch: the solver loop's kernels are launched with
// programmatic stream serialisation, so the next kernel's blocks are
// scheduled while this one drains; each kernel lets its dependent launch at
// once and waits for its predecessor's completion (and memory) before it
// reads anything the predecessor wrote.  Both are no-ops in a plain launch.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}


constexpr int kLB = 256;  // threads per block (points of one plane)
constexpr int kKC = 4;    // planes per thread

struct Col {  // per-column (fixed i,j) data of one component
  int i, j;
  bool ok, gij;  // inside the field; ghost in x or y
};

// The (i,j) columns of a plane are split into the INNER set -- columns that
// are neither ghosts nor boundary nodes of a node-located direction, where
// no BC or wall rule applies -- and the PERIMETER ring around it.  Blocks
// 0..npbI-1 of a plane take 256 inner columns each, the next npbP blocks the
// perimeter, so the BC-specific code paths never diverge inside a warp of
// inner columns.
struct PlaneSplit {
  int ilo, ihi, jlo, jhi;
  unsigned wI, nI, nP, npbI, npbP;
};
MG_HD PlaneSplit plane_split(int s0, int s1, int dl) {
  PlaneSplit q;
  q.ilo = n_along(dl, 1) ? 3 : 2;
  q.jlo = n_along(dl, 2) ? 3 : 2;
  q.ihi = s0 + 1 - q.ilo;
  q.jhi = s1 + 1 - q.jlo;
  const int w = q.ihi - q.ilo + 1, h = q.jhi - q.jlo + 1;
  q.wI = w > 0 ? (unsigned)w : 0u;
  q.nI = (w > 0 && h > 0) ? (unsigned)(w * h) : 0u;
  q.nP = (unsigned)(s0 * s1) - q.nI;
  q.npbI = (q.nI + kLB - 1) / kLB;
  q.npbP = (q.nP + kLB - 1) / kLB;
  return q;
}

// pb: index of the 256-column block of the plane
__device__ __forceinline__ Col col_of(const DF& a, unsigned pb) {
  Col c;
  const PlaneSplit q = plane_split(a.s0, a.s1, a.dl);
  if (pb < q.npbI) {
    const unsigned t = pb * kLB + threadIdx.x;
    const unsigned r = t / q.wI;
    c.ok = t < q.nI;
    c.j = q.jlo + (int)r;
    c.i = q.ilo + (int)(t - r * q.wI);
  } else {
    unsigned t = (pb - q.npbI) * kLB + threadIdx.x;
    c.ok = t < q.nP;
    const unsigned s0 = (unsigned)a.s0;
    const unsigned nb = (unsigned)(q.jlo - 1) * s0;            // rows below the inner set
    const unsigned nt = (unsigned)(a.s1 - q.jhi) * s0;         // rows above it
    if (t < nb) {
      const unsigned r = t / s0;
      c.j = 1 + (int)r;
      c.i = 1 + (int)(t - r * s0);
    } else if (t < nb + nt) {
      t -= nb;
      const unsigned r = t / s0;
      c.j = q.jhi + 1 + (int)r;
      c.i = 1 + (int)(t - r * s0);
    } else {  // left and right bands of the inner rows
      t -= nb + nt;
      const unsigned wl = (unsigned)(q.ilo - 1), ws = wl + (unsigned)(a.s0 - q.ihi);
      const unsigned r = t / ws, u = t - r * ws;
      c.j = q.jlo + (int)r;
      c.i = u < wl ? 1 + (int)u : q.ihi + 1 + (int)(u - wl);
    }
  }
  if (!c.ok) c.i = c.j = 1;
  c.gij = c.i == 1 || c.i == a.s0 || c.j == 1 || c.j == a.s1;
  return c;
}
// plain (coherent) loads: the persistent solver reads data other blocks
// wrote earlier in the same launch, after a grid barrier
__device__ __forceinline__ double ld(const double* p) { return *p; }

// cell-volume share of one axis (volume_DL_GF, GF_distributions.f90:61-88)
MG_HD double vol_axis(const DCoord& c, bool N, int t) { return N ? c.dhc[t - 1] : c.dhn[t]; }

// wall-mask factor and zeroing of the x,y position of a column
__device__ __forceinline__ void wall_xy(const DF& A, const FBC& b, int i, int j, double& f, bool& zero) {
  f = 1.0;
  zero = false;
  int t[2] = {i, j};
  int s[2] = {A.s0, A.s1};
#pragma unroll
  for (int d = 0; d < 2; d++) {
    if (((b.wall_neu >> (2 * d)) & 1) && t[d] == 2) f *= 0.5;
    if (((b.wall_neu >> (2 * d + 1)) & 1) && t[d] == s[d] - 1) f *= 0.5;
    if (((b.wall_dir >> (2 * d)) & 1) && t[d] == 2) zero = true;
    if (((b.wall_dir >> (2 * d + 1)) & 1) && t[d] == s[d] - 1) zero = true;
    if (((b.wall_per >> d) & 1) && t[d] == s[d] - 1) zero = true;
  }
}
__device__ __forceinline__ void wall_z(const DF& A, const FBC& b, bool Nz, int k, double& f, bool& zero) {
  if (!Nz) return;
  if (((b.wall_neu >> 4) & 1) && k == 2) f *= 0.5;
  if (((b.wall_neu >> 5) & 1) && k == A.s2 - 1) f *= 0.5;
  if ((((b.wall_dir >> 4) & 1) && k == 2) || (((b.wall_dir >> 5) & 1) && k == A.s2 - 1) ||
      (((b.wall_per >> 2) & 1) && k == A.s2 - 1))
    zero = true;
}
__device__ __forceinline__ bool dot_xy(const DF& A, const FBC& b, int i, int j) {
  return !(((b.dot_wall & 1) && i == 2) || ((b.dot_wall & 2) && i == A.s0 - 1) || ((b.dot_wall & 4) && j == 2) ||
           ((b.dot_wall & 8) && j == A.s1 - 1));
}
__device__ __forceinline__ bool dot_z(const DF& A, const FBC& b, int k) {
  return !(((b.dot_wall & 16) && k == 2) || ((b.dot_wall & 32) && k == A.s2 - 1));
}

// the 1-D second-difference coefficients of one axis at t: the reference's
// two-gradient composition part = (pm*a1 + p0*a2)*o1 + (p0*b1 + pp*b2)*o2
struct Ax6 {
  double a1, a2, b1, b2, o1, o2;
};
__device__ __forceinline__ Ax6 axis_coef(const DCoord& c, bool N, int t) {
  Ax6 r;
  if (!N) {
    r.a1 = c.cc2nD[t - 1]; r.a2 = c.cc2nU[t - 1]; r.b1 = c.cc2nD[t]; r.b2 = c.cc2nU[t];
    r.o1 = c.n2ccD[t]; r.o2 = c.n2ccU[t];
  } else {
    r.a1 = c.n2ccD[t - 1]; r.a2 = c.n2ccU[t - 1]; r.b1 = c.n2ccD[t]; r.b2 = c.n2ccU[t];
    r.o1 = c.cc2nD[t - 1]; r.o2 = c.cc2nU[t - 1];
  }
  return r;
}

// ---- K1: LAP_UNIFORM (MODE 0), LAP_PROPS (1), MOM_DIFFUSION (2), NRG_DIFFUSION (3)
// all k chunks of this block's columns (blockIdx.y strides over them)
template <int MODE>
__device__ __forceinline__ double lap_col(const DF& A, const DF& p, const FBC& b, const DGrid& g, const DF& kx,
                                          const DF& ky, const DF& kz, double coeff) {
  const Col cl = col_of(A, blockIdx.x);
  if (!cl.ok) return 0.0;
  const int i = cl.i, j = cl.j;
  const size_t sy = (size_t)A.s0, sz = (size_t)A.s0 * A.s1;
  const int nkc = (A.s2 + kKC - 1) / kKC;
  if (cl.gij) {  // ghost columns: Ap = vol*... = 0
    for (int kc = blockIdx.y; kc < nkc; kc += gridDim.y) {
      const int k0 = kc * kKC + 1;
      const size_t idx0 = A.at(i, j, k0);
#pragma unroll
      for (int q = 0; q < kKC; q++)
        if (k0 + q <= A.s2) A.f[idx0 + q * sz] = 0.0;
    }
    return 0.0;
  }
  const bool Nx = n_along(A.dl, 1), Ny = n_along(A.dl, 2), Nz = n_along(A.dl, 3);
  const Ax6 X = axis_coef(g.c[0], Nx, i), Y = axis_coef(g.c[1], Ny, j);
  const double vxy = vol_axis(g.c[0], Nx, i) * vol_axis(g.c[1], Ny, j);
  double fxy;
  bool zxy;
  wall_xy(A, b, i, j, fxy, zxy);
  const bool dxy = dot_xy(A, b, i, j);
  double acc = 0.0;
  for (int kc = blockIdx.y; kc < nkc; kc += gridDim.y) {
    const int k0 = kc * kKC + 1, k1 = min(k0 + kKC - 1, A.s2);
    const size_t idx0 = A.at(i, j, k0);
    const double* pbase = p.f + idx0;
    // loads: p on planes k0-1 .. k1+1, x and y neighbours on k0 .. k1
    double pc[kKC + 2], xm[kKC], xp[kKC], ym[kKC], yp[kKC];
#pragma unroll
    for (int q = 0; q < kKC + 2; q++) {
      const int k = k0 - 1 + q;
      pc[q] = (k >= 1 && k <= k1 + 1 && k <= A.s2) ? ld(pbase + (ptrdiff_t)(q - 1) * (ptrdiff_t)sz) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < kKC; q++) {
      const int k = k0 + q;
      const bool in = k > 1 && k < A.s2 && k <= k1;
      const double* c = pbase + (size_t)q * sz;
      xm[q] = in ? ld(c - 1) : 0.0;
      xp[q] = in ? ld(c + 1) : 0.0;
      ym[q] = in ? ld(c - sy) : 0.0;
      yp[q] = in ? ld(c + sy) : 0.0;
    }
    // coefficient fields have their own (face) extents
    size_t ix = 0, iy = 0, iz = 0, szx = 0, szy = 0, szz = 0;
    if (MODE == 1 || MODE == 3) {
      ix = kx.at(i, j, k0);
      iy = ky.at(i, j, k0);
      iz = kz.at(i, j, k0);
      szx = (size_t)kx.s0 * kx.s1;
      szy = (size_t)ky.s0 * ky.s1;
      szz = (size_t)kz.s0 * kz.s1;
    }
#pragma unroll
    for (int q = 0; q < kKC; q++) {
      const int k = k0 + q;
      if (k > k1) break;
      const size_t idx = idx0 + (size_t)q * sz;
      if (k == 1 || k == A.s2) {
        A.f[idx] = 0.0;
        continue;
      }
      const double pm = pc[q], p0 = pc[q + 1], pp = pc[q + 2];
      const Ax6 Z = axis_coef(g.c[2], Nz, k);
      double gl = xm[q] * X.a1 + p0 * X.a2, gr = p0 * X.b1 + xp[q] * X.b2;
      if ((MODE == 1 || MODE == 3) && !Nx) { gl = gl * ld(kx.f + ix + q * szx); gr = gr * ld(kx.f + ix + q * szx + 1); }
      double v = gl * X.o1 + gr * X.o2;
      gl = ym[q] * Y.a1 + p0 * Y.a2;
      gr = p0 * Y.b1 + yp[q] * Y.b2;
      if ((MODE == 1 || MODE == 3) && !Ny) { gl = gl * ld(ky.f + iy + q * szy); gr = gr * ld(ky.f + iy + q * szy + ky.s0); }
      v = v + (gl * Y.o1 + gr * Y.o2);
      gl = pm * Z.a1 + p0 * Z.a2;
      gr = p0 * Z.b1 + pp * Z.b2;
      if ((MODE == 1 || MODE == 3) && !Nz) { gl = gl * ld(kz.f + iz + q * szz); gr = gr * ld(kz.f + iz + (q + 1) * szz); }
      v = v + (gl * Z.o1 + gr * Z.o2);
      if (MODE == 2 || MODE == 3) {
        v = v * coeff;
        v = v + p0;
      }
      double f = fxy;
      bool zero = zxy;
      wall_z(A, b, Nz, k, f, zero);
      if (f != 1.0) v = v * f;
      if (zero) v = 0.0;
      v = v * (vxy * vol_axis(g.c[2], Nz, k));
      A.f[idx] = v;
      if (dxy && dot_z(A, b, k)) acc += p0 * v;
    }
  }
  return acc;
}

template <int MODE>
__global__ void __launch_bounds__(kLB, 2) k_l_lap(FComp Ap, FComp P, DGrid g, FBC b0, FBC b1, FBC b2, DF kx, DF ky,
                                                   DF kz, double coeff, PcgScalars* S, double* partial,
                                                   unsigned* ticket) {
  pdl_enter();
  if (S->done) return;
  double acc;
  if (blockIdx.z == 0) acc = lap_col<MODE>(Ap.f[0], P.f[0], b0, g, kx, ky, kz, coeff);
  else if (blockIdx.z == 1) acc = lap_col<MODE>(Ap.f[1], P.f[1], b1, g, kx, ky, kz, coeff);
  else acc = lap_col<MODE>(Ap.f[2], P.f[2], b2, g, kx, ky, kz, coeff);
  finish_alpha(acc, S, partial, ticket);
}

// ---- K1 curl-curl: E_l = sig_l * curl_l(p) on edges (raw p) --------------------
// l=0: d/dy(pz) - d/dz(py) ; l=1: d/dz(px) - d/dx(pz) ; l=2: d/dx(py) - d/dy(px)
// (curl_SF with del assign/subtract: the CC->N passes are 0 at their end nodes)
// planes per thread of the curl-curl kernels: two (fewer registers, more
// resident warps) measured 2 % faster per duct step than four
constexpr int kKCc = 2;
template <int L>
__device__ __forceinline__ void curl_sig_col(const DF& E, const DF& pa, const DF& pb, const DF& sg, const DGrid& g) {
  constexpr int da = L == 0 ? 2 : (L == 1 ? 3 : 1);
  constexpr int db = L == 0 ? 3 : (L == 1 ? 1 : 2);
  const Col cl = col_of(E, blockIdx.x);
  if (!cl.ok) return;
  const int i = cl.i, j = cl.j;
  const DCoord& ca = g.c[da - 1];
  const DCoord& cb = g.c[db - 1];
  const size_t stride_a = da == 1 ? 1 : (da == 2 ? (size_t)pa.s0 : (size_t)pa.s0 * pa.s1);
  const size_t stride_b = db == 1 ? 1 : (db == 2 ? (size_t)pb.s0 : (size_t)pb.s0 * pb.s1);
  const int nkc = (E.s2 + kKCc - 1) / kKCc;
  for (int kc = blockIdx.y; kc < nkc; kc += gridDim.y) {
    const int k0 = kc * kKCc + 1, k1 = min(k0 + kKCc - 1, E.s2);
    double va[kKCc], vb[kKCc], sv[kKCc];
#pragma unroll
    for (int q = 0; q < kKCc; q++) {
      const int k = k0 + q;
      va[q] = 0.0;
      vb[q] = 0.0;
      sv[q] = 0.0;
      if (k > k1) continue;
      const int ta = da == 1 ? i : (da == 2 ? j : k);
      const int tb = db == 1 ? i : (db == 2 ? j : k);
      if (!(ta == 1 || ta == E.s(da))) {
        const size_t ia = pa.at(i, j, k);
        va[q] = ld(pa.f + ia - stride_a) * ca.cc2nD[ta - 1] + ld(pa.f + ia) * ca.cc2nU[ta - 1];
      }
      if (!(tb == 1 || tb == E.s(db))) {
        const size_t ib = pb.at(i, j, k);
        vb[q] = ld(pb.f + ib - stride_b) * cb.cc2nD[tb - 1] + ld(pb.f + ib) * cb.cc2nU[tb - 1];
      }
      sv[q] = ld(sg.f + sg.at(i, j, k));
    }
#pragma unroll
    for (int q = 0; q < kKCc; q++) {
      const int k = k0 + q;
      if (k > k1) break;
      const int tb = db == 1 ? i : (db == 2 ? j : k);
      const double v = (tb == 1 || tb == E.s(db)) ? 0.0 : va[q] - vb[q];
      E(i, j, k) = v * sv[q];
    }
  }
}
__global__ void __launch_bounds__(kLB) k_l_curl_sig(DF E0, DF E1, DF E2, FComp P, DF s0, DF s1, DF s2, DGrid g,
                                                     PcgScalars* S) {
  pdl_enter();
  if (S->done) return;
  if (blockIdx.z == 0) curl_sig_col<0>(E0, P.f[2], P.f[1], s0, g);
  else if (blockIdx.z == 1) curl_sig_col<1>(E1, P.f[0], P.f[2], s1, g);
  else curl_sig_col<2>(E2, P.f[1], P.f[0], s2, g);
}
// Ap_c = vol*mask(coeff*curl_c(E) + p) and p.Ap (edges -> faces: N->CC passes)
template <int C>
__device__ __forceinline__ double curl_ap_col(const DF& A, const DF& p, const FBC& b, const DF& Ea, const DF& Eb,
                                              const DGrid& g, double coeff) {
  constexpr int da = C == 0 ? 2 : (C == 1 ? 3 : 1);
  constexpr int db = C == 0 ? 3 : (C == 1 ? 1 : 2);
  const Col cl = col_of(A, blockIdx.x);
  if (!cl.ok) return 0.0;
  const int i = cl.i, j = cl.j;
  const DCoord& ca = g.c[da - 1];
  const DCoord& cb = g.c[db - 1];
  const size_t stride_a = da == 1 ? 1 : (da == 2 ? (size_t)Ea.s0 : (size_t)Ea.s0 * Ea.s1);
  const size_t stride_b = db == 1 ? 1 : (db == 2 ? (size_t)Eb.s0 : (size_t)Eb.s0 * Eb.s1);
  const bool Nx = n_along(A.dl, 1), Ny = n_along(A.dl, 2), Nz = n_along(A.dl, 3);
  const double vxy = vol_axis(g.c[0], Nx, i) * vol_axis(g.c[1], Ny, j);
  const int nkc = (A.s2 + kKCc - 1) / kKCc;
  double acc = 0.0;
  for (int kc = blockIdx.y; kc < nkc; kc += gridDim.y) {
    const int k0 = kc * kKCc + 1, k1 = min(k0 + kKCc - 1, A.s2);
    double e0[kKCc], e1[kKCc], f0[kKCc], f1[kKCc], pv[kKCc];
#pragma unroll
    for (int q = 0; q < kKCc; q++) {
      const int k = k0 + q;
      const bool in = k <= k1 && !(cl.gij || k == 1 || k == A.s2);
      e0[q] = e1[q] = f0[q] = f1[q] = pv[q] = 0.0;
      if (in) {
        const size_t ia = Ea.at(i, j, k), ib = Eb.at(i, j, k);
        e0[q] = ld(Ea.f + ia);
        e1[q] = ld(Ea.f + ia + stride_a);
        f0[q] = ld(Eb.f + ib);
        f1[q] = ld(Eb.f + ib + stride_b);
        pv[q] = ld(p.f + p.at(i, j, k));
      }
    }
#pragma unroll
    for (int q = 0; q < kKCc; q++) {
      const int k = k0 + q;
      if (k > k1) break;
      const bool ghost = cl.gij || k == 1 || k == A.s2;
      double v = 0.0;
      if (!ghost) {
        const int ta = da == 1 ? i : (da == 2 ? j : k);
        const int tb = db == 1 ? i : (db == 2 ? j : k);
        double w = e0[q] * ca.n2ccD[ta] + e1[q] * ca.n2ccU[ta];
        w = w - (f0[q] * cb.n2ccD[tb] + f1[q] * cb.n2ccU[tb]);
        w = w * coeff;
        w = w + pv[q];
        bool zero;
        const double f = wall_fac(A, b, i, j, k, zero);
        if (f != 1.0) w = w * f;
        if (zero) w = 0.0;
        v = w * (vxy * vol_axis(g.c[2], Nz, k));
        if (in_dot(A, i, j, k, b.dot_wall)) acc += pv[q] * v;
      }
      A(i, j, k) = v;
    }
  }
  return acc;
}
__global__ void __launch_bounds__(kLB) k_l_curl_ap(FComp Ap, FComp P, DF E0, DF E1, DF E2, DGrid g, FBC b0, FBC b1,
                                                    FBC b2, double coeff, PcgScalars* S, double* partial,
                                                    unsigned* ticket) {
  pdl_enter();
  if (S->done) return;
  double acc;
  if (blockIdx.z == 0) acc = curl_ap_col<0>(Ap.f[0], P.f[0], b0, E2, E1, g, coeff);
  else if (blockIdx.z == 1) acc = curl_ap_col<1>(Ap.f[1], P.f[1], b1, E0, E2, g, coeff);
  else acc = curl_ap_col<2>(Ap.f[2], P.f[2], b2, E1, E0, g, coeff);
  finish_alpha(acc, S, partial, ticket);
}

// ---- K2: x += alpha p ; r -= alpha Ap ; z = Minv r ; r.r, z.r ; exit test ; beta ----
// Minv at a point, MM = 0: stored (PCG%Minv); 1: prec_Lap, 2: prec_mom
// (coeff), formed from the per-axis tables exactly as k_prec stores it
// (minv_at): 1/(((dx + dy) + dz) * ((hx*hy)*hz)).  The x,y parts are formed
// once per column (dxy, vxy).
struct MinvCol {
  double dxy, vxy;
};
template <int MM>
__device__ __forceinline__ MinvCol minv_col(const DGrid& g, int dl, int i, int j) {
  MinvCol c{0.0, 0.0};
  if (MM != 0) {
    const bool Nx = n_along(dl, 1), Ny = n_along(dl, 2);
    c.dxy = (Nx ? g.c[0].diagN[i] : g.c[0].diagC[i]) + (Ny ? g.c[1].diagN[j] : g.c[1].diagC[j]);
    c.vxy = vol_axis(g.c[0], Nx, i) * vol_axis(g.c[1], Ny, j);
  }
  return c;
}
template <int MM>
__device__ __forceinline__ double minv_k(const MinvCol& c, const DGrid& g, int dl, int k, double coeff) {
  const bool Nz = n_along(dl, 3);
  double d = c.dxy + (Nz ? g.c[2].diagN[k] : g.c[2].diagC[k]);
  if (MM == 2) {
    d = d * coeff;
    d = d + 1.0;
  }
  return 1.0 / (d * (c.vxy * vol_axis(g.c[2], Nz, k)));
}

// SZ: also store z = Minv r at every non-ghost point (the fused CC iteration
// forms the next p from it in its operator kernel)
template <int KC, int MM, bool SZ = false>
__device__ __forceinline__ void update_col(const DF& x, const DF& p, const DF& r, const DF& Ap, const DF& M,
                                           const FBC& b, const DGrid& g, double coeff, double alpha, double& arr,
                                           double& azr, const DF& zo = DF{}) {
  const Col cl = col_of(x, blockIdx.x);
  if (!cl.ok) return;
  const int i = cl.i, j = cl.j;
  const bool inxy = !cl.gij && dot_xy(x, b, i, j);
  const size_t sz = (size_t)x.s0 * x.s1;
  const int nkc = (x.s2 + KC - 1) / KC;
  const MinvCol mc = minv_col<MM>(g, x.dl, i, j);
  // a chunk's loads; with SZ (two arrays a point) the next chunk's loads are
  // issued before this chunk's stores (2 % per over-L2 iteration; the
  // three-array form would spill)
  auto load = [&](int kc, double* xv, double* pv, double* rv, double* av, double* mv) {
    const int k0 = kc * KC + 1, k1 = min(k0 + KC - 1, x.s2);
    const size_t idx0 = x.at(i, j, min(k0, x.s2));
#pragma unroll
    for (int q = 0; q < KC; q++) {
      const bool in = kc < nkc && k0 + q <= k1;
      const size_t idx = idx0 + (size_t)q * sz;
      xv[q] = (!SZ && in) ? x.f[idx] : 0.0;
      pv[q] = (!SZ && in) ? ld(p.f + idx) : 0.0;
      rv[q] = in ? r.f[idx] : 0.0;
      av[q] = in ? ld(Ap.f + idx) : 0.0;
      mv[q] = (MM == 0 && in) ? ld(M.f + idx) : 0.0;
    }
  };
  double xv[KC], pv[KC], rv[KC], av[KC], mv[KC];
  if constexpr (SZ) load(blockIdx.y, xv, pv, rv, av, mv);
  for (int kc = blockIdx.y; kc < nkc; kc += gridDim.y) {
    double nx[KC], np[KC], nr[KC], na[KC], nm[KC];
    if constexpr (SZ) load(kc + gridDim.y, nx, np, nr, na, nm);
    else load(kc, xv, pv, rv, av, mv);
    const int k0 = kc * KC + 1, k1 = min(k0 + KC - 1, x.s2);
    const size_t idx0 = x.at(i, j, k0);
#pragma unroll
    for (int q = 0; q < KC; q++) {
      const int k = k0 + q;
      if (k > k1) break;
      const size_t idx = idx0 + (size_t)q * sz;
      if (!SZ) x.f[idx] = xv[q] + pv[q] * alpha;  // SZ: x is updated by the next operator kernel
      const double rn = rv[q] + av[q] * (-alpha);
      r.f[idx] = rn;
      if (SZ) {
        if (!cl.gij && k != 1 && k != x.s2) {
          const double m = MM == 0 ? mv[q] : minv_k<MM>(mc, g, x.dl, k, coeff);
          const double zv = m * rn;
          zo.f[idx] = zv;
          if (inxy && dot_z(x, b, k)) {
            arr += rn * rn;
            azr += zv * rn;
          }
        }
      } else if (inxy && k != 1 && k != x.s2 && dot_z(x, b, k)) {
        const double m = MM == 0 ? mv[q] : minv_k<MM>(mc, g, x.dl, k, coeff);
        const double zv = m * rn;
        arr += rn * rn;
        azr += zv * rn;
      }
    }
    if constexpr (SZ) {
#pragma unroll
      for (int q = 0; q < KC; q++) {
        rv[q] = nr[q];
        av[q] = na[q];
        mv[q] = nm[q];
      }
    }
  }
}
template <int KC, int MM, bool SZ = false>
__global__ void __launch_bounds__(kLB, 5) k_l_update(FComp X, FComp P, FComp R, FComp Ap, FComp M, FBC b0, FBC b1,
                                                   FBC b2, DGrid g, double coeff, PcgScalars* S, double* partial,
                                                   unsigned* ticket, DF zo, int half) {
  pdl_enter();
  if (S->done) return;
  double arr = 0.0, azr = 0.0;
  const double alpha = S->alpha;
  if (blockIdx.z == 0)
    update_col<KC, MM, SZ>(X.f[0], P.f[0], R.f[0], Ap.f[0], M.f[0], b0, g, coeff, alpha, arr, azr, zo);
  else if (blockIdx.z == 1)
    update_col<KC, MM, SZ>(X.f[1], P.f[1], R.f[1], Ap.f[1], M.f[1], b1, g, coeff, alpha, arr, azr, zo);
  else update_col<KC, MM, SZ>(X.f[2], P.f[2], R.f[2], Ap.f[2], M.f[2], b2, g, coeff, alpha, arr, azr, zo);
  const double s_rr = block_sum(arr);
  const double s_zr = block_sum(azr);
  const unsigned fb = flat_block(), nb = n_blocks();
  if (threadIdx.x == 0) {
    partial[fb] = s_rr;
    partial[nb + fb] = s_zr;
  }
  if (last_block_any(ticket)) {
    const double rr = sum_partials(partial, nb);
    const double zr = sum_partials(partial + nb, nb);
    if (threadIdx.x == 0) {
      *ticket = 0;
      S->rr = rr;
      S->zr = zr;
      S->iter += 1;
      S->iter_total += 1;
      bool stop = false;
      if (S->iter % S->nskip == 0) {
        const double res = sqrt(fabs(rr));
        S->res = res;
        const bool e1 = res / S->res0 < S->tol_rel;
        const bool e2 = res < S->tol_abs;
        const bool e3 = S->iter >= S->iter_max;
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
      if (SZ && stop) S->last_half = half;
    }
  }
}

// fused CC iteration, after the loop: the update x += alpha p of the
// iteration that ended it (interior points; apply_BCs of x follows)
__global__ void k_cc_xfinal(DF x, DF p, DF p2, const PcgScalars* S) {
  const int h = S->last_half;
  if (h < 0) return;
  const DF& pl = h == 0 ? p2 : p;
  const double alpha = S->alpha;
  const size_t n = x.n();
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(idx, x, i, j, k);
    if (i == 1 || i == x.s0 || j == 1 || j == x.s1 || k == 1 || k == x.s2) continue;
    x.f[idx] = x.f[idx] + pl.f[idx] * alpha;
  }
}

// ---- K3: p' = p*beta + Minv r at every point (BC points: k_l_bcfill) -------------
template <int KC, int MM>
__device__ __forceinline__ void pupd_col(const DF& p, const DF& pn, const DF& r, const DF& M, const DGrid& g,
                                         double coeff, double beta) {
  const Col cl = col_of(p, blockIdx.x);
  if (!cl.ok) return;
  const size_t sz = (size_t)p.s0 * p.s1;
  const int nkc = (p.s2 + KC - 1) / KC;
  const MinvCol mc = minv_col<MM>(g, p.dl, cl.i, cl.j);
  for (int kc = blockIdx.y; kc < nkc; kc += gridDim.y) {
    const int k0 = kc * KC + 1, k1 = min(k0 + KC - 1, p.s2);
    const size_t idx0 = p.at(cl.i, cl.j, k0);
    double pv[KC], rv[KC], mv[KC];
#pragma unroll
    for (int q = 0; q < KC; q++) {
      const bool in = k0 + q <= k1;
      const size_t idx = idx0 + (size_t)q * sz;
      pv[q] = in ? ld(p.f + idx) : 0.0;
      rv[q] = in ? ld(r.f + idx) : 0.0;
      mv[q] = (MM == 0 && in) ? ld(M.f + idx) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < KC; q++) {
      const int k = k0 + q;
      if (k > k1) break;
      // Minv is 0 on the ghost points (k_prec)
      const double m = MM == 0 ? mv[q] : ((cl.gij || k == 1 || k == p.s2) ? 0.0 : minv_k<MM>(mc, g, p.dl, k, coeff));
      pn.f[idx0 + (size_t)q * sz] = pv[q] * beta + m * rv[q];
    }
  }
}
template <int KC, int MM>
__global__ void __launch_bounds__(kLB, 6) k_l_pupd(FComp P, FComp Pn, FComp R, FComp M, DGrid g, double coeff,
                                                 PcgScalars* S) {
  pdl_enter();
  if (S->done) return;
  const double beta = S->beta;
  if (blockIdx.z == 0) pupd_col<KC, MM>(P.f[0], Pn.f[0], R.f[0], M.f[0], g, coeff, beta);
  else if (blockIdx.z == 1) pupd_col<KC, MM>(P.f[1], Pn.f[1], R.f[1], M.f[1], g, coeff, beta);
  else pupd_col<KC, MM>(P.f[2], Pn.f[2], R.f[2], M.f[2], g, coeff, beta);
}

// ---- p's implicit BC values (apply_BCs_implicit, PCG_solver_algorithm.f90:70) ----
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
#pragma unroll
    for (int d = 1; d <= 3; d++) {
      const int t = I[d], n = p.s(d);
      const bool N = n_along(p.dl, d);
      const int fmin = 2 * d - 1, fmax = 2 * d;
      if (!N) {
        if (t == 1 || t == n) {
          const int ty = b.type[t == 1 ? fmin : fmax];
          const int in = t == 1 ? 2 : n - 1;
          if (ty == MOONS_BC_DIRICHLET) { I[d] = in; s.fac = -s.fac; }
          else if (ty == MOONS_BC_NEUMANN) I[d] = in;
          else if (ty == MOONS_BC_PERIODIC) I[d] = t == 1 ? n - 1 : 2;
          else if (ty == MOONS_BC_ROBIN) { I[d] = in; s.fac *= b.rc[t == 1 ? fmin : fmax]; }
        }
      } else {
        const bool many = n > 4;
        const bool per = b.type[fmin] == MOONS_BC_PERIODIC && b.type[fmax] == MOONS_BC_PERIODIC;
        if (t == 1) {
          const int ty = b.type[fmin];
          if (ty == MOONS_BC_DIRICHLET) { I[d] = 3; s.fac = -s.fac; }
          else if (ty == MOONS_BC_NEUMANN) I[d] = 3;
          else if (ty == MOONS_BC_PERIODIC) I[d] = n - 2;
          else if (ty == MOONS_BC_ROBIN) { I[d] = 3; rd = d; rb = 2; s.rc = b.rc[fmin]; }
        } else if (t == n) {
          const int ty = b.type[fmax];
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
#pragma unroll
    for (int d = 1; d <= 3; d++) {  // a source on a Dirichlet boundary plane is 0
      if (!n_along(p.dl, d)) continue;
      const int n = p.s(d);
      if ((I[d] == 2 && b.type[2 * d - 1] == MOONS_BC_DIRICHLET) || (I[d] == n - 1 && b.type[2 * d] == MOONS_BC_DIRICHLET))
        s.zero = true;
    }
  }
  s.I = I[1];
  s.J = I[2];
  s.K = I[3];
  s.rI = rd == 1 ? rb : I[1];
  s.rJ = rd == 2 ? rb : I[2];
  s.rK = rd == 3 ? rb : I[3];
  return s;
}

// rewrite one BC point from its source(s); sources are never points this
// kernel changes, so the order of the writes is free
__device__ __forceinline__ void bcfill_point(const DF& p, const FBC& b, int i, int j, int k) {
  const Src s = src_of(p, b, i, j, k);
  if (s.zero) {
    p(i, j, k) = 0.0;
    return;
  }
  if (s.I == i && s.J == j && s.K == k && s.fac == 1.0 && s.rc == 0.0) return;
  double v = p(s.I, s.J, s.K);
  if (s.rc != 0.0) v = v + p(s.rI, s.rJ, s.rK) * s.rc;
  p(i, j, k) = s.fac * v;
}
// block x < npbP: perimeter columns, every plane (strided over blockIdx.y);
// block x >= npbP: inner columns, one ghost plane or node-located boundary
// plane per blockIdx.y = 0..3
__device__ __forceinline__ void bcfill_col(const DF& p, const FBC& b, unsigned npbP) {
  if (!b.defined) return;
  const PlaneSplit q = plane_split(p.s0, p.s1, p.dl);
  if (blockIdx.x < npbP) {
    if (blockIdx.x >= q.npbP) return;
    const Col cl = col_of(p, q.npbI + blockIdx.x);
    if (!cl.ok) return;
    for (int k = blockIdx.y + 1; k <= p.s2; k += gridDim.y) bcfill_point(p, b, cl.i, cl.j, k);
  } else {
    const unsigned pi = blockIdx.x - npbP;
    const bool Nz = n_along(p.dl, 3);
    if (pi >= q.npbI || blockIdx.y >= (Nz ? 4u : 2u)) return;
    const Col cl = col_of(p, pi);
    if (!cl.ok) return;
    const int k = blockIdx.y == 0 ? 1 : (blockIdx.y == 1 ? p.s2 : (blockIdx.y == 2 ? 2 : p.s2 - 1));
    bcfill_point(p, b, cl.i, cl.j, k);
  }
}
__global__ void __launch_bounds__(kLB) k_l_bcfill(FComp P, FBC b0, FBC b1, FBC b2, unsigned npbP, PcgScalars* S) {
  pdl_enter();
  if (S->done) return;
  if (blockIdx.z == 0) bcfill_col(P.f[0], b0, npbP);
  else if (blockIdx.z == 1) bcfill_col(P.f[1], b1, npbP);
  else bcfill_col(P.f[2], b2, npbP);
}

}  // namespace mg
