// kernels.cuh -- generic sm_100a kernels of the MOONS hot path: staggered
// and collocated derivatives, the fused centred Laplacian, interpolation,
// ghost-cell BCs, wall masks, pointwise algebra and deterministic
// reductions.  One thread per output point, x-contiguous threads, so every
// warp reads and writes whole 256-byte rows of the x-fastest arrays.
#pragma once
#include "core.cuh"

namespace mg {

// ===========================================================================
// del (HW/ops/ops_del.f90:59-288 + HW/stencils/stencils.f90:47-206)
//
// The reference applies a 1-D stencil per pencil.  Each output point here
// computes what its pencil loop leaves in it, including the stencil quirks:
//  * staggered ops zero both end entries first, also for add/subtract, so an
//    end entry the loop does not write is 0 and one it writes loses what was
//    accumulated before (stag_add/stag_subtract :108-181);
//  * collocated ops zero both end entries after the loop (col_*_assign/add);
//  * pencils with transverse index outside [1+pad, s-pad] are untouched and,
//    for assign with pad>0, transverse ghost planes are zeroed (ops_del.f90:215-229).
// diffType: 1 col CC, 2 col N, 3 stag CC->N, 4 stag N->CC.  gen 1/2/3 =
// assign/add/subtract.
// ===========================================================================
__device__ __forceinline__ double del_point(const DF& in, const DCoord& c, int dir, int diffType, int n,
                                            int gen, int t, int sd, int ia, int ib, double prior, bool& write) {
  // returns the new value at pencil position t (write=false -> untouched)
  // ia/ib: transverse indices; the input pencil is read through lambda-like index math
  auto IN = [&](int tt) -> double {
    int i = dir == 1 ? tt : ia;
    int j = dir == 2 ? tt : (dir == 1 ? ia : ib);
    int k = dir == 3 ? tt : ib;
    return in(i, j, k);
  };
  write = true;
  double sgn = gen == 3 ? -1.0 : 1.0;
  if (diffType >= 3) {
    int gt = diffType == 3 ? 1 : 0;
    const double* D = diffType == 3 ? c.cc2nD : c.n2ccD;
    const double* U = diffType == 3 ? c.cc2nU : c.n2ccU;
    int s = in.s(dir);
    double base = (t == 1 || t == sd) ? 0.0 : prior;
    int i = t - gt;
    if (i >= 1 && i <= s - 1) {
      double v = IN(i) * D[i] + IN(i + 1) * U[i];
      if (gen == 1) return v;
      return gen == 2 ? base + v : base - v;
    }
    return base;
  } else {
    bool cc = diffType == 1;
    int s = in.s(dir);
    const double* L = cc ? c.colCC_L[n - 1] : c.colN_L[n - 1];
    const double* D = cc ? c.colCC_D[n - 1] : c.colN_D[n - 1];
    const double* U = cc ? c.colCC_U[n - 1] : c.colN_U[n - 1];
    if (t == 1 || t == s) return 0.0;
    double acc = prior;
    bool any = false;
    double v = 0.0;
    if (t >= 3 && t <= s - 2) {
      v = IN(t - 1) * L[t - 1] + IN(t) * D[t - 1] + IN(t + 1) * U[t - 1];
      acc = (gen == 1) ? v : acc + sgn * v;
      any = true;
    }
    if (t == 2) {
      if (cc) v = 0.5 * (IN(1) + IN(2)) * L[1] + IN(2) * D[1] + IN(3) * U[1];
      else v = IN(2) * L[1] + IN(3) * D[1] + IN(4) * U[1];
      acc = (gen == 1) ? v : acc + sgn * v;
      any = true;
    }
    if (t == s - 1) {
      if (cc) v = IN(s - 2) * L[s - 2] + IN(s - 1) * D[s - 2] + 0.5 * (IN(s - 1) + IN(s)) * U[s - 2];
      else v = IN(s - 3) * L[s - 2] + IN(s - 2) * D[s - 2] + IN(s - 1) * U[s - 2];
      acc = (gen == 1) ? v : acc + sgn * v;
      any = true;
    }
    if (!any) write = false;
    return acc;
  }
}

__global__ void k_del(DF out, DF in, DCoord c, int dir, int diffType, int n, int pad, int gen) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= out.n()) return;
  int i, j, k;
  ijk_of(idx, out, i, j, k);
  int a = dir == 1 ? 2 : 1, b = dir == 3 ? 2 : 3;
  int ia = pick(a, i, j, k), ib = pick(b, i, j, k);
  int t = pick(dir, i, j, k);
  bool tghost = (ia == 1 || ia == out.s(a) || ib == 1 || ib == out.s(b));
  if (ia < 1 + pad || ia > in.s(a) - pad || ib < 1 + pad || ib > in.s(b) - pad) {
    if (gen == 1 && pad > 0 && tghost) out.f[idx] = 0.0;
    return;
  }
  if (gen == 1 && pad > 0 && tghost) {
    out.f[idx] = 0.0;
    return;
  }
  bool write;
  double v = del_point(in, c, dir, diffType, n, gen, t, out.s(dir), ia, ib, out.f[idx], write);
  if (write) out.f[idx] = v;
}

// ===========================================================================
// Fused centred Laplacian: lap_centered_SF_new (grad then div, CC data,
// ops_discrete.f90:124-132) and lap_centered_SF_given_both (staggered data,
// :112-122), composed per point with the del semantics above:
//   along d where u is CC: N->CC of CC->N   (ends of the CC->N pass are 0)
//   along d where u is N:  CC->N of N->CC   (ends of the CC->N pass are 0)
// the x pass assigns, y and z add; for ghost points along y/z an add pass
// restarts (N->CC) or zeroes (CC->N) the value, as stag_add does.
// ghost_zero: bit f-1 set -> ghost plane of face f set to 0
// (assign_ghost_XPeriodic of div_SF; only the CC form applies it).
// Then out = coeff*lap + (add_x ? u : 0) (mom_diffusion_explicit :176-188)
// when scale_mode != 0.
// ===========================================================================
__device__ __forceinline__ double lap_dir_cc(const DF& u, const DCoord& c, int d, int i, int j, int k, int t,
                                             int s) {
  // CC along d: g(tt) = (u(tt)-u(tt-1))/dhc(tt-1) for tt=2..s, 0 at 1 and s+1
  // result (g(t+1)-g(t))/dhn(t) = g(t)*D + g(t+1)*U
  auto U = [&](int tt) -> double {
    return d == 1 ? u(tt, j, k) : (d == 2 ? u(i, tt, k) : u(i, j, tt));
  };
  double gl = 0.0, gr = 0.0;
  if (t >= 2) gl = U(t - 1) * c.cc2nD[t - 1] + U(t) * c.cc2nU[t - 1];
  if (t + 1 <= s) gr = U(t) * c.cc2nD[t] + U(t + 1) * c.cc2nU[t];
  return gl * c.n2ccD[t] + gr * c.n2ccU[t];
}
__device__ __forceinline__ double lap_dir_n(const DF& u, const DCoord& c, int d, int i, int j, int k, int t,
                                            int s) {
  // N along d: tx(tt) = (u(tt+1)-u(tt))/dhn(tt) for tt=1..s-1;
  // result at t (2..s-1) = tx(t-1)*D(t-1) + tx(t)*U(t-1) with CC2N coeffs
  auto U = [&](int tt) -> double {
    return d == 1 ? u(tt, j, k) : (d == 2 ? u(i, tt, k) : u(i, j, tt));
  };
  double tl = U(t - 1) * c.n2ccD[t - 1] + U(t) * c.n2ccU[t - 1];
  double tr = U(t) * c.n2ccD[t] + U(t + 1) * c.n2ccU[t];
  return tl * c.cc2nD[t - 1] + tr * c.cc2nU[t - 1];
}

__device__ __forceinline__ double lap_centered_point(const DF& u, const DGrid& g, int i, int j, int k) {
  double v = 0.0;
  for (int d = 1; d <= 3; d++) {
    int t = pick(d, i, j, k);
    int s = u.s(d);
    bool nd = n_along(u.dl, d);
    bool end = (t == 1 || t == s);
    double part;
    if (nd) {
      part = end ? 0.0 : lap_dir_n(u, g.c[d - 1], d, i, j, k, t, s);
      v = (d == 1) ? part : (end ? 0.0 : v + part);
    } else {
      part = lap_dir_cc(u, g.c[d - 1], d, i, j, k, t, s);
      v = (d == 1) ? part : (end ? part : v + part);
    }
  }
  return v;
}

__global__ void k_lap_centered(DF out, DF u, DGrid g, int ghost_zero, int scale_mode, double coeff) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= out.n()) return;
  int i, j, k;
  ijk_of(idx, out, i, j, k);
  if (ghost_zero) {
    if (((ghost_zero & 1) && i == 1) || ((ghost_zero & 2) && i == out.s0) || ((ghost_zero & 4) && j == 1) ||
        ((ghost_zero & 8) && j == out.s1) || ((ghost_zero & 16) && k == 1) || ((ghost_zero & 32) && k == out.s2)) {
      out.f[idx] = scale_mode ? (0.0 * coeff + u.f[idx]) : 0.0;
      return;
    }
  }
  double v = lap_centered_point(u, g, i, j, k);
  if (scale_mode) {
    v = v * coeff;
    v = v + u.f[idx];
  }
  out.f[idx] = v;
}

// ===========================================================================
// interpolation: interp_C2N_GF / interp_N2C_GF (GF_interp.f90:19-76) and
// extrap_staggered_GF (GF_extrap.f90:17-46)
// ===========================================================================
__global__ void k_interp_c2n(DF N, DF C, DCoord c, int dir) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= N.n()) return;
  int i, j, k;
  ijk_of(idx, N, i, j, k);
  int t = pick(dir, i, j, k);
  int sN = N.s(dir);
  int di = dir == 1, dj = dir == 2, dk = dir == 3;
  if (t >= 2 && t <= sN - 1) {
    int tt = t - 1;  // theta index
    N.f[idx] = C(i, j, k) * c.thD[tt] + C(i - di, j - dj, k - dk) * c.thU[tt];
  }
}
// end planes: N(1) = 2C(1) - N(2); N(s) = 2C(sc) - N(s-1)  (after interior)
__global__ void k_extrap(DF N, DF C, int dir) {
  int a = dir == 1 ? 2 : 1, b = dir == 3 ? 2 : 3;
  int na = N.s(a), nb = N.s(b);
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= na * nb) return;
  int x = p % na + 1, y = p / na + 1;
  int ia[4];
  ia[a] = x;
  ia[b] = y;
  ia[dir] = 2;
  double n2 = N(ia[1], ia[2], ia[3]);
  ia[dir] = 1;
  double c1 = C(ia[1], ia[2], ia[3]);
  N(ia[1], ia[2], ia[3]) = 2.0 * c1 - n2;
  int sN = N.s(dir);
  ia[dir] = sN - 1;
  double nm = N(ia[1], ia[2], ia[3]);
  ia[dir] = C.s(dir);
  double cs = C(ia[1], ia[2], ia[3]);
  ia[dir] = sN;
  N(ia[1], ia[2], ia[3]) = 2.0 * cs - nm;
}
__global__ void k_interp_n2c(DF C, DF N, int dir) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= C.n()) return;
  int i, j, k;
  ijk_of(idx, C, i, j, k);
  int di = dir == 1, dj = dir == 2, dk = dir == 3;
  C.f[idx] = 0.5 * (N(i, j, k) + N(i + di, j + dj, k + dk));
}

// ===========================================================================
// ghost-cell BCs of one face (HW/BCs/direct/apply_BCs_faces_raw.f90,
// HW/BCs/implicit/apply_BCs_faces_raw_implicit.f90; index sets of
// HW/sub_domain/face_SD_extend.f90:37-84).  One thread per plane point.
// ===========================================================================
__global__ void k_bc_face(DF u, DBC bc, int f, int implicit) {
  int d = (f + 1) / 2;
  bool mn = (f & 1);
  int a = d == 1 ? 2 : 1, b = d == 3 ? 2 : 3;
  int na = u.s(a), nb = u.s(b);
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= na * nb) return;
  int ia[4];
  ia[a] = p % na + 1;
  ia[b] = p / na + 1;
  int s = u.s(d);
  bool N = n_along(u.dl, d);
  int G, B, I, Iopp, Gp, Ip;
  if (!N) {
    G = mn ? 1 : s; I = mn ? 2 : s - 1; Iopp = mn ? s - 1 : 2; B = 0; Gp = G; Ip = Iopp;
  } else {
    G = mn ? 1 : s; B = mn ? 2 : s - 1; I = mn ? 3 : s - 2; Iopp = mn ? s - 2 : 3;
    if (!mn && s > 4) { Gp = s - 1; Ip = 2; } else { Gp = G; Ip = Iopp; }
  }
  auto A = [&](int t) -> double& {
    ia[d] = t;
    return u(ia[1], ia[2], ia[3]);
  };
  double bv = implicit ? 0.0 : bc.value[f];
  double dh = bc.dh[f], nhat = bc.nhat[f], cw = bc.c_w[f];
  switch (bc.type[f]) {
    case MOONS_BC_DIRICHLET:
      if (!N) {
        double ui = A(I);
        A(G) = implicit ? -ui : 2.0 * bv - ui;
      } else {
        double ui = A(I);
        if (implicit) { A(B) = 0.0; A(G) = -ui; }
        else { A(B) = bv; A(G) = 2.0 * bv - ui; }
      }
      break;
    case MOONS_BC_NEUMANN: {
      double ui = A(I);
      if (implicit) A(G) = ui;
      else if (!N) A(G) = ui + bv * (dh * nhat);
      else A(G) = ui + 2.0 * bv * (dh * nhat);
    } break;
    case MOONS_BC_PERIODIC:
      if (bc.prescribed[f] && !implicit) A(G) = bv;
      else if (!N) { double v = A(Iopp); A(G) = v; }
      else { double v = A(Ip); A(Gp) = v; }
      break;
    case MOONS_BC_ROBIN:
      if (!N) {
        double c1 = (2.0 * cw * nhat / dh - 1.0) / (2.0 * cw * nhat / dh + 1.0);
        A(G) = A(I) * c1 + (implicit ? 0.0 : bv * 0.0);
      } else {
        double ui = A(I), ub = A(B);
        if (implicit) A(G) = ui + ub * (-2.0 * dh * nhat / cw);
        else A(G) = ui + ub * (-2.0 * dh / cw * nhat) + bv * (2.0 * dh / cw * nhat);
      }
      break;
    default: break;
  }
}

// ===========================================================================
// plane masks (HW/grid_field/GF_2D/GF_assign_wall.f90, GF_multiply_wall.f90,
// GF_assign_ghost.f90): mode 0 assign v, 1 multiply by v
// ===========================================================================
__global__ void k_plane(DF u, int d, int idx_plane, double v, int mode) {
  int a = d == 1 ? 2 : 1, b = d == 3 ? 2 : 3;
  int na = u.s(a), nb = u.s(b);
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= na * nb) return;
  int ia[4];
  ia[a] = p % na + 1;
  ia[b] = p / na + 1;
  ia[d] = idx_plane;
  double& r = u(ia[1], ia[2], ia[3]);
  r = mode ? r * v : v;
}

// ===========================================================================
// pointwise algebra (HW/grid_field/GF_3D/*) -- whole arrays incl. ghosts
// ===========================================================================
enum PwOp { PW_FILL, PW_COPY, PW_ADD, PW_SUB, PW_MUL, PW_SCALE, PW_ADD_PRODUCT, PW_PRODUCT_ADD, PW_INV };
__global__ void k_pw(int op, double* __restrict__ a, const double* __restrict__ b, double c, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  switch (op) {
    case PW_FILL: a[i] = c; break;
    case PW_COPY: a[i] = b[i]; break;
    case PW_ADD: a[i] = a[i] + b[i]; break;
    case PW_SUB: a[i] = a[i] - b[i]; break;
    case PW_MUL: a[i] = a[i] * b[i]; break;
    case PW_SCALE: a[i] = a[i] * c; break;
    case PW_ADD_PRODUCT: a[i] = a[i] + b[i] * c; break;   // add_product(a,b,c)
    case PW_PRODUCT_ADD: a[i] = a[i] * c + b[i]; break;   // product_add(a,c,b)
    case PW_INV: a[i] = c / a[i]; break;                  // divide(c,a)
  }
}

// ===========================================================================
// deterministic reductions.  Each block reduces a grid-stride share into
// partial[blockIdx.x]; the last block to finish (atomic ticket) sums the
// partials in index order, so the result is independent of block timing.
// ===========================================================================
constexpr int kRedBlocks = 592;  // 4 x 148 SMs
__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ unsigned lin_tid() { return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z); }
__device__ __forceinline__ unsigned lin_nthreads() { return blockDim.x * blockDim.y * blockDim.z; }
// block-wide sum (any block shape, <= 1024 threads); valid in thread 0
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double sh[32];
  unsigned t = lin_tid();
  int lane = t & 31, w = t >> 5;
  v = warp_sum(v);
  if (lane == 0) sh[w] = v;
  __syncthreads();
  unsigned nw = (lin_nthreads() + 31) >> 5;
  v = (t < nw) ? sh[t] : 0.0;
  if (w == 0) v = warp_sum(v);
  __syncthreads();
  return v;
}
// (call after thread 0 wrote this block's partial; only thread 0 fences)
__device__ __forceinline__ bool last_block(unsigned* ticket) {
  __shared__ bool amlast;
  if (lin_tid() == 0) {
    __threadfence();
    unsigned t = atomicAdd(ticket, 1u);
    amlast = (t == gridDim.x - 1);
  }
  __syncthreads();
  return amlast;
}
__device__ __forceinline__ double sum_partials(const double* partial, int n) {
  // fixed-order: each thread sums a strided set, then a fixed tree
  double v = 0.0;
  for (int i = lin_tid(); i < n; i += lin_nthreads()) v += ((volatile const double*)partial)[i];
  return block_sum(v);
}

// interior (pad=1) mask test with Dirichlet-wall planes removed
// (dot_product_SF: multiply, assign_wall_Dirichlet, sum(.,1))
MG_HD bool dot_keep(const DF& a, int i, int j, int k, int wallmask) {
  if (i < 2 || i > a.s0 - 1 || j < 2 || j > a.s1 - 1 || k < 2 || k > a.s2 - 1) return false;
  if (wallmask) {
    if ((wallmask & 1) && i == 2) return false;
    if ((wallmask & 2) && i == a.s0 - 1) return false;
    if ((wallmask & 4) && j == 2) return false;
    if ((wallmask & 8) && j == a.s1 - 1) return false;
    if ((wallmask & 16) && k == 2) return false;
    if ((wallmask & 32) && k == a.s2 - 1) return false;
  }
  return true;
}

}  // namespace mg
