// mgrid.cuh -- geometric multigrid V-cycle for cell-centred Poisson
// problems, used as the preconditioner of (flexible) CG.
//
// Building blocks follow the reference's multigrid pieces
// (code/handwritten/grid_field/GF_MG/GF_restrict.f90:22-82,
// GF_MG/GF_prolongate.f90:22-106, coordinates_extend.f90:336-391 restrict_c,
// solvers/SOR/SOR.f90:234-314 redBlack/init_r) and the V-cycle design of
// code_not_compiled/9.6.2017/MG/MG.f90:241-396 (not compiled in the
// reference):
//  * coarse grids keep every other node of the fine grid along each axis
//    whose interior count is even (stretching kept; other axes unchanged);
//  * prolongation is the reference's prolongate_C: each fine cell takes the
//    mean of its parent's value and the theta-interpolated value at the
//    parent's face nearest to it (linear interpolation on stretched grids);
//  * restriction is the exact transpose of that prolongation (built from the
//    same 1-D weights on the host), so the V-cycle is a symmetric operator
//    and plain CG may use it (the reference's restrict_C is the
//    volume-weighted average; its index expressions for the transverse
//    directions read `i` where `j`/`k` are meant, GF_restrict.f90:38-39);
//  * smoothing is red-black SOR (redBlack, omega = 1.15) on the
//    volume-weighted operator, two forward sweeps (red, black) before the
//    coarse correction and two backward ones (black, red) after it;
//  * ghost values are never stored: a neighbour index on a ghost plane is
//    resolved through the level's homogeneous BCs (Dirichlet -u, Neumann u,
//    periodic opposite side), exactly as apply_BCs_implicit fills them;
//  * the coarsest level is solved directly (dense inverse built on the host,
//    regularised on the constants when no face is Dirichlet), or by a fixed
//    number of symmetric red-black sweeps inside one block when too large.
// Everything is templated on the arithmetic type: T = double for the plain
// path, T = float for the mixed-precision path (V-cycle in FP32 inside an
// FP64 flexible CG).
#pragma once
#include "lean.cuh"

namespace mg {

template <typename T>
struct MGAxis {
  const T *cD, *cU;  // stagCC2N D/U (index 1..sc-1)
  const T *nD, *nU;  // stagN2CC D/U (index 1..sn-1)
  const T* dg;       // laplacian diagonal share of CC data (index 2..sc-1)
  const T* hv;       // cell widths dhn (index 1..sc)
};

template <typename T>
struct MGLev {
  T *e, *r, *t;      // correction, right-hand side, residual (CC, with ghosts)
  int s0, s1, s2;
  MGAxis<T> ax[3];
  const T* w[3];     // face weights of the operator per axis (face arrays): (A e)(c) = sum_f W_f (e_nb - e_c)
  const T* kx;       // face coefficients (LAP_PROPS) or null
  const T* ky;
  const T* kz;
  int bt[7];         // BC type per face (MOONS_BC_*)
};

// prolongation tables of one axis: for fine index f, two coarse interior
// indices (ghosts already resolved) and their weights
template <typename T>
struct MGProl {
  const int* i0;
  const int* i1;
  const T* w0;
  const T* w1;
};
// restriction (transpose) tables of one axis: for coarse interior index I,
// entries off[I] .. off[I+1]-1 of (fi, fw)
template <typename T>
struct MGRest {
  const int* off;
  const int* fi;
  const T* fw;
};

template <typename T>
__device__ __forceinline__ size_t lidx(const MGLev<T>& L, int i, int j, int k) {
  return (size_t)((unsigned)(i - 1) + (unsigned)L.s0 * ((unsigned)(j - 1) + (unsigned)L.s1 * (unsigned)(k - 1)));
}

// value at (i,j,k) of a field whose ghost entries are implied by the level's
// homogeneous BCs
template <typename T>
__device__ __forceinline__ T ev(const MGLev<T>& L, const T* e, int i, int j, int k) {
  T fac = T(1);
  int I[3] = {i, j, k};
  const int s[3] = {L.s0, L.s1, L.s2};
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (I[d] == 1) {
      const int ty = L.bt[2 * d + 1];
      if (ty == MOONS_BC_PERIODIC) I[d] = s[d] - 1;
      else {
        I[d] = 2;
        if (ty == MOONS_BC_DIRICHLET) fac = -fac;
      }
    } else if (I[d] == s[d]) {
      const int ty = L.bt[2 * d + 2];
      if (ty == MOONS_BC_PERIODIC) I[d] = 2;
      else {
        I[d] = s[d] - 1;
        if (ty == MOONS_BC_DIRICHLET) fac = -fac;
      }
    }
  }
  return fac * e[lidx(L, I[0], I[1], I[2])];
}

// index of face (i,j,k) of a face-`d` array on the level's grid (the face
// array has one more entry along d)
template <typename T>
__device__ __forceinline__ size_t fidx(const MGLev<T>& L, int d, int i, int j, int k) {
  const unsigned f0 = (unsigned)L.s0 + (d == 0), f1 = (unsigned)L.s1 + (d == 1);
  return (size_t)((unsigned)(i - 1) + f0 * ((unsigned)(j - 1) + f1 * (unsigned)(k - 1)));
}

// (A e)(i,j,k) = vol * div(k grad e) at an interior point (k = 1 without
// face coefficients) as a sum over the cell's six faces, sum_f W_f (e_nb -
// e0), with the level's precomputed face weights W (the volume-weighted
// operator is symmetric, so one weight per face), and its true diagonal D
// (the smoother's divisor).  A ghost neighbour is implied by the level's
// homogeneous BCs: periodic reads the opposite cell, Neumann repeats the
// point (the face drops out), Dirichlet negates it (-2 W e0 and -2 W in D).
template <typename T>
__device__ __forceinline__ T apply_A(const MGLev<T>& L, const T* e, int i, int j, int k, T& D) {
  const size_t id = lidx(L, i, j, k);
  const size_t sy = (size_t)L.s0, sz = (size_t)L.s0 * L.s1;
  const size_t fx = id + (size_t)(j - 1) + (size_t)L.s1 * (size_t)(k - 1);  // x face (i,j,k)
  const size_t fy = id + (size_t)L.s0 * (size_t)(k - 1);                       // y face (i,j,k)
  const T w[6] = {L.w[0][fx], L.w[0][fx + 1], L.w[1][fy], L.w[1][fy + sy], L.w[2][id], L.w[2][id + sz]};
  const T e0 = e[id];
  // points two or more away from every boundary read no ghost value
  if (i > 2 && i < L.s0 - 1 && j > 2 && j < L.s1 - 1 && k > 2 && k < L.s2 - 1) {
    const T s = ((w[0] + w[1]) + (w[2] + w[3])) + (w[4] + w[5]);
    const T nb = ((w[0] * e[id - 1] + w[1] * e[id + 1]) + (w[2] * e[id - sy] + w[3] * e[id + sy])) +
                 (w[4] * e[id - sz] + w[5] * e[id + sz]);
    D = -s;
    return nb - s * e0;
  }
  const int ii[3] = {i, j, k};
  const int s[3] = {L.s0, L.s1, L.s2};
  const size_t st[3] = {1, sy, sz};
  T acc = T(0), dg = T(0);
#pragma unroll
  for (int d = 0; d < 3; d++) {
#pragma unroll
    for (int hi = 0; hi < 2; hi++) {
      const T wf = w[2 * d + hi];
      const int nbi = ii[d] + (hi ? 1 : -1);
      if (nbi >= 2 && nbi <= s[d] - 1) {
        acc = acc + wf * (hi ? e[id + st[d]] : e[id - st[d]]) - wf * e0;
        dg = dg - wf;
      } else {
        const int ty = L.bt[2 * d + 1 + hi];
        if (ty == MOONS_BC_PERIODIC) {
          const long long off = (long long)(hi ? 2 - ii[d] : s[d] - 1 - ii[d]) * (long long)st[d];
          acc = acc + wf * e[(size_t)((long long)id + off)] - wf * e0;
          dg = dg - wf;
        } else if (ty == MOONS_BC_DIRICHLET) {
          acc = acc - T(2) * wf * e0;
          dg = dg - T(2) * wf;
        }  // Neumann: the ghost repeats the point, the face drops out
      }
    }
  }
  D = dg;
  return acc;
}

// the diagonal D alone
template <typename T>
__device__ __forceinline__ T diag_A(const MGLev<T>& L, int i, int j, int k) {
  const size_t id = lidx(L, i, j, k);
  const size_t sy = (size_t)L.s0, sz = (size_t)L.s0 * L.s1;
  const size_t fx = id + (size_t)(j - 1) + (size_t)L.s1 * (size_t)(k - 1);
  const size_t fy = id + (size_t)L.s0 * (size_t)(k - 1);
  const T w[6] = {L.w[0][fx], L.w[0][fx + 1], L.w[1][fy], L.w[1][fy + sy], L.w[2][id], L.w[2][id + sz]};
  const int ii[3] = {i, j, k};
  const int s[3] = {L.s0, L.s1, L.s2};
  T dg = T(0);
#pragma unroll
  for (int d = 0; d < 3; d++) {
#pragma unroll
    for (int hi = 0; hi < 2; hi++) {
      const int nbi = ii[d] + (hi ? 1 : -1);
      if (nbi >= 2 && nbi <= s[d] - 1) {
        dg = dg - w[2 * d + hi];
      } else {
        const int ty = L.bt[2 * d + 1 + hi];
        if (ty == MOONS_BC_PERIODIC) dg = dg - w[2 * d + hi];
        else if (ty == MOONS_BC_DIRICHLET) dg = dg - T(2) * w[2 * d + hi];
      }
    }
  }
  return dg;
}

// ---- V-cycle steps as grid-stride point loops (thread t0 of nt) ----------

// one red-black half sweep of colour `color` (points with (i+j+k)&1 == color).
// first != 0: e starts at zero (both colours are written).
template <typename T>
__device__ __forceinline__ void mg_smooth_pts(const MGLev<T>& L, int color, int first, T omega, unsigned t0,
                                              unsigned nt) {
  const int nx = L.s0 - 2, ny = L.s1 - 2, nz = L.s2 - 2;
  const int nxh = (nx + 1) / 2;
  const unsigned n = (unsigned)nxh * (unsigned)ny * (unsigned)nz;
  // point t of this colour: (i, j, k), false past the row's end
  auto point = [&](unsigned t, int& i, int& j, int& k) -> bool {
    const unsigned q = t / (unsigned)nxh;
    const int ih = (int)(t - q * (unsigned)nxh);
    const unsigned kk = q / (unsigned)ny;
    j = (int)(q - kk * (unsigned)ny) + 2;
    k = (int)kk + 2;
    i = 2 + ((color + j + k) & 1) + 2 * ih;
    return i <= L.s0 - 1;
  };
  if (first) {
    for (unsigned t = t0; t < n; t += nt) {
      int i, j, k;
      const bool in = point(t, i, j, k);
      // the other colour of this pair starts at zero
      const int io = 2 + ((color + 1 + j + k) & 1) + (i - 2 - ((color + j + k) & 1));
      if (io <= L.s0 - 1) L.e[lidx(L, io, j, k)] = T(0);
      // e = 0 everywhere before this sweep, so A e = 0 and e = r / D
      if (in) L.e[lidx(L, i, j, k)] = omega * L.r[lidx(L, i, j, k)] / diag_A<T>(L, i, j, k);
    }
    return;
  }
  // two points of the colour per trip (t and t + nt): the points of one
  // colour are independent, and both points' loads are in flight together
  for (unsigned t = t0; t < n; t += 2 * nt) {
    int ia, ja, ka, ib = 2, jb = 2, kb = 2;
    const bool a = point(t, ia, ja, ka);
    const bool b = t + nt < n && point(t + nt, ib, jb, kb);
    T Da = T(1), Db = T(1), Aea = T(0), Aeb = T(0), ra = T(0), rb = T(0), ea = T(0), eb = T(0);
    const size_t ida = lidx(L, ia, ja, ka), idb = lidx(L, ib, jb, kb);
    if (a) {
      Aea = apply_A<T>(L, L.e, ia, ja, ka, Da);
      ra = L.r[ida];
      ea = L.e[ida];
    }
    if (b) {
      Aeb = apply_A<T>(L, L.e, ib, jb, kb, Db);
      rb = L.r[idb];
      eb = L.e[idb];
    }
    if (a) L.e[ida] = ea + omega * (ra - Aea) / Da;
    if (b) L.e[idb] = eb + omega * (rb - Aeb) / Db;
  }
}

// t = r - A e at interior points
template <typename T>
__device__ __forceinline__ void mg_resid_pts(const MGLev<T>& L, unsigned t0, unsigned nt) {
  const int nx = L.s0 - 2, ny = L.s1 - 2, nz = L.s2 - 2;
  const unsigned n = (unsigned)nx * (unsigned)ny * (unsigned)nz;
  for (unsigned t = t0; t < n; t += nt) {
    const unsigned q = t / (unsigned)nx;
    const int i = (int)(t - q * (unsigned)nx) + 2;
    const unsigned kk = q / (unsigned)ny;
    const int j = (int)(q - kk * (unsigned)ny) + 2, k = (int)kk + 2;
    T D;
    const T Ae = apply_A<T>(L, L.e, i, j, k, D);
    const size_t id = lidx(L, i, j, k);
    L.t[id] = L.r[id] - Ae;
  }
}

// coarse r = R (fine t), R the transpose of the prolongation
template <typename T>
__device__ __forceinline__ void mg_restrict_pts(const MGLev<T>& F, const MGLev<T>& C, const MGRest<T>& Rx,
                                                const MGRest<T>& Ry, const MGRest<T>& Rz, unsigned t0, unsigned nt) {
  const int nx = C.s0 - 2, ny = C.s1 - 2, nz = C.s2 - 2;
  const unsigned n = (unsigned)nx * (unsigned)ny * (unsigned)nz;
  for (unsigned t = t0; t < n; t += nt) {
    const unsigned q = t / (unsigned)nx;
    const int I = (int)(t - q * (unsigned)nx) + 2;
    const unsigned kk = q / (unsigned)ny;
    const int J = (int)(q - kk * (unsigned)ny) + 2, K = (int)kk + 2;
    T acc = T(0);
    for (int c = Rz.off[K]; c < Rz.off[K + 1]; c++) {
      const int fk = Rz.fi[c];
      const T wz = Rz.fw[c];
      for (int b = Ry.off[J]; b < Ry.off[J + 1]; b++) {
        const int fj = Ry.fi[b];
        const T wyz = Ry.fw[b] * wz;
        T row = T(0);
        for (int a = Rx.off[I]; a < Rx.off[I + 1]; a++) row = row + Rx.fw[a] * F.t[lidx(F, Rx.fi[a], fj, fk)];
        acc = acc + wyz * row;
      }
    }
    C.r[lidx(C, I, J, K)] = acc;
  }
}

// fine e += P (coarse e)
template <typename T>
__device__ __forceinline__ void mg_prolong_pts(const MGLev<T>& F, const MGLev<T>& C, const MGProl<T>& Px,
                                               const MGProl<T>& Py, const MGProl<T>& Pz, unsigned t0, unsigned nt) {
  const int nx = F.s0 - 2, ny = F.s1 - 2, nz = F.s2 - 2;
  const unsigned n = (unsigned)nx * (unsigned)ny * (unsigned)nz;
  for (unsigned t = t0; t < n; t += nt) {
    const unsigned q = t / (unsigned)nx;
    const int i = (int)(t - q * (unsigned)nx) + 2;
    const unsigned kk = q / (unsigned)ny;
    const int j = (int)(q - kk * (unsigned)ny) + 2, k = (int)kk + 2;
    const int ix[2] = {Px.i0[i], Px.i1[i]}, jy[2] = {Py.i0[j], Py.i1[j]}, kz[2] = {Pz.i0[k], Pz.i1[k]};
    const T wx[2] = {Px.w0[i], Px.w1[i]}, wy[2] = {Py.w0[j], Py.w1[j]}, wz[2] = {Pz.w0[k], Pz.w1[k]};
    T acc = T(0);
#pragma unroll
    for (int c = 0; c < 2; c++)
#pragma unroll
      for (int b = 0; b < 2; b++) {
        const T w = wy[b] * wz[c];
        acc = acc + w * (wx[0] * C.e[lidx(C, ix[0], jy[b], kz[c])] + wx[1] * C.e[lidx(C, ix[1], jy[b], kz[c])]);
      }
    const size_t id = lidx(F, i, j, k);
    F.e[id] = F.e[id] + acc;
  }
}

constexpr size_t kRsepMin = 262144;  // fine levels of at least this many cells restrict separably
// separable restriction of a large level, R = Rz Ry Rx applied one axis at a
// time (three 4-tap passes instead of one 64-tap gather per coarse cell):
// x pass F.t -> T1 (cx, fy, fz), y pass T1 -> T2 (cx, cy, fz), z pass
// T2 -> C.r.  T1, T2 are compact interior arrays (x fastest).
template <typename T>
__device__ __forceinline__ void mg_rx_pts(const MGLev<T>& F, const MGRest<T>& Rx, T* t1, int cx, unsigned t0,
                                          unsigned nt) {
  const int fy = F.s1 - 2, fz = F.s2 - 2;
  const unsigned n = (unsigned)cx * (unsigned)fy * (unsigned)fz;
  for (unsigned t = t0; t < n; t += nt) {
    const unsigned q = t / (unsigned)cx;
    const int I = (int)(t - q * (unsigned)cx) + 2;
    const unsigned kk = q / (unsigned)fy;
    const int j = (int)(q - kk * (unsigned)fy) + 2, k = (int)kk + 2;
    T row = T(0);
    for (int a = Rx.off[I]; a < Rx.off[I + 1]; a++) row = row + Rx.fw[a] * F.t[lidx(F, Rx.fi[a], j, k)];
    t1[t] = row;
  }
}
template <typename T>
__device__ __forceinline__ void mg_ry_pts(const T* t1, int cx, int fy, int cy, int fz, const MGRest<T>& Ry, T* t2,
                                          unsigned t0, unsigned nt) {
  const unsigned n = (unsigned)cx * (unsigned)cy * (unsigned)fz;
  for (unsigned t = t0; t < n; t += nt) {
    const unsigned q = t / (unsigned)cx;
    const int I = (int)(t - q * (unsigned)cx);
    const unsigned kk = q / (unsigned)cy;
    const int J = (int)(q - kk * (unsigned)cy) + 2, k = (int)kk;
    T acc = T(0);
    for (int b = Ry.off[J]; b < Ry.off[J + 1]; b++)
      acc = acc + Ry.fw[b] * t1[(size_t)I + (size_t)cx * ((size_t)(Ry.fi[b] - 2) + (size_t)fy * (size_t)k)];
    t2[t] = acc;
  }
}
template <typename T>
__device__ __forceinline__ void mg_rz_pts(const T* t2, const MGLev<T>& C, const MGRest<T>& Rz, unsigned t0,
                                          unsigned nt) {
  const int cx = C.s0 - 2, cy = C.s1 - 2, cz = C.s2 - 2;
  const unsigned n = (unsigned)cx * (unsigned)cy * (unsigned)cz;
  for (unsigned t = t0; t < n; t += nt) {
    const unsigned q = t / (unsigned)cx;
    const int I = (int)(t - q * (unsigned)cx) + 2;
    const unsigned kk = q / (unsigned)cy;
    const int J = (int)(q - kk * (unsigned)cy) + 2, K = (int)kk + 2;
    T acc = T(0);
    for (int c = Rz.off[K]; c < Rz.off[K + 1]; c++)
      acc = acc + Rz.fw[c] * t2[(size_t)(I - 2) + (size_t)cx * ((size_t)(J - 2) + (size_t)cy * (size_t)(Rz.fi[c] - 2))];
    C.r[lidx(C, I, J, K)] = acc;
  }
}

// coarsest level solved directly: e = Minv r over the n interior cells
// (Minv: the inverse of the level's operator, regularised on the constant
// mode when no face is Dirichlet; built on the host, row-major).  Each block
// gathers r into shared memory (rs, n entries) in the inverse's order; warp
// w0, w0 + nw, ... forms one row's dot product each.  Minv and the sum are
// FP64 on every level type: a stretched, high-contrast coarsest operator can
// have a condition number at which an FP32 inverse is no solve at all.
constexpr int kDirectMax = 1024;        // largest coarsest level solved by the dense inverse
constexpr int kDirectRowsPerBlock = 8;  // one warp per row of the inverse
template <typename T>
__device__ __forceinline__ void mg_direct_rows(const MGLev<T>& L, const double* Minv, int n, double* rs, int w0,
                                               int nw) {
  const int nx = L.s0 - 2, ny = L.s1 - 2;
  for (int c = threadIdx.x; c < n; c += blockDim.x) {
    const int i = c % nx + 2, q = c / nx, j = q % ny + 2, k = q / ny + 2;
    rs[c] = (double)L.r[lidx(L, i, j, k)];
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  for (int row = w0; row < n; row += nw) {
    const double* mr = Minv + (size_t)row * n;
    double acc = 0.0;
    for (int c = lane; c < n; c += 32) acc += mr[c] * rs[c];
#pragma unroll
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      const int i = row % nx + 2, q = row / nx, j = q % ny + 2, k = q / ny + 2;
      L.e[lidx(L, i, j, k)] = (T)acc;
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_mg_smooth(MGLev<T> L, int color, int first, T omega, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  mg_smooth_pts(L, color, first, omega, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_mg_resid(MGLev<T> L, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  mg_resid_pts(L, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_mg_restrict(MGLev<T> F, MGLev<T> C, MGRest<T> Rx, MGRest<T> Ry,
                                                     MGRest<T> Rz, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  mg_restrict_pts(F, C, Rx, Ry, Rz, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_mg_rx(MGLev<T> F, MGRest<T> Rx, T* t1, int cx, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  mg_rx_pts(F, Rx, t1, cx, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
template <typename T>
__global__ void __launch_bounds__(256) k_mg_ry(const T* t1, int cx, int fy, int cy, int fz, MGRest<T> Ry, T* t2,
                                               const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  mg_ry_pts(t1, cx, fy, cy, fz, Ry, t2, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}
template <typename T>
__global__ void __launch_bounds__(256) k_mg_rz(const T* t2, MGLev<T> C, MGRest<T> Rz, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  mg_rz_pts(t2, C, Rz, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <typename T>
__global__ void __launch_bounds__(256) k_mg_prolong(MGLev<T> F, MGLev<T> C, MGProl<T> Px, MGProl<T> Py,
                                                    MGProl<T> Pz, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  mg_prolong_pts(F, C, Px, Py, Pz, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// coarsest level: e = 0, then `sweeps` forward red-black sweeps and as many
// backward ones (symmetric), all inside one block
template <typename T>
__global__ void __launch_bounds__(256) k_mg_coarse(MGLev<T> L, int sweeps, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  const int nx = L.s0 - 2, ny = L.s1 - 2, nz = L.s2 - 2;
  const int n = nx * ny * nz;
  for (int t = threadIdx.x; t < n; t += blockDim.x) {
    const int i = t % nx + 2, q = t / nx, j = q % ny + 2, k = q / ny + 2;
    L.e[lidx(L, i, j, k)] = T(0);
  }
  __syncthreads();
  for (int s = 0; s < 4 * sweeps; s++) {
    // forward: colours 0,1,0,1,... ; backward: 1,0,1,0,...
    const int color = s < 2 * sweeps ? (s & 1) : 1 - (s & 1);
    for (int t = threadIdx.x; t < n; t += blockDim.x) {
      const int i = t % nx + 2, q = t / nx, j = q % ny + 2, k = q / ny + 2;
      if (((i + j + k) & 1) != color) continue;
      T D;
      const T Ae = apply_A<T>(L, L.e, i, j, k, D);
      const size_t id = lidx(L, i, j, k);
      L.e[id] = L.e[id] + (L.r[id] - Ae) / D;
    }
    __syncthreads();
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_mg_direct(MGLev<T> L, const double* Minv, int n, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  __shared__ double rs[kDirectMax];
  mg_direct_rows(L, Minv, n, rs, blockIdx.x * kDirectRowsPerBlock + (threadIdx.x >> 5), n);
}

// ---- the learned + mixed (two-stage) preconditioner's scaling -------------
// z = V(r) + gamma N(t), t = r - A V(r): gamma = (N.t) / (N.A N) minimises the
// energy norm of the remaining error e - V(r) - gamma N along N (A e = r, so
// A (e - V(r)) = t).  N is in the finest level's e array; t and the sums are
// FP64; fixed block partition and summation order.
constexpr int kTsBlocks = 296;
template <typename T>
__global__ void __launch_bounds__(256) k_ts_dots(MGLev<T> L, const double* t, double* part, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  const int nx = L.s0 - 2, ny = L.s1 - 2, nz = L.s2 - 2;
  const unsigned n = (unsigned)nx * (unsigned)ny * (unsigned)nz;
  double a = 0.0, b = 0.0;
  for (unsigned q0 = blockIdx.x * blockDim.x + threadIdx.x; q0 < n; q0 += gridDim.x * blockDim.x) {
    const unsigned q = q0 / (unsigned)nx;
    const int i = (int)(q0 - q * (unsigned)nx) + 2;
    const unsigned kk = q / (unsigned)ny;
    const int j = (int)(q - kk * (unsigned)ny) + 2, k = (int)kk + 2;
    T D;
    const T An = apply_A<T>(L, L.e, i, j, k, D);
    const size_t id = lidx(L, i, j, k);
    const double nv = (double)L.e[id];
    a += nv * t[id];
    b += nv * (double)An;
  }
  __shared__ double sa[8], sb[8];
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sa[threadIdx.x >> 5] = a;
    sb[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) {
      ta += sa[w];
      tb += sb[w];
    }
    part[2 * blockIdx.x] = ta;
    part[2 * blockIdx.x + 1] = tb;
  }
}

__global__ void k_ts_gamma(const double* part, int nb, double* gamma, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  const int lane = threadIdx.x & 31;
  double a = 0.0, b = 0.0;
  for (int q = lane; q < nb; q += 32) {
    a += part[2 * q];
    b += part[2 * q + 1];
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  if (lane == 0) {
    const double g = a / b;
    *gamma = (b != 0.0 && isfinite(g)) ? g : 0.0;  // A may be negative definite; no usable direction: z = V(r)
  }
}

__global__ void k_ts_axpy(double* z, const double* N, const double* gamma, size_t n, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  const double g = *gamma;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    z[i] = z[i] + g * N[i];
}

// dst = (Tdst) src over n entries
template <typename Td, typename Ts>
__global__ void k_mg_cast(Td* dst, const Ts* src, size_t n, const PcgScalars* S) {
  pdl_enter();
  if (S && S->done) return;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (Td)src[i];
}

// ---- the outer (flexible) CG around the V-cycle (mgpcg.cu) ----------------

// x += alpha p ; r -= alpha Ap ; r_prev = old r (flexible) ; r.r over the
// interior; the last block runs update_exit_loop
__global__ void __launch_bounds__(kLB) k_m_update(DF x, DF p, DF r, DF Ap, double* rprev, PcgScalars* S,
                                                  double* partial, unsigned* ticket) {
  pdl_enter();
  if (S->done) return;
  const double alpha = S->alpha;
  if (S->stag_window > 0 && !(isfinite(alpha) && alpha > 0.0)) {
    // learned preconditioner broke down: alpha = z.r / p.Ap must be positive
    // and finite (z.r and p.Ap share the operator's sign when the
    // preconditioner is definite like the operator).  Leave x and r as they
    // are and hand over to the fallback (exit_reason 4); every block sees
    // the same alpha and returns here
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      S->exit_reason = 4;
      S->done = 1;
    }
    return;
  }
  double arr = 0.0;
  const unsigned n = (unsigned)x.n();
  for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
    const double rv = r.f[id];
    if (rprev) rprev[id] = rv;
    x.f[id] = x.f[id] + p.f[id] * alpha;
    const double rn = rv + Ap.f[id] * (-alpha);
    r.f[id] = rn;
    int i, j, k;
    ijk_of(id, x, i, j, k);
    if (i > 1 && i < x.s0 && j > 1 && j < x.s1 && k > 1 && k < x.s2) arr += rn * rn;
  }
  const double s_rr = block_sum(arr);
  if (threadIdx.x == 0) partial[blockIdx.x] = s_rr;
  if (last_block(ticket)) {
    const double rr = sum_partials(partial, gridDim.x);
    if (threadIdx.x == 0) {
      *ticket = 0;
      S->rr = rr;
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
      if (!stop && S->iter >= S->iter_max) {
        stop = true;
        S->exit_reason = 3;
      }
      if (!stop && S->stag_window > 0 && S->iter % S->stag_window == 0) {
        const double res = sqrt(fabs(rr));
        if (res > S->stag_factor * S->stag_ref) {
          stop = true;
          S->res = res;
          S->exit_reason = 4;
        }
        S->stag_ref = res;
      }
      S->done = stop ? 1 : 0;
    }
  }
}

// rho' = z.r (interior), flexible: minus z.r_prev; beta = that / rho
__global__ void __launch_bounds__(kLB) k_m_beta(DF z, DF r, const double* rprev, PcgScalars* S, double* partial,
                                                unsigned* ticket) {
  pdl_enter();
  if (S->done) return;
  double azr = 0.0, azp = 0.0;
  const unsigned n = (unsigned)z.n();
  for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x) {
    int i, j, k;
    ijk_of(id, z, i, j, k);
    if (i > 1 && i < z.s0 && j > 1 && j < z.s1 && k > 1 && k < z.s2) {
      const double zv = z.f[id];
      azr += zv * r.f[id];
      if (rprev) azp += zv * rprev[id];
    }
  }
  const double s1 = block_sum(azr);
  const double s2 = block_sum(azp);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = s1;
    partial[gridDim.x + blockIdx.x] = s2;
  }
  if (last_block(ticket)) {
    const double zr = sum_partials(partial, gridDim.x);
    const double zp = sum_partials(partial + gridDim.x, gridDim.x);
    if (threadIdx.x == 0) {
      *ticket = 0;
      S->zr = zr;
      S->beta = (rprev ? zr - zp : zr) / S->rhok;
      S->rhok = zr;
    }
  }
}

// p' = z + beta p (every point; BC points are rewritten by k_l_bcfill)
__global__ void __launch_bounds__(kLB) k_m_pupd(DF pn, DF p, DF z, const PcgScalars* S) {
  pdl_enter();
  if (S->done) return;
  const double beta = S->beta;
  const unsigned n = (unsigned)p.n();
  for (unsigned id = blockIdx.x * blockDim.x + threadIdx.x; id < n; id += gridDim.x * blockDim.x)
    pn.f[id] = z.f[id] + p.f[id] * beta;
}

}  // namespace mg
