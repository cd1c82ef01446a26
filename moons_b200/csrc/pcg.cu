// pcg.cu -- matrix-free Jacobi-PCG (PCG_solver_algorithm.f90:37-179) with
// every scalar of the recurrence kept on the device.
//
// One iteration is a fixed sequence of launches (implicit BCs of p, the
// operator, a fused mask*vol + dot(p,Ap) kernel whose last block forms
// alpha, a fused x/r/z update + dot(r,r) + dot(z,r) kernel whose last block
// runs the exit test of update_exit_loop and forms beta, and p = beta p + z).
// The whole loop is captured once into a CUDA graph whose WHILE node repeats
// the body until the device-side exit flag is set; the flag also comes up
// when the iteration count reaches iter_max, so the loop always ends.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "kernels.cuh"
#include "runtime.cuh"

namespace mg {

struct PcgScalars {
  double rhok, alpha, res, res0, beta, pap, rr, zr, mean;
  int iter, done, exit_reason, nan;
  int iter_max, nskip;
  double tol_rel, tol_abs;
  int body_runs;  // executions of the loop body (second bound on the loop)
};

struct WallMask {  // masks applied to Ap, from the BCs of x_BC (PCG_solver_algorithm.f90:72-75)
  int neu, dir, per;  // face bits (Neumann x0.5, Dirichlet =0); dir bits for periodic_single
};

struct Comp3 {
  DF a[3];
  int nc;
};

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
__device__ __forceinline__ double wall_factor(const DF& a, int i, int j, int k, const WallMask& w, bool& zero) {
  // multiply_wall_Neumann(0.5) then assign_wall_Dirichlet(0) then assign_wall_Periodic_single(0)
  double f = 1.0;
  zero = false;
  int t[4] = {0, i, j, k};
  for (int d = 1; d <= 3; d++) {
    int s = a.s(d);
    if ((w.neu >> (2 * d - 2)) & 1 && t[d] == 2) f *= 0.5;
    if ((w.neu >> (2 * d - 1)) & 1 && t[d] == s - 1) f *= 0.5;
    if ((w.dir >> (2 * d - 2)) & 1 && t[d] == 2) zero = true;
    if ((w.dir >> (2 * d - 1)) & 1 && t[d] == s - 1) zero = true;
    if ((w.per >> (d - 1)) & 1 && t[d] == s - 1) zero = true;
  }
  return f;
}

// Ap <- mask(Ap)*vol ; pap = dot(p,Ap) over the interior minus Dirichlet walls of x;
// last block: alpha = rhok/pap
__global__ void k_pcg_ap(Comp3 Ap, Comp3 p, Comp3 vol, WallMask wm0, WallMask wm1, WallMask wm2, int dw0, int dw1,
                         int dw2, PcgScalars* S, double* partial, unsigned* ticket) {
  if (S->done) return;
  const WallMask wm[3] = {wm0, wm1, wm2};
  const int dw[3] = {dw0, dw1, dw2};
  double acc = 0.0;
  size_t off = 0;
  for (int c = 0; c < Ap.nc; c++) {
    const DF& A = Ap.a[c];
    size_t n = A.n();
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
      int i, j, k;
      ijk_of(idx, A, i, j, k);
      bool zero;
      double f = wall_factor(A, i, j, k, wm[c], zero);
      double v = A.f[idx];
      if (f != 1.0) v = v * f;
      if (zero) v = 0.0;
      v = v * vol.a[c].f[idx];
      A.f[idx] = v;
      if (dot_keep(A, i, j, k, dw[c])) acc += p.a[c].f[idx] * v;
    }
    off += n;
  }
  double bs = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
  if (last_block(ticket)) {
    double tot = sum_partials(partial, gridDim.x);
    if (threadIdx.x == 0) {
      S->pap = tot;
      S->alpha = S->rhok / tot;
      *ticket = 0;
    }
  }
}

// x += alpha p ; r -= alpha Ap ; z = Minv r ; rr = dot(r,r), zr = dot(z,r);
// last block: iteration count, exit test, beta
__global__ void k_pcg_update(Comp3 x, Comp3 p, Comp3 r, Comp3 Ap, Comp3 z, Comp3 Minv, int dw0, int dw1, int dw2,
                             PcgScalars* S, double* partial, unsigned* ticket) {
  if (S->done) return;
  const int dw[3] = {dw0, dw1, dw2};
  double alpha = S->alpha;
  double arr = 0.0, azr = 0.0;
  for (int c = 0; c < x.nc; c++) {
    const DF& X = x.a[c];
    size_t n = X.n();
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
      X.f[idx] = X.f[idx] + p.a[c].f[idx] * alpha;
      double rv = r.a[c].f[idx] + Ap.a[c].f[idx] * (-alpha);
      r.a[c].f[idx] = rv;
      double zv = Minv.a[c].f[idx] * rv;
      z.a[c].f[idx] = zv;
      int i, j, k;
      ijk_of(idx, X, i, j, k);
      if (dot_keep(X, i, j, k, dw[c])) {
        arr += rv * rv;
        azr += zv * rv;
      }
    }
  }
  double b1 = block_sum(arr);
  double b2 = block_sum(azr);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = b1;
    partial[kRedBlocks + blockIdx.x] = b2;
  }
  if (last_block(ticket)) {
    double rr = sum_partials(partial, gridDim.x);
    double zr = sum_partials(partial + kRedBlocks, gridDim.x);
    if (threadIdx.x == 0) {
      *ticket = 0;
      S->rr = rr;
      S->zr = zr;
      S->iter += 1;
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

// p = p*beta + z  (product_add)
__global__ void k_pcg_p(Comp3 p, Comp3 z, PcgScalars* S) {
  if (S->done) return;
  double beta = S->beta;
  for (int c = 0; c < p.nc; c++) {
    size_t n = p.a[c].n();
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x)
      p.a[c].f[idx] = p.a[c].f[idx] * beta + z.a[c].f[idx];
  }
}

// generic two-level reduction: mode 0 dot(a,b) masked interior, 1 sum(a^2) whole array,
// 2 sum(a*b) over interior pad 1 (no wall mask)
__global__ void k_reduce(Comp3 a, Comp3 b, int mode, int dw0, int dw1, int dw2, double* out, double* partial,
                         unsigned* ticket) {
  const int dw[3] = {dw0, dw1, dw2};
  double acc = 0.0;
  for (int c = 0; c < a.nc; c++) {
    const DF& A = a.a[c];
    size_t n = A.n();
    for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
      if (mode == 1) {
        double v = A.f[idx];
        acc += v * v;
      } else {
        int i, j, k;
        ijk_of(idx, A, i, j, k);
        if (dot_keep(A, i, j, k, mode == 0 ? dw[c] : 0)) acc += A.f[idx] * b.a[c].f[idx];
      }
    }
  }
  double bs = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
  if (last_block(ticket)) {
    double tot = sum_partials(partial, gridDim.x);
    if (threadIdx.x == 0) {
      *out = tot;
      *ticket = 0;
    }
  }
}

// start of the solve, after res0 (=sum r^2) and rhok (=dot(r,z)) were reduced
__global__ void k_pcg_start(PcgScalars* S) {
  S->res0 = sqrt(S->res0);
  S->res = sqrt(fabs(S->rhok));
  S->iter = 0;
  S->body_runs = 0;
  S->nan = isnan(S->res0) ? 1 : 0;
  S->exit_reason = 0;
  bool e2 = S->res < S->tol_abs;  // only exit_loop(2) skips the loop (PCG_solver_algorithm.f90:68)
  S->done = (e2 || S->iter_max <= 0 || S->nan) ? 1 : 0;
  if (e2) {
    S->exit_reason = 2;
    S->iter = 1;  // update_iter in the else branch
  }
}

// r -= mean, mean = sum(r*vol, pad 1)/vol%vol (subtract_phys_mean_vol_SF)
__global__ void k_sub_mean(DF r, const double* sum, double volsum) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= r.n()) return;
  double mean = *sum / volsum;
  r.f[idx] = r.f[idx] - mean;
}

// volume_DL_GF (GF_distributions.f90:61-88)
__global__ void k_volume(DF u, DGrid g) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= u.n()) return;
  int i, j, k;
  ijk_of(idx, u, i, j, k);
  if (i < 2 || i > u.s0 - 1 || j < 2 || j > u.s1 - 1 || k < 2 || k > u.s2 - 1) {
    u.f[idx] = 0.0;
    return;
  }
  int ex = n_along(u.dl, 1), ey = n_along(u.dl, 2), ez = n_along(u.dl, 3);
  double hx = ex ? g.c[0].dhc[i - 1] : g.c[0].dhn[i];
  double hy = ey ? g.c[1].dhc[j - 1] : g.c[1].dhn[j];
  double hz = ez ? g.c[2].dhc[k - 1] : g.c[2].dhn[k];
  u.f[idx] = hx * hy * hz;
}

// Jacobi preconditioners (preconditioners.f90:55-129, GF_diagonals.f90:15-71):
// mode 1 Lap: 1/(diag*vol); 2 mom: 1/((diag*c+1)*vol); 3 ind: 1/((cc_diag*c+1)*vol);
// ghost planes 0 (Minv carries no BCs, so assign_ghost_XPeriodic zeroes all six).
__global__ void k_prec(DF M, DGrid g, int mode, double coeff, int comp, DF sx, DF sy, DF sz) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= M.n()) return;
  int i, j, k;
  ijk_of(idx, M, i, j, k);
  bool ghost = (i == 1 || i == M.s0 || j == 1 || j == M.s1 || k == 1 || k == M.s2);
  if (mode == 0) {  // prec_Identity_SF: assign(Minv,1)
    M.f[idx] = 1.0;
    return;
  }
  if (ghost) {
    M.f[idx] = 0.0;
    return;
  }
  const DCoord &c1 = g.c[0], &c2 = g.c[1], &c3 = g.c[2];
  double d;
  if (mode == 1 || mode == 2) {
    int px = n_along(M.dl, 1), py = n_along(M.dl, 2), pz = n_along(M.dl, 3);
    d = c1.n2ccD[i] * c1.cc2nU[i - 1] + c1.n2ccU[i - px] * c1.cc2nD[i - px] + c2.n2ccD[j] * c2.cc2nU[j - 1] +
        c2.n2ccU[j - py] * c2.cc2nD[j - py] + c3.n2ccD[k] * c3.cc2nU[k - 1] + c3.n2ccU[k - pz] * c3.cc2nD[k - pz];
  } else {
    if (comp == 0)
      d = -c2.n2ccD[j] * sz(i, j, k) * c2.cc2nU[j - 1] - c2.n2ccU[j] * sz(i, j + 1, k) * c2.cc2nD[j] -
          c3.n2ccD[k] * sy(i, j, k) * c3.cc2nU[k - 1] - c3.n2ccU[k] * sy(i, j, k + 1) * c3.cc2nD[k];
    else if (comp == 1)
      d = -c1.n2ccD[i] * sz(i, j, k) * c1.cc2nU[i - 1] - c1.n2ccU[i] * sz(i + 1, j, k) * c1.cc2nD[i] -
          c3.n2ccD[k] * sx(i, j, k) * c3.cc2nU[k - 1] - c3.n2ccU[k] * sx(i, j, k + 1) * c3.cc2nD[k];
    else
      d = -c1.n2ccD[i] * sy(i, j, k) * c1.cc2nU[i - 1] - c1.n2ccU[i] * sy(i + 1, j, k) * c1.cc2nD[i] -
          c2.n2ccD[j] * sx(i, j, k) * c2.cc2nU[j - 1] - c2.n2ccU[j] * sx(i, j + 1, k) * c2.cc2nD[j];
  }
  if (mode >= 2) {
    d = d * coeff;
    d = d + 1.0;
  }
  int ex = n_along(M.dl, 1), ey = n_along(M.dl, 2), ez = n_along(M.dl, 3);
  double vol = (ex ? c1.dhc[i - 1] : c1.dhn[i]) * (ey ? c2.dhc[j - 1] : c2.dhn[j]) * (ez ? c3.dhc[k - 1] : c3.dhn[k]);
  M.f[idx] = 1.0 / (d * vol);
}

__global__ void k_set_cond(cudaGraphConditionalHandle h, PcgScalars* S) {
  S->body_runs += 1;
  bool go = !S->done && S->body_runs < S->iter_max + 2;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

}  // namespace mg

using namespace mg;

// ---------------------------------------------------------------------------
// the PCG object
// ---------------------------------------------------------------------------
struct moons_pcg {
  moons_mesh* m = nullptr;
  int op = 0, prec = 0, nc = 1;
  double coeff = 0.0;
  DF p[3]{}, xbc[3]{}, r[3]{}, Ax[3]{}, vol[3]{}, z[3]{}, Minv[3]{}, tempx[3]{}, k[3]{}, tempk[3]{};
  DBC xbc_bc[3]{};   // BCs of x_BC
  DBC x_bc[3]{};     // BCs of x, copied to p
  int x_dl[3] = {0, 0, 0};
  int all_neumann = 0;
  double volsum[3] = {0, 0, 0};
  PcgScalars* S = nullptr;   // device
  PcgScalars* hS = nullptr;  // pinned host
  std::vector<void*> allocs;
  // graph of the loop (rebuilt when x changes)
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double* gx[3] = {nullptr, nullptr, nullptr};
  long long body_launches = 0;  // kernels per execution of the loop body
};

namespace {
int alloc_df(moons_pcg* s, DF& f, int dl) {
  f = make_df(s->m, dl, nullptr);
  if (cudaMalloc(&f.f, f.n() * sizeof(double)) != cudaSuccess) {
    set_error("moons_pcg: device allocation failed");
    return MOONS_ERR_NOMEM;
  }
  cudaMemsetAsync(f.f, 0, f.n() * sizeof(double), s->m->stream);
  s->allocs.push_back(f.f);
  return MOONS_OK;
}
Comp3 c3(const DF* a, int nc) {
  Comp3 r{};
  r.nc = nc;
  for (int c = 0; c < nc; c++) r.a[c] = a[c];
  return r;
}
unsigned red_grid(const DF* a, int nc) {
  size_t n = 0;
  for (int c = 0; c < nc; c++) n += a[c].n();
  return (unsigned)std::min<size_t>(kRedBlocks, std::max<size_t>(1, (n + kBlock - 1) / kBlock));
}
WallMask wall_mask_of(const DBC& b, int dl, int s[4]) {
  WallMask w{0, 0, 0};
  for (int f = 1; f <= 6; f++) {
    int d = (f + 1) / 2;
    if (!n_along(dl, d)) continue;
    bool def = b.defined != 0;
    if (def ? b.type[f] == MOONS_BC_NEUMANN : true) w.neu |= 1 << (f - 1);
    if (def ? b.type[f] == MOONS_BC_DIRICHLET : true) w.dir |= 1 << (f - 1);
  }
  if (b.defined)
    for (int d = 1; d <= 3; d++)
      if (n_along(dl, d) && b.type[2 * d - 1] == MOONS_BC_PERIODIC && b.type[2 * d] == MOONS_BC_PERIODIC && s[d] > 4)
        w.per |= 1 << (d - 1);
  return w;
}

// operator_explicit of matrix_free_operators.f90 on component fields
int apply_op_explicit(moons_pcg* s, DF* out, DF* x) {
  moons_mesh* m = s->m;
  int r = MOONS_OK;
  switch (s->op) {
    case MOONS_OP_LAP_UNIFORM:
      for (int c = 0; c < s->nc && !r; c++) {
        int gz = (x[c].dl == MOONS_CC) ? ghost_zero_bits(nullptr) : 0;  // Ax carries no BCs
        r = launch_lap_centered(m, out[c], x[c], gz, 0, 0.0);
      }
      break;
    case MOONS_OP_MOM_DIFFUSION:
      for (int c = 0; c < s->nc && !r; c++) {
        int gz = (x[c].dl == MOONS_CC) ? ghost_zero_bits(nullptr) : 0;
        if (gz) {
          r = launch_lap_centered(m, out[c], x[c], gz, 0, 0.0);
          if (!r) r = launch_pw(m, PW_PRODUCT_ADD, out[c], &x[c], s->coeff);
        } else {
          r = launch_lap_centered(m, out[c], x[c], 0, 1, s->coeff);
        }
      }
      break;
    case MOONS_OP_LAP_PROPS: {
      for (int d = 0; d < 3 && !r; d++) r = launch_del(m, s->tempk[d], x[0], 1, d + 1, 0, 1);
      for (int d = 0; d < 3 && !r; d++) r = launch_pw(m, PW_MUL, s->tempk[d], &s->k[d], 0.0);
      if (!r) r = launch_del(m, out[0], s->tempk[0], 1, 1, 0, 1);
      if (!r) r = launch_del(m, out[0], s->tempk[1], 1, 2, 0, 2);
      if (!r) r = launch_del(m, out[0], s->tempk[2], 1, 3, 0, 2);
      if (!r) r = mask_ghost_XPeriodic(m, out[0], nullptr);
    } break;
    case MOONS_OP_IND_DIFFUSION: {
      DF* t = s->tempk;
      // curl(tempk, x): faces -> edges
      if (!r) r = launch_del(m, t[0], x[2], 1, 2, 0, 1);
      if (!r) r = launch_del(m, t[0], x[1], 1, 3, 0, 3);
      if (!r) r = launch_del(m, t[1], x[0], 1, 3, 0, 1);
      if (!r) r = launch_del(m, t[1], x[2], 1, 1, 0, 3);
      if (!r) r = launch_del(m, t[2], x[1], 1, 1, 0, 1);
      if (!r) r = launch_del(m, t[2], x[0], 1, 2, 0, 3);
      for (int d = 0; d < 3 && !r; d++) r = launch_pw(m, PW_MUL, t[d], &s->k[d], 0.0);
      // curl(Ax, tempk): edges -> faces
      if (!r) r = launch_del(m, out[0], t[2], 1, 2, 0, 1);
      if (!r) r = launch_del(m, out[0], t[1], 1, 3, 0, 3);
      if (!r) r = launch_del(m, out[1], t[0], 1, 3, 0, 1);
      if (!r) r = launch_del(m, out[1], t[2], 1, 1, 0, 3);
      if (!r) r = launch_del(m, out[2], t[1], 1, 1, 0, 1);
      if (!r) r = launch_del(m, out[2], t[0], 1, 2, 0, 3);
      for (int c = 0; c < 3 && !r; c++) r = launch_pw(m, PW_PRODUCT_ADD, out[c], &x[c], s->coeff);
    } break;
    default:
      set_error("moons_pcg: unknown operator");
      return MOONS_ERR_ARG;
  }
  return r;
}

int compute_prec(moons_pcg* s) {
  moons_mesh* m = s->m;
  int mode = s->prec;
  DF dummy{};
  for (int c = 0; c < s->nc; c++) {
    DF sx = s->op == MOONS_OP_IND_DIFFUSION ? s->k[0] : dummy;
    DF sy = s->op == MOONS_OP_IND_DIFFUSION ? s->k[1] : dummy;
    DF sz = s->op == MOONS_OP_IND_DIFFUSION ? s->k[2] : dummy;
    if (mode == MOONS_PREC_IND && s->op != MOONS_OP_IND_DIFFUSION) {
      set_error("moons_pcg: prec_ind needs the induction operator's sigma^-1 edge fields");
      return MOONS_ERR_ARG;
    }
    MG_LAUNCH(k_prec, nblocks(s->Minv[c].n()), kBlock, m->stream, s->Minv[c], m->dg, mode, s->coeff, c, sx, sy, sz);
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// one PCG iteration (PCG_solver_algorithm.f90:69-96), enqueued on the mesh stream
int enqueue_iteration(moons_pcg* s, DF* x) {
  moons_mesh* m = s->m;
  int r = MOONS_OK;
  for (int c = 0; c < s->nc && !r; c++) r = launch_bcs(m, s->p[c], s->x_bc[c], true);
  if (!r) r = apply_op_explicit(s, s->Ax, s->p);
  if (r) return r;
  int sarr[3][4];
  WallMask wm[3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
  int dw[3] = {0, 0, 0};
  for (int c = 0; c < s->nc; c++) {
    sarr[c][1] = s->Ax[c].s0;
    sarr[c][2] = s->Ax[c].s1;
    sarr[c][3] = s->Ax[c].s2;
    wm[c] = wall_mask_of(s->xbc_bc[c], s->xbc[c].dl, sarr[c]);
    dw[c] = dirichlet_wall_bits(s->x_bc[c].defined ? &s->x_bc[c] : nullptr, s->x_dl[c]);
  }
  unsigned G = red_grid(s->Ax, s->nc);
  MG_LAUNCH(k_pcg_ap, G, kBlock, m->stream, c3(s->Ax, s->nc), c3(s->p, s->nc), c3(s->vol, s->nc), wm[0], wm[1], wm[2],
                                        dw[0], dw[1], dw[2], s->S, m->d_partial, m->d_ticket);
  MG_LAUNCH(k_pcg_update, G, kBlock, m->stream, c3(x, s->nc), c3(s->p, s->nc), c3(s->r, s->nc), c3(s->Ax, s->nc),
                                            c3(s->z, s->nc), c3(s->Minv, s->nc), dw[0], dw[1], dw[2], s->S,
                                            m->d_partial + 2 * kRedBlocks, m->d_ticket + 1);
  MG_LAUNCH(k_pcg_p, G, kBlock, m->stream, c3(s->p, s->nc), c3(s->z, s->nc), s->S);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

int build_graph(moons_pcg* s, DF* x) {
  moons_mesh* m = s->m;
  if (s->exec) {
    cudaGraphExecDestroy(s->exec);
    s->exec = nullptr;
  }
  if (s->graph) {
    cudaGraphDestroy(s->graph);
    s->graph = nullptr;
  }
  MG_CUDA(cudaGraphCreate(&s->graph, 0));
  cudaGraphConditionalHandle h;
  MG_CUDA(cudaGraphConditionalHandleCreate(&h, s->graph, 1, cudaGraphCondAssignDefault));
  cudaGraphNodeParams cp = {};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = h;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t node;
  MG_CUDA(cudaGraphAddNode(&node, s->graph, nullptr, 0, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  MG_CUDA(cudaStreamBeginCaptureToGraph(m->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  long long before = g_launch_count;  // captured launches run later, once per body execution
  int r = enqueue_iteration(s, x);
  MG_LAUNCH(k_set_cond, 1, 1, m->stream, h, s->S);
  s->body_launches = g_launch_count - before;
  g_launch_count = before;
  cudaGraph_t captured = nullptr;
  cudaError_t e = cudaStreamEndCapture(m->stream, &captured);
  if (r) return r;
  MG_CUDA(e);
  MG_CUDA(cudaGraphInstantiate(&s->exec, s->graph, 0));
  for (int c = 0; c < s->nc; c++) s->gx[c] = x[c].f;
  return MOONS_OK;
}
}  // namespace

extern "C" {

int moons_pcg_create(moons_mesh* m, int op, int prec, int nc, moons_sf* const* x, moons_sf* const* x_bc,
                     moons_sf* const* k, moons_pcg** out) {
  if (!m || !x || !x_bc || !out) {
    set_error("moons_pcg_create: null pointer");
    return MOONS_ERR_ARG;
  }
  if (nc != 1 && nc != 3) {
    set_error("moons_pcg_create: ncomp must be 1 or 3");
    return MOONS_ERR_ARG;
  }
  if (op < MOONS_OP_LAP_UNIFORM || op > MOONS_OP_MOM_DIFFUSION || prec < 0 || prec > MOONS_PREC_IND) {
    set_error("moons_pcg_create: bad operator/preconditioner");
    return MOONS_ERR_ARG;
  }
  if ((op == MOONS_OP_LAP_PROPS && nc != 1) || (op == MOONS_OP_IND_DIFFUSION && nc != 3)) {
    set_error("moons_pcg_create: operator/component count mismatch");
    return MOONS_ERR_ARG;
  }
  bool needk = (op == MOONS_OP_LAP_PROPS || op == MOONS_OP_IND_DIFFUSION);
  if (needk && (!k || !k[0] || !k[1] || !k[2])) {
    set_error("moons_pcg_create: operator needs three coefficient fields");
    return MOONS_ERR_ARG;
  }
  cudaSetDevice(m->device);
  auto* s = new moons_pcg();
  s->m = m;
  s->op = op;
  s->prec = prec;
  s->nc = nc;
  int r = MOONS_OK;
  for (int c = 0; c < nc && !r; c++) {
    if (!x[c] || !x_bc[c] || x[c]->m != m) {
      set_error("moons_pcg_create: bad x field");
      r = MOONS_ERR_ARG;
      break;
    }
    int dl = x[c]->f.dl;
    s->x_dl[c] = dl;
    s->x_bc[c] = x[c]->bc;
    s->xbc_bc[c] = x_bc[c]->bc;
    if (!r) r = alloc_df(s, s->p[c], dl);
    if (!r) r = alloc_df(s, s->xbc[c], x_bc[c]->f.dl);
    if (!r) r = alloc_df(s, s->r[c], dl);
    if (!r) r = alloc_df(s, s->Ax[c], dl);
    if (!r) r = alloc_df(s, s->vol[c], dl);
    if (!r) r = alloc_df(s, s->z[c], dl);
    if (!r) r = alloc_df(s, s->Minv[c], dl);
    if (!r) r = alloc_df(s, s->tempx[c], dl);
  }
  s->all_neumann = (nc == 1) ? x[0]->all_neumann : 0;
  if (!r && needk) {
    for (int d = 0; d < 3 && !r; d++) {
      r = alloc_df(s, s->k[d], k[d]->f.dl);
      if (!r) r = alloc_df(s, s->tempk[d], k[d]->f.dl);
      if (!r)
        if (cudaMemcpyAsync(s->k[d].f, k[d]->f.f, k[d]->f.n() * sizeof(double), cudaMemcpyDeviceToDevice,
                            m->stream) != cudaSuccess)
          r = MOONS_ERR_CUDA;
    }
  }
  if (!r) {
    void* p;
    if (cudaMalloc(&p, sizeof(PcgScalars)) != cudaSuccess) r = MOONS_ERR_NOMEM;
    else {
      s->S = (PcgScalars*)p;
      s->allocs.push_back(p);
    }
    if (!r && cudaMallocHost(&p, sizeof(PcgScalars)) != cudaSuccess) r = MOONS_ERR_NOMEM;
    else if (!r) s->hS = (PcgScalars*)p;
  }
  if (!r) {
    for (int c = 0; c < nc; c++) MG_LAUNCH(k_volume, nblocks(s->vol[c].n()), kBlock, m->stream, s->vol[c], m->dg);
    // coeff_implicit is not known here; Lap needs none and mom/ind set it through update_mfp
    r = compute_prec(s);
  }
  if (!r) {
    // plain sums of vol (ghosts are 0, so interior sum == whole sum)
    for (int c = 0; c < nc; c++) {
      std::vector<double> hv(s->vol[c].n());
      if (cudaMemcpyAsync(hv.data(), s->vol[c].f, hv.size() * sizeof(double), cudaMemcpyDeviceToHost, m->stream) !=
          cudaSuccess) {
        r = MOONS_ERR_CUDA;
        break;
      }
      cudaStreamSynchronize(m->stream);
      double t = 0;
      for (double v : hv) t += v;
      s->volsum[c] = t;
    }
  }
  if (!r && cudaStreamSynchronize(m->stream) != cudaSuccess) r = cuda_fail(cudaGetLastError(), "pcg create");
  if (r) {
    moons_pcg_destroy(s);
    return r;
  }
  *out = s;
  return MOONS_OK;
}

int moons_pcg_destroy(moons_pcg* s) {
  if (!s) return MOONS_OK;
  cudaSetDevice(s->m->device);
  cudaStreamSynchronize(s->m->stream);
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  for (void* p : s->allocs) cudaFree(p);
  if (s->hS) cudaFreeHost(s->hS);
  delete s;
  return MOONS_OK;
}

int moons_pcg_update_mfp(moons_pcg* s, double c, int upd) {
  if (!s) {
    set_error("null pcg");
    return MOONS_ERR_ARG;
  }
  s->coeff = c;
  if (s->exec) {  // the coefficient is baked into the captured launches
    cudaGraphExecDestroy(s->exec);
    s->exec = nullptr;
    cudaGraphDestroy(s->graph);
    s->graph = nullptr;
  }
  if (upd) {
    int r = compute_prec(s);
    if (r) return r;
  }
  return MOONS_OK;
}

int moons_pcg_solve(moons_pcg* s, moons_sf* const* x, moons_sf* const* b, const moons_isp* isp,
                    moons_solve_info* info) {
  if (!s || !x || !b || !isp) {
    set_error("moons_pcg_solve: null pointer");
    return MOONS_ERR_ARG;
  }
  if (isp->n_skip_check_res < 1) {
    set_error("moons_pcg_solve: n_skip_check_res must be >= 1");
    return MOONS_ERR_ARG;
  }
  moons_mesh* m = s->m;
  cudaSetDevice(m->device);
  DF X[3], B[3];
  for (int c = 0; c < s->nc; c++) {
    if (!x[c] || !b[c] || x[c]->f.dl != s->x_dl[c] || b[c]->f.n() != x[c]->f.n()) {
      set_error("moons_pcg_solve: field does not match the solver");
      return MOONS_ERR_SHAPE;
    }
    X[c] = x[c]->f;
    B[c] = b[c]->f;
  }
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, m->stream);
  int r = MOONS_OK;
  int nc = s->nc;
  // ---- modify_RHS (PCG_aux.f90:30-79)
  for (int c = 0; c < nc && !r; c++) r = launch_pw(m, PW_COPY, s->r[c], &B[c], 0.0);
  if (!r && s->all_neumann) {
    // tempx = r*vol; mean = sum(tempx,1)/vol%vol; r -= mean; assign_ghost_XPeriodic(r,0)
    MG_LAUNCH(k_reduce, red_grid(&s->r[0], 1), kBlock, m->stream, c3(&s->r[0], 1), c3(&s->vol[0], 1), 2, 0, 0, 0,
                                                               m->d_scal, m->d_partial, m->d_ticket);
    MG_LAUNCH(k_sub_mean, nblocks(s->r[0].n()), kBlock, m->stream, s->r[0], m->d_scal, s->volsum[0]);
    r = mask_ghost_XPeriodic(m, s->r[0], nullptr);
  }
  for (int c = 0; c < nc && !r; c++) {
    r = launch_pw(m, PW_FILL, s->xbc[c], nullptr, 0.0);
    if (!r) r = launch_bcs(m, s->xbc[c], s->xbc_bc[c], false);
    if (!r) r = mask_ghost_N_XPeriodic(m, s->xbc[c], &s->xbc_bc[c], s->xbc[c].dl);
  }
  if (!r) r = apply_op_explicit(s, s->tempx, s->xbc);
  for (int c = 0; c < nc && !r; c++) {
    r = mask_ghost_XPeriodic(m, s->tempx[c], s->x_bc[c].defined ? &s->x_bc[c] : nullptr);
    if (!r) r = launch_pw(m, PW_SUB, s->r[c], &s->tempx[c], 0.0);
  }
  for (int c = 0; c < nc && !r; c++) r = launch_bcs(m, X[c], s->x_bc[c], true);
  if (!r) r = apply_op_explicit(s, s->Ax, X);
  for (int c = 0; c < nc && !r; c++) {
    r = launch_pw(m, PW_SUB, s->r[c], &s->Ax[c], 0.0);
    if (!r) r = launch_pw(m, PW_MUL, s->r[c], &s->vol[c], 0.0);
    if (!r && s->r[c].dl != MOONS_CC) {
      const DBC* w = s->xbc_bc[c].defined ? &s->xbc_bc[c] : nullptr;
      int dlw = s->xbc[c].dl;
      r = mask_wall_Periodic_single(m, s->r[c], w, dlw, 0.0);
      if (!r) r = mask_wall_Dirichlet(m, s->r[c], w, dlw, 0.0);
      if (!r) r = mask_wall_Neumann(m, s->r[c], w, dlw, 0.5);
    }
  }
  if (r) return r;
  // ---- scalars
  PcgScalars h{};
  h.iter_max = isp->iter_max;
  h.nskip = isp->n_skip_check_res;
  h.tol_rel = isp->tol_rel;
  h.tol_abs = isp->tol_abs;
  *s->hS = h;
  MG_CUDA(cudaMemcpyAsync(s->S, s->hS, sizeof(PcgScalars), cudaMemcpyHostToDevice, m->stream));
  // res0 = sqrt(sum r^2) whole array
  MG_LAUNCH(k_reduce, red_grid(s->r, nc), kBlock, m->stream, c3(s->r, nc), c3(s->r, nc), 1, 0, 0, 0, &s->S->res0,
                                                         m->d_partial, m->d_ticket);
  // z = Minv r ; p = z ; rhok = dot(r,z)
  for (int c = 0; c < nc; c++) {
    launch_pw(m, PW_COPY, s->z[c], &s->Minv[c], 0.0);
    launch_pw(m, PW_MUL, s->z[c], &s->r[c], 0.0);
    launch_pw(m, PW_COPY, s->p[c], &s->z[c], 0.0);
  }
  int dw[3] = {0, 0, 0};
  for (int c = 0; c < nc; c++) dw[c] = dirichlet_wall_bits(s->x_bc[c].defined ? &s->x_bc[c] : nullptr, s->x_dl[c]);
  MG_LAUNCH(k_reduce, red_grid(s->r, nc), kBlock, m->stream, c3(s->r, nc), c3(s->z, nc), 0, dw[0], dw[1], dw[2],
                                                         &s->S->rhok, m->d_partial, m->d_ticket);
  MG_LAUNCH(k_pcg_start, 1, 1, m->stream, s->S);
  MG_CUDA(cudaGetLastError());
  // ---- the loop: one graph launch (WHILE node) unless the solve is trivial
  bool need_graph = !s->exec;
  for (int c = 0; c < nc; c++)
    if (s->gx[c] != X[c].f) need_graph = true;
  if (need_graph) {
    r = build_graph(s, X);
    if (r) return r;
  }
  MG_CUDA(cudaGraphLaunch(s->exec, m->stream));
  // x: apply_BCs (the reference applies them after every update; they only
  // rewrite ghost/boundary entries, which no update reads)
  for (int c = 0; c < nc && !r; c++) r = launch_bcs(m, X[c], s->x_bc[c], false);
  if (r) return r;
  MG_CUDA(cudaMemcpyAsync(s->hS, s->S, sizeof(PcgScalars), cudaMemcpyDeviceToHost, m->stream));
  cudaEventRecord(e1, m->stream);
  MG_CUDA(cudaStreamSynchronize(m->stream));
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const PcgScalars& H = *s->hS;
  g_launch_count += s->body_launches * (long long)H.body_runs;
  if (info) {
    info->iterations = H.iter;
    info->res0 = H.res0;
    info->res = H.res;
    info->rel = (H.res0 == 0.0) ? H.res : H.res / H.res0;
    info->exit_reason = H.exit_reason;
    info->ms = ms;
  }
  if (H.nan || std::isnan(H.res0) || std::isnan(H.res)) {
    set_error("moons_pcg_solve: NaN in residual norms");
    return MOONS_ERR_NAN;
  }
  return MOONS_OK;
}

}  // extern "C"
