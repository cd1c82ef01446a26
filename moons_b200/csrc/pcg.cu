// pcg.cu -- matrix-free Jacobi-PCG (PCG_solver_algorithm.f90:37-179) with
// every scalar of the recurrence kept on the device.
//
// modify_RHS (PCG_aux.f90:30-79) runs once per solve with the generic
// kernels.  The iteration is the lean kernels of lean.cuh (grid-stride, one
// resident wave each); the loop is captured once into a CUDA graph whose
// WHILE node repeats a two-iteration body until the device-side exit flag is
// set (the flag also comes up at iter_max, and the node stops after
// iter_max+2 body runs in any case, so the loop always ends).
// MOONS_PCG_HOSTLOOP=1 launches the same kernels from the host instead (for
// profilers).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "lean_cc.cuh"
#include "mgrid.cuh"
#include "runtime.cuh"

namespace mg {

struct Comp3 {
  DF a[3];
  int nc;
};

// generic two-level reduction: mode 0 dot(a,b) masked interior, 1 sum(a^2) whole array,
// 2 sum(a*b) over interior pad 1 (no wall mask)
__global__ void k_reduce(Comp3 a, Comp3 b, int mode, int dw0, int dw1, int dw2, double* out, double* partial,
                         unsigned* ticket) {
  double acc = 0.0;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (c >= a.nc) break;
    const DF& A = a.a[c];
    const DF& Bf = b.a[c];
    int dw = c == 0 ? dw0 : (c == 1 ? dw1 : dw2);
    unsigned n = (unsigned)A.n();
    for (unsigned idx = blockIdx.x * blockDim.x + threadIdx.x; idx < n; idx += gridDim.x * blockDim.x) {
      if (mode == 1) {
        double v = A.f[idx];
        acc += v * v;
      } else {
        unsigned q = idx / (unsigned)A.s0;
        int i = (int)(idx - q * (unsigned)A.s0) + 1;
        unsigned kk = q / (unsigned)A.s1;
        int j = (int)(q - kk * (unsigned)A.s1) + 1;
        int k = (int)kk + 1;
        if (dot_keep(A, i, j, k, mode == 0 ? dw : 0)) acc += A.f[idx] * Bf.f[idx];
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
  S->stag_ref = S->res0;
  S->res = sqrt(fabs(S->rhok));
  if (S->stag_window > 0 && !(fabs(S->rhok) > 0.0) && S->res0 > 0.0) {
    // learned preconditioner: z.r = 0 (or NaN) gives no search direction;
    // hand over to the fallback (exit_reason 4) before the first iteration.
    // (Its sign is not tested: the Laplacians are negative definite, and a
    // good preconditioner then has z.r < 0, as the Jacobi one does.)
    S->iter = 0;
    S->body_runs = 0;
    S->nan = 0;
    S->res = S->res0;
    S->exit_reason = 4;
    S->done = 1;
    return;
  }
  S->iter = 0;
  S->body_runs = 0;
  S->beta = 0.0;  // the fused iteration's first p is 0 * p + z
  S->alpha = 0.0;  // ... and its first x update adds 0 * p
  S->last_half = -1;
  S->nan = isnan(S->res0) ? 1 : 0;
  if (S->nan) S->nan_any = 1;
  S->exit_reason = 0;
  bool e2 = S->res < S->tol_abs;  // only exit_loop(2) skips the loop (PCG_solver_algorithm.f90:68)
  S->done = (e2 || S->iter_max <= 0 || S->nan) ? 1 : 0;
  if (e2) {
    S->exit_reason = 2;
    S->iter = 1;  // update_iter in the else branch
    S->iter_total += 1;
  }
}

// host-side parameters of the next solve (the accumulators are kept)
// stagnation test of the learned preconditioner (window 0 = off)
__global__ void k_stag_params(PcgScalars* S, int window, double factor) {
  S->stag_window = window;
  S->stag_factor = factor;
}

__global__ void k_pcg_params(PcgScalars* S, int iter_max, int nskip, double tol_rel, double tol_abs) {
  S->iter_max = iter_max;
  S->nskip = nskip;
  S->tol_rel = tol_rel;
  S->tol_abs = tol_abs;
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
  int i, j, k;
  if (!point_of(u, i, j, k)) return;
  bool ghost = (i == 1 || i == u.s0 || j == 1 || j == u.s1 || k == 1 || k == u.s2);
  u(i, j, k) = ghost ? 0.0 : vol_at(g, u.dl, i, j, k);
}

// Jacobi preconditioners (preconditioners.f90:55-129, GF_diagonals.f90:15-71):
// mode 0 identity (1 everywhere); 1 Lap: 1/(diag*vol); 2 mom: 1/((diag*c+1)*vol);
// 3 ind: 1/((cc_diag*c+1)*vol); ghost planes 0 (Minv carries no BCs, so
// assign_ghost_XPeriodic zeroes all six).
__global__ void k_prec(DF M, DGrid g, int mode, double coeff, int comp, DF sx, DF sy, DF sz) {
  int i, j, k;
  if (!point_of(M, i, j, k)) return;
  if (mode == 0) {
    M(i, j, k) = 1.0;
    return;
  }
  bool ghost = (i == 1 || i == M.s0 || j == 1 || j == M.s1 || k == 1 || k == M.s2);
  if (ghost) {
    M(i, j, k) = 0.0;
    return;
  }
  if (mode != 3) {
    M(i, j, k) = minv_at(mode, g, M, M.dl, i, j, k, false, coeff);
    return;
  }
  const DCoord &c1 = g.c[0], &c2 = g.c[1], &c3 = g.c[2];
  double d;
  if (comp == 0)
    d = -c2.n2ccD[j] * sz(i, j, k) * c2.cc2nU[j - 1] - c2.n2ccU[j] * sz(i, j + 1, k) * c2.cc2nD[j] -
        c3.n2ccD[k] * sy(i, j, k) * c3.cc2nU[k - 1] - c3.n2ccU[k] * sy(i, j, k + 1) * c3.cc2nD[k];
  else if (comp == 1)
    d = -c1.n2ccD[i] * sz(i, j, k) * c1.cc2nU[i - 1] - c1.n2ccU[i] * sz(i + 1, j, k) * c1.cc2nD[i] -
        c3.n2ccD[k] * sx(i, j, k) * c3.cc2nU[k - 1] - c3.n2ccU[k] * sx(i, j, k + 1) * c3.cc2nD[k];
  else
    d = -c1.n2ccD[i] * sy(i, j, k) * c1.cc2nU[i - 1] - c1.n2ccU[i] * sy(i + 1, j, k) * c1.cc2nD[i] -
        c2.n2ccD[j] * sx(i, j, k) * c2.cc2nU[j - 1] - c2.n2ccU[j] * sx(i, j + 1, k) * c2.cc2nD[j];
  d = d * coeff;
  d = d + 1.0;
  M(i, j, k) = 1.0 / (d * vol_at(g, M.dl, i, j, k));
}


__global__ void k_set_cond(cudaGraphConditionalHandle h, PcgScalars* S) {
  pdl_enter();
  S->body_runs += 1;
  S->runs_total += 1;
  bool go = !S->done && S->body_runs < S->iter_max + 2;
  cudaGraphSetConditional(h, go ? 1u : 0u);
}

// grids of the lean kernels: (plane blocks, k stride, component)
struct LeanGrids {
  dim3 gA, gB, gC, gD, gE;  // K1 (op), K2 (update), K3 (p update), BC fill, curl-curl edge pass
  unsigned npbP;            // perimeter plane blocks (BC fill)
  bool bc;
  // one CC unknown under LAP_UNIFORM / LAP_PROPS / NRG_DIFFUSION: K1 is the
  // shared-memory staged k_cc_lap (ghost values formed from the interior, no
  // BC fill of p); grid gF, klen planes per block
  bool cc;
  dim3 gF;
  int klen;
  bool tm;             // the staged operator loads p through tensor maps (even s0)
  CUtensorMap tmap[3];  // of p, p2 and z
  // fused iteration (cc, prec_Lap / prec_mom / identity): the operator kernel
  // forms p' = beta p + z and the update kernel stores z, two kernels per
  // iteration instead of three
  bool fz;
  int mm;  // Minv of K2/K3: 0 stored, 1 prec_Lap, 2 prec_mom (formed per point)
};

}  // namespace mg

using namespace mg;

// multigrid preconditioner (mgpcg.cu)
struct MGHier;
// flexible CG with the learned preconditioner stops (and the multigrid
// fallback takes over) when 10 iterations fail to halve the residual
constexpr int kStagWindow = 10;
constexpr double kStagFactor = 0.5;

struct moons_pcg;
namespace mg {
int unet_apply_dev(moons_unet* u, double* z, const double* r, const int* skip);
int unet_prepare(moons_unet* u);
moons_mesh* unet_mesh(moons_unet* u);
}  // namespace mg
int mg_build(moons_pcg* s, moons_mesh* m, int mixed, const mg::DBC& bc, const mg::DF* kf, MGHier** out);
int fd_build(moons_pcg* s, moons_mesh* m, const mg::DBC& bc, MGHier** out);
void mg_free(MGHier* h);
int mg_vcycle(MGHier* h, mg::DF z, mg::DF r, cudaStream_t st, const mg::PcgScalars* S);
int mg_vcycle_resid_f64(MGHier* h, mg::DF t, cudaStream_t st, const mg::PcgScalars* S);
int mg_two_stage_combine(MGHier* h, mg::DF z, const double* N, const double* t, cudaStream_t st,
                         const mg::PcgScalars* S);
double* mg_rprev(MGHier* h);

// ---------------------------------------------------------------------------
// the PCG object
// ---------------------------------------------------------------------------
struct moons_pcg {
  moons_mesh* m = nullptr;
  int op = 0, prec = 0, nc = 1;
  double coeff = 0.0;
  DF p[3]{}, p2[3]{}, xbc[3]{}, r[3]{}, Ax[3]{}, vol[3]{}, z[3]{}, Minv[3]{}, tempx[3]{}, k[3]{}, tempk[3]{};
  DBC xbc_bc[3]{};   // BCs of x_BC
  DBC x_bc[3]{};     // BCs of x, copied to p
  int x_dl[3] = {0, 0, 0};
  int all_neumann = 0;
  double volsum[3] = {0, 0, 0};
  PcgScalars* S = nullptr;   // device
  PcgScalars* hS = nullptr;  // pinned host
  double* partial = nullptr; // fused-kernel block partials (2 x max blocks)
  unsigned* ticket = nullptr;
  size_t max_blocks = 0;
  std::vector<void*> allocs;
  // lean kernels: grids, and the CUDA graph of the loop (rebuilt when x changes)
  int nsm = 0;
  LeanGrids lg{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double* gx[3] = {nullptr, nullptr, nullptr};
  long long body_launches = 0;  // kernels per execution of the loop body
  MGHier* mgh = nullptr;        // MOONS_PREC_MG / MG_MIXED / UNET: the V-cycle hierarchy
  // MOONS_PREC_UNET: the network (not owned) and the multigrid fallback mode
  moons_unet* unet = nullptr;
  bool learned = false;
  bool two_stage = false;       // MOONS_PREC_UNET_MG: z = V(r) + N(r - A V(r))
  bool fb = false;              // true while the fallback (FP32 V-cycle) runs
  // the other mode's loop graph (swapped in and out with the fields above)
  cudaGraph_t graph_alt = nullptr;
  cudaGraphExec_t exec_alt = nullptr;
  double* gx_alt[3] = {nullptr, nullptr, nullptr};
  long long body_launches_alt = 0;
};

namespace {
// internal fields carry 64 doubles of padding past their last point: a bulk
// row copy of k_cc_lap (a fixed 36 doubles from an even element) may end up
// to 33 doubles past the field
constexpr size_t kFieldPad = 64;
int alloc_df(moons_pcg* s, DF& f, int dl) {
  f = make_df(s->m, dl, nullptr);
  if (cudaMalloc(&f.f, (f.n() + kFieldPad) * sizeof(double)) != cudaSuccess) {
    set_error("moons_pcg: device allocation failed");
    return MOONS_ERR_NOMEM;
  }
  cudaMemsetAsync(f.f, 0, (f.n() + kFieldPad) * sizeof(double), s->m->stream);
  s->allocs.push_back(f.f);
  return MOONS_OK;
}
Comp3 c3(const DF* a, int nc) {
  Comp3 r{};
  r.nc = nc;
  for (int c = 0; c < nc; c++) r.a[c] = a[c];
  return r;
}
FComp fc(const DF* a, int nc) {
  FComp r{};
  r.nc = nc;
  for (int c = 0; c < nc; c++) r.f[c] = a[c];
  for (int c = nc; c < 3; c++) r.f[c] = a[0];
  return r;
}
unsigned red_grid(const DF* a, int nc) {
  size_t n = 0;
  for (int c = 0; c < nc; c++) n += a[c].n();
  return (unsigned)std::min<size_t>(kRedBlocks, std::max<size_t>(1, (n + kBlock - 1) / kBlock));
}
// (plane chunk, k, component) grid covering nc fields
dim3 fgrid(const DF* a, int nc) {
  unsigned px = 0, kz = 0;
  for (int c = 0; c < nc; c++) {
    px = std::max(px, (unsigned)(((size_t)a[c].s0 * a[c].s1 + kBlock - 1) / kBlock));
    kz = std::max(kz, (unsigned)a[c].s2);
  }
  return dim3(px, kz, nc);
}

FBC fbc_of(const DBC& xb, const DBC& xbcb, int dl, const DF& shape) {
  int ext[4] = {0, shape.s0, shape.s1, shape.s2};
  return make_fbc(xb, xbcb, dl, ext);
}

// operator_explicit of matrix_free_operators.f90 on component fields (generic
// kernels; used by modify_RHS, once per solve)
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
    case MOONS_OP_LAP_PROPS:
    case MOONS_OP_NRG_DIFFUSION: {
      for (int d = 0; d < 3 && !r; d++) r = launch_del(m, s->tempk[d], x[0], 1, d + 1, 0, 1);
      for (int d = 0; d < 3 && !r; d++) r = launch_pw(m, PW_MUL, s->tempk[d], &s->k[d], 0.0);
      if (!r) r = launch_del(m, out[0], s->tempk[0], 1, 1, 0, 1);
      if (!r) r = launch_del(m, out[0], s->tempk[1], 1, 2, 0, 2);
      if (!r) r = launch_del(m, out[0], s->tempk[2], 1, 3, 0, 2);
      if (!r) r = mask_ghost_XPeriodic(m, out[0], nullptr);
      // nrg_diffusion_explicit (matrix_free_operators.f90:148-162): Ax*coeff + x
      if (!r && s->op == MOONS_OP_NRG_DIFFUSION) r = launch_pw(m, PW_PRODUCT_ADD, out[0], &x[0], s->coeff);
    } break;
    case MOONS_OP_IND_DIFFUSION: {
      DF* t = s->tempk;
      if (!r) r = launch_del(m, t[0], x[2], 1, 2, 0, 1);
      if (!r) r = launch_del(m, t[0], x[1], 1, 3, 0, 3);
      if (!r) r = launch_del(m, t[1], x[0], 1, 3, 0, 1);
      if (!r) r = launch_del(m, t[1], x[2], 1, 1, 0, 3);
      if (!r) r = launch_del(m, t[2], x[1], 1, 1, 0, 1);
      if (!r) r = launch_del(m, t[2], x[0], 1, 2, 0, 3);
      for (int d = 0; d < 3 && !r; d++) r = launch_pw(m, PW_MUL, t[d], &s->k[d], 0.0);
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
  if (mode == MOONS_PREC_MG || mode == MOONS_PREC_MG_MIXED || mode == MOONS_PREC_UNET || mode == MOONS_PREC_FD ||
      mode == MOONS_PREC_UNET_MG)
    mode = MOONS_PREC_IDENTITY;  // Minv unused
  DF dummy{};
  if (mode == MOONS_PREC_IND && s->op != MOONS_OP_IND_DIFFUSION) {
    set_error("moons_pcg: prec_ind needs the induction operator's sigma^-1 edge fields");
    return MOONS_ERR_ARG;
  }
  for (int c = 0; c < s->nc; c++) {
    DF sx = s->op == MOONS_OP_IND_DIFFUSION ? s->k[0] : dummy;
    DF sy = s->op == MOONS_OP_IND_DIFFUSION ? s->k[1] : dummy;
    DF sz = s->op == MOONS_OP_IND_DIFFUSION ? s->k[2] : dummy;
    MG_LAUNCH(k_prec, fgrid(&s->Minv[c], 1), kBlock, m->stream, s->Minv[c], m->dg, mode, s->coeff, c, sx, sy, sz);
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}


// one PCG iteration (PCG_solver_algorithm.f90:69-96), enqueued on the mesh stream
#ifndef MOONS_KCU
#define MOONS_KCU 2
#endif
constexpr int kKCU = MOONS_KCU;  // planes per thread of the pointwise kernels

// grid of a grid-stride kernel: every block resident, at most one per item
unsigned resident_grid(const moons_pcg* s, const void* kern, size_t items) {
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLB, 0);
  size_t g = (size_t)std::max(occ, 1) * (size_t)std::max(s->nsm, 1);
  return (unsigned)std::max<size_t>(1, std::min(g, items));
}

// one PCG iteration (PCG_solver_algorithm.f90:69-96) as five grid-stride
// kernels, twice: p -> p2 -> p (K3 reads one buffer and writes the other)
int enqueue_mg_iteration(moons_pcg* s, DF* x);

// the cell-centred operator step k_cc_lap on the direction of this half
// (p for half 0, p2 for half 1): Ap, p.Ap and alpha; with the fused
// iteration (L.fz) also p' = beta p + z into pn and x += alpha_prev p
int enqueue_cc_lap(moons_pcg* s, int half, DF* pc, DF* pn, DF* x, const FBC& b0, unsigned* tA) {
  moons_mesh* m = s->m;
  const LeanGrids& L = s->lg;
  DF z0{};
  const bool ev = (s->Ax[0].s0 & 1) == 0;
  const CUtensorMap& tm = L.tmap[half];
  const CUtensorMap& tz = L.tmap[2];
  const size_t sm = cc_smem(L.klen, L.fz);
#define MG_CC_LAP(MD, EV, T, F, KX, KY, KZ, CF)                                                            \
  MG_LAUNCH_PDL_SMEM((k_cc_lap<MD, EV, T, F>), L.gF, kCThreads, sm, m->stream, tm, tz, s->Ax[0], pc[0], s->z[0], \
                     pn[0], x[0], m->dg, b0, KX, KY, KZ, CF, L.klen, s->S, s->partial, tA)
#define MG_CC_LAP_F(MD, KX, KY, KZ, CF)                                            \
  if (L.fz) {                                                                      \
    if (L.tm) MG_CC_LAP(MD, true, true, true, KX, KY, KZ, CF);                     \
    else if (ev) MG_CC_LAP(MD, true, false, true, KX, KY, KZ, CF);                 \
    else MG_CC_LAP(MD, false, false, true, KX, KY, KZ, CF);                        \
  } else {                                                                         \
    if (L.tm) MG_CC_LAP(MD, true, true, false, KX, KY, KZ, CF);                    \
    else if (ev) MG_CC_LAP(MD, true, false, false, KX, KY, KZ, CF);                \
    else MG_CC_LAP(MD, false, false, false, KX, KY, KZ, CF);                       \
  }
  switch (s->op) {
    case MOONS_OP_LAP_UNIFORM:
      MG_CC_LAP_F(0, z0, z0, z0, 0.0);
      break;
    case MOONS_OP_LAP_PROPS:
      MG_CC_LAP_F(1, s->k[0], s->k[1], s->k[2], 0.0);
      break;
    default:
      MG_CC_LAP_F(3, s->k[0], s->k[1], s->k[2], s->coeff);
      break;
  }
#undef MG_CC_LAP_F
#undef MG_CC_LAP
  return MOONS_OK;
}

int enqueue_iteration(moons_pcg* s, DF* x) {
  if (s->mgh) return enqueue_mg_iteration(s, x);
  moons_mesh* m = s->m;
  FBC b[3];
  for (int c = 0; c < 3; c++) {
    int cc = c < s->nc ? c : 0;
    b[c] = fbc_of(s->x_bc[cc], s->xbc_bc[cc], s->x_dl[cc], s->Ax[cc]);
  }
  const LeanGrids& L = s->lg;
  unsigned* tA = s->ticket;
  unsigned* tB = s->ticket + 1;
  DF z0{};
  const int nc = s->nc;
  for (int half = 0; half < 2; half++) {
    DF* pc = half == 0 ? s->p : s->p2;
    DF* pn = half == 0 ? s->p2 : s->p;
    if (L.cc) {
      int r = enqueue_cc_lap(s, half, pc, pn, x, b[0], tA);
      if (r) return r;
    } else switch (s->op) {
      case MOONS_OP_LAP_UNIFORM:
        MG_LAUNCH_PDL(k_l_lap<0>, L.gA, kLB, m->stream, fc(s->Ax, nc), fc(pc, nc), m->dg, b[0], b[1], b[2], z0, z0, z0,
                  0.0, s->S, s->partial, tA);
        break;
      case MOONS_OP_LAP_PROPS:
        MG_LAUNCH_PDL(k_l_lap<1>, L.gA, kLB, m->stream, fc(s->Ax, nc), fc(pc, nc), m->dg, b[0], b[1], b[2], s->k[0],
                  s->k[1], s->k[2], 0.0, s->S, s->partial, tA);
        break;
      case MOONS_OP_NRG_DIFFUSION:
        MG_LAUNCH_PDL(k_l_lap<3>, L.gA, kLB, m->stream, fc(s->Ax, nc), fc(pc, nc), m->dg, b[0], b[1], b[2], s->k[0],
                      s->k[1], s->k[2], s->coeff, s->S, s->partial, tA);
        break;
      case MOONS_OP_MOM_DIFFUSION:
        MG_LAUNCH_PDL(k_l_lap<2>, L.gA, kLB, m->stream, fc(s->Ax, nc), fc(pc, nc), m->dg, b[0], b[1], b[2], z0, z0, z0,
                  s->coeff, s->S, s->partial, tA);
        break;
      case MOONS_OP_IND_DIFFUSION:
        MG_LAUNCH_PDL(k_l_curl_sig, L.gE, kLB, m->stream, s->tempk[0], s->tempk[1], s->tempk[2], fc(pc, 3), s->k[0],
                  s->k[1], s->k[2], m->dg, s->S);
        MG_LAUNCH_PDL(k_l_curl_ap, L.gA, kLB, m->stream, fc(s->Ax, 3), fc(pc, 3), s->tempk[0], s->tempk[1], s->tempk[2],
                  m->dg, b[0], b[1], b[2], s->coeff, s->S, s->partial, tA);
        break;
    }
    if (L.fz) {
      // fused: K2 reads the p' the operator kernel just wrote (pn) and stores z
      if (L.mm == 1)
        MG_LAUNCH_PDL((k_l_update<kKCU, 1, true>), L.gB, kLB, m->stream, fc(x, 1), fc(pn, 1), fc(s->r, 1),
                      fc(s->Ax, 1), fc(s->Minv, 1), b[0], b[1], b[2], m->dg, s->coeff, s->S, s->partial, tB, s->z[0],
                      half);
      else if (L.mm == 2)
        MG_LAUNCH_PDL((k_l_update<kKCU, 2, true>), L.gB, kLB, m->stream, fc(x, 1), fc(pn, 1), fc(s->r, 1),
                      fc(s->Ax, 1), fc(s->Minv, 1), b[0], b[1], b[2], m->dg, s->coeff, s->S, s->partial, tB, s->z[0],
                      half);
      else
        MG_LAUNCH_PDL((k_l_update<kKCU, 0, true>), L.gB, kLB, m->stream, fc(x, 1), fc(pn, 1), fc(s->r, 1),
                      fc(s->Ax, 1), fc(s->Minv, 1), b[0], b[1], b[2], m->dg, s->coeff, s->S, s->partial, tB, s->z[0],
                      half);
      continue;
    }
    if (L.mm == 1) {
      MG_LAUNCH_PDL((k_l_update<kKCU, 1>), L.gB, kLB, m->stream, fc(x, nc), fc(pc, nc), fc(s->r, nc),
                    fc(s->Ax, nc), fc(s->Minv, nc), b[0], b[1], b[2], m->dg, s->coeff, s->S, s->partial, tB, z0, 0);
      MG_LAUNCH_PDL((k_l_pupd<kKCU, 1>), L.gC, kLB, m->stream, fc(pc, nc), fc(pn, nc), fc(s->r, nc),
                    fc(s->Minv, nc), m->dg, s->coeff, s->S);
    } else if (L.mm == 2) {
      MG_LAUNCH_PDL((k_l_update<kKCU, 2>), L.gB, kLB, m->stream, fc(x, nc), fc(pc, nc), fc(s->r, nc),
                    fc(s->Ax, nc), fc(s->Minv, nc), b[0], b[1], b[2], m->dg, s->coeff, s->S, s->partial, tB, z0, 0);
      MG_LAUNCH_PDL((k_l_pupd<kKCU, 2>), L.gC, kLB, m->stream, fc(pc, nc), fc(pn, nc), fc(s->r, nc),
                    fc(s->Minv, nc), m->dg, s->coeff, s->S);
    } else {
      MG_LAUNCH_PDL((k_l_update<kKCU, 0>), L.gB, kLB, m->stream, fc(x, nc), fc(pc, nc), fc(s->r, nc),
                    fc(s->Ax, nc), fc(s->Minv, nc), b[0], b[1], b[2], m->dg, s->coeff, s->S, s->partial, tB, z0, 0);
      MG_LAUNCH_PDL((k_l_pupd<kKCU, 0>), L.gC, kLB, m->stream, fc(pc, nc), fc(pn, nc), fc(s->r, nc),
                    fc(s->Minv, nc), m->dg, s->coeff, s->S);
    }
    if (L.bc && !L.cc) MG_LAUNCH_PDL(k_l_bcfill, L.gD, kLB, m->stream, fc(pn, nc), b[0], b[1], b[2], L.npbP, s->S);
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// z = M(r) of a multigrid-family solver: the V-cycle, the U-Net, or (two-
// stage) the V-cycle then the U-Net on what it leaves:
// z = V(r) + gamma N(r - A V(r)), with r - A V(r) the FP32 finest level's
// residual and gamma the energy-optimal multiple of the network's output
// (work arrays: tempx, xbc)
int apply_prec_dev(moons_pcg* s, const int* skip, const PcgScalars* S) {
  moons_mesh* m = s->m;
  if (s->learned && !s->fb && !s->two_stage) return unet_apply_dev(s->unet, s->z[0].f, s->r[0].f, skip);
  int r = mg_vcycle(s->mgh, s->z[0], s->r[0], m->stream, S);
  if (r || !(s->learned && s->two_stage && !s->fb)) return r;
  if ((r = mg_vcycle_resid_f64(s->mgh, s->tempx[0], m->stream, S))) return r;
  // the network writes interior cells only: its output buffer's ghosts are 0
  MG_CUDA(cudaMemsetAsync(s->xbc[0].f, 0, s->xbc[0].n() * sizeof(double), m->stream));
  if ((r = unet_apply_dev(s->unet, s->xbc[0].f, s->tempx[0].f, skip))) return r;
  return mg_two_stage_combine(s->mgh, s->z[0], s->xbc[0].f, s->tempx[0].f, m->stream, S);
}

// one multigrid-preconditioned CG iteration, twice (p -> p2 -> p)
int enqueue_mg_iteration(moons_pcg* s, DF* x) {
  moons_mesh* m = s->m;
  FBC b[3];
  for (int c = 0; c < 3; c++) b[c] = fbc_of(s->x_bc[0], s->xbc_bc[0], s->x_dl[0], s->Ax[0]);
  const LeanGrids& L = s->lg;
  unsigned* tA = s->ticket;
  unsigned* tB = s->ticket + 1;
  DF z0{};
  const unsigned gF = resident_grid(s, (const void*)k_m_update, nblocks(s->r[0].n()));
  double* rprev = mg_rprev(s->mgh);
  for (int half = 0; half < 2; half++) {
    DF* pc = half == 0 ? s->p : s->p2;
    DF* pn = half == 0 ? s->p2 : s->p;
    if (L.cc) {
      // shared-memory staged operator with the ghost values formed from the
      // interior: p needs no BC fill
      int r = enqueue_cc_lap(s, half, pc, pn, x, b[0], tA);
      if (r) return r;
    } else if (s->op == MOONS_OP_LAP_PROPS) {
      MG_LAUNCH_PDL(k_l_lap<1>, L.gA, kLB, m->stream, fc(s->Ax, 1), fc(pc, 1), m->dg, b[0], b[1], b[2], s->k[0], s->k[1],
                s->k[2], 0.0, s->S, s->partial, tA);
    } else {
      MG_LAUNCH_PDL(k_l_lap<0>, L.gA, kLB, m->stream, fc(s->Ax, 1), fc(pc, 1), m->dg, b[0], b[1], b[2], z0, z0, z0, 0.0,
                s->S, s->partial, tA);
    }
    MG_LAUNCH_PDL(k_m_update, gF, kLB, m->stream, x[0], pc[0], s->r[0], s->Ax[0], rprev, s->S, s->partial, tB);
    int r = apply_prec_dev(s, &s->S->done, s->S);
    if (r) return r;
    MG_LAUNCH_PDL(k_m_beta, gF, kLB, m->stream, s->z[0], s->r[0], rprev, s->S, s->partial, tA);
    MG_LAUNCH_PDL(k_m_pupd, gF, kLB, m->stream, pn[0], pc[0], s->z[0], s->S);
    if (L.bc && !L.cc) MG_LAUNCH_PDL(k_l_bcfill, L.gD, kLB, m->stream, fc(pn, 1), b[0], b[1], b[2], L.npbP, s->S);
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// (plane blocks, k stride, component) grid of a lean kernel over fields a[0..nc):
// the k stride fills one resident wave (SMs x occupancy)
dim3 lean_grid(const moons_pcg* s, const void* kern, const DF* a, int nc, int kc) {
  unsigned npb = 0, nkc = 0;
  for (int c = 0; c < nc; c++) {
    const PlaneSplit q = plane_split(a[c].s0, a[c].s1, a[c].dl);
    npb = std::max(npb, q.npbI + q.npbP);
    nkc = std::max(nkc, (unsigned)((a[c].s2 + kc - 1) / kc));
  }
  int occ = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kLB, 0);
  const size_t wave = (size_t)std::max(occ, 1) * (size_t)std::max(s->nsm, 1);
  const size_t per = (size_t)npb * nc;
  const unsigned gy = (unsigned)std::max<size_t>(1, std::min<size_t>(nkc, wave / per));  // never a partial 2nd wave
  return dim3(npb, gy, (unsigned)nc);
}

// grids of the lean kernels (set once at create)
void plan_lean(moons_pcg* s) {
  LeanGrids& L = s->lg;
  const int nc = s->nc;
  const void* ka = s->op == MOONS_OP_LAP_UNIFORM ? (const void*)k_l_lap<0>
                   : s->op == MOONS_OP_LAP_PROPS ? (const void*)k_l_lap<1>
                   : s->op == MOONS_OP_MOM_DIFFUSION ? (const void*)k_l_lap<2>
                   : s->op == MOONS_OP_NRG_DIFFUSION ? (const void*)k_l_lap<3>
                                                    : (const void*)k_l_curl_ap;
  L.gA = lean_grid(s, ka, s->Ax, nc, s->op == MOONS_OP_IND_DIFFUSION ? kKCc : kKC);
  L.mm = (s->prec == MOONS_PREC_LAP) ? 1 : (s->prec == MOONS_PREC_MOM ? 2 : 0);
  // grids sized with the variant that runs (its occupancy sets the wave)
  const void* kB = L.mm == 1 ? (const void*)k_l_update<kKCU, 1>
                   : L.mm == 2 ? (const void*)k_l_update<kKCU, 2> : (const void*)k_l_update<kKCU, 0>;
  const void* kC = L.mm == 1 ? (const void*)k_l_pupd<kKCU, 1>
                   : L.mm == 2 ? (const void*)k_l_pupd<kKCU, 2> : (const void*)k_l_pupd<kKCU, 0>;
  L.gB = lean_grid(s, kB, s->Ax, nc, kKCU);
  L.gC = lean_grid(s, kC, s->Ax, nc, kKCU);
  L.cc = nc == 1 && s->x_dl[0] == MOONS_CC && s->Ax[0].s0 >= 3 && s->Ax[0].s1 >= 3 && s->Ax[0].s2 >= 3 &&
         (s->op == MOONS_OP_LAP_UNIFORM || s->op == MOONS_OP_LAP_PROPS || s->op == MOONS_OP_NRG_DIFFUSION);
  L.gF = dim3(1, 1, 1);
  L.klen = 1;
  if (L.cc) {
    const bool ev = (s->Ax[0].s0 & 1) == 0;
    std::memset(L.tmap, 0, sizeof(L.tmap));
    L.fz = s->prec == MOONS_PREC_LAP || s->prec == MOONS_PREC_MOM || s->prec == MOONS_PREC_IDENTITY;
    L.tm = ev && cc_tensor_map(&L.tmap[0], s->p[0]) && cc_tensor_map(&L.tmap[1], s->p2[0]) &&
           cc_tensor_map(&L.tmap[2], s->z[0]);
    const int md = s->op == MOONS_OP_LAP_UNIFORM ? 0 : (s->op == MOONS_OP_LAP_PROPS ? 1 : 3);
    const void* kf = nullptr;
#define MG_CC_PICK1(MD, F)                                                                                 \
  kf = L.tm ? (const void*)k_cc_lap<MD, true, true, F>                                                     \
            : (ev ? (const void*)k_cc_lap<MD, true, false, F> : (const void*)k_cc_lap<MD, false, false, F>)
#define MG_CC_PICK(MD)      \
  if (L.fz) MG_CC_PICK1(MD, true); \
  else MG_CC_PICK1(MD, false)
    if (md == 0) { MG_CC_PICK(0); }
    else if (md == 1) { MG_CC_PICK(1); }
    else { MG_CC_PICK(3); }
#undef MG_CC_PICK
#undef MG_CC_PICK1
    L.gF = cc_lap_grid(s->Ax[0], s->nsm, kf, L.fz, L.klen);
    if (L.fz) {
      const void* kb2 = L.mm == 1 ? (const void*)k_l_update<kKCU, 1, true>
                        : L.mm == 2 ? (const void*)k_l_update<kKCU, 2, true> : (const void*)k_l_update<kKCU, 0, true>;
      L.gB = lean_grid(s, kb2, s->Ax, 1, kKCU);
    }
  }
  L.gE = dim3(1, 1, 1);
  if (s->op == MOONS_OP_IND_DIFFUSION) L.gE = lean_grid(s, (const void*)k_l_curl_sig, s->tempk, 3, kKCc);
  // BC fill: perimeter blocks over every plane, then inner blocks (ghost planes)
  unsigned npbP = 0, npbI = 0, smax = 0;
  L.bc = false;
  for (int c = 0; c < nc; c++) {
    const PlaneSplit q = plane_split(s->Ax[c].s0, s->Ax[c].s1, s->Ax[c].dl);
    npbP = std::max(npbP, q.npbP);
    npbI = std::max(npbI, q.npbI);
    smax = std::max(smax, (unsigned)s->Ax[c].s2);
    if (s->x_bc[c].defined) L.bc = true;
  }
  L.npbP = npbP;
  const unsigned gyD = std::max(4u, std::min(smax, (unsigned)(2 * std::max(s->nsm, 1)) / std::max(1u, npbP * nc)));
  L.gD = dim3(npbP + npbI, gyD, (unsigned)nc);
}

// destroy both loop graphs (they are rebuilt on the next solve)
void drop_graphs(moons_pcg* s) {
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  if (s->exec_alt) cudaGraphExecDestroy(s->exec_alt);
  if (s->graph_alt) cudaGraphDestroy(s->graph_alt);
  s->exec = s->exec_alt = nullptr;
  s->graph = s->graph_alt = nullptr;
  for (int c = 0; c < 3; c++) s->gx[c] = s->gx_alt[c] = nullptr;
}

// switch between the learned and the fallback preconditioner (each mode
// keeps its own loop graph)
void set_fallback(moons_pcg* s, bool fb) {
  if (s->fb == fb) return;
  std::swap(s->graph, s->graph_alt);
  std::swap(s->exec, s->exec_alt);
  for (int c = 0; c < 3; c++) std::swap(s->gx[c], s->gx_alt[c]);
  std::swap(s->body_launches, s->body_launches_alt);
  s->fb = fb;
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
  // the body: two iterations (p -> p2 -> p), eight for the fused two-kernel
  // CC iteration, whose launches are short enough that the conditional node
  // between bodies shows (kernels after the exit skip themselves)
  const int reps = (s->lg.fz && !s->mgh) ? 4 : 1;
  int r = MOONS_OK;
  for (int q = 0; q < reps && !r; q++) r = enqueue_iteration(s, x);
  if (!r) {
    cudaError_t e_ = launch_pdl(k_set_cond, dim3(1), dim3(1), m->stream, h, s->S);
    if (e_ != cudaSuccess) r = cuda_fail(e_, "k_set_cond");
  }
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
  if (op < MOONS_OP_LAP_UNIFORM || op > MOONS_OP_NRG_DIFFUSION || prec < 0 || prec > MOONS_PREC_UNET_MG) {
    set_error("moons_pcg_create: bad operator/preconditioner");
    return MOONS_ERR_ARG;
  }
  if (((op == MOONS_OP_LAP_PROPS || op == MOONS_OP_NRG_DIFFUSION) && nc != 1) || (op == MOONS_OP_IND_DIFFUSION && nc != 3)) {
    set_error("moons_pcg_create: operator/component count mismatch");
    return MOONS_ERR_ARG;
  }
  bool needk = (op == MOONS_OP_LAP_PROPS || op == MOONS_OP_IND_DIFFUSION || op == MOONS_OP_NRG_DIFFUSION);
  if (needk && (!k || !k[0] || !k[1] || !k[2])) {
    set_error("moons_pcg_create: operator needs three coefficient fields");
    return MOONS_ERR_ARG;
  }
  const bool use_mg = prec == MOONS_PREC_MG || prec == MOONS_PREC_MG_MIXED || prec == MOONS_PREC_UNET ||
                      prec == MOONS_PREC_FD || prec == MOONS_PREC_UNET_MG;
  if (use_mg) {
    bool ok = nc == 1 && (op == MOONS_OP_LAP_UNIFORM || (op == MOONS_OP_LAP_PROPS && prec != MOONS_PREC_FD)) && x[0] &&
              x[0]->f.dl == MOONS_CC;
    if (ok && x[0]->bc.defined)
      for (int f = 1; f <= 6; f++) {
        const int t = x[0]->bc.type[f];
        if (t != MOONS_BC_DIRICHLET && t != MOONS_BC_NEUMANN && t != MOONS_BC_PERIODIC) ok = false;
      }
    if (!ok) {
      set_error(prec == MOONS_PREC_FD
                    ? "moons_pcg_create: fast diagonalization needs one CC unknown, LAP_UNIFORM, and "
                      "Dirichlet/Neumann/periodic BCs"
                    : "moons_pcg_create: multigrid needs one CC unknown, LAP_UNIFORM or LAP_PROPS, and "
                      "Dirichlet/Neumann/periodic BCs");
      return MOONS_ERR_ARG;
    }
  }
  cudaSetDevice(m->device);
  auto* s = new moons_pcg();
  s->m = m;
  mesh_ref(m);
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
    if (!r) r = alloc_df(s, s->p2[c], dl);
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
    int nsm = 0;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, m->device);
    s->nsm = nsm;
    plan_lean(s);
    const LeanGrids& L = s->lg;
    dim3 G2 = fgrid(s->Ax, nc);
    size_t nb = (size_t)G2.x * G2.y * G2.z;
    for (const dim3& g : {L.gA, L.gB, L.gC, L.gD, L.gE, L.gF}) nb = std::max(nb, (size_t)g.x * g.y * g.z);
    nb = std::max<size_t>(nb, kRedBlocks);
    s->max_blocks = nb;
    void* p;
    if (cudaMalloc(&p, sizeof(PcgScalars)) != cudaSuccess) r = MOONS_ERR_NOMEM;
    else {
      s->S = (PcgScalars*)p;
      s->allocs.push_back(p);
      cudaMemsetAsync(p, 0, sizeof(PcgScalars), m->stream);
    }
    if (!r && cudaMalloc(&p, sizeof(double) * 2 * nb) != cudaSuccess) r = MOONS_ERR_NOMEM;
    else if (!r) {
      s->partial = (double*)p;
      s->allocs.push_back(p);
    }
    if (!r && cudaMalloc(&p, sizeof(unsigned) * 4) != cudaSuccess) r = MOONS_ERR_NOMEM;
    else if (!r) {
      s->ticket = (unsigned*)p;
      s->allocs.push_back(p);
      cudaMemsetAsync(p, 0, sizeof(unsigned) * 4, m->stream);
    }
    if (!r && cudaMallocHost(&p, sizeof(PcgScalars)) != cudaSuccess) r = MOONS_ERR_NOMEM;
    else if (!r) s->hS = (PcgScalars*)p;
    if (r) set_error("moons_pcg_create: device allocation failed");
  }
  if (!r) {
    for (int c = 0; c < nc; c++) MG_LAUNCH(k_volume, fgrid(&s->vol[c], 1), kBlock, m->stream, s->vol[c], m->dg);
    // coeff_implicit is not known here; Lap needs none and mom/ind set it through update_mfp
    r = compute_prec(s);
  }
  if (!r) {
    // SF%vol: plain sum of the volume field (ghosts are 0)
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
  if (!r && use_mg) {
    r = prec == MOONS_PREC_FD
            ? fd_build(s, m, s->x_bc[0], &s->mgh)
            : mg_build(s, m, prec != MOONS_PREC_MG, s->x_bc[0], op == MOONS_OP_LAP_PROPS ? s->k : nullptr, &s->mgh);
    s->learned = prec == MOONS_PREC_UNET || prec == MOONS_PREC_UNET_MG;
    s->two_stage = prec == MOONS_PREC_UNET_MG;
    if (r == MOONS_ERR_NOMEM) set_error("moons_pcg_create: device allocation failed (multigrid levels)");
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
  if (s && s->exec) cudaGraphExecDestroy(s->exec);
  if (s && s->graph) cudaGraphDestroy(s->graph);
  if (s && s->exec_alt) cudaGraphExecDestroy(s->exec_alt);
  if (s && s->graph_alt) cudaGraphDestroy(s->graph_alt);
  if (!s) return MOONS_OK;
  cudaSetDevice(s->m->device);
  cudaStreamSynchronize(s->m->stream);
  if (s->mgh) mg_free(s->mgh);
  for (void* p : s->allocs) cudaFree(p);
  if (s->hS) cudaFreeHost(s->hS);
  moons_mesh* m = s->m;
  delete s;
  mesh_unref(m);
  return MOONS_OK;
}

int moons_pcg_update_mfp(moons_pcg* s, double c, int upd) {
  if (!s) {
    set_error("null pcg");
    return MOONS_ERR_ARG;
  }
  s->coeff = c;
  drop_graphs(s);  // the coefficient is baked into the captured launches
  if (upd) {
    int r = compute_prec(s);
    if (r) return r;
  }
  return MOONS_OK;
}

}  // extern "C"

namespace mg {
__global__ void k_pcg_clear_acc(PcgScalars* S) {
  S->iter_total = 0;
  S->runs_total = 0;
  S->nan_any = 0;
}
}  // namespace mg

// zero the accumulators (enqueued)
int mg_pcg_clear_totals(moons_pcg* s) {
  MG_LAUNCH(k_pcg_clear_acc, 1, 1, s->m->stream, s->S);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
// read the accumulators after the stream drained (syncs)
int mg_pcg_totals(moons_pcg* s, int* iters, int* nan_any, double* last_rel) {
  moons_mesh* m = s->m;
  MG_CUDA(cudaMemcpyAsync(s->hS, s->S, sizeof(PcgScalars), cudaMemcpyDeviceToHost, m->stream));
  MG_CUDA(cudaStreamSynchronize(m->stream));
  const PcgScalars& H = *s->hS;
  g_launch_count += s->body_launches * (long long)H.runs_total;
  *iters = H.iter_total;
  *nan_any = H.nan_any;
  if (last_rel) *last_rel = (H.res0 == 0.0) ? H.res : H.res / H.res0;
  return MOONS_OK;
}

int modify_rhs(moons_pcg* s, DF* X, DF* B);

// modify_RHS (PCG_aux.f90:30-79) and the initial residual of
// PCG_solver_algorithm.f90:55-66: s->r = vol * (b - A x_BC - A x), the mean
// removed for an all-Neumann problem, wall masks applied; x gets its
// implicit BCs.  Enqueued, no host sync.
int modify_rhs(moons_pcg* s, DF* X, DF* B) {
  moons_mesh* m = s->m;
  const int nc = s->nc;
  int r = MOONS_OK;
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
  return r;
}

// fused CC iteration: the x update of the iteration that ended the loop
int cc_xfinal(moons_pcg* s, DF* X) {
  moons_mesh* m = s->m;
  MG_LAUNCH(k_cc_xfinal, resident_grid(s, (const void*)k_cc_xfinal, nblocks(X[0].n())), kLB, m->stream, X[0], s->p[0],
            s->p2[0], s->S);
  return MOONS_OK;
}

// enqueue a whole solve (modify_RHS + loop + final BCs of x); no host sync
int mg_pcg_enqueue(moons_pcg* s, moons_sf* const* x, moons_sf* const* b, const moons_isp* isp) {
  moons_mesh* m = s->m;
  DF X[3], B[3];
  for (int c = 0; c < s->nc; c++) {
    if (!x[c] || !b[c] || x[c]->f.dl != s->x_dl[c] || b[c]->f.n() != x[c]->f.n()) {
      set_error("moons_pcg_solve: field does not match the solver");
      return MOONS_ERR_SHAPE;
    }
    X[c] = x[c]->f;
    B[c] = b[c]->f;
  }
  int nc = s->nc;
  int r = modify_rhs(s, X, B);
  if (r) return r;
  // ---- scalars
  MG_LAUNCH(k_pcg_params, 1, 1, m->stream, s->S, isp->iter_max, isp->n_skip_check_res, isp->tol_rel, isp->tol_abs);
  // res0 = sqrt(sum r^2) whole array
  MG_LAUNCH(k_reduce, red_grid(s->r, nc), kBlock, m->stream, c3(s->r, nc), c3(s->r, nc), 1, 0, 0, 0, &s->S->res0,
            m->d_partial, m->d_ticket);
  const bool learned = s->learned && !s->fb;
  MG_LAUNCH(k_stag_params, 1, 1, m->stream, s->S, learned ? kStagWindow : 0, kStagFactor);
  // z = Minv r ; p = z ; rhok = dot(r,z)
  if (learned) {
    if (!s->unet) {
      set_error("moons_pcg_solve: MOONS_PREC_UNET / MOONS_PREC_UNET_MG needs a network (moons_pcg_set_unet)");
      return MOONS_ERR_STATE;
    }
    r = apply_prec_dev(s, nullptr, nullptr);
    if (r) return r;
  } else if (s->mgh) {
    r = mg_vcycle(s->mgh, s->z[0], s->r[0], m->stream, nullptr);
    if (r) return r;
  }
  for (int c = 0; c < nc; c++) {
    if (!s->mgh) {
      launch_pw(m, PW_COPY, s->z[c], &s->Minv[c], 0.0);
      launch_pw(m, PW_MUL, s->z[c], &s->r[c], 0.0);
    }
    if (s->lg.fz && !s->mgh) {
      // fused iteration: the first operator kernel forms p = 0 * p + z
      launch_pw(m, PW_FILL, s->p[c], nullptr, 0.0);
    } else {
      launch_pw(m, PW_COPY, s->p[c], &s->z[c], 0.0);
      launch_bcs(m, s->p[c], s->x_bc[c], true);  // the iteration kernels read p with its implicit BCs
    }
  }
  int dw[3] = {0, 0, 0};
  for (int c = 0; c < nc; c++) dw[c] = dirichlet_wall_bits(s->x_bc[c].defined ? &s->x_bc[c] : nullptr, s->x_dl[c]);
  MG_LAUNCH(k_reduce, red_grid(s->r, nc), kBlock, m->stream, c3(s->r, nc), c3(s->z, nc), 0, dw[0], dw[1], dw[2],
            &s->S->rhok, m->d_partial, m->d_ticket);
  MG_LAUNCH(k_pcg_start, 1, 1, m->stream, s->S);
  // k_cc_lap writes Ap on interior points only: its ghost points stay 0
  if (s->lg.cc) MG_CUDA(cudaMemsetAsync(s->Ax[0].f, 0, s->Ax[0].n() * sizeof(double), m->stream));
  MG_CUDA(cudaGetLastError());
  // ---- the loop.  MOONS_PCG_HOSTLOOP=1 launches the iteration as separate
  // kernels from the host in chunks of 32 iterations (kernels skip
  // themselves once the exit flag is up), so a profiler sees each step.
  static const bool hostloop = [] {
    const char* e = getenv("MOONS_PCG_HOSTLOOP");
    return e && e[0] == '1';
  }();
  if (hostloop) {
    for (int it = 0; it < isp->iter_max + 1; it += 32) {
      for (int q = 0; q < 16 && !r; q++) r = enqueue_iteration(s, X);  // 2 iterations each
      if (r) return r;
      MG_CUDA(cudaMemcpyAsync(s->hS, s->S, sizeof(PcgScalars), cudaMemcpyDeviceToHost, m->stream));
      MG_CUDA(cudaStreamSynchronize(m->stream));
      if (s->hS->done) break;
    }
    if (!r && s->lg.fz && !s->mgh) r = cc_xfinal(s, X);
    for (int c = 0; c < nc && !r; c++) r = launch_bcs(m, X[c], s->x_bc[c], false);
    return r;
  }
  bool need_graph = !s->exec;
  for (int c = 0; c < nc; c++)
    if (s->gx[c] != X[c].f) need_graph = true;
  if (need_graph) r = build_graph(s, X);
  if (!r) {
    cudaError_t e = cudaGraphLaunch(s->exec, m->stream);
    if (e != cudaSuccess) r = cuda_fail(e, "cudaGraphLaunch");
  }
  if (r) return r;
  if (s->lg.fz && !s->mgh) r = cc_xfinal(s, X);
  if (r) return r;
  // x: apply_BCs (the reference applies them after every update; they only
  // rewrite ghost/boundary entries, which no update reads)
  for (int c = 0; c < nc && !r; c++) r = launch_bcs(m, X[c], s->x_bc[c], false);
  return r;
}

// read back what the last enqueued solve left in the device scalars (syncs)
int mg_pcg_collect(moons_pcg* s, moons_solve_info* info, float ms) {
  moons_mesh* m = s->m;
  MG_CUDA(cudaMemcpyAsync(s->hS, s->S, sizeof(PcgScalars), cudaMemcpyDeviceToHost, m->stream));
  MG_CUDA(cudaStreamSynchronize(m->stream));
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
  if (H.wait_err) {
    const int code = H.wait_err;
    cudaMemsetAsync(&s->S->wait_err, 0, sizeof(int), m->stream);
    set_error("moons_pcg_solve: a bounded shared-memory stage wait ran out (site " + std::to_string(code) + ")");
    return MOONS_ERR_CUDA;
  }
  if (H.nan || std::isnan(H.res0) || std::isnan(H.res)) {
    set_error("moons_pcg_solve: NaN in residual norms");
    return MOONS_ERR_NAN;
  }
  return MOONS_OK;
}

extern "C" {

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
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  mg_pcg_clear_totals(s);
  set_fallback(s, false);
  cudaEventRecord(e0, m->stream);
  int r = mg_pcg_enqueue(s, x, b, isp);
  cudaEventRecord(e1, m->stream);
  cudaError_t e = cudaStreamSynchronize(m->stream);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  if (!r) r = e == cudaSuccess ? MOONS_OK : cuda_fail(e, "moons_pcg_solve");
  moons_solve_info i1{};
  if (!r) r = mg_pcg_collect(s, &i1, ms);
  if (!r && s->learned && i1.exit_reason == 4) {
    // the learned preconditioner stagnated: continue from the current x with
    // the FP32 V-cycle, to the original target (relative to the first res0)
    moons_isp isp2 = *isp;
    isp2.iter_max = std::max(0, isp->iter_max - i1.iterations);
    const double target = isp->tol_rel * i1.res0;
    isp2.tol_rel = i1.res > 0.0 ? target / i1.res : isp->tol_rel;
    set_fallback(s, true);
    cudaEventRecord(e0, m->stream);
    r = mg_pcg_enqueue(s, x, b, &isp2);
    cudaEventRecord(e1, m->stream);
    e = cudaStreamSynchronize(m->stream);
    float ms2 = 0;
    cudaEventElapsedTime(&ms2, e0, e1);
    if (!r) r = e == cudaSuccess ? MOONS_OK : cuda_fail(e, "moons_pcg_solve (fallback)");
    moons_solve_info i2{};
    if (!r) r = mg_pcg_collect(s, &i2, ms2);
    set_fallback(s, false);
    if (!r) {
      i2.iterations += i1.iterations;
      i2.res0 = i1.res0;
      i2.rel = i1.res0 == 0.0 ? i2.res : i2.res / i1.res0;
      i2.exit_reason += 10;
      i2.ms += i1.ms;
      i1 = i2;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!r && info) *info = i1;
  return r;
}

int moons_pcg_residual(moons_pcg* s, moons_sf* const* x, moons_sf* const* b, moons_sf* const* rout) {
  if (!s || !x || !b || !rout) {
    set_error("moons_pcg_residual: null pointer");
    return MOONS_ERR_ARG;
  }
  DF X[3], B[3];
  for (int c = 0; c < s->nc; c++) {
    if (!x[c] || !b[c] || !rout[c] || x[c]->f.dl != s->x_dl[c] || b[c]->f.n() != x[c]->f.n() ||
        rout[c]->f.n() != x[c]->f.n()) {
      set_error("moons_pcg_residual: field does not match the solver");
      return MOONS_ERR_SHAPE;
    }
    X[c] = x[c]->f;
    B[c] = b[c]->f;
  }
  moons_mesh* m = s->m;
  cudaSetDevice(m->device);
  int r = modify_rhs(s, X, B);
  for (int c = 0; c < s->nc && !r; c++) r = launch_pw(m, PW_COPY, rout[c]->f, &s->r[c], 0.0);
  if (!r) MG_CUDA(cudaStreamSynchronize(m->stream));
  return r;
}

int moons_pcg_apply_op(moons_pcg* s, moons_sf* const* out, moons_sf* const* x) {
  if (!s || !out || !x) {
    set_error("moons_pcg_apply_op: null argument");
    return MOONS_ERR_ARG;
  }
  moons_mesh* m = s->m;
  cudaSetDevice(m->device);
  DF O[3], X[3];
  for (int c = 0; c < s->nc; c++) {
    if (!out[c] || !x[c] || out[c]->f.n() != s->Ax[c].n() || x[c]->f.n() != s->Ax[c].n() ||
        out[c]->f.dl != s->x_dl[c] || x[c]->f.dl != s->x_dl[c]) {
      set_error("moons_pcg_apply_op: field does not match the solver's unknown");
      return MOONS_ERR_SHAPE;
    }
    O[c] = out[c]->f;
    X[c] = x[c]->f;
  }
  const int rc = apply_op_explicit(s, O, X);
  if (rc) return rc;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_pcg_apply_prec(moons_pcg* s, moons_sf* const* z, moons_sf* const* r) {
  if (!s || !z || !r) {
    set_error("moons_pcg_apply_prec: null argument");
    return MOONS_ERR_ARG;
  }
  moons_mesh* m = s->m;
  cudaSetDevice(m->device);
  for (int c = 0; c < s->nc; c++)
    if (!z[c] || !r[c] || z[c]->f.n() != s->r[c].n() || r[c]->f.n() != s->r[c].n()) {
      set_error("moons_pcg_apply_prec: field does not match the solver");
      return MOONS_ERR_SHAPE;
    }
  int rc = MOONS_OK;
  if (s->mgh) {
    rc = mg_vcycle(s->mgh, z[0]->f, r[0]->f, m->stream, nullptr);
  } else {
    for (int c = 0; c < s->nc && !rc; c++) {
      rc = launch_pw(m, PW_COPY, z[c]->f, &s->Minv[c], 0.0);
      if (!rc) rc = launch_pw(m, PW_MUL, z[c]->f, &r[c]->f, 0.0);
    }
  }
  if (rc) return rc;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_pcg_set_unet(moons_pcg* s, moons_unet* u) {
  if (!s || !u) {
    set_error("moons_pcg_set_unet: null argument");
    return MOONS_ERR_ARG;
  }
  if (!s->learned) {
    set_error("moons_pcg_set_unet: the solver was not created with MOONS_PREC_UNET or MOONS_PREC_UNET_MG");
    return MOONS_ERR_ARG;
  }
  if (unet_mesh(u) != s->m) {
    set_error("moons_pcg_set_unet: the network lives on another mesh");
    return MOONS_ERR_SHAPE;
  }
  int r = unet_prepare(u);
  if (r) return r;
  s->unet = u;
  drop_graphs(s);
  return MOONS_OK;
}

}  // extern "C"

namespace mg {
MGHier* pcg_mg_hier(moons_pcg* s) { return s ? s->mgh : nullptr; }
moons_mesh* pcg_mesh(moons_pcg* s) { return s ? s->m : nullptr; }
}  // namespace mg
