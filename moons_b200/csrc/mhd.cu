// mhd.cu -- the MOONS MHD time step on one B200 (HW/MOONS/MOONS_solver.f90:47-144).
//
// All fields stay in HBM for the whole run; the host only enqueues kernels
// and the four PCG solves per step (U, p, B, phi).  The sequence follows the
// reference routine by routine; pointwise chains the reference runs as
// separate whole-array passes (AB2 RHS build, projection update, cross
// products) are fused into single kernels that perform the same operations
// in the same order per point.
#include <cmath>
#include <cstring>
#include <vector>

#include "kernels.cuh"
#include "runtime.cuh"
#include "schemes.cuh"

namespace mg {

// ---- fused pointwise kernels ----------------------------------------------
// Predictor RHS of the time schemes (time_marching_methods.f90,
// time_marching_methods_SF.f90) in one pass: the point arithmetic of each
// form is in schemes.cuh (scheme_increment, the wall mask, scheme_rhs):
//  6 Euler_time_AB2_sources (:137-142); 4 the AB2 schemes without diffusion
//  (:289-292, :342-345) and the SF AB2 schemes; 5 Euler_time_Euler_sources
//  and the Euler schemes without diffusion (:70-73, :321-323, :362-364);
//  7 O2_BDF_time_AB2_sources (:104-108); 8 Euler_time_RK_sources (:217-222)
//  with a = (dt gamma, dt zeta, dt 2 alpha) (dt alpha for the SF scheme).
// Then Xnm1 = X when set_nm1 (every scheme but the "no_correction" ones,
// whose t is X itself: X = X + increment).  dts is dt, or the product 2/3*dt
// for form 7.  t may alias X: each point reads X and Xnm1 before writing t.
__global__ void k_ab2_rhs(DF t, DF F, DF Fm, DF L, DF X, DF Xnm1, double dts, int wallbits, int form,
                          int set_nm1, double a0, double a1, double a2) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= t.n()) return;
  int i, j, k;
  ijk_of(idx, t, i, j, k);
  const double fm = form == kFormEuler ? 0.0 : Fm.f[idx];
  const double l = (form == kFormAB2L || form == kFormRK) ? L.f[idx] : 0.0;
  double v = scheme_increment(form, F.f[idx], fm, l, dts, a0, a1, a2);
  if (wallbits) {
    if (((wallbits & 1) && i == 2) || ((wallbits & 2) && i == t.s0 - 1) || ((wallbits & 4) && j == 2) ||
        ((wallbits & 8) && j == t.s1 - 1) || ((wallbits & 16) && k == 2) || ((wallbits & 32) && k == t.s2 - 1))
      v = 0.0;
  }
  const double x = X.f[idx];
  const double xnm1 = form == kFormBDF2 ? Xnm1.f[idx] : 0.0;
  t.f[idx] = scheme_rhs(form, v, x, xnm1);
  if (set_nm1) Xnm1.f[idx] = x;
}
// clean_div tail: temp_F = grad(phi) ; temp_F *= 1/scale ; X = Xstar - temp_F
__global__ void k_project(DF X, DF Xstar, DF g, double inv_scale) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= X.n()) return;
  double gv = g.f[idx] * inv_scale;
  X.f[idx] = Xstar.f[idx] - gv;
}
// cross_product_x/y/z (HW/grid_field/GF_3D/GF_cross_product.f90:17-70)
__global__ void k_cross(DF o, DF a1, DF a2, DF b1, DF b2, int neg) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= o.n()) return;
  double v = a1.f[idx] * b2.f[idx] - a2.f[idx] * b1.f[idx];
  o.f[idx] = neg ? -v : v;
}
// embed (ind <- mom) / extract (mom <- ind) over the physical region of the
// fluid-mesh field (indices 2..s-1), offset o (ops_embedExtract.f90)
__global__ void k_embed_extract(DF dst, DF src, int o0, int o1, int o2, int embed) {
  const DF& mom = embed ? src : dst;
  int ni = mom.s0 - 2, nj = mom.s1 - 2, nk = mom.s2 - 2;
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (size_t)ni * nj * nk) return;
  int i = (int)(idx % ni) + 2;
  size_t r = idx / ni;
  int j = (int)(r % nj) + 2;
  int k = (int)(r / nj) + 2;
  if (embed) dst(i + o0, j + o1, k + o2) = src(i, j, k);
  else dst(i, j, k) = src(i + o0, j + o1, k + o2);
}
// t(i,j,k) = prof[j-1] over the whole array (a profile along y)
__global__ void k_fill_y(DF t, const double* prof) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= t.n()) return;
  int i, j, k;
  ijk_of(idx, t, i, j, k);
  t.f[idx] = prof[j - 1];
}
// u += c everywhere (compute_add_MPG: add(U%x, scale*dt))
__global__ void k_add_scalar(double* a, double c, size_t n) {
  size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = a[i] + c;
}
__global__ void k_sumsq(DF a, double* partial, unsigned* ticket, double* out) {
  double acc = 0.0;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < a.n(); idx += (size_t)gridDim.x * blockDim.x) {
    double v = a.f[idx];
    acc += v * v;
  }
  double bs = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = bs;
  if (last_block(ticket)) {
    double t = sum_partials(partial, gridDim.x);
    if (threadIdx.x == 0) {
      *out = t;
      *ticket = 0;
    }
  }
}

}  // namespace mg

using namespace mg;

namespace {
inline int orth(int a, int b) { return 6 - a - b; }  // 1-based directions
// solve_method of the momentum / induction step: 1 to 9, 0 selects the
// default, 6.  Euler_time_AB2_sources_FFT (9, time_marching_methods.f90:
// 152-185) is 6 with its cleaning Poisson equation solved directly
// (clean_div_FFT, clean_divergence.f90:61-83): the step runs 6 and the
// solver of that equation is created with the direct solve (MOONS_PREC_FD).
inline bool time_method_ok(int m) { return m >= 0 && m <= 9; }
// RK_Params of one stage (init_RKP, RK_params_extend.f90:22-55): the
// three-stage coefficients of Lundbladh et al. (1999), or all 1 when the
// step has one stage (RK inactive); beta = alpha
struct RKStage {
  double gamma, zeta, alpha, beta;
};
inline RKStage rk_stage(int stages, int n) {
  if (stages != 3) return {1.0, 1.0, 1.0, 1.0};
  static const double g[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
  static const double z[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
  static const double a[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
  return {g[n - 1], z[n - 1], a[n - 1], a[n - 1]};
}
inline int time_method(int m) { return m == 0 || m == 9 ? 6 : m; }
}

struct moons_mhd {
  moons_mesh* mm = nullptr;  // fluid mesh
  moons_mesh* mi = nullptr;  // induction mesh
  bool same = true;
  moons_mhd_params P{};
  std::vector<moons_sf*> owned;
  // momentum
  moons_sf *U[3], *Ustar[3], *Unm1[3], *F[3], *Fnm1[3], *L[3], *tF1[3], *tF2[3], *tF3[3], *tCC, *p, *UCC[3], *divU;
  moons_sf* UE[3][3];
  moons_pcg *pcgU = nullptr, *pcgP = nullptr;
  moons_unet* unet[2] = {nullptr, nullptr};  // networks of the learned + mixed pressure / potential solves
  // induction
  moons_sf *B[3], *Bstar[3], *Bnm1[3], *B0[3], *Btot[3], *Fi[3], *Fnm1i[3], *Li[3], *J[3], *jxb[3], *sig[3], *phi,
      *tCCi, *tFi1[3], *tFi2[3], *tE[3], *curlUxB[3], *divB, *Ui[3], *E[3];
  moons_sf *UEi[3][3], *BE[3][3], *TF1[3][3], *TF2[3][3];
  moons_pcg *pcgB = nullptr, *pcgPhi = nullptr;
  // energy (on the induction mesh)
  moons_sf *T = nullptr, *Tnm1 = nullptr, *FT = nullptr, *FnmT = nullptr, *LT = nullptr, *tCCT = nullptr,
           *tCCT2 = nullptr, *tmpT = nullptr, *kT[3] = {}, *grav[3] = {}, *tFT[3] = {}, *UFT[3] = {};
  // nrg%U_CC, ind%sigmaInv_CC, nrg%temp_CC2, nrg%temp_CC1_VF (KE diffusion,
  // viscous dissipation, Joule heating)
  moons_sf *UCCn[3] = {}, *sigInvCC = nullptr, *tCCT3 = nullptr, *tVFT[3] = {};
  moons_pcg* pcgT = nullptr;
  double* heat_prof = nullptr;  // add_volumetric_heating_Nuclear profile per y index (device)
  double coefU = NAN, coefB = NAN, coefT = NAN;
  int iters[5] = {0, 0, 0, 0, 0};
  double res_p = 0, res_phi = 0;
  double* d_red = nullptr;
  cudaStream_t mi_stream_saved = nullptr;  // the induction mesh runs on the fluid mesh's stream
};

namespace {

int mk(moons_mhd* s, moons_mesh* m, int dl, moons_sf** out) {
  int r = moons_sf_create(m, dl, out);
  if (!r) s->owned.push_back(*out);
  return r;
}

int set_bcs_from(moons_sf* f, const moons_bc_spec& b) { return moons_sf_set_bcs(f, &b); }

// moons_sf view helpers
inline DF& D(moons_sf* f) { return f->f; }

int launch_cross3(moons_mesh* m, moons_sf* const* o, moons_sf* A[3][3], moons_sf* Bt[3][3]) {
  // cross_product_TF (TF_extend.f90:385-401)
  MG_LAUNCH(k_cross, nblocks(D(o[0]).n()), kBlock, m->stream, D(o[0]), D(A[1][0]), D(A[2][0]), D(Bt[1][0]), D(Bt[2][0]), 0);
  MG_LAUNCH(k_cross, nblocks(D(o[1]).n()), kBlock, m->stream, D(o[1]), D(A[0][1]), D(A[2][1]), D(Bt[0][1]), D(Bt[2][1]), 1);
  MG_LAUNCH(k_cross, nblocks(D(o[2]).n()), kBlock, m->stream, D(o[2]), D(A[0][2]), D(A[1][2]), D(Bt[0][2]), D(Bt[1][2]), 0);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

int face2edge_nd(moons_mesh* m, moons_sf* E[3][3], moons_sf* const* Fc) {
  int r = MOONS_OK;
  for (int c = 0; c < 3 && !r; c++)
    for (int l = 0; l < 3 && !r; l++)
      if (c != l) r = launch_interp(m, D(E[c][l]), D(Fc[c]), orth(c + 1, l + 1));
  return r;
}
int edge2face_nd(moons_mesh* m, moons_sf* Fo[3][3], moons_sf* const* Ec) {
  return face2edge_nd(m, Fo, Ec);  // same index pattern: interp along the orthogonal direction
}
int face2face_nd(moons_mesh* m, moons_sf* Fo[3][3], moons_sf* const* Fc, moons_sf* tCC) {
  int r = MOONS_OK;
  for (int c = 0; c < 3 && !r; c++)
    for (int l = 0; l < 3 && !r; l++)
      if (c != l) {
        r = launch_interp(m, D(tCC), D(Fc[c]), c + 1);
        if (!r) r = launch_interp(m, D(Fo[c][l]), D(tCC), l + 1);
      }
  return r;
}
int curl3(moons_mesh* m, moons_sf* const* o, moons_sf* const* u) {
  int r;
  if ((r = launch_del(m, D(o[0]), D(u[2]), 1, 2, 0, 1))) return r;
  if ((r = launch_del(m, D(o[0]), D(u[1]), 1, 3, 0, 3))) return r;
  if ((r = launch_del(m, D(o[1]), D(u[0]), 1, 3, 0, 1))) return r;
  if ((r = launch_del(m, D(o[1]), D(u[2]), 1, 1, 0, 3))) return r;
  if ((r = launch_del(m, D(o[2]), D(u[1]), 1, 1, 0, 1))) return r;
  return launch_del(m, D(o[2]), D(u[0]), 1, 2, 0, 3);
}
int div3(moons_mesh* m, moons_sf* o, moons_sf* const* u) {
  int r;
  if ((r = launch_del(m, D(o), D(u[0]), 1, 1, 0, 1))) return r;
  if ((r = launch_del(m, D(o), D(u[1]), 1, 2, 0, 2))) return r;
  if ((r = launch_del(m, D(o), D(u[2]), 1, 3, 0, 2))) return r;
  return mask_ghost_XPeriodic(m, D(o), o->bc.defined ? &o->bc : nullptr);
}
int grad3(moons_mesh* m, moons_sf* const* g, moons_sf* u) {
  int r;
  for (int d = 0; d < 3; d++)
    if ((r = launch_del(m, D(g[d]), D(u), 1, d + 1, 0, 1))) return r;
  return MOONS_OK;
}
int embed_extract(moons_mesh* m, moons_sf* dst, moons_sf* src, const int o[3], bool embed) {
  const DF& mom = embed ? D(src) : D(dst);
  size_t n = (size_t)(mom.s0 - 2) * (mom.s1 - 2) * (mom.s2 - 2);
  MG_LAUNCH(k_embed_extract, nblocks(n), kBlock, m->stream, D(dst), D(src), o[0], o[1], o[2], embed ? 1 : 0);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
int copy(moons_mesh* m, moons_sf* dst, moons_sf* src) {
  MG_CUDA(cudaMemcpyAsync(D(dst).f, D(src).f, D(src).n() * sizeof(double), cudaMemcpyDeviceToDevice, m->stream));
  return MOONS_OK;
}

// solves are enqueued without a host sync; iteration counts, NaN flags and
// the last residual are read once per moons_mhd_step (mg_pcg_totals)
int solve(moons_pcg* s, moons_sf* const* x, moons_sf* const* b, const moons_isp& isp, int* iters, double* rel) {
  (void)iters;
  (void)rel;
  if (isp.n_skip_check_res < 1) {
    set_error("moons_mhd: n_skip_check_res must be >= 1");
    return MOONS_ERR_ARG;
  }
  return mg_pcg_enqueue(s, x, b, &isp);
}

// One solve_momentum / solve_induction time step for solve_method 1 to 8
// (time_marching_methods.f90:47-208, :266-366, clean_divergence.f90:37-59):
//  5 to 8:  the scheme's RHS, update_MFP with its implicit factor, the PCG
//           solve for X*, then clean_div;
//  3, 4:    X* = X + dt F (Euler) or X + dt AB2(F, Fnm1), then clean_div;
//  1, 2:    X = X + dt F or X + dt AB2(F, Fnm1), then apply_BCs(X).
// clean_div's scale is 1/dt for method 6 and 1 for the others.
int time_scheme_step(moons_mhd* s, moons_mesh* m, moons_pcg* pv, moons_pcg* ps, const moons_isp& iv, const moons_isp& is,
              moons_sf** X, moons_sf** Xstar, moons_sf** Xnm1, moons_sf* ph, moons_sf** Fn, moons_sf** Fm,
              moons_sf** Lx, moons_sf** t1, moons_sf* tcc, double coeff_implicit, double* coef_cache, int slot_v,
              int slot_s, double* res_s, int method, const RKStage& rk) {
  double dt = s->P.dt;
  double dts = method == 7 ? (2.0 / 3.0) * dt : dt;
  // multiply(temp_F1,F,dt*gamma) ; add_product(temp_F1,Fnm1,dt*zeta) ;
  // add_product(temp_F1,L,dt*2*alpha)
  const double a0 = dt * rk.gamma, a1 = dt * rk.zeta, a2 = dt * 2.0 * rk.alpha;
  const int form = (method == 1 || method == 3 || method == 5) ? 5 : (method == 2 || method == 4) ? 4 : method;
  const bool no_correction = method <= 2, implicit = method >= 5;  // 5 to 8
  moons_sf** out = no_correction ? X : implicit ? t1 : Xstar;
  for (int c = 0; c < 3; c++) {
    int wb = dirichlet_wall_bits(X[c]->bc.defined ? &X[c]->bc : nullptr, D(X[c]).dl);
    MG_LAUNCH(k_ab2_rhs, nblocks(D(out[c]).n()), kBlock, m->stream, D(out[c]), D(Fn[c]), D(Fm[c]), D(Lx[c]),
              D(X[c]), D(Xnm1[c]), dts, wb, form, no_correction ? 0 : 1, a0, a1, a2);
  }
  int r;
  if (no_correction) {
    for (int k = 0; k < 3; k++)
      if ((r = launch_bcs(m, D(X[k]), X[k]->bc, false))) return r;
    MG_CUDA(cudaGetLastError());
    return MOONS_OK;
  }
  MG_CUDA(cudaGetLastError());
  // update_MFP(PCG, m, dt*f*coeff_implicit, ...) with f = 1, 2/3 or, for
  // method 8, 2*beta; the preconditioner only changes with c, so it is rebuilt
  // when c changes (methods 5 and 7 rebuild it on the first steps only,
  // TMP%n_step <= 2, which is the same thing for a fixed dt)
  double c = method == 7   ? dt * (2.0 / 3.0) * coeff_implicit
             : method == 8 ? dt * 2.0 * rk.beta * coeff_implicit
                           : dt * 1.0 * coeff_implicit;
  if (implicit && !(c == *coef_cache)) {
    if ((r = moons_pcg_update_mfp(pv, c, 1))) return r;
    *coef_cache = c;
  }
  if (implicit && (r = solve(pv, Xstar, t1, iv, &s->iters[slot_v], nullptr))) return r;
  double scale = method == 6 ? 1.0 / dt : 1.0;
  if ((r = div3(m, tcc, Xstar))) return r;
  if ((r = launch_pw(m, PW_SCALE, D(tcc), nullptr, scale))) return r;
  moons_sf* xp[1] = {ph};
  moons_sf* bp[1] = {tcc};
  if ((r = solve(ps, xp, bp, is, &s->iters[slot_s], res_s))) return r;
  if ((r = grad3(m, t1, ph))) return r;
  for (int k = 0; k < 3; k++) {
    MG_LAUNCH(k_project, nblocks(D(X[k]).n()), kBlock, m->stream, D(X[k]), D(Xstar[k]), D(t1[k]), 1.0 / scale);
    if ((r = launch_bcs(m, D(X[k]), X[k]->bc, false))) return r;
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

int compute_J(moons_mhd* s) {
  moons_mesh* m = s->mi;
  int r = curl3(m, s->J, s->B);
  for (int c = 0; c < 3 && !r; c++) r = launch_pw(m, PW_SCALE, D(s->J[c]), nullptr, s->P.scale_current);
  return r;
}
int compute_Btot(moons_mhd* s) {
  moons_mesh* m = s->mi;
  int r = MOONS_OK;
  for (int c = 0; c < 3 && !r; c++) {
    r = copy(m, s->Btot[c], s->B0[c]);
    if (!r && s->P.finite_Rem) r = launch_pw(m, PW_ADD, D(s->Btot[c]), &D(s->B[c]), 0.0);
  }
  return r;
}
int compute_JxB(moons_mhd* s) {
  moons_mesh* m = s->mi;
  int r;
  if (s->P.induction == MOONS_IND_B) r = edge2face_nd(m, s->TF1, s->J);
  else r = face2face_nd(m, s->TF1, s->J, s->tCCi);
  if (!r) r = face2face_nd(m, s->TF2, s->Btot, s->tCCi);
  if (!r) r = launch_cross3(m, s->jxb, s->TF1, s->TF2);
  for (int c = 0; c < 3 && !r; c++) r = launch_pw(m, PW_SCALE, D(s->jxb[c]), nullptr, s->P.scale_JxB);
  return r;
}
int potential_solve(moons_mhd* s) {
  moons_mesh* m = s->mi;
  int r = MOONS_OK;
  for (int c = 0; c < 3 && !r; c++) {
    if (s->same) r = copy(m, s->Ui[c], s->U[c]);
    else r = embed_extract(m, s->Ui[c], s->U[c], s->P.ind_offset, true);
  }
  if (!r) r = face2face_nd(m, s->TF1, s->Ui, s->tCCi);
  if (!r) r = face2face_nd(m, s->TF2, s->Btot, s->tCCi);
  if (!r) r = launch_cross3(m, s->E, s->TF1, s->TF2);
  for (int c = 0; c < 3 && !r; c++) {
    r = copy(m, s->tFi1[c], s->E[c]);
    if (!r) r = launch_pw(m, PW_MUL, D(s->tFi1[c]), &D(s->sig[c]), 0.0);
  }
  if (!r) r = div3(m, s->tCCi, s->tFi1);
  if (r) return r;
  moons_sf* xf[1] = {s->phi};
  moons_sf* bf[1] = {s->tCCi};
  if ((r = solve(s->pcgPhi, xf, bf, s->P.isp_phi, &s->iters[3], &s->res_phi))) return r;
  if ((r = grad3(m, s->tFi2, s->phi))) return r;
  for (int c = 0; c < 3 && !r; c++) {
    r = copy(m, s->J[c], s->E[c]);
    if (!r) r = launch_pw(m, PW_SUB, D(s->J[c]), &D(s->tFi2[c]), 0.0);
    if (!r) r = launch_pw(m, PW_MUL, D(s->J[c]), &D(s->sig[c]), 0.0);
  }
  return r;
}

// advect_U_convection1 (ops_advect.f90:71-127) into tF3
int advect_U_convection1(moons_mhd* s) {
  moons_mesh* m = s->mm;
  int r = MOONS_OK;
  for (int c = 0; c < 3 && !r; c++) {
    r = launch_interp(m, D(s->tCC), D(s->U[c]), c + 1);
    if (!r) r = launch_del(m, D(s->tF3[c]), D(s->tCC), 1, c + 1, 0, 1);
    if (!r) r = launch_pw(m, PW_MUL, D(s->tF3[c]), &D(s->U[c]), 0.0);
  }
  struct T {
    int c, e, d, v;
  };
  const T terms[6] = {{0, 2, 2, 1}, {0, 1, 3, 2}, {1, 2, 1, 0}, {1, 0, 3, 2}, {2, 1, 1, 0}, {2, 0, 2, 1}};
  for (const T& t : terms) {
    if (r) break;
    r = launch_del(m, D(s->tF1[t.c]), D(s->UE[t.c][t.e]), 1, t.d, 0, 1);
    if (!r) r = launch_interp(m, D(s->tCC), D(s->U[t.v]), t.v + 1);
    if (!r) r = launch_interp(m, D(s->tF2[t.c]), D(s->tCC), t.c + 1);
    if (!r) r = launch_pw(m, PW_MUL, D(s->tF1[t.c]), &D(s->tF2[t.c]), 0.0);
    if (!r) r = launch_pw(m, PW_ADD, D(s->tF3[t.c]), &D(s->tF1[t.c]), 0.0);
  }
  return r;
}

// ---- energy equation ---------------------------------------------------------
// add_KE_diffusion, add_viscous_dissipation, add_joule_heating
// (energy_sources.f90:51-94) as add_all_energy_sources calls them
// (add_all_energy_sources.f90:30-32, 51-62).  Each assigns its scratch
// (add(f,g,h,...) is f = g + h + ... in GF_add.f90:41-86,137-160), so no
// term carries state from an earlier one.
int energy_sources_KE_visc_joule(moons_mhd* s) {
  moons_mesh* mi = s->mi;
  const moons_mhd_params& P = s->P;
  int r = MOONS_OK;
  if (P.scale_KE_diffusion_T != 0.0 || P.scale_viscous_dissipation_T != 0.0) {
    // embedCC(nrg%U_CC, mom%U_CC, nrg%MD)
    for (int c = 0; c < 3 && !r; c++) {
      if (s->same) r = copy(mi, s->UCCn[c], s->UCC[c]);
      else r = embed_extract(mi, s->UCCn[c], s->UCC[c], P.ind_offset, true);
    }
  }
  // temp = (a0 + a1) + a2 over three CC fields (add_GF_GF_GF_GF)
  auto sum3 = [&](moons_sf* out, moons_sf* const* a) -> int {
    int q = copy(mi, out, a[0]);
    if (!q) q = launch_pw(mi, PW_ADD, D(out), &D(a[1]), 0.0);
    if (!q) q = launch_pw(mi, PW_ADD, D(out), &D(a[2]), 0.0);
    return q;
  };
  if (!r && P.scale_KE_diffusion_T != 0.0) {
    // temp_CC1_VF = U_CC ; square ; temp_CC1 = x + y + z ; temp_CC2 = lap(temp_CC1) ; F += s temp_CC2
    for (int c = 0; c < 3 && !r; c++) {
      r = copy(mi, s->tVFT[c], s->UCCn[c]);
      if (!r) r = launch_pw(mi, PW_MUL, D(s->tVFT[c]), &D(s->tVFT[c]), 0.0);
    }
    if (!r) r = sum3(s->tCCT, s->tVFT);
    if (!r) r = launch_del(mi, D(s->tCCT3), D(s->tCCT), 2, 1, 0, 1);  // lapUniformCoeff_SF
    if (!r) r = launch_del(mi, D(s->tCCT3), D(s->tCCT), 2, 2, 0, 2);
    if (!r) r = launch_del(mi, D(s->tCCT3), D(s->tCCT), 2, 3, 0, 2);
    if (!r) r = launch_pw(mi, PW_ADD_PRODUCT, D(s->FT), &D(s->tCCT3), P.scale_KE_diffusion_T);
  }
  if (!r && P.scale_viscous_dissipation_T != 0.0) {
    // temp_CC_TF = grad(U_CC) (collocated first derivatives, CC -> CC) ;
    // square ; temp_CC1 = g%x%x + g%y%x + g%z%x + g%x%y + ... + g%z%z
    // (add_SF_TF, TF_extend.f90:248-255) ; F += s temp_CC1
    bool first = true;
    for (int d = 0; d < 3 && !r; d++)
      for (int c = 0; c < 3 && !r; c++) {
        r = launch_del(mi, D(s->tCCT2), D(s->UCCn[c]), 1, d + 1, 0, 1);
        if (!r) r = launch_pw(mi, PW_MUL, D(s->tCCT2), &D(s->tCCT2), 0.0);
        if (!r) r = first ? copy(mi, s->tCCT, s->tCCT2) : launch_pw(mi, PW_ADD, D(s->tCCT), &D(s->tCCT2), 0.0);
        first = false;
      }
    if (!r) r = launch_pw(mi, PW_ADD_PRODUCT, D(s->FT), &D(s->tCCT), P.scale_viscous_dissipation_T);
  }
  if (!r && P.scale_joule_heating_T != 0.0) {
    // temp_CC1_VF = edge2CellCenter(J) (edge -> face along the face direction
    // (x: y, y: z, z: x), then face -> CC; ops_interp.f90:415-431, 688-696);
    // the potential form keeps J on faces: face -> CC
    const bool pot = P.induction == MOONS_IND_POTENTIAL;
    for (int c = 0; c < 3 && !r; c++) {
      if (pot) {
        r = launch_interp(mi, D(s->tVFT[c]), D(s->J[c]), c + 1);
      } else {
        const int edir = c + 1, fdir = edir == 1 ? 2 : (edir == 2 ? 3 : 1);
        moons_sf* tf = s->tFT[fdir - 1];
        r = launch_interp(mi, D(tf), D(s->J[c]), 6 - edir - fdir);
        if (!r) r = launch_interp(mi, D(s->tVFT[c]), D(tf), fdir);
      }
      if (!r) r = launch_pw(mi, PW_MUL, D(s->tVFT[c]), &D(s->tVFT[c]), 0.0);
    }
    if (!r) r = sum3(s->tCCT, s->tVFT);
    if (!r) r = launch_pw(mi, PW_MUL, D(s->tCCT), &D(s->sigInvCC), 0.0);
    if (!r) r = launch_pw(mi, PW_ADD_PRODUCT, D(s->FT), &D(s->tCCT), P.scale_joule_heating_T);
  }
  return r;
}

// add_all_energy_sources (add_all_energy_sources.f90:21-67) with the
// advection, diffusion and volumetric-heating terms (energy_sources.f90),
// then solve_energy (energy_extend.f90:236-262), methods 2 and 3
// add_all_energy_sources + solve_energy (add_all_energy_sources.f90:21-67,
// energy_extend.f90:236-262) for one stage of the step
int energy_step(moons_mhd* s, const RKStage& rk) {
  moons_mesh* mi = s->mi;
  const moons_mhd_params& P = s->P;
  const bool rk_active = P.rk_stages == 3;
  int r = copy(mi, s->FnmT, s->FT);
  if (!r && rk_active) r = launch_pw(mi, PW_FILL, D(s->LT), nullptr, 0.0);
  if (!r) r = launch_pw(mi, PW_FILL, D(s->FT), nullptr, 0.0);
  if (!r && P.scale_advection_T != 0.0) {
    // add_advection: S += scale * (-div(face(T) * U_F)), U_F = embedFace(U)
    for (int c = 0; c < 3 && !r; c++) {
      if (s->same) r = copy(mi, s->UFT[c], s->U[c]);
      else r = embed_extract(mi, s->UFT[c], s->U[c], P.ind_offset, true);
    }
    for (int c = 0; c < 3 && !r; c++) {
      r = launch_interp(mi, D(s->tFT[c]), D(s->T), c + 1);
      if (!r) r = launch_pw(mi, PW_MUL, D(s->tFT[c]), &D(s->UFT[c]), 0.0);
    }
    if (!r) r = div3(mi, s->tCCT, s->tFT);
    if (!r) r = launch_pw(mi, PW_SCALE, D(s->tCCT), nullptr, -1.0);
    if (!r) r = launch_pw(mi, PW_ADD_PRODUCT, D(s->FT), &D(s->tCCT), P.scale_advection_T);
  }
  if (!r && P.scale_diffusion_T != 0.0) {
    // add_diffusion: S += scale * lap(T) (lapUniformCoeff_SF), into L when
    // the RK stages are active
    r = launch_del(mi, D(s->tCCT), D(s->T), 2, 1, 0, 1);
    if (!r) r = launch_del(mi, D(s->tCCT), D(s->T), 2, 2, 0, 2);
    if (!r) r = launch_del(mi, D(s->tCCT), D(s->T), 2, 3, 0, 2);
    if (!r) r = launch_pw(mi, PW_ADD_PRODUCT, rk_active ? D(s->LT) : D(s->FT), &D(s->tCCT), P.scale_diffusion_T);
  }
  if (!r) r = energy_sources_KE_visc_joule(s);
  if (!r && P.scale_heating_T != 0.0) {
    // add_volumetric_heating_Nuclear: temp = scale*F0*exp(-m (y_c + 1)); S += scale * temp
    MG_LAUNCH(k_fill_y, nblocks(D(s->tCCT).n()), kBlock, mi->stream, D(s->tCCT), s->heat_prof);
    r = launch_pw(mi, PW_ADD_PRODUCT, D(s->FT), &D(s->tCCT), P.scale_heating_T);
  }
  if (r) return r;
  // the energy time schemes (solve_energy's select case, energy_extend.f90:
  // 244-257; time_marching_methods_SF.f90), RHS forms of k_ab2_rhs:
  //  1 Euler_time_no_diff_Euler_sources_SF (:154-170): X += dt F
  //  2 Euler_time_no_diff_AB2_sources_SF (:135-152): X += dt AB2(F, Fnm1)
  //  3 Euler_time_AB2_sources_SF (:71-98): solve (I + dt c A) X = X + dt AB2
  //  4 O2_BDF_time_AB2_sources_SF (:42-69): solve (I + 2/3 dt c A) X =
  //    4/3 X - 1/3 Xnm1 + 2/3 dt AB2
  //  5 Euler_time_RK_sources_SF (:100-133): solve (I + beta dt c A) X =
  //    X + dt (gamma F + zeta Fnm1 + alpha L)
  // (increments on wall-Dirichlet points zeroed; CC data has none)
  const int mT = P.solve_method_T;
  const int wb = dirichlet_wall_bits(s->T->bc.defined ? &s->T->bc : nullptr, D(s->T).dl);
  const int form = mT == 1 ? 5 : mT == 4 ? 7 : mT == 5 ? 8 : 4;
  const double dts = mT == 4 ? (2.0 / 3.0) * P.dt : P.dt;
  moons_sf* out = mT <= 2 ? s->T : s->tmpT;  // 1, 2: X = X + increment
  MG_LAUNCH(k_ab2_rhs, nblocks(D(out).n()), kBlock, mi->stream, D(out), D(s->FT), D(s->FnmT), D(s->LT), D(s->T),
            D(s->Tnm1), dts, wb, form, mT <= 2 ? 0 : 1, P.dt * rk.gamma, P.dt * rk.zeta, P.dt * rk.alpha);
  MG_CUDA(cudaGetLastError());
  if (mT <= 2) return MOONS_OK;
  // update_MFP: 3 and 4 rebuild the preconditioner while TMP%n_step <= 2,
  // 5 every stage; it only changes with c, so it is rebuilt when c changes
  const double c = mT == 4   ? P.dt * (2.0 / 3.0) * P.coeff_implicit_T
                   : mT == 5 ? P.dt * rk.beta * P.coeff_implicit_T
                             : P.dt * 1.0 * P.coeff_implicit_T;
  if (!(c == s->coefT)) {
    if ((r = moons_pcg_update_mfp(s->pcgT, c, 1))) return r;
    s->coefT = c;
  }
  moons_sf* xt[1] = {s->T};
  moons_sf* bt[1] = {s->tmpT};
  return solve(s->pcgT, xt, bt, P.isp_T, &s->iters[4], nullptr);
}

// compute_add_buoyancy (momentum_sources.f90:133-150): F += scale extractFace(face(T g))
int add_buoyancy(moons_mhd* s) {
  moons_mesh *m = s->mm, *mi = s->mi;
  int r = MOONS_OK;
  for (int c = 0; c < 3 && !r; c++) {
    r = copy(mi, s->tCCT2, s->T);
    if (!r) r = launch_pw(mi, PW_MUL, D(s->tCCT2), &D(s->grav[c]), 0.0);
    if (!r) r = launch_interp(mi, D(s->tFT[c]), D(s->tCCT2), c + 1);
    if (!r) {
      if (s->same) r = copy(m, s->tF1[c], s->tFT[c]);
      else r = embed_extract(m, s->tF1[c], s->tFT[c], s->P.ind_offset, false);
    }
    if (!r) r = launch_pw(m, PW_ADD_PRODUCT, D(s->F[c]), &D(s->tF1[c]), s->P.scale_buoyancy);
  }
  return r;
}

// One stage of the step (the body of the RK stage loop, MOONS_solver.f90:73-97)
int step_once(moons_mhd* s, const RKStage& rk) {
  moons_mesh* m = s->mm;
  const moons_mhd_params& P = s->P;
  double dt = P.dt;
  int r = MOONS_OK;
  // ---- energy (solve_MOONS: energy sources and solve before momentum)
  if (P.energy && (r = energy_step(s, rk))) return r;
  // ---- add_all_momentum_sources
  if (P.mpg_dir >= 1 && P.mpg_dir <= 3) {
    DF u = D(s->U[P.mpg_dir - 1]);
    MG_LAUNCH(k_add_scalar, nblocks(u.n()), kBlock, m->stream, u.f, P.mpg_scale * dt, u.n());
    for (int c = 0; c < 3 && !r; c++) r = launch_bcs(m, D(s->U[c]), s->U[c]->bc, false);
  }
  for (int c = 0; c < 3 && !r; c++) {
    r = copy(m, s->Fnm1[c], s->F[c]);
    if (!r) r = launch_pw(m, PW_FILL, D(s->L[c]), nullptr, 0.0);
    if (!r) r = launch_pw(m, PW_FILL, D(s->F[c]), nullptr, 0.0);
  }
  if (!r) r = advect_U_convection1(s);
  for (int c = 0; c < 3 && !r; c++) r = launch_pw(m, PW_ADD_PRODUCT, D(s->F[c]), &D(s->tF3[c]), P.scale_advection_U);
  if (!r && P.scale_diffusion_U != 0.0) {
    for (int c = 0; c < 3 && !r; c++) {
      r = launch_del(m, D(s->tF1[c]), D(s->U[c]), 2, 1, 0, 1);
      if (!r) r = launch_del(m, D(s->tF1[c]), D(s->U[c]), 2, 2, 0, 2);
      if (!r) r = launch_del(m, D(s->tF1[c]), D(s->U[c]), 2, 3, 0, 2);
      if (!r) r = launch_pw(m, PW_ADD_PRODUCT, D(s->F[c]), &D(s->tF1[c]), P.scale_diffusion_U);
    }
  }
  if (!r && P.scale_diffusion_linear_U != 0.0) {  // diffusion_linear: compute_add_diffusion(L, ...)
    for (int c = 0; c < 3 && !r; c++) {
      r = launch_del(m, D(s->tF1[c]), D(s->U[c]), 2, 1, 0, 1);
      if (!r) r = launch_del(m, D(s->tF1[c]), D(s->U[c]), 2, 2, 0, 2);
      if (!r) r = launch_del(m, D(s->tF1[c]), D(s->U[c]), 2, 3, 0, 2);
      if (!r) r = launch_pw(m, PW_ADD_PRODUCT, D(s->L[c]), &D(s->tF1[c]), P.scale_diffusion_linear_U);
    }
  }
  if (!r && P.induction != MOONS_IND_OFF) {
    for (int c = 0; c < 3 && !r; c++) {
      if (s->same) r = copy(m, s->tF1[c], s->jxb[c]);
      else r = embed_extract(m, s->tF1[c], s->jxb[c], P.ind_offset, false);
      if (!r) r = mask_ghost_XPeriodic(m, D(s->tF1[c]), nullptr);
      if (!r) r = launch_pw(m, PW_ADD_PRODUCT, D(s->F[c]), &D(s->tF1[c]), 1.0);
    }
  }
  if (!r && P.energy && P.scale_buoyancy != 0.0) r = add_buoyancy(s);
  if (r) return r;
  // ---- solve_momentum (solve_method 1 to 9)
  r = time_scheme_step(s, m, s->pcgU, s->pcgP, P.isp_U, P.isp_p, s->U, s->Ustar, s->Unm1, s->p, s->F, s->Fnm1, s->L, s->tF1,
                s->tCC, P.coeff_implicit_U, &s->coefU, 0, 1, &s->res_p, time_method(P.solve_method_U), rk);
  if (r) return r;
  for (int c = 0; c < 3 && !r; c++) r = launch_interp(m, D(s->UCC[c]), D(s->U[c]), c + 1);
  if (!r) r = face2edge_nd(m, s->UE, s->U);
  if (r) return r;
  // ---- induction
  moons_mesh* mi = s->mi;
  if (P.induction == MOONS_IND_B) {
    for (int c = 0; c < 3 && !r; c++) {
      r = copy(mi, s->Fnm1i[c], s->Fi[c]);
      if (!r) r = launch_pw(mi, PW_FILL, D(s->Li[c]), nullptr, 0.0);
      if (!r) r = launch_pw(mi, PW_FILL, D(s->Fi[c]), nullptr, 0.0);
    }
    for (int c = 0; c < 3 && !r; c++)
      for (int l = 0; l < 3 && !r; l++)
        if (c != l) {
          if (s->same) r = copy(mi, s->UEi[c][l], s->UE[c][l]);
          else r = embed_extract(mi, s->UEi[c][l], s->UE[c][l], P.ind_offset, true);
        }
    if (!r) r = face2edge_nd(mi, s->BE, s->Btot);
    if (!r) r = launch_cross3(mi, s->tE, s->UEi, s->BE);
    if (!r) r = curl3(mi, s->curlUxB, s->tE);
    for (int c = 0; c < 3 && !r; c++)
      r = launch_pw(mi, PW_ADD_PRODUCT, D(s->Fi[c]), &D(s->curlUxB[c]), P.scale_advection_B);
    if (!r && P.scale_diffusion_linear_B != 0.0) {  // diffusion_linear: add_curl_J(L, ...)
      for (int c = 0; c < 3 && !r; c++) {
        r = copy(mi, s->tE[c], s->J[c]);
        if (!r) r = launch_pw(mi, PW_MUL, D(s->tE[c]), &D(s->sig[c]), 0.0);
      }
      if (!r) r = curl3(mi, s->tFi2, s->tE);
      for (int c = 0; c < 3 && !r; c++)
        r = launch_pw(mi, PW_ADD_PRODUCT, D(s->Li[c]), &D(s->tFi2[c]), P.scale_diffusion_linear_B);
    }
    if (!r && P.scale_diffusion_B != 0.0) {
      for (int c = 0; c < 3 && !r; c++) {
        r = copy(mi, s->tE[c], s->J[c]);
        if (!r) r = launch_pw(mi, PW_MUL, D(s->tE[c]), &D(s->sig[c]), 0.0);
      }
      if (!r) r = curl3(mi, s->tFi2, s->tE);
      for (int c = 0; c < 3 && !r; c++)
        r = launch_pw(mi, PW_ADD_PRODUCT, D(s->Fi[c]), &D(s->tFi2[c]), P.scale_diffusion_B);
    }
    if (r) return r;
    r = time_scheme_step(s, mi, s->pcgB, s->pcgPhi, P.isp_B, P.isp_phi, s->B, s->Bstar, s->Bnm1, s->phi, s->Fi, s->Fnm1i,
                  s->Li, s->tFi1, s->tCCi, P.coeff_implicit_B, &s->coefB, 2, 3, &s->res_phi,
                  time_method(P.solve_method_B), rk);
    if (!r) r = compute_J(s);
    if (!r) r = compute_Btot(s);
    if (!r) r = compute_JxB(s);
  } else if (P.induction == MOONS_IND_POTENTIAL) {
    r = compute_Btot(s);
    if (!r) r = potential_solve(s);
    if (!r) r = compute_JxB(s);
  }
  return r;
}

}  // namespace

extern "C" {

int moons_mhd_create(moons_mesh* mm, moons_mesh* mi, const moons_mhd_params* prm, moons_mhd** out) {
  if (!mm || !mi || !prm || !out) {
    set_error("moons_mhd_create: null pointer");
    return MOONS_ERR_ARG;
  }
  if (mm->device != mi->device) {
    set_error("moons_mhd_create: meshes on different devices");
    return MOONS_ERR_ARG;
  }
  if (prm->induction < MOONS_IND_OFF || prm->induction > MOONS_IND_POTENTIAL || !(prm->dt > 0)) {
    set_error("moons_mhd_create: bad induction mode or dt");
    return MOONS_ERR_ARG;
  }
  if (prm->energy && (prm->solve_method_T < 1 || prm->solve_method_T > 5)) {
    set_error("moons_mhd_create: solve_method_T must be 1 to 5");
    return MOONS_ERR_ARG;
  }
  if (!time_method_ok(prm->solve_method_U) || !time_method_ok(prm->solve_method_B)) {
    set_error("moons_mhd_create: solve_method_U and solve_method_B must be 0 to 9");
    return MOONS_ERR_ARG;
  }
  {
    const int pq = prm->prec_poisson;  // the Poisson solvers the step can use
    if (!(pq == 0 || pq == MOONS_PREC_LAP || pq == MOONS_PREC_MG || pq == MOONS_PREC_MG_MIXED ||
          pq == MOONS_PREC_FD || pq == MOONS_PREC_UNET_MG)) {
      set_error("moons_mhd_create: prec_poisson must be 0, LAP, MG, MG_MIXED, FD or UNET_MG");
      return MOONS_ERR_ARG;
    }
  }
  if (prm->rk_stages != 0 && prm->rk_stages != 1 && prm->rk_stages != 3) {
    set_error("moons_mhd_create: rk_stages must be 0, 1 or 3");
    return MOONS_ERR_ARG;
  }
  auto* s = new moons_mhd();
  s->mm = mm;
  s->mi = mi;
  mesh_ref(mm);
  mesh_ref(mi);
  s->same = (mm == mi);
  s->P = *prm;
  if (!s->same) {
    for (int d = 0; d < 3; d++)
      if (prm->ind_offset[d] < 0 || mm->sn[d] + prm->ind_offset[d] > mi->sn[d]) {
        mesh_unref(mm);
        mesh_unref(mi);
        delete s;
        set_error("moons_mhd_create: fluid mesh does not fit inside the induction mesh at ind_offset");
        return MOONS_ERR_SHAPE;
      }
    // one stream for both meshes: the induction step reads what the momentum
    // step wrote (embed/extract), so the two must not overlap
    s->mi_stream_saved = mi->stream;
    mi->stream = mm->stream;
  } else {
    for (int d = 0; d < 3; d++) s->P.ind_offset[d] = 0;
  }
  int r = MOONS_OK;
  auto F = [&](moons_mesh* m, int dl, moons_sf** o) {
    if (!r) r = mk(s, m, dl, o);
  };
  for (int c = 0; c < 3; c++) {
    for (moons_sf** f : {&s->U[c], &s->Ustar[c], &s->Unm1[c], &s->F[c], &s->Fnm1[c], &s->L[c], &s->tF1[c], &s->tF2[c],
                         &s->tF3[c]})
      F(mm, MOONS_FX + c, f);
    F(mm, MOONS_CC, &s->UCC[c]);
    for (int l = 0; l < 3; l++) {
      s->UE[c][l] = s->UEi[c][l] = s->BE[c][l] = s->TF1[c][l] = s->TF2[c][l] = nullptr;
      if (c != l) {
        F(mm, MOONS_EX + l, &s->UE[c][l]);
        F(mi, MOONS_EX + l, &s->UEi[c][l]);
        F(mi, MOONS_EX + l, &s->BE[c][l]);
        F(mi, MOONS_FX + l, &s->TF1[c][l]);
        F(mi, MOONS_FX + l, &s->TF2[c][l]);
      }
    }
  }
  F(mm, MOONS_CC, &s->tCC);
  F(mm, MOONS_CC, &s->p);
  F(mm, MOONS_CC, &s->divU);
  bool pot = prm->induction == MOONS_IND_POTENTIAL;
  for (int c = 0; c < 3; c++) {
    for (moons_sf** f : {&s->B[c], &s->Bstar[c], &s->Bnm1[c], &s->B0[c], &s->Btot[c], &s->Fi[c], &s->Fnm1i[c],
                         &s->Li[c], &s->jxb[c], &s->tFi1[c], &s->tFi2[c], &s->curlUxB[c], &s->Ui[c], &s->E[c]})
      F(mi, MOONS_FX + c, f);
    F(mi, pot ? MOONS_FX + c : MOONS_EX + c, &s->J[c]);
    F(mi, pot ? MOONS_FX + c : MOONS_EX + c, &s->sig[c]);
    F(mi, MOONS_EX + c, &s->tE[c]);
  }
  F(mi, MOONS_CC, &s->phi);
  F(mi, MOONS_CC, &s->tCCi);
  F(mi, MOONS_CC, &s->divB);
  if (prm->energy) {
    for (moons_sf** f : {&s->T, &s->Tnm1, &s->FT, &s->FnmT, &s->LT, &s->tCCT, &s->tCCT2, &s->tmpT, &s->sigInvCC,
                         &s->tCCT3})
      F(mi, MOONS_CC, f);
    for (int c = 0; c < 3; c++) {
      F(mi, MOONS_FX + c, &s->kT[c]);
      F(mi, MOONS_CC, &s->grav[c]);
      F(mi, MOONS_FX + c, &s->tFT[c]);
      F(mi, MOONS_FX + c, &s->UFT[c]);
      F(mi, MOONS_CC, &s->UCCn[c]);
      F(mi, MOONS_CC, &s->tVFT[c]);
    }
    if (!r) r = set_bcs_from(s->T, prm->bc_T);
    if (!r && prm->scale_heating_T != 0.0) {
      // add_volumetric_heating_Nuclear (energy_sources.f90:98-114): a = L = 1,
      // m = a/L, F = scale 2m/(1-exp(-2m)), temp(j) = F exp(-m (hc(j)+1))
      const std::vector<double>& hy = mi->hn[1];
      const double a = 1.0, Lh = 1.0, mm_ = a / Lh;
      const double Fh = prm->scale_heating_T * 2.0 * mm_ / (1.0 - std::exp(-2.0 * mm_));
      std::vector<double> prof(hy.size() - 1);
      for (size_t j = 0; j + 1 < hy.size(); j++) prof[j] = Fh * std::exp(-mm_ * (0.5 * (hy[j] + hy[j + 1]) + 1.0));
      if (cudaMalloc((void**)&s->heat_prof, prof.size() * sizeof(double)) != cudaSuccess) r = MOONS_ERR_NOMEM;
      else if (cudaMemcpy(s->heat_prof, prof.data(), prof.size() * sizeof(double), cudaMemcpyHostToDevice) !=
               cudaSuccess)
        r = MOONS_ERR_CUDA;
    }
  }
  // BCs
  for (int c = 0; c < 3 && !r; c++) {
    r = set_bcs_from(s->U[c], prm->bc_U[c]);
    if (!r) {
      s->Ustar[c]->bc = s->U[c]->bc;
      if (prm->prescribed_Ustar)
        for (int f = 1; f <= 6; f++) {
          int d = (f + 1) / 2;
          int sz = D(s->U[c]).s(d);
          bool many = n_along(D(s->U[c]).dl, d) ? sz > 4 : sz > 3;
          if (many) s->Ustar[c]->bc.prescribed[f] = 1;
        }
    }
  }
  if (!r) r = set_bcs_from(s->p, prm->bc_p);
  if (!r && prm->induction != MOONS_IND_OFF) {
    for (int c = 0; c < 3 && !r; c++) {
      r = set_bcs_from(s->B[c], prm->bc_B[c]);
      if (!r) {
        s->Bstar[c]->bc = s->B[c]->bc;
        for (int f = 1; f <= 6; f++) {
          s->Bstar[c]->bc.value[f] = 0.0;  // set_BCs_homogeneous
          int d = (f + 1) / 2;
          int sz = D(s->B[c]).s(d);
          bool many = n_along(D(s->B[c]).dl, d) ? sz > 4 : sz > 3;
          if (prm->prescribed_Bstar && many) s->Bstar[c]->bc.prescribed[f] = 1;
        }
      }
    }
    if (!r) r = set_bcs_from(s->phi, prm->bc_phi);
  }
  if (!r && cudaMalloc((void**)&s->d_red, 2 * sizeof(double)) != cudaSuccess) r = MOONS_ERR_NOMEM;
  if (r) {
    moons_mhd_destroy(s);
    return r;
  }
  *out = s;
  return MOONS_OK;
}

int moons_mhd_destroy(moons_mhd* s) {
  if (!s) return MOONS_OK;
  for (moons_pcg* p : {s->pcgU, s->pcgP, s->pcgB, s->pcgPhi, s->pcgT})
    if (p) moons_pcg_destroy(p);
  for (moons_sf* f : s->owned) moons_sf_destroy(f);
  if (s->d_red) cudaFree(s->d_red);
  if (s->heat_prof) cudaFree(s->heat_prof);
  if (s->mi_stream_saved) s->mi->stream = s->mi_stream_saved;
  moons_mesh *mm = s->mm, *mi = s->mi;
  delete s;
  mesh_unref(mm);
  mesh_unref(mi);
  return MOONS_OK;
}

int moons_mhd_field(moons_mhd* s, int which, int comp, moons_sf** out) {
  if (!s || !out || comp < 0 || comp > 2) {
    set_error("moons_mhd_field: bad argument");
    return MOONS_ERR_ARG;
  }
  moons_sf* f = nullptr;
  switch (which) {
    case MOONS_MHD_U: f = s->U[comp]; break;
    case MOONS_MHD_P: f = s->p; break;
    case MOONS_MHD_B: f = s->B[comp]; break;
    case MOONS_MHD_B0: f = s->B0[comp]; break;
    case MOONS_MHD_PHI: f = s->phi; break;
    case MOONS_MHD_J: f = s->J[comp]; break;
    case MOONS_MHD_SIGMA_INV: f = s->sig[comp]; break;
    case MOONS_MHD_JXB: f = s->jxb[comp]; break;
    case MOONS_MHD_DIVU: f = s->divU; break;
    case MOONS_MHD_DIVB: f = s->divB; break;
    case MOONS_MHD_T: f = s->T; break;
    case MOONS_MHD_KT: f = s->kT[comp]; break;
    case MOONS_MHD_GRAVITY: f = s->grav[comp]; break;
    case MOONS_MHD_SIGMA_INV_CC: f = s->sigInvCC; break;
    case MOONS_MHD_U_CC: f = s->UCCn[comp]; break;
    default:
      set_error("moons_mhd_field: unknown field");
      return MOONS_ERR_ARG;
  }
  *out = f;
  return MOONS_OK;
}

int moons_mhd_init(moons_mhd* s) {
  if (!s) {
    set_error("null mhd");
    return MOONS_ERR_ARG;
  }
  moons_mesh* m = s->mm;
  cudaSetDevice(m->device);
  int r = launch_bcs(m, D(s->p), s->p->bc, false);
  for (int c = 0; c < 3 && !r; c++) {
    r = launch_bcs(m, D(s->U[c]), s->U[c]->bc, false);
    if (!r) r = copy(m, s->Unm1[c], s->U[c]);
    if (!r) r = copy(m, s->Ustar[c], s->U[c]);
  }
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  // solvers (init_mom :160-169, init_induction :203-215)
  if (!s->pcgU) {
    moons_sf* xbu[3] = {s->U[0], s->U[1], s->U[2]};
    if ((r = moons_pcg_create(m, MOONS_OP_MOM_DIFFUSION, MOONS_PREC_MOM, 3, s->Ustar, xbu, nullptr, &s->pcgU))) return r;
    moons_sf* xp[1] = {s->p};
    const int pq = s->P.prec_poisson;
    const int pp = pq == MOONS_PREC_MG || pq == MOONS_PREC_MG_MIXED || pq == MOONS_PREC_FD ||
                           pq == MOONS_PREC_UNET_MG
                       ? pq
                       : MOONS_PREC_LAP;
    // the sigma-weighted potential solve is not separable (multigrid under
    // FD), and the networks are trained for the constant-coefficient solves
    const int pv = pp == MOONS_PREC_FD || pp == MOONS_PREC_UNET_MG ? MOONS_PREC_MG_MIXED : pp;
    const int ppU = s->P.solve_method_U == 9 ? MOONS_PREC_FD : pp;  // FFT_P of solve_method 9
    if ((r = moons_pcg_create(m, MOONS_OP_LAP_UNIFORM, ppU, 1, xp, xp, nullptr, &s->pcgP))) return r;
    if (ppU == MOONS_PREC_UNET_MG && s->unet[0] && (r = moons_pcg_set_unet(s->pcgP, s->unet[0]))) return r;
    if (s->P.induction == MOONS_IND_B) {
      if ((r = moons_pcg_create(s->mi, MOONS_OP_IND_DIFFUSION, MOONS_PREC_IND, 3, s->Bstar, s->B, s->sig, &s->pcgB)))
        return r;
      moons_sf* xf[1] = {s->phi};
      const int ppB = s->P.solve_method_B == 9 ? MOONS_PREC_FD : pp;  // FFT_cleanB of solve_method 9
      if ((r = moons_pcg_create(s->mi, MOONS_OP_LAP_UNIFORM, ppB, 1, xf, xf, nullptr, &s->pcgPhi))) return r;
      if (ppB == MOONS_PREC_UNET_MG && s->unet[1] && (r = moons_pcg_set_unet(s->pcgPhi, s->unet[1]))) return r;
    } else if (s->P.induction == MOONS_IND_POTENTIAL) {
      moons_sf* xf[1] = {s->phi};
      if ((r = moons_pcg_create(s->mi, MOONS_OP_LAP_PROPS, pv, 1, xf, xf, s->sig, &s->pcgPhi))) return r;
    }
    if (s->P.energy && s->P.solve_method_T >= 3) {
      // init(nrg%PCG_T, nrg_diffusion, nrg_diffusion_explicit, prec_lap_SF, ...) (energy_extend.f90:129)
      moons_sf* xt[1] = {s->T};
      if ((r = moons_pcg_create(s->mi, MOONS_OP_NRG_DIFFUSION, MOONS_PREC_LAP, 1, xt, xt, s->kT, &s->pcgT))) return r;
    }
  }
  if (s->P.energy) {  // init_energy tail (energy_extend.f90:119-120): apply_BCs(T); Tnm1 = T
    r = launch_bcs(s->mi, D(s->T), s->T->bc, false);
    if (!r) r = copy(s->mi, s->Tnm1, s->T);
    if (r) return r;
  }
  moons_mesh* mi = s->mi;
  if (s->P.induction == MOONS_IND_B) {
    for (int c = 0; c < 3 && !r; c++) {
      r = copy(mi, s->Bnm1[c], s->B[c]);
      if (!r) r = launch_bcs(mi, D(s->B[c]), s->B[c]->bc, false);
      if (!r) r = copy(mi, s->Bstar[c], s->B[c]);
    }
    if (!r) r = compute_J(s);
    if (!r) r = compute_Btot(s);
    if (!r) r = compute_JxB(s);
    if (!r) r = compute_J(s);
  }
  for (int c = 0; c < 3 && !r; c++) r = launch_interp(m, D(s->UCC[c]), D(s->U[c]), c + 1);
  if (!r) r = face2edge_nd(m, s->UE, s->U);
  if (!r && s->P.induction == MOONS_IND_POTENTIAL) {
    r = compute_Btot(s);
    if (!r) r = potential_solve(s);
    if (!r) r = compute_JxB(s);
  }
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  if (mi != m) MG_CUDA(cudaStreamSynchronize(mi->stream));
  return MOONS_OK;
}

int moons_mhd_step(moons_mhd* s, int nsteps, moons_step_info* info) {
  if (!s || nsteps < 0) {
    set_error("moons_mhd_step: bad argument");
    return MOONS_ERR_ARG;
  }
  if (!s->pcgU) {
    set_error("moons_mhd_step: call moons_mhd_init first");
    return MOONS_ERR_STATE;
  }
  moons_mesh* m = s->mm;
  cudaSetDevice(m->device);
  for (int k = 0; k < 5; k++) s->iters[k] = 0;
  moons_pcg* solvers[5] = {s->pcgU, s->pcgP, s->pcgB, s->pcgPhi, s->pcgT};
  for (moons_pcg* p : solvers)
    if (p) mg_pcg_clear_totals(p);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, m->stream);
  int r = MOONS_OK;
  const int stages = s->P.rk_stages == 3 ? 3 : 1;
  for (int n = 0; n < nsteps && !r; n++)
    for (int st = 1; st <= stages && !r; st++) r = step_once(s, rk_stage(stages, st));
  cudaEventRecord(e1, m->stream);
  cudaError_t e = cudaStreamSynchronize(m->stream);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (r) return r;
  MG_CUDA(e);
  int nan = 0;
  for (int k = 0; k < 5; k++) {
    if (!solvers[k]) continue;
    int it = 0, na = 0;
    double rel = 0;
    if ((r = mg_pcg_totals(solvers[k], &it, &na, &rel))) return r;
    s->iters[k] = it;
    nan |= na;
    if (k == 1) s->res_p = rel;
    if (k == 3) s->res_phi = rel;
  }
  if (nan) {
    set_error("moons_mhd_step: NaN in a solver's residual norms");
    return MOONS_ERR_NAN;
  }
  if (info) {
    info->steps = nsteps;
    info->iters_U = s->iters[0];
    info->iters_p = s->iters[1];
    info->iters_B = s->iters[2];
    info->iters_phi = s->iters[3];
    info->iters_T = s->iters[4];
    info->res_p = s->res_p;
    info->res_phi = s->res_phi;
    info->ms = ms;
  }
  return MOONS_OK;
}

int moons_clean_div(moons_pcg* p, moons_sf* const* X, moons_sf* const* Xstar, moons_sf* phi, double scale,
                    moons_sf* const* temp_F, moons_sf* temp_CC, const moons_isp* isp, moons_solve_info* info) {
  if (!p || !X || !Xstar || !phi || !temp_F || !temp_CC || !isp || !(scale != 0.0)) {
    set_error("moons_clean_div: null argument or zero scale");
    return MOONS_ERR_ARG;
  }
  moons_mesh* m = mg::pcg_mesh(p);
  for (int k = 0; k < 3; k++) {
    const int dl = k == 0 ? MOONS_FX : (k == 1 ? MOONS_FY : MOONS_FZ);
    if (!X[k] || !Xstar[k] || !temp_F[k] || D(X[k]).dl != dl || D(Xstar[k]).dl != dl || D(temp_F[k]).dl != dl) {
      set_error("moons_clean_div: X, Xstar and temp_F must be x, y, z face fields");
      return MOONS_ERR_SHAPE;
    }
  }
  if (D(phi).dl != MOONS_CC || D(temp_CC).dl != MOONS_CC) {
    set_error("moons_clean_div: phi and temp_CC must be cell-centred");
    return MOONS_ERR_SHAPE;
  }
  cudaSetDevice(m->device);
  // div(temp_CC, Xstar) ; temp_CC *= scale ; solve(PCG, phi, temp_CC)
  int r = div3(m, temp_CC, Xstar);
  if (!r) r = launch_pw(m, PW_SCALE, D(temp_CC), nullptr, scale);
  if (r) return r;
  moons_sf* xp[1] = {phi};
  moons_sf* bp[1] = {temp_CC};
  if ((r = moons_pcg_solve(p, xp, bp, isp, info))) return r;
  // grad(temp_F, phi) ; temp_F *= 1/scale ; X = Xstar - temp_F ; apply_BCs(X)
  if ((r = grad3(m, temp_F, phi))) return r;
  for (int k = 0; k < 3; k++) {
    MG_LAUNCH(k_project, nblocks(D(X[k]).n()), kBlock, m->stream, D(X[k]), D(Xstar[k]), D(temp_F[k]), 1.0 / scale);
    if ((r = launch_bcs(m, D(X[k]), X[k]->bc, false))) return r;
  }
  MG_CUDA(cudaGetLastError());
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_mhd_set_unet(moons_mhd* s, int which, moons_unet* u) {
  if (!s || !u || which < 0 || which > 1) {
    set_error("moons_mhd_set_unet: bad argument");
    return MOONS_ERR_ARG;
  }
  if (s->P.prec_poisson != MOONS_PREC_UNET_MG) {
    set_error("moons_mhd_set_unet: prec_poisson is not MOONS_PREC_UNET_MG");
    return MOONS_ERR_STATE;
  }
  if (unet_mesh(u) != (which == 0 ? s->mm : s->mi)) {
    set_error("moons_mhd_set_unet: the network lives on another mesh");
    return MOONS_ERR_SHAPE;
  }
  s->unet[which] = u;
  moons_pcg* p = which == 0 ? s->pcgP : s->pcgPhi;
  if (p && !(which == 1 && s->P.induction != MOONS_IND_B)) return moons_pcg_set_unet(p, u);
  return MOONS_OK;
}

int moons_mhd_divergence(moons_mhd* s, double* du, double* db) {
  if (!s || !du || !db) {
    set_error("moons_mhd_divergence: null pointer");
    return MOONS_ERR_ARG;
  }
  moons_mesh* m = s->mm;
  int r = div3(m, s->divU, s->U);
  if (r) return r;
  MG_LAUNCH(k_sumsq, std::min<unsigned>(kRedBlocks, nblocks(D(s->divU).n())), kBlock, m->stream, 
      D(s->divU), m->d_partial, m->d_ticket, s->d_red);
  MG_CUDA(cudaStreamSynchronize(m->stream));
  double h[2] = {0, 0};
  if (s->P.induction == MOONS_IND_B) {
    moons_mesh* mi = s->mi;
    if ((r = div3(mi, s->divB, s->B))) return r;
    MG_LAUNCH(k_sumsq, std::min<unsigned>(kRedBlocks, nblocks(D(s->divB).n())), kBlock, mi->stream, 
        D(s->divB), mi->d_partial, mi->d_ticket, s->d_red + 1);
    MG_CUDA(cudaStreamSynchronize(mi->stream));
  } else {
    MG_CUDA(cudaMemsetAsync(s->d_red + 1, 0, sizeof(double), m->stream));
  }
  MG_CUDA(cudaMemcpy(h, s->d_red, 2 * sizeof(double), cudaMemcpyDeviceToHost));
  *du = h[0];
  *db = h[1];
  return MOONS_OK;
}

}  // extern "C"
