// moons_oracle_mhd.cpp -- CPU restatement of one MOONS MHD time step
// (TEST ORACLE; see moons_oracle.hpp).
//
// HW/MOONS/MOONS_solver.f90:47-144 with one RK stage:
//   add_all_momentum_sources  (HW/solvers/momentum/add_all_momentum_sources.f90:22-86)
//   solve_momentum, method 6  (HW/governing_equations/momentum_extend.f90:326-374,
//                              HW/solvers/time_marching_methods.f90:117-150,
//                              HW/solvers/clean_divergence.f90:37-59)
//   add_all_induction_sources (HW/solvers/induction/add_all_induction_sources.f90:24-60)
//   solve_induction, method 6 (HW/governing_equations/induction_extend.f90:475-525)
// and the low-Rem electric-potential form (new; composed of reference ops).
#include <cstring>

#include "../include/moons_gpu.h"
#include "moons_oracle.hpp"

namespace mo {

void set_bcs_spec(SF& u, const Grid& g, const moons_bc_spec& b) {
  set_bcs(u, g, b.type, b.prescribed, b.value, b.c_w, b.order);
  u.bc->all_neumann = b.all_neumann != 0;
}

static int dl_face(int c) { return 1 + c; }  // FX,FY,FZ
static int dl_edge(int c) { return 4 + c; }  // EX,EY,EZ

// pointwise helpers
static void cross_x(SF& o, const SF& Ay, const SF& Az, const SF& By, const SF& Bz) {  // GF_cross_product.f90:17-33
  for (size_t i = 0; i < o.n(); i++) o.f[i] = Ay.f[i] * Bz.f[i] - Az.f[i] * By.f[i];
}
static void cross_y(SF& o, const SF& Ax, const SF& Az, const SF& Bx, const SF& Bz) {
  for (size_t i = 0; i < o.n(); i++) o.f[i] = -(Ax.f[i] * Bz.f[i] - Az.f[i] * Bx.f[i]);
}
static void cross_z(SF& o, const SF& Ax, const SF& Ay, const SF& Bx, const SF& By) {
  for (size_t i = 0; i < o.n(); i++) o.f[i] = Ax.f[i] * By.f[i] - Ay.f[i] * Bx.f[i];
}

struct TF {  // off-diagonal tensor field: t[c][loc], c != loc
  SF t[3][3];
  void init(const Grid& g, bool edges) {
    for (int c = 0; c < 3; c++)
      for (int l = 0; l < 3; l++)
        if (c != l) t[c][l].init(g, edges ? dl_edge(l) : dl_face(l));
  }
};

// cross_product_TF (HW/fields/TF_extend.f90:385-401)
static void cross_TF(SF* o, const TF& A, const TF& B) {
  cross_x(o[0], A.t[1][0], A.t[2][0], B.t[1][0], B.t[2][0]);
  cross_y(o[1], A.t[0][1], A.t[2][1], B.t[0][1], B.t[2][1]);
  cross_z(o[2], A.t[0][2], A.t[1][2], B.t[0][2], B.t[1][2]);
}

static int orth(int a, int b) { return 6 - a - b; }  // 1-based dirs

// face2Edge_TF_no_diag (ops_interp.f90:531-544)
static void face2edge_nd(TF& E, SF* const* F, const Grid& g) {
  for (int c = 0; c < 3; c++)
    for (int l = 0; l < 3; l++)
      if (c != l) interp(E.t[c][l], *F[c], g, orth(c + 1, l + 1));
}
// edge2Face_no_diag_TF (ops_interp.f90:698-709)
static void edge2face_nd(TF& Fo, SF* const* E, const Grid& g) {
  for (int c = 0; c < 3; c++)
    for (int l = 0; l < 3; l++)
      if (c != l) interp(Fo.t[c][l], *E[c], g, orth(c + 1, l + 1));
}
// face2Face_no_diag_TF (ops_interp.f90:496-510): face2CellCenter then cellCenter2Face
static void face2face_nd(TF& Fo, SF* const* F, const Grid& g, SF& tCC) {
  for (int c = 0; c < 3; c++)
    for (int l = 0; l < 3; l++)
      if (c != l) {
        interp(tCC, *F[c], g, c + 1);
        interp(Fo.t[c][l], tCC, g, l + 1);
      }
}

// physical region of a field (interior cells, boundary nodes; no ghosts) and
// its copy between the fluid mesh and the induction mesh (offset o).
// embed: ind <- mom ; extract: mom <- ind (ops_embedExtract.f90)
static void embed_extract(SF& dst, const SF& src, const int o[3], bool embed) {
  const SF& mom = embed ? src : dst;
  for (int k = 2; k <= mom.s[3] - 1; k++)
    for (int j = 2; j <= mom.s[2] - 1; j++)
      for (int i = 2; i <= mom.s[1] - 1; i++) {
        if (embed) dst(i + o[0], j + o[1], k + o[2]) = src(i, j, k);
        else dst(i, j, k) = src(i + o[0], j + o[1], k + o[2]);
      }
}

// RK_Params of one stage (init_RKP, RK_params_extend.f90:22-55): the
// three-stage coefficients of Lundbladh et al. (1999), or all 1 when the
// step has one stage (RK inactive); beta = alpha
struct RKStage {
  double gamma, zeta, alpha, beta;
};
// solve_method 0 is the default, 6; 9 runs 6 (the direct cleaning solve is
// a solver choice, not a different arithmetic of the step)
inline int time_method(int m) { return m == 0 || m == 9 ? 6 : m; }
inline RKStage rk_stage(int stages, int n) {
  if (stages != 3) return {1.0, 1.0, 1.0, 1.0};
  const double g[3] = {8.0 / 15.0, 5.0 / 12.0, 3.0 / 4.0};
  const double z[3] = {0.0, -17.0 / 60.0, -5.0 / 12.0};
  const double a[3] = {4.0 / 15.0, 1.0 / 15.0, 1.0 / 6.0};
  return {g[n - 1], z[n - 1], a[n - 1], a[n - 1]};
}

struct MHD {
  Grid gm, gi;
  bool same = true;
  int off[3] = {0, 0, 0};
  moons_mhd_params P{};
  // momentum
  SF U[3], Ustar[3], Unm1[3], F[3], Fnm1[3], L[3], tF1[3], tF2[3], tF3[3], tCC, p, UCC[3], divU;
  TF UE;
  PCG pcgU, pcgP;
  ISP ispU, ispP;
  // induction
  SF B[3], Bstar[3], Bnm1[3], B0[3], Btot[3], Fi[3], Fnm1i[3], Li[3], J[3], jxb[3], sig[3], phi, tCCi, tFi1[3],
      tFi2[3], tE[3], curlUxB[3], divB;
  TF UEi, BE, TF1, TF2;
  PCG pcgB, pcgPhi;
  ISP ispB, ispPhi;
  // energy (on the induction mesh)
  SF T, Tnm1, FT, FnmT, LT, tCCT, tCCT2, tmpT, kT[3], grav[3], tFT[3], UFT[3];
  // nrg%U_CC, ind%sigmaInv_CC, nrg%temp_CC2, nrg%temp_CC1_VF
  SF UCCn[3], sigInvCC, tCCT3, tVFT[3];
  PCG pcgT;
  ISP ispT;
  bool pcgT_made = false;
  int iters[5] = {0, 0, 0, 0, 0};
  double res_p = 0, res_phi = 0;
  int n_step = 0;  // TMP%n_step: steps taken (time_marching_params_extend.f90:43,59)

  void create(const Grid& gmom, const Grid& gind, const moons_mhd_params& prm) {
    gm = gmom;
    gi = gind;
    P = prm;
    for (int d = 0; d < 3; d++) off[d] = prm.ind_offset[d];
    for (int c = 0; c < 3; c++) {
      for (SF* f : {&U[c], &Ustar[c], &Unm1[c], &F[c], &Fnm1[c], &L[c], &tF1[c], &tF2[c], &tF3[c]})
        f->init(gm, dl_face(c));
      UCC[c].init(gm, 0);
    }
    tCC.init(gm, 0);
    p.init(gm, 0);
    divU.init(gm, 0);
    UE.init(gm, true);
    for (int c = 0; c < 3; c++) {
      set_bcs_spec(U[c], gm, P.bc_U[c]);
      // init(Ustar,U) copies BCs; set_prescribed_BCs when SS%prescribed_BCs
      auto sb = std::make_shared<BCs>(*U[c].bc);
      if (P.prescribed_Ustar)
        for (int f = 1; f <= 6; f++)
          if (sb->many_cell[(f + 1) / 2]) sb->prescribed[f] = 1;
      Ustar[c].bc = sb;
    }
    set_bcs_spec(p, gm, P.bc_p);
    const Grid& g = gi;
    for (int c = 0; c < 3; c++) {
      for (SF* f : {&B[c], &Bstar[c], &Bnm1[c], &B0[c], &Btot[c], &Fi[c], &Fnm1i[c], &Li[c], &jxb[c], &tFi1[c],
                    &tFi2[c], &curlUxB[c]})
        f->init(g, dl_face(c));
      if (P.induction == MOONS_IND_POTENTIAL) {
        J[c].init(g, dl_face(c));
        sig[c].init(g, dl_face(c));
      } else {
        J[c].init(g, dl_edge(c));
        sig[c].init(g, dl_edge(c));
      }
      tE[c].init(g, dl_edge(c));
    }
    phi.init(g, 0);
    tCCi.init(g, 0);
    divB.init(g, 0);
    UEi.init(g, true);
    BE.init(g, true);
    TF1.init(g, false);
    TF2.init(g, false);
    if (P.induction != MOONS_IND_OFF) {
      for (int c = 0; c < 3; c++) {
        set_bcs_spec(B[c], g, P.bc_B[c]);
        // Bstar: init(Bstar,B) + set_BCs_homogeneous (induction_extend.f90:171-174)
        auto hb = std::make_shared<BCs>(*B[c].bc);
        for (int f = 1; f <= 6; f++) {
          hb->value[f] = 0.0;
          if (P.prescribed_Bstar && hb->many_cell[(f + 1) / 2]) hb->prescribed[f] = 1;
        }
        Bstar[c].bc = hb;
      }
      set_bcs_spec(phi, g, P.bc_phi);
    }
    if (P.energy) {
      for (SF* f : {&T, &Tnm1, &FT, &FnmT, &LT, &tCCT, &tCCT2, &tmpT, &sigInvCC, &tCCT3}) f->init(g, 0);
      for (int c = 0; c < 3; c++) {
        UCCn[c].init(g, 0);
        tVFT[c].init(g, 0);
      }
      for (int c = 0; c < 3; c++) {
        kT[c].init(g, dl_face(c));
        grav[c].init(g, 0);
        tFT[c].init(g, dl_face(c));
        UFT[c].init(g, dl_face(c));
      }
      set_bcs_spec(T, g, P.bc_T);
    }
    for (auto* I : {&ispU, &ispP, &ispB, &ispPhi, &ispT}) *I = ISP();
    auto cp = [](ISP& d, const moons_isp& s) {
      d.iter_max = s.iter_max;
      d.tol_rel = s.tol_rel;
      d.tol_abs = s.tol_abs;
      d.n_skip_check_res = s.n_skip_check_res;
    };
    cp(ispU, P.isp_U);
    cp(ispP, P.isp_p);
    cp(ispB, P.isp_B);
    cp(ispPhi, P.isp_phi);
    cp(ispT, P.isp_T);
  }

  void make_solvers() {
    SF* xu[3] = {&Ustar[0], &Ustar[1], &Ustar[2]};
    SF* xbu[3] = {&U[0], &U[1], &U[2]};
    pcgU.init(gm, OP_MOM_DIFFUSION, PREC_MOM, 3, xu, xbu, nullptr, P.coeff_implicit_U);
    SF* xp[1] = {&p};
    pcgP.init(gm, OP_LAP_UNIFORM, PREC_LAP, 1, xp, xp, nullptr, 0.0);
    if (P.induction == MOONS_IND_B) {
      SF* xb[3] = {&Bstar[0], &Bstar[1], &Bstar[2]};
      SF* xbb[3] = {&B[0], &B[1], &B[2]};
      SF* ks[3] = {&sig[0], &sig[1], &sig[2]};
      pcgB.init(gi, OP_IND_DIFFUSION, PREC_IND, 3, xb, xbb, ks, P.coeff_implicit_B);
      SF* xf[1] = {&phi};
      pcgPhi.init(gi, OP_LAP_UNIFORM, PREC_LAP, 1, xf, xf, nullptr, 0.0);
    } else if (P.induction == MOONS_IND_POTENTIAL) {
      SF* xf[1] = {&phi};
      SF* ks[3] = {&sig[0], &sig[1], &sig[2]};
      pcgPhi.init(gi, OP_LAP_PROPS, PREC_LAP, 1, xf, xf, ks, 0.0);
    }
    if (P.energy && P.solve_method_T >= 3) {
      // init(nrg%PCG_T, nrg_diffusion, nrg_diffusion_explicit, prec_lap_SF, ...) (energy_extend.f90:129)
      SF* xt[1] = {&T};
      SF* ks[3] = {&kT[0], &kT[1], &kT[2]};
      pcgT.init(gi, OP_NRG_DIFFUSION, PREC_LAP, 1, xt, xt, ks, P.coeff_implicit_T);
      pcgT_made = true;
    }
  }

  // ---- energy: add_all_energy_sources (add_all_energy_sources.f90:21-67),
  // advection / diffusion / volumetric heating (energy_sources.f90), then
  // solve_energy methods 2 and 3 (energy_extend.f90:236-262,
  // time_marching_methods_SF.f90:71-160)
  // add_all_energy_sources + solve_energy (add_all_energy_sources.f90:21-67,
  // energy_extend.f90:236-262) for one stage of the step
  void energy_step(const RKStage& rk) {
    const bool rk_active = P.rk_stages == 3;
    assign(FnmT, FT);
    if (rk_active) assign(LT, 0.0);
    assign(FT, 0.0);
    if (P.scale_advection_T != 0.0) {  // add_advection (energy_sources.f90:22-35)
      for (int c = 0; c < 3; c++) {
        if (same) assign(UFT[c], U[c]);
        else embed_extract(UFT[c], U[c], off, true);
      }
      for (int c = 0; c < 3; c++) {
        interp(tFT[c], T, gi, c + 1);  // cellCenter2Face
        multiply(tFT[c], UFT[c]);
      }
      div(tCCT, tFT[0], tFT[1], tFT[2], gi);
      multiply(tCCT, -1.0);
      add_product(FT, tCCT, P.scale_advection_T);
    }
    if (P.scale_diffusion_T != 0.0) {  // add_diffusion: lap = lapUniformCoeff_SF, into L when RK is active
      lap_uniform_coeff(tCCT, T, gi);
      add_product(rk_active ? LT : FT, tCCT, P.scale_diffusion_T);
    }
    if (P.scale_KE_diffusion_T != 0.0 || P.scale_viscous_dissipation_T != 0.0) {
      // embedCC(nrg%U_CC, mom%U_CC, nrg%MD) (add_all_energy_sources.f90:30-32)
      for (int c = 0; c < 3; c++) {
        if (same) assign(UCCn[c], UCC[c]);
        else embed_extract(UCCn[c], UCC[c], off, true);
      }
    }
    if (P.scale_KE_diffusion_T != 0.0) {  // add_KE_diffusion (energy_sources.f90:51-64)
      for (int c = 0; c < 3; c++) {
        assign(tVFT[c], UCCn[c]);
        multiply(tVFT[c], tVFT[c]);  // square
      }
      // add(temp_CC1, temp_CC_VF): temp_CC1 = x + y + z (GF_add.f90:63-86)
      for (size_t i = 0; i < tCCT.n(); i++) tCCT.f[i] = tVFT[0].f[i] + tVFT[1].f[i] + tVFT[2].f[i];
      lap_uniform_coeff(tCCT3, tCCT, gi);  // lap = lapUniformCoeff_SF
      add_product(FT, tCCT3, P.scale_KE_diffusion_T);
    }
    if (P.scale_viscous_dissipation_T != 0.0) {  // add_viscous_dissipation (energy_sources.f90:66-78)
      // grad_TF (ops_discrete.f90:313-321): g%c%d = d U_CC,c / d x_d, CC -> CC
      SF g[3][3];
      for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) {
          g[c][d].init(gi, 0);
          del(g[c][d], UCCn[c], gi, 1, d + 1, 0, 1);
          multiply(g[c][d], g[c][d]);  // square_TF
        }
      // add_SF_TF (TF_extend.f90:248-255): x%x + y%x + z%x + x%y + ... + z%z
      for (size_t i = 0; i < tCCT.n(); i++)
        tCCT.f[i] = g[0][0].f[i] + g[1][0].f[i] + g[2][0].f[i] + g[0][1].f[i] + g[1][1].f[i] + g[2][1].f[i] +
                    g[0][2].f[i] + g[1][2].f[i] + g[2][2].f[i];
      add_product(FT, tCCT, P.scale_viscous_dissipation_T);
    }
    if (P.scale_joule_heating_T != 0.0) {  // add_joule_heating (energy_sources.f90:80-94)
      // edge2CellCenter_VF (ops_interp.f90:415-431, 688-696); faces in the potential form
      const bool pot = P.induction == MOONS_IND_POTENTIAL;
      for (int c = 0; c < 3; c++) {
        if (pot) {
          interp(tVFT[c], J[c], gi, c + 1);
        } else {
          const int edir = c + 1, fdir = edir == 1 ? 2 : (edir == 2 ? 3 : 1);
          interp(tFT[fdir - 1], J[c], gi, 6 - edir - fdir);  // edge2Face
          interp(tVFT[c], tFT[fdir - 1], gi, fdir);          // face2CellCenter
        }
        multiply(tVFT[c], tVFT[c]);
      }
      for (size_t i = 0; i < tCCT.n(); i++) tCCT.f[i] = tVFT[0].f[i] + tVFT[1].f[i] + tVFT[2].f[i];
      multiply(tCCT, sigInvCC);
      add_product(FT, tCCT, P.scale_joule_heating_T);
    }
    if (P.scale_heating_T != 0.0) {  // add_volumetric_heating_Nuclear (energy_sources.f90:98-114)
      const double a = 1.0, Lh = 1.0, m_ = a / Lh;
      const double Fh = P.scale_heating_T * 2.0 * m_ / (1.0 - std::exp(-2.0 * m_));
      const Coord& cy = gi.c[1];
      for (int k = 1; k <= tCCT.s[3]; k++)
        for (int j = 1; j <= tCCT.s[2]; j++)
          for (int i = 1; i <= tCCT.s[1]; i++) tCCT(i, j, k) = Fh * std::exp(-m_ * (cy.hc(j) + 1.0));
      add_product(FT, tCCT, P.scale_heating_T);
    }
    // the energy time schemes (solve_energy, energy_extend.f90:244-257;
    // time_marching_methods_SF.f90)
    const double two_thirds = 2.0 / 3.0, four_thirds = 4.0 / 3.0, neg_one_third = -1.0 / 3.0;
    const int mT = P.solve_method_T;
    // AB2_SF: temp = Fn*1.5 ; temp += Fnm1*(-0.5)
    auto ab2 = [&]() {
      for (size_t i = 0; i < tmpT.n(); i++) tmpT.f[i] = FT.f[i] * 1.5;
      add_product(tmpT, FnmT, -0.5);
    };
    if (mT == 1) {  // Euler_time_no_diff_Euler_sources_SF (:154-170)
      assign(tmpT, FT);  // multiply(Xstar,F,dt)
      multiply(tmpT, P.dt);
      assign_wall_Dirichlet(tmpT, 0.0, &T);
      add(T, tmpT);
      return;
    }
    if (mT == 2) {  // Euler_time_no_diff_AB2_sources_SF (:135-152)
      ab2();
      multiply(tmpT, P.dt);
      assign_wall_Dirichlet(tmpT, 0.0, &T);
      add(T, tmpT);
      return;
    }
    if (mT == 3) {  // Euler_time_AB2_sources_SF (:71-98)
      ab2();
      multiply(tmpT, P.dt);
      assign_wall_Dirichlet(tmpT, 0.0, &T);
      add(tmpT, T);
      assign(Tnm1, T);
      pcgT.update_MFP(P.dt * 1.0 * P.coeff_implicit_T, n_step <= 2);
    } else if (mT == 4) {  // O2_BDF_time_AB2_sources_SF (:42-69)
      ab2();
      multiply(tmpT, two_thirds * P.dt);
      assign_wall_Dirichlet(tmpT, 0.0, &T);
      add_product(tmpT, T, four_thirds);
      add_product(tmpT, Tnm1, neg_one_third);
      assign(Tnm1, T);
      pcgT.update_MFP(P.dt * two_thirds * P.coeff_implicit_T, n_step <= 2);
    } else {  // Euler_time_RK_sources_SF (:100-133)
      for (size_t i = 0; i < tmpT.n(); i++) tmpT.f[i] = FT.f[i] * (P.dt * rk.gamma);
      add_product(tmpT, FnmT, P.dt * rk.zeta);
      add_product(tmpT, LT, P.dt * rk.alpha);
      assign_wall_Dirichlet(tmpT, 0.0, &T);
      add(tmpT, T);
      assign(Tnm1, T);
      pcgT.update_MFP(P.dt * rk.beta * P.coeff_implicit_T, true);
    }
    SF* xt[1] = {&T};
    SF* bt[1] = {&tmpT};
    SolveInfo si = pcgT.solve(xt, bt, ispT);
    iters[4] += si.iterations;
  }

  // compute_add_buoyancy (momentum_sources.f90:133-150)
  void add_buoyancy() {
    for (int c = 0; c < 3; c++) {
      assign(tCCT2, T);
      multiply(tCCT2, grav[c]);
      interp(tFT[c], tCCT2, gi, c + 1);
      if (same) assign(tF1[c], tFT[c]);
      else embed_extract(tF1[c], tFT[c], off, false);
      add_product(F[c], tF1[c], P.scale_buoyancy);
    }
  }

  // ---- induction helpers
  void compute_J() {  // compute_J (induction_aux.f90:80-88)
    curl(J[0], J[1], J[2], B[0], B[1], B[2], gi);
    for (int c = 0; c < 3; c++) multiply(J[c], P.scale_current);
  }
  void compute_Btot() {  // induction_extend.f90:527-536
    for (int c = 0; c < 3; c++) {
      assign(Btot[c], B0[c]);
      if (P.finite_Rem) add(Btot[c], B[c]);
    }
  }
  void compute_JxB() {  // compute_JCrossB (induction_sources.f90:70-84)
    SF* Jp[3] = {&J[0], &J[1], &J[2]};
    SF* Bp[3] = {&Btot[0], &Btot[1], &Btot[2]};
    if (P.induction == MOONS_IND_B) edge2face_nd(TF1, Jp, gi);
    else face2face_nd(TF1, Jp, gi, tCCi);
    face2face_nd(TF2, Bp, gi, tCCi);
    cross_TF(jxb, TF1, TF2);
    for (int c = 0; c < 3; c++) multiply(jxb[c], P.scale_JxB);
  }
  void embed_UE() {  // embedVelocity_E (induction_aux.f90:135-143)
    for (int c = 0; c < 3; c++)
      for (int l = 0; l < 3; l++)
        if (c != l) {
          if (same) assign(UEi.t[c][l], UE.t[c][l]);
          else embed_extract(UEi.t[c][l], UE.t[c][l], off, true);
        }
  }
  // low-Rem potential: E = u x Btot at faces, div(sigma grad phi) = div(sigma E), J = sigma(E - grad phi)
  void potential_solve() {
    SF Ui[3];
    for (int c = 0; c < 3; c++) {
      Ui[c].init(gi, dl_face(c));
      if (same) assign(Ui[c], U[c]);
      else embed_extract(Ui[c], U[c], off, true);
    }
    SF* Up[3] = {&Ui[0], &Ui[1], &Ui[2]};
    SF* Bp[3] = {&Btot[0], &Btot[1], &Btot[2]};
    face2face_nd(TF1, Up, gi, tCCi);
    face2face_nd(TF2, Bp, gi, tCCi);
    SF E[3];
    for (int c = 0; c < 3; c++) E[c].init(gi, dl_face(c));
    cross_TF(E, TF1, TF2);
    for (int c = 0; c < 3; c++) {
      assign(tFi1[c], E[c]);
      multiply(tFi1[c], sig[c]);
    }
    div(tCCi, tFi1[0], tFi1[1], tFi1[2], gi);
    SF* xf[1] = {&phi};
    SF* bf[1] = {&tCCi};
    SolveInfo si = pcgPhi.solve(xf, bf, ispPhi);
    iters[3] += si.iterations;
    res_phi = si.rel;
    grad(tFi2[0], tFi2[1], tFi2[2], phi, gi);
    for (int c = 0; c < 3; c++) {
      assign(J[c], E[c]);
      subtract(J[c], tFi2[c]);
      multiply(J[c], sig[c]);
    }
  }

  void init() {
    if (P.energy) {  // init_energy tail (energy_extend.f90:119-120)
      apply_BCs(T);
      assign(Tnm1, T);
    }
    // init_mom tail (momentum_extend.f90:139-181)
    apply_BCs(p);
    for (int c = 0; c < 3; c++) {
      apply_BCs(U[c]);
      assign(Unm1[c], U[c]);
      assign(Ustar[c], U[c]);
    }
    make_solvers();
    if (P.induction == MOONS_IND_B) {
      for (int c = 0; c < 3; c++) {
        assign(Bnm1[c], B[c]);
        apply_BCs(B[c]);
        assign(Bstar[c], B[c]);
      }
      compute_J();
      compute_Btot();
      compute_JxB();
    }
    // solve_MOONS start (MOONS_solver.f90:51-53)
    if (P.induction == MOONS_IND_B) compute_J();
    for (int c = 0; c < 3; c++) interp(UCC[c], U[c], gm, c + 1);
    SF* Up[3] = {&U[0], &U[1], &U[2]};
    face2edge_nd(UE, Up, gm);
    if (P.induction == MOONS_IND_POTENTIAL) {
      compute_Btot();
      potential_solve();
      compute_JxB();
    }
  }

  // The time schemes of solve_momentum / solve_induction
  // (momentum_extend.f90:335-367, induction_extend.f90:484-514), selected by
  // solve_method (time_marching_methods.f90):
  //   1 Euler_time_no_diff_Euler_sources_no_correction (:349-366)
  //   2 Euler_time_no_diff_AB2_sources_no_correction (:329-347)
  //   3 Euler_time_no_diff_Euler_sources (:298-327)
  //   4 Euler_time_no_diff_AB2_sources (:266-296)
  //   5 Euler_time_Euler_sources (:47-79)
  //   6 Euler_time_AB2_sources (:117-150)
  //   7 O2_BDF_time_AB2_sources (:81-115)
  //   8 Euler_time_RK_sources (:186-208), with the stage's RK_Params
  //   9 Euler_time_AB2_sources_FFT (:152-185): 6 with clean_div_FFT's direct
  //     solve of the cleaning equation; here that equation is solved by the
  //     PCG of 6 to its tolerance (the caller maps 9 to 6)
  // 3 to 8 end in clean_div_PCG (clean_divergence.f90:37-59).
  void time_scheme_step(PCG& pv, PCG& ps, ISP& iv, ISP& is, SF* X, SF* Xstar, SF* Xnm1, SF& ph, SF* Fn, SF* Fm, SF* Lx,
                 SF* t1, SF& tcc, const Grid& g, double coeff_implicit, int slot_v, int slot_s, double* res_s,
                 int method, const RKStage& rk) {
    const double two_thirds = 2.0 / 3.0, four_thirds = 4.0 / 3.0, neg_one_third = -1.0 / 3.0;
    double dt = P.dt;
    // AB2_VF (AB2.f90:53-64): AB2 = Fn*1.5 ; AB2 += Fnm1*(-0.5)
    auto ab2 = [&](SF& o, int c) {
      for (size_t i = 0; i < o.n(); i++) o.f[i] = Fn[c].f[i] * 1.5;
      add_product(o, Fm[c], -0.5);
    };
    if (method <= 4) {
      for (int c = 0; c < 3; c++) {
        if (method == 1 || method == 3) {
          assign(Xstar[c], Fn[c]);  // multiply(Xstar,F,dt)
          multiply(Xstar[c], dt);
        } else {
          ab2(Xstar[c], c);
          multiply(Xstar[c], dt);
        }
        assign_wall_Dirichlet(Xstar[c], 0.0, &X[c]);
        if (method <= 2) {
          add(X[c], Xstar[c]);
          apply_BCs(X[c]);
        } else {
          add(Xstar[c], X[c]);
          assign(Xnm1[c], X[c]);
        }
      }
      if (method <= 2) return;
    } else {
      for (int c = 0; c < 3; c++) {
        if (method == 5) {
          assign(t1[c], Fn[c]);
          multiply(t1[c], dt);
          assign_wall_Dirichlet(t1[c], 0.0, &X[c]);
          add(t1[c], X[c]);
        } else if (method == 6) {
          ab2(t1[c], c);
          add(t1[c], Lx[c]);
          multiply(t1[c], dt);
          assign_wall_Dirichlet(t1[c], 0.0, &X[c]);
          add(t1[c], X[c]);
        } else if (method == 8) {
          // multiply(temp_F1,F,dt*gamma) ; add_product(temp_F1,Fnm1,dt*zeta) ;
          // add_product(temp_F1,L,dt*2*alpha)
          for (size_t i = 0; i < t1[c].n(); i++) t1[c].f[i] = Fn[c].f[i] * (dt * rk.gamma);
          add_product(t1[c], Fm[c], dt * rk.zeta);
          add_product(t1[c], Lx[c], dt * 2.0 * rk.alpha);
          assign_wall_Dirichlet(t1[c], 0.0, &X[c]);
          add(t1[c], X[c]);
        } else {
          ab2(t1[c], c);
          multiply(t1[c], two_thirds * dt);
          assign_wall_Dirichlet(t1[c], 0.0, &X[c]);
          add_product(t1[c], X[c], four_thirds);
          add_product(t1[c], Xnm1[c], neg_one_third);
        }
        assign(Xnm1[c], X[c]);
      }
      // update_MFP: methods 6 and 8 rebuild the preconditioner every call,
      // methods 5 and 7 while TMP%n_step <= 2
      if (method == 6) pv.update_MFP(dt * 1.0 * coeff_implicit, true);
      else if (method == 8) pv.update_MFP(dt * 2.0 * rk.beta * coeff_implicit, true);
      else if (method == 5) pv.update_MFP(dt * 1.0 * coeff_implicit, n_step <= 2);
      else pv.update_MFP(dt * two_thirds * coeff_implicit, n_step <= 2);
      SF* xs[3] = {&Xstar[0], &Xstar[1], &Xstar[2]};
      SF* bs[3] = {&t1[0], &t1[1], &t1[2]};
      SolveInfo si = pv.solve(xs, bs, iv);
      iters[slot_v] += si.iterations;
    }
    // clean_div_PCG (clean_divergence.f90:37-59), scale = 1/dt for method 6,
    // 1 for the others
    double scale = method == 6 ? 1.0 / dt : 1.0;
    div(tcc, Xstar[0], Xstar[1], Xstar[2], g);
    multiply(tcc, scale);
    SF* xp[1] = {&ph};
    SF* bp[1] = {&tcc};
    SolveInfo sp = ps.solve(xp, bp, is);
    iters[slot_s] += sp.iterations;
    *res_s = sp.rel;
    grad(t1[0], t1[1], t1[2], ph, g);
    for (int c = 0; c < 3; c++) {
      multiply(t1[c], 1.0 / scale);
      // subtract(X,Xstar,temp_F): X = Xstar - temp_F
      for (size_t i = 0; i < X[c].n(); i++) X[c].f[i] = Xstar[c].f[i] - t1[c].f[i];
      apply_BCs(X[c]);
    }
  }

  // solve_MOONS's stage loop (MOONS_solver.f90:73-97): every stage runs the
  // sources and solves of the whole step; TMP%n_step advances once per step
  void step() {
    const int stages = P.rk_stages == 3 ? 3 : 1;
    for (int n = 1; n <= stages; n++) step_stage(rk_stage(stages, n));
    n_step++;
  }

  void step_stage(const RKStage& rk) {
    double dt = P.dt;
    if (P.energy) energy_step(rk);
    // ---- add_all_momentum_sources
    if (P.mpg_dir >= 1 && P.mpg_dir <= 3) {  // compute_add_MPG (momentum_sources.f90:97-109)
      SF& u = U[P.mpg_dir - 1];
      for (auto& v : u.f) v += P.mpg_scale * dt;
      for (int c = 0; c < 3; c++) apply_BCs(U[c]);
    }
    for (int c = 0; c < 3; c++) {
      assign(Fnm1[c], F[c]);
      assign(L[c], 0.0);
      assign(F[c], 0.0);
    }
    advect_U_convection1();
    for (int c = 0; c < 3; c++) add_product(F[c], tF3[c], P.scale_advection_U);
    if (P.scale_diffusion_U != 0.0) {  // compute_add_diffusion: lap (lapUniformCoeff_VF) * scale
      for (int c = 0; c < 3; c++) {
        lap_uniform_coeff(tF1[c], U[c], gm);
        add_product(F[c], tF1[c], P.scale_diffusion_U);
      }
    }
    if (P.scale_diffusion_linear_U != 0.0) {  // diffusion_linear: compute_add_diffusion into L
      for (int c = 0; c < 3; c++) {
        lap_uniform_coeff(tF1[c], U[c], gm);
        add_product(L[c], tF1[c], P.scale_diffusion_linear_U);
      }
    }
    if (P.induction != MOONS_IND_OFF) {  // extract_add_JCrossB (momentum_sources.f90:111-121)
      for (int c = 0; c < 3; c++) {
        if (same) assign(tF1[c], jxb[c]);
        else embed_extract(tF1[c], jxb[c], off, false);
        assign_ghost_XPeriodic(tF1[c], 0.0, nullptr);
        add_product(F[c], tF1[c], 1.0);
      }
    }
    if (P.energy && P.scale_buoyancy != 0.0) add_buoyancy();
    // ---- solve_momentum (solve_method 1 to 9; 0 = 6)
    time_scheme_step(pcgU, pcgP, ispU, ispP, U, Ustar, Unm1, p, F, Fnm1, L, tF1, tCC, gm, P.coeff_implicit_U, 0, 1, &res_p,
              time_method(P.solve_method_U), rk);
    for (int c = 0; c < 3; c++) interp(UCC[c], U[c], gm, c + 1);
    SF* Up[3] = {&U[0], &U[1], &U[2]};
    face2edge_nd(UE, Up, gm);
    // ---- induction
    if (P.induction == MOONS_IND_B) {
      for (int c = 0; c < 3; c++) {
        assign(Fnm1i[c], Fi[c]);
        assign(Li[c], 0.0);
        assign(Fi[c], 0.0);
      }
      embed_UE();
      // advect_B (ops_advect.f90:186-218): E = U_E x face2Edge(Btot); curl(E)
      SF* Bp[3] = {&Btot[0], &Btot[1], &Btot[2]};
      face2edge_nd(BE, Bp, gi);
      cross_TF(tE, UEi, BE);
      curl(curlUxB[0], curlUxB[1], curlUxB[2], tE[0], tE[1], tE[2], gi);
      for (int c = 0; c < 3; c++) add_product(Fi[c], curlUxB[c], P.scale_advection_B);
      if (P.scale_diffusion_linear_B != 0.0) {  // diffusion_linear: add_curl_J into L
        for (int c = 0; c < 3; c++) {
          assign(tE[c], J[c]);
          multiply(tE[c], sig[c]);
        }
        curl(tFi2[0], tFi2[1], tFi2[2], tE[0], tE[1], tE[2], gi);
        for (int c = 0; c < 3; c++) add_product(Li[c], tFi2[c], P.scale_diffusion_linear_B);
      }
      if (P.scale_diffusion_B != 0.0) {  // add_curl_J (induction_sources.f90:40-49)
        for (int c = 0; c < 3; c++) {
          assign(tE[c], J[c]);
          multiply(tE[c], sig[c]);
        }
        curl(tFi2[0], tFi2[1], tFi2[2], tE[0], tE[1], tE[2], gi);
        for (int c = 0; c < 3; c++) add_product(Fi[c], tFi2[c], P.scale_diffusion_B);
      }
      time_scheme_step(pcgB, pcgPhi, ispB, ispPhi, B, Bstar, Bnm1, phi, Fi, Fnm1i, Li, tFi1, tCCi, gi, P.coeff_implicit_B,
                2, 3, &res_phi, time_method(P.solve_method_B), rk);
      compute_J();
      compute_Btot();
      compute_JxB();
    } else if (P.induction == MOONS_IND_POTENTIAL) {
      compute_Btot();
      potential_solve();
      compute_JxB();
    }
  }

  // advect_U_convection1 (ops_advect.f90:71-127) into tF3
  void advect_U_convection1() {
    SF* div_ = tF3;
    for (int c = 0; c < 3; c++) {
      interp(tCC, U[c], gm, c + 1);       // face2CellCenter(temp_CC,U%c,m,c)
      del(div_[c], tCC, gm, 1, c + 1, 0, 1);
      multiply(div_[c], U[c]);
    }
    // (component, edge used, derivative dir, velocity comp for face2Face)
    struct T { int c, e, d, v; };
    const T terms[6] = {{0, 2, 2, 1}, {0, 1, 3, 2}, {1, 2, 1, 0}, {1, 0, 3, 2}, {2, 1, 1, 0}, {2, 0, 2, 1}};
    for (const T& t : terms) {
      del(tF1[t.c], UE.t[t.c][t.e], gm, 1, t.d, 0, 1);
      // face2Face(temp_F2%c, U%v, m, temp_CC, v, c): face2CellCenter along v then cellCenter2Face along c
      interp(tCC, U[t.v], gm, t.v + 1);
      interp(tF2[t.c], tCC, gm, t.c + 1);
      multiply(tF1[t.c], tF2[t.c]);
      add(div_[t.c], tF1[t.c]);
    }
  }

  void divergence(double* l2u, double* l2b) {
    div(divU, U[0], U[1], U[2], gm);
    double s = 0;
    for (double v : divU.f) s += v * v;
    *l2u = s;
    if (P.induction == MOONS_IND_B) {
      div(divB, B[0], B[1], B[2], gi);
      s = 0;
      for (double v : divB.f) s += v * v;
      *l2b = s;
    } else {
      *l2b = 0;
    }
  }

  SF* field(int which, int comp) {
    switch (which) {
      case MOONS_MHD_U: return &U[comp];
      case MOONS_MHD_P: return &p;
      case MOONS_MHD_B: return &B[comp];
      case MOONS_MHD_B0: return &B0[comp];
      case MOONS_MHD_PHI: return &phi;
      case MOONS_MHD_J: return &J[comp];
      case MOONS_MHD_SIGMA_INV: return &sig[comp];
      case MOONS_MHD_JXB: return &jxb[comp];
      case MOONS_MHD_DIVU: return &divU;
      case MOONS_MHD_DIVB: return &divB;
      case MOONS_MHD_T: return &T;
      case MOONS_MHD_KT: return &kT[comp];
      case MOONS_MHD_GRAVITY: return &grav[comp];
      case MOONS_MHD_SIGMA_INV_CC: return &sigInvCC;
      case MOONS_MHD_U_CC: return &UCCn[comp];
    }
    return nullptr;
  }
};

}  // namespace mo

// ---------------------------------------------------------------------------
// C entry points (or_mhd_*), mirroring moons_mhd_* of include/moons_gpu.h
// ---------------------------------------------------------------------------
namespace {
struct OMeshView {
  mo::Grid g;
};
struct OSFView {
  mo::SF f;
  const mo::Grid* g;
};
}  // namespace

extern "C" {
void* or_mhd_create(void* mesh_mom, void* mesh_ind, const moons_mhd_params* prm) {
  for (int m : {prm->solve_method_U, prm->solve_method_B})
    if (m < 0 || m > 9) return nullptr;  // solve_method 1 to 9 (0 = 6)
  if (prm->rk_stages != 0 && prm->rk_stages != 1 && prm->rk_stages != 3) return nullptr;
  if (prm->energy && (prm->solve_method_T < 1 || prm->solve_method_T > 5)) return nullptr;
  auto* s = new mo::MHD();
  const mo::Grid& gm = ((OMeshView*)mesh_mom)->g;
  const mo::Grid& gi = ((OMeshView*)mesh_ind)->g;
  s->same = (mesh_mom == mesh_ind);
  s->create(gm, gi, *prm);
  return s;
}
void or_mhd_destroy(void* s) { delete (mo::MHD*)s; }
// upload/download through host arrays (the oracle keeps fields inside the object)
int or_mhd_upload(void* s, int which, int comp, const double* h, long long n) {
  mo::SF* f = ((mo::MHD*)s)->field(which, comp);
  if (!f || (size_t)n != f->n()) return MOONS_ERR_SHAPE;
  std::memcpy(f->f.data(), h, n * sizeof(double));
  return MOONS_OK;
}
int or_mhd_download(void* s, int which, int comp, double* h, long long n) {
  mo::SF* f = ((mo::MHD*)s)->field(which, comp);
  if (!f || (size_t)n != f->n()) return MOONS_ERR_SHAPE;
  std::memcpy(h, f->f.data(), n * sizeof(double));
  return MOONS_OK;
}
int or_mhd_shape(void* s, int which, int comp, int* out) {
  mo::SF* f = ((mo::MHD*)s)->field(which, comp);
  if (!f) return MOONS_ERR_ARG;
  for (int d = 0; d < 3; d++) out[d] = f->s[d + 1];
  return MOONS_OK;
}
int or_mhd_init(void* s) {
  ((mo::MHD*)s)->init();
  return MOONS_OK;
}
int or_mhd_step(void* s, int n, moons_step_info* info) {
  auto* m = (mo::MHD*)s;
  for (int k = 0; k < 5; k++) m->iters[k] = 0;
  for (int i = 0; i < n; i++) m->step();
  if (info) {
    info->steps = n;
    info->iters_U = m->iters[0];
    info->iters_p = m->iters[1];
    info->iters_B = m->iters[2];
    info->iters_phi = m->iters[3];
    info->iters_T = m->iters[4];
    info->res_p = m->res_p;
    info->res_phi = m->res_phi;
    info->ms = 0;
  }
  return MOONS_OK;
}
int or_mhd_divergence(void* s, double* a, double* b) {
  ((mo::MHD*)s)->divergence(a, b);
  return MOONS_OK;
}
}
