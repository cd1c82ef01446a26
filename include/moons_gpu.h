/*
 * moons_gpu.h -- C-ABI of the B200 (sm_100a) implementation of the MOONS
 * time-step hot path.
 *
 * Every entry point is extern "C", takes plain pointers and sizes, returns an
 * int status (MOONS_OK == 0) and never exits the process; the caller (the
 * Fortran host through ISO_C_BINDING, or Python through ctypes) decides what
 * to do with an error, reading the text with moons_last_error().
 *
 * Layout contract: a field is the reference's grid_field array f(sx,sy,sz),
 * Fortran column-major (x fastest), one ghost layer per side, FP64.  With N
 * interior cells on an axis the node extent is N+3 and the cell extent N+2
 * (code/generated_code/grid_field/grid_field.f90:39-43,
 *  code/handwritten/grid_field/grid_field_extend.f90:89-133).
 * Uploads and downloads copy such arrays verbatim; between calls the fields
 * stay resident in HBM.
 *
 * Calls on one mesh are not re-entrant; all work of a mesh is enqueued on one
 * CUDA stream and a call returns after its work completed, unless stated.
 */
#ifndef MOONS_GPU_H
#define MOONS_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
  MOONS_OK = 0,
  MOONS_ERR_ARG = 1,     /* bad argument (null pointer, bad enum)            */
  MOONS_ERR_SHAPE = 2,   /* field shapes / data locations do not fit the op  */
  MOONS_ERR_CUDA = 3,    /* a CUDA call failed                               */
  MOONS_ERR_NAN = 4,     /* NaN in solver norms (PCG_solver_algorithm.f90:223-248) */
  MOONS_ERR_STATE = 5,   /* object used before it was set up                 */
  MOONS_ERR_NOMEM = 6,   /* device allocation failed                         */
  MOONS_ERR_LIMIT = 7    /* size beyond a compiled-in maximum                */
};

/* ---- data locations (code/handwritten/fields/data_location_extend.f90) -- */
enum {
  MOONS_CC = 0,
  MOONS_FX = 1, MOONS_FY = 2, MOONS_FZ = 3, /* face data, normal x/y/z       */
  MOONS_EX = 4, MOONS_EY = 5, MOONS_EZ = 6, /* edge data, edge along x/y/z   */
  MOONS_NODE = 7
};

/* ---- boundary-condition types (bctype, code/handwritten/BCs/base/bctype_extend.f90) */
enum {
  MOONS_BC_NONE = 0,       /* field carries no BCs (reference: BCs not defined) */
  MOONS_BC_DIRICHLET = 1,
  MOONS_BC_NEUMANN = 2,
  MOONS_BC_PERIODIC = 3,
  MOONS_BC_ROBIN = 4
};

/* Per-field BC description.  Faces are numbered as in the reference:
 * 1=xmin 2=xmax 3=ymin 4=ymax 5=zmin 6=zmax (face_edge_corner_indexing.f90).
 * value[] is the uniform boundary value b of each face; order[] is
 * apply_BC_order (sim_params_aux.f90:37-55), a permutation of 1..6.
 * Replaces init_Dirichlet/init_Neumann/init_periodic/init_Robin +
 * init_BC_props + set_prescribed (boundary_conditions_extend.f90:120-340). */
typedef struct {
  int type[6];
  int prescribed[6];
  double value[6];
  double c_w[6];
  int order[6];
  int all_neumann;   /* SF%all_Neumann, set by hand in the reference
                        (init_P_BCs.f90:26, init_phi_BCs.f90:27): the PCG
                        removes the RHS mean (PCG_aux.f90:45) when set */
} moons_bc_spec;

/* iter_solver_params (code/handwritten/var_set/iter_solver_params_extend.f90:44-63) */
typedef struct {
  int iter_max;
  double tol_rel;
  double tol_abs;
  int n_skip_check_res;
} moons_isp;

/* What a solve reports (PCG_solver_algorithm.f90:180-220 print/export data). */
typedef struct {
  int iterations;      /* ISP%iter_per_call                                  */
  double res0;         /* L2 of the modified RHS over the whole array        */
  double res;          /* sqrt|dot(r,r)| at exit                             */
  double rel;          /* res/res0 (res when res0 == 0)                      */
  int exit_reason;     /* 1 tol_rel, 2 tol_abs, 3 iter_max; 11/12/13: the same
                          reached by the multigrid fallback after the learned
                          preconditioner stagnated (MOONS_PREC_UNET)        */
  double ms;           /* device time of the solve, CUDA events              */
} moons_solve_info;

/* Operators a PCG object applies (matrix_free_operators.f90). */
enum {
  MOONS_OP_LAP_UNIFORM = 1,   /* Lap_uniform_SF/VF      :35-90              */
  MOONS_OP_LAP_PROPS = 2,     /* Lap_nonuniform_props   :92-118  div(k grad) */
  MOONS_OP_IND_DIFFUSION = 3, /* ind_diffusion          :120-146             */
  MOONS_OP_MOM_DIFFUSION = 4, /* mom_diffusion          :176-202             */
  MOONS_OP_NRG_DIFFUSION = 5  /* nrg_diffusion          :148-174  I + c div(k grad) */
};
/* Diagonal preconditioners (preconditioners.f90). */
enum {
  MOONS_PREC_IDENTITY = 0,    /* prec_Identity_SF/VF :27-51                  */
  MOONS_PREC_LAP = 1,         /* prec_Lap_SF/VF      :55-82                  */
  MOONS_PREC_MOM = 2,         /* prec_mom_SF/VF      :85-113                 */
  MOONS_PREC_IND = 3,         /* prec_ind_VF         :115-129                */
  /* Multigrid V-cycle preconditioners (one CC unknown, LAP_UNIFORM or
   * LAP_PROPS, Dirichlet/Neumann/periodic BCs).  The reference has the
   * building blocks (GF_restrict.f90, GF_prolongate.f90, SOR.f90) but no
   * compiled V-cycle (code_not_compiled/9.6.2017/MG/MG.f90:241-396). */
  MOONS_PREC_MG = 4,          /* FP64 V-cycle inside CG                      */
  MOONS_PREC_MG_MIXED = 5,    /* FP32 V-cycle inside FP64 flexible CG         */
  MOONS_PREC_UNET = 6,        /* learned: the U-Net (moons_pcg_set_unet) inside
                                 FP64 flexible CG, FP32 V-cycle as the fallback
                                 when 10 iterations fail to halve the residual */
  /* Direct solve of the separable operator by fast diagonalization (one CC
   * unknown, LAP_UNIFORM, Dirichlet/Neumann/periodic BCs): the B200 form of
   * the reference's FFT Poisson (FFT_poisson.f90:107-189, solve_method 9),
   * exact for stretched meshes too; CG converges in one or two iterations. */
  MOONS_PREC_FD = 7,
  /* learned + mixed (no reference counterpart): z = V(r) + N(r - A V(r)),
   * the FP32 V-cycle followed by the U-Net (moons_pcg_set_unet) on what the
   * V-cycle leaves, inside FP64 flexible CG; the same stagnation fallback to
   * the V-cycle alone as MOONS_PREC_UNET */
  MOONS_PREC_UNET_MG = 8
};

typedef struct moons_mesh moons_mesh;
typedef struct moons_sf moons_sf;
typedef struct moons_pcg moons_pcg;
typedef struct moons_mhd moons_mhd;

/* ---- error text -------------------------------------------------------- */
/* Last error message of the calling thread ("" if none). */
const char* moons_last_error(void);
/* Diagnostic (no reference counterpart): number of kernels the library has
 * run in this process, host launches plus the launches a solver's
 * device-side loop executed. */
long long moons_kernel_launches(void);
/* Diagnostic (no reference counterpart): runs one bounded in-kernel wait on
 * an mbarrier that nothing completes, with the given limit (0 < limit_ns <=
 * 1e9); returns MOONS_ERR_CUDA with "bounded wait ran out (site 900)" in
 * moons_last_error once the limit has passed.  It exercises, without any
 * fault, the path every bounded wait of the library takes when it runs out:
 * the kernel records the site and returns, and the CUDA context stays
 * usable.  Synchronizes the device. */
int moons_debug_bounded_wait(unsigned long long limit_ns);

/* ---- mesh: single block (coordinates_extend.f90:78-173 init_c,
 *      :506-523 init_stencils_c).  hn_* are the node coordinates including
 *      the ghost nodes, sn_* their counts; stencil coefficients are built
 *      from them exactly as init_stencils_c does.  device < 0 keeps the
 *      current CUDA device. ------------------------------------------------ */
int moons_mesh_create(moons_mesh** out, const double* hn_x, int sn_x,
                      const double* hn_y, int sn_y, const double* hn_z,
                      int sn_z, int device);
int moons_mesh_destroy(moons_mesh* m);
int moons_mesh_sync(moons_mesh* m);

/* ---- fields (SF with one block; GEN/fields/SF.f90:43-51) --------------- */
int moons_sf_create(moons_mesh* m, int data_loc, moons_sf** out);
int moons_sf_destroy(moons_sf* f);
int moons_sf_shape(const moons_sf* f, int s[3]);
/* n must equal s1*s2*s3; host arrays in Fortran order. */
int moons_sf_upload(moons_sf* f, const double* host, long long n);
int moons_sf_download(const moons_sf* f, double* host, long long n);
int moons_sf_fill(moons_sf* f, double val);   /* assign(f,val) */
/* Attach BCs to the field (init_BC_mesh + init_* + init_BC_props). */
int moons_sf_set_bcs(moons_sf* f, const moons_bc_spec* spec);

/* ---- BCs (code/handwritten/BCs/apply/apply_BCs.f90:31-64,
 *      apply_BCs_implicit.f90:18-60) -------------------------------------- */
int moons_apply_bcs(moons_sf* f);
int moons_apply_bcs_implicit(moons_sf* f);

/* ---- discrete operators (code/handwritten/ops) ------------------------- */
/* del%assign/add/subtract (ops_del.f90:236-261): gen 1=assign 2=add
 * 3=subtract, n=1,2 derivative order, dir 1..3, pad 0/1. */
int moons_del(moons_sf* out, const moons_sf* in, int n, int dir, int pad,
              int gen);
/* grad_SF (ops_discrete.f90:173-182): CC -> 3 faces (or any staggered set). */
int moons_grad(moons_sf* gx, moons_sf* gy, moons_sf* gz, const moons_sf* u);
/* div_SF (ops_discrete.f90:158-171) incl. assign_ghost_XPeriodic. */
int moons_div(moons_sf* out, const moons_sf* ux, const moons_sf* uy,
              const moons_sf* uz);
/* curl_VF (ops_discrete.f90:357-365): faces->edges or edges->faces. */
int moons_curl(moons_sf* ox, moons_sf* oy, moons_sf* oz, const moons_sf* ux,
               const moons_sf* uy, const moons_sf* uz);
/* lap_centered_SF_new (ops_discrete.f90:124-132) for CC data and
 * lap_centered_SF_given_both (:112-122) for staggered data, fused. */
int moons_lap_centered(moons_sf* out, const moons_sf* u);
/* lapVarCoeff_VF (ops_discrete.f90:275-285): div(k grad u), k on faces. */
int moons_lap_var(moons_sf* out, const moons_sf* u, const moons_sf* kx,
                  const moons_sf* ky, const moons_sf* kz);
/* interpO2_SF (ops_interp.f90:190-220): C->N (with extrapolation) or N->C
 * along dir. */
int moons_interp(moons_sf* out, const moons_sf* in, int dir);

/* moons_lap_var without device allocation.  No counterpart in the
 * reference: it exists for host codes that cannot allocate device memory at
 * the point of the call (their own pool already holds the free memory, or
 * they keep allocator traffic out of a timed loop).  Same result as
 * moons_lap_var; the three face temporaries come from one built-in device
 * array instead of the allocator.
 *  - each temporary holds at most MOONS_LAP_VAR_NOALLOC_MAX_POINTS doubles;
 *    larger fields are rejected with MOONS_ERR_LIMIT (use moons_lap_var);
 *  - the first call on a device looks up the array's address on that
 *    device (the caller's current device is left as it was) and later calls
 *    reuse it: make the first call before any stream capture;
 *  - every call synchronizes the mesh's stream before it returns;
 *  - the array needs no initial contents (every element read is written
 *    earlier in the same call);
 *  - the array is shared per device: calls that overlap in time race. */
#define MOONS_LAP_VAR_NOALLOC_MAX_POINTS 131072
int moons_lap_var_noalloc(moons_sf* out, const moons_sf* u, const moons_sf* kx,
                          const moons_sf* ky, const moons_sf* kz);

/* ---- PCG (code/handwritten/PCG/PCG_solver_extend.f90:51-291,
 *      code/handwritten/solvers/PCG/PCG_solver_algorithm.f90:37-179) ------ */
/* ncomp = 1 (SF) or 3 (VF).  x[] are the unknown's fields (their BCs are
 * copied, as init(PCG%p,x) does), x_bc[] the fields whose BCs define x_BC,
 * k[] the coefficient fields the operator reads (faces for LAP_PROPS,
 * edges for IND_DIFFUSION; NULL otherwise). */
int moons_pcg_create(moons_mesh* m, int op, int prec, int ncomp,
                     moons_sf* const* x, moons_sf* const* x_bc,
                     moons_sf* const* k, moons_pcg** out);
int moons_pcg_destroy(moons_pcg* s);
/* update_MFP (PCG_solver_extend.f90:269-291). */
int moons_pcg_update_mfp(moons_pcg* s, double coeff_implicit_time_split,
                         int update_preconditioner);
/* solve (PCG_solver_extend.f90:182-206): x[] updated in place. */
int moons_pcg_solve(moons_pcg* s, moons_sf* const* x, moons_sf* const* b,
                    const moons_isp* isp, moons_solve_info* info);

/* clean_div (clean_divergence.f90:37-59) with PCG_phi: temp_CC = scale *
 * div(Xstar); solve(PCG, phi, temp_CC); temp_F = grad(phi) / scale;
 * X = Xstar - temp_F; apply_BCs(X).  X, Xstar, temp_F: x, y, z face fields;
 * phi, temp_CC: cell-centred, all on the solver's mesh; the caller's
 * temporaries are overwritten (as the reference's temp_F, temp_CC are). */
int moons_clean_div(moons_pcg* pcg, moons_sf* const* X, moons_sf* const* Xstar, moons_sf* phi, double scale,
                    moons_sf* const* temp_F, moons_sf* temp_CC, const moons_isp* isp, moons_solve_info* info);

/* ---- the MHD time step (HW/MOONS/MOONS_solver.f90:47-144, one RK stage) --
 * Momentum: add_all_momentum_sources (add_all_momentum_sources.f90:22-86)
 * + Euler_time_AB2_sources (time_marching_methods.f90:117-150) with PCG_U
 * (mom_diffusion, prec_mom_VF) and clean_div (clean_divergence.f90:37-59)
 * with PCG_P (Lap_uniform_SF, prec_Lap_SF).
 * Induction, MOONS_IND_B: add_all_induction_sources
 * (add_all_induction_sources.f90:24-60, constrained-transport curl(u x B))
 * + Euler_time_AB2_sources with PCG_B (ind_diffusion, prec_ind_VF) and
 * clean_div with PCG_phi; then compute_J, compute_Btot, compute_JCrossB
 * (induction_extend.f90:441-536).
 * Induction, MOONS_IND_POTENTIAL: low-Rem electric-potential form (new; not
 * in the reference): div(sigma grad phi) = div(sigma u x B0) with
 * Lap_nonuniform_props, J = sigma(-grad phi + u x B0), F += N J x B0. */
enum { MOONS_IND_OFF = 0, MOONS_IND_B = 1, MOONS_IND_POTENTIAL = 2 };

typedef struct {
  double dt;
  int induction;            /* MOONS_IND_*                                  */
  int finite_Rem;           /* Btot = B0 + B (else B0)                      */
  int mpg_dir;              /* compute_add_MPG direction (0 = off)          */
  double mpg_scale;         /* SP%MT%mean_pressure_grad%scale               */
  double scale_advection_U; /* SP%MT%advection_convection%scale (-1)        */
  double scale_diffusion_U; /* SP%MT%diffusion%scale = coeff_explicit       */
  double scale_JxB;         /* SP%MT%JCrossB%scale (N = Ha^2/Re)            */
  double scale_advection_B; /* SP%IT%advection%scale (1)                    */
  double scale_diffusion_B; /* SP%IT%diffusion%scale (-beta)                */
  double scale_current;     /* SP%IT%current%scale (1/Rem)                  */
  double coeff_implicit_U;  /* SP%VS%U%MFP%coeff_implicit (-1/Re)... see
                               assign_coeff_implicit_VS: -coeff_natural*alpha */
  double coeff_implicit_B;  /* SP%VS%B%MFP%coeff_implicit (1/Rem)           */
  moons_isp isp_U, isp_p, isp_B, isp_phi;
  moons_bc_spec bc_U[3], bc_p, bc_B[3], bc_phi;
  int ind_offset[3];        /* first fluid cell inside the induction mesh, minus 1
                               (0 when both meshes coincide)                  */
  int prescribed_Ustar;     /* SP%VS%U%SS%prescribed_BCs: Ustar gets prescribed
                               BCs (set_prescribed_BCs, block_field_extend.f90:810-821) */
  int prescribed_Bstar;     /* SP%VS%B%SS%prescribed_BCs                      */
  int prec_poisson;         /* preconditioner of the pressure and potential
                               solves: 0 (default) = the reference's prec_Lap,
                               or MOONS_PREC_MG / MOONS_PREC_MG_MIXED (no
                               reference counterpart: same system, same exit
                               tests, far fewer iterations), or MOONS_PREC_FD
                               (direct solve of the separable pressure and
                               cleaning potential; the sigma-weighted potential
                               of the low-Rem form takes MG_MIXED), or
                               MOONS_PREC_UNET_MG (learned + mixed, networks
                               from moons_mhd_set_unet); MOONS_PREC_LAP is
                               the same as 0; other values are refused
                               (MOONS_ERR_ARG)                                */
  /* energy equation (energy_extend.f90:236-262, add_all_energy_sources.f90:
   * 21-67), solved on the induction mesh before the momentum step as
   * solve_MOONS does (MOONS_solver.f90:81-85); fields MOONS_MHD_T, _KT,
   * _GRAVITY */
  int energy;               /* 1: solve for T                               */
  int solve_method_T;       /* solve_energy's select case (energy_extend.f90:
                               244-257), time_marching_methods_SF.f90:
                               1: Euler_time_no_diff_Euler_sources_SF (:154-170),
                               2: Euler_time_no_diff_AB2_sources_SF (:135-152),
                                  X += dt F or dt AB2(F, Fnm1), no solve;
                               3: Euler_time_AB2_sources_SF (:71-98),
                               4: O2_BDF_time_AB2_sources_SF (:42-69),
                               5: Euler_time_RK_sources_SF (:100-133), with
                                  the rk_stages coefficients: PCG_T solves
                                  (nrg_diffusion, prec_lap_SF)              */
  double coeff_implicit_T;  /* SP%VS%T%MFP%coeff_implicit                    */
  double scale_advection_T; /* SP%ET%advection%scale: F += s (-div(u T))     */
  double scale_diffusion_T; /* SP%ET%diffusion%scale: F += s lap(T) (explicit) */
  double scale_heating_T;   /* SP%ET%volumetric_heating%scale
                               (add_volumetric_heating_Nuclear)              */
  double scale_buoyancy;    /* SP%MT%Buoyancy%scale: F_U += s face(T g)      */
  moons_isp isp_T;
  moons_bc_spec bc_T;
  /* further energy sources (energy_sources.f90:51-94), with U_CC the cell-centre
   * velocity embedded in the induction mesh (embedCC of face2CellCenter(U),
   * add_all_energy_sources.f90:30-32): */
  double scale_KE_diffusion_T;        /* SP%ET%KE_diffusion%scale: F += s lap(sum_c U_CC,c^2) */
  double scale_viscous_dissipation_T; /* SP%ET%viscous_dissipation%scale: F += s sum_cd (d_d U_CC,c)^2 */
  double scale_joule_heating_T;       /* SP%ET%joule_heating%scale: F += s (sum_c J_CC,c^2) sigmaInv_CC,
                                         J_CC = edge2CellCenter(J) (faces in the potential form) */
  /* time schemes of the momentum and (B form) induction steps, the
   * solve_method switch of solve_momentum (momentum_extend.f90:335-367) and
   * solve_induction (induction_extend.f90:484-514), time_marching_methods.f90:
   *   0 or 6: Euler_time_AB2_sources (:117-150), (I + dt c A) X* =
   *           X + dt (AB2(F, Fnm1) + L), clean_div scale 1/dt;
   *   5:      Euler_time_Euler_sources (:47-79), (I + dt c A) X* = X + dt F,
   *           clean_div scale 1;
   *   7:      O2_BDF_time_AB2_sources (:81-115), (I + 2/3 dt c A) X* =
   *           4/3 X - 1/3 Xnm1 + 2/3 dt AB2(F, Fnm1), clean_div scale 1;
   *   3, 4:   Euler_time_no_diff_Euler_sources (:298-327) and
   *           Euler_time_no_diff_AB2_sources (:266-296), no diffusion solve:
   *           X* = X + dt F or X + dt AB2(F, Fnm1), clean_div scale 1;
   *   1, 2:   the same without the projection (:329-366): X += dt F or
   *           dt AB2(F, Fnm1), then X's BCs;
   *   8:      Euler_time_RK_sources (:186-208), with rk_stages below;
   *   9:      Euler_time_AB2_sources_FFT (:152-185): 6 with the cleaning
   *           Poisson equation solved directly (clean_div_FFT), which here
   *           is the fast-diagonalization solve, MOONS_PREC_FD, in place of
   *           prec_poisson for that equation (pressure for solve_method_U,
   *           the B-cleaning potential for solve_method_B).
   * Source terms on wall-normal Dirichlet faces are zeroed in all of them. */
  int solve_method_U;
  int solve_method_B;
  /* Runge-Kutta stages of the step (RKP%n_stages, the stage loop of
   * solve_MOONS, MOONS_solver.f90:73-97): 0 or 1 = one stage with the
   * inactive coefficients (all 1), 3 = the three-stage low-storage scheme of
   * init_RKP (RK_params_extend.f90:22-55).  Every stage runs the sources and
   * the solves of the whole step; solve_method 8 (Euler_time_RK_sources,
   * time_marching_methods.f90:186-208) uses the stage's coefficients:
   * (I + 2 beta dt c A) X* = X + dt (gamma F + zeta Fnm1 + 2 alpha L),
   * clean_div scale 1.  With three stages the energy's explicit diffusion
   * goes into its L (add_all_energy_sources.f90:35-48), which only
   * solve_method_T 5 reads. */
  int rk_stages;
  /* SP%MT%diffusion_linear / SP%IT%diffusion_linear: the diffusion term into
   * L instead of F (add_all_momentum_sources.f90:49-51,
   * add_all_induction_sources.f90:39-41), with the diffusion scale:
   * L_U += s lap(U), L_B += s curl(sigma^-1 J).  Only Euler_time_AB2_sources
   * (6) and Euler_time_RK_sources (8) read L. */
  double scale_diffusion_linear_U;
  double scale_diffusion_linear_B;
} moons_mhd_params;

typedef struct {
  int steps;
  int iters_U, iters_p, iters_B, iters_phi;  /* summed over the steps       */
  double res_p, res_phi;                     /* last relative residuals     */
  double ms;                                 /* device time of the steps    */
  int iters_T;                               /* energy PCG (solve_method 3) */
} moons_step_info;

/* Field handles of an MHD object (for upload / download / probes). */
enum {
  MOONS_MHD_U = 0,        /* comp 0..2, faces on the fluid mesh              */
  MOONS_MHD_P = 1,        /* CC on the fluid mesh                            */
  MOONS_MHD_B = 2,        /* comp 0..2, faces on the induction mesh          */
  MOONS_MHD_B0 = 3,       /* comp 0..2, faces                                */
  MOONS_MHD_PHI = 4,      /* CC on the induction mesh                        */
  MOONS_MHD_J = 5,        /* comp 0..2: edges (B form) / faces (potential)   */
  MOONS_MHD_SIGMA_INV = 6,/* comp 0..2: edges (B form) / sigma on faces (potential) */
  MOONS_MHD_JXB = 7,      /* comp 0..2, faces on the induction mesh          */
  MOONS_MHD_DIVU = 8,     /* CC on the fluid mesh (probe)                    */
  MOONS_MHD_DIVB = 9,     /* CC on the induction mesh (probe)                */
  MOONS_MHD_T = 10,       /* temperature, CC on the induction mesh           */
  MOONS_MHD_KT = 11,      /* comp 0..2: thermal conductivity on the faces    */
  MOONS_MHD_GRAVITY = 12, /* comp 0..2: gravity vector field, CC             */
  MOONS_MHD_SIGMA_INV_CC = 13, /* sigma^-1 at cell centres on the induction mesh,
                               the factor of the Joule heating; 0 until uploaded
                               (the reference's ind%sigmaInv_CC starts at 0 and
                               its step never sets it)                       */
  MOONS_MHD_U_CC = 14     /* comp 0..2: the energy equation's cell-centre
                             velocity on the induction mesh (probe)           */
};

/* mesh_ind may equal mesh_mom.  Fields start at 0; upload initial U, B, B0
 * and sigma through moons_mhd_field, then call moons_mhd_init. */
int moons_mhd_create(moons_mesh* mesh_mom, moons_mesh* mesh_ind,
                     const moons_mhd_params* prm, moons_mhd** out);
int moons_mhd_destroy(moons_mhd* s);
int moons_mhd_field(moons_mhd* s, int which, int comp, moons_sf** out);
/* init_mom/init_induction tail + the start of solve_MOONS: apply BCs,
 * J, Btot, J x B, U at cell centres and edges. */
int moons_mhd_init(moons_mhd* s);
int moons_mhd_step(moons_mhd* s, int nsteps, moons_step_info* info);
/* probes: div U and div B over the whole array (compute_Ln L2, as the
 * divU/divB probes export) */
int moons_mhd_divergence(moons_mhd* s, double* l2_divU, double* l2_divB);

/* Diagnostics (no reference counterpart): the building blocks of an
 * MOONS_PREC_MG solver's FP64 multigrid hierarchy, one at a time, on host
 * arrays, so each can be checked against a CPU restatement of the
 * reference's prolongate_C (grid_field/GF_MG/GF_prolongate.f90:22-56), its
 * transpose, and the point update of redBlack (solvers/SOR/SOR.f90:234-268).
 * Level 0 is the solver's mesh; moons_mg_level_shape gives a level's
 * cell-centred extents (ghosts included) and the level count.  Arrays are
 * Fortran-ordered level arrays with ghosts (ghost entries are implied by the
 * homogeneous BCs: not read, returned as zeros).
 *  op 0: out(level) = P a, a on level+1 (prolongation of a correction)
 *  op 1: out(level+1) = P^T a, a on level (restriction of a residual)
 *  op 2: out(level) = e after one red (i+j+k even) and one black SOR sweep
 *        from e = a, right-hand side b (the V-cycle's omega)
 *  op 3: out(level) = b - A a with A the level's volume-weighted operator */
int moons_mg_level_shape(moons_pcg* s, int level, int* shape3, int* nlevels);
int moons_mg_debug(moons_pcg* s, int op, int level, const double* a, const double* b, double* out);

/* ---- learned preconditioner: 3-D U-Net -------------------------------------
 * No reference counterpart (the reference's preconditioners are the Jacobi
 * family of code/handwritten/solvers/preconditioners/preconditioners.f90:
 * 55-129).  A network on a mesh's cell-centred interior (cell counts
 * multiples of 8): z = M(r) ~ A^-1 r, inputs r / rms(r) and one per-cell
 * feature of the operator's coefficients, BF16 activations and weights,
 * FP32 accumulation on the tensor cores (tcgen05).  It is trained on
 * (r, e) pairs with A e = r by moons_unet_train_step (forward, backward and
 * Adam on the GPU) and used inside flexible CG through moons_pcg_set_unet.
 * Parameters: one flat FP32 array; per convolution W[co][ci][dz][dy][dx]
 * then b[co] (layers enc0a 8->16, enc0b 16->16, enc1a 16->32, enc1b 32->32,
 * enc2a 32->64, enc2b 64->64, enc3a 64->128, enc3b 128->128,
 * dec2a 192->64, dec2b 64->64, dec1a 96->32, dec1b 32->32, dec0a 48->16,
 * dec0b 16->16), then the 1x1 head w[16], b. */
typedef struct moons_unet moons_unet;
int moons_unet_create(moons_mesh* m, unsigned long long seed, moons_unet** out);
/* networks of the learned + mixed Poisson solves (prec_poisson =
 * MOONS_PREC_UNET_MG; no reference counterpart): which = 0 the pressure
 * (net on the fluid mesh), 1 the B-form cleaning potential (net on the
 * induction mesh); before or after moons_mhd_init.  The low-Rem potential
 * (sigma-weighted) takes MOONS_PREC_MG_MIXED under this setting.  A step
 * whose learned solver has no network returns MOONS_ERR_STATE.  The
 * simulation does not own the network: keep it alive while the simulation
 * steps (one network may serve both solves when the meshes coincide). */
int moons_mhd_set_unet(moons_mhd* s, int which, moons_unet* u);
int moons_unet_destroy(moons_unet* u);
int moons_unet_nparams(const moons_unet* u, long long* n);
int moons_unet_get_params(moons_unet* u, float* host, long long n);
int moons_unet_set_params(moons_unet* u, const float* host, long long n);  /* resets Adam */
/* z = out_scale * rms(r) * y: the scale c of the network's output */
int moons_unet_set_out_scale(moons_unet* u, double c);
int moons_unet_get_out_scale(const moons_unet* u, double* c);
/* per-cell feature (ghosts included, cell-centred layout), e.g.
 * log10(mean face coefficient) / 3 */
int moons_unet_set_feature(moons_unet* u, const float* host, long long n);
/* z = M(r); r, z cell-centred fields of the net's mesh (z's ghosts = 0) */
int moons_unet_apply(moons_unet* u, moons_sf* z, const moons_sf* r);
/* training loss: kind 0 relative L2, |y - t|^2 / |t|^2 with
 * t = e / (out_scale * rms(r)); kind 1 (default) cosine, 1 - y.t / (|y| |t|),
 * invariant to a positive scale of the output, as flexible CG is; */
int moons_unet_set_loss(moons_unet* u, int kind);
/* kind 2: cosine in the energy norm of the solver's operator A (the norm CG
 * minimises), 1 - y.A e / sqrt(y.A y  e.A e) with A e = r; the operator is
 * the FP32 finest multigrid level of a MOONS_PREC_MG_MIXED / MOONS_PREC_UNET
 * solver on the net's mesh, set (per case) by moons_unet_set_operator */
int moons_unet_set_operator(moons_unet* u, moons_pcg* s);
/* the training loss and its gradient (grads_host may be null; n = nparams) */
int moons_unet_loss_grad(moons_unet* u, const moons_sf* r, const moons_sf* e, float* loss, float* grads_host,
                         long long n);
/* one Adam step (beta 0.9 / 0.999) on one (r, e) pair; loss may be null */
int moons_unet_train_step(moons_unet* u, const moons_sf* r, const moons_sf* e, float lr, float* loss);
/* per-cell feature from face coefficients: log10(mean of the six faces)/3 */
int moons_unet_set_coeff(moons_unet* u, const moons_sf* kx, const moons_sf* ky, const moons_sf* kz);
/* the solver's own residual for the iterate x (modify_RHS + the initial
 * residual of PCG_solver_algorithm.f90:55-66): r = vol*(b - A x_BC - A x),
 * mean removed for all-Neumann problems; what a preconditioner is applied to */
int moons_pcg_residual(moons_pcg* s, moons_sf* const* x, moons_sf* const* b, moons_sf* const* r);
/* attach a network to a solver created with MOONS_PREC_UNET or
 * MOONS_PREC_UNET_MG (same mesh; the solver does not own it and reads its
 * current weights at every solve) */
int moons_pcg_set_unet(moons_pcg* s, moons_unet* u);
/* out = A x with the solver's operator in its explicit form, the abstract
 * op_SF / op_VF of matrix_free_operators_interfaces.f90:14-60 as
 * operator_explicit binds it (matrix_free_operators.f90: Lap_uniform,
 * Lap_nonuniform_props, mom_diffusion, ind_diffusion, nrg_diffusion
 * _explicit): the values in x's ghost cells are used as they are, no
 * volume weighting; out and x are fields of the solver's unknown's layout */
int moons_pcg_apply_op(moons_pcg* s, moons_sf* const* out, moons_sf* const* x);
/* z = M(r) with the solver's preconditioner (no reference counterpart): the
 * Jacobi Minv r, or one multigrid V-cycle (MOONS_PREC_MG / _MG_MIXED /
 * _UNET / _UNET_MG: the V-cycle alone), or the direct solve (MOONS_PREC_FD);
 * used to form the training targets of the two-stage learned form */
int moons_pcg_apply_prec(moons_pcg* s, moons_sf* const* z, moons_sf* const* r);
/* kernel self-check of one layer on host data ([C][Z][Y][X] FP32, interior,
 * rounded to BF16 on upload): op 0 out = conv(in) (+bias, ReLU if relu);
 * op 1 out = transposed conv of dout (gradient w.r.t. the input); op 2 out =
 * weight gradient [cout][cin][27] followed by the bias gradient [cout] */
int moons_unet_layer_check(int op, int X, int Y, int Z, int cinA, int cinB, int cout, const float* in,
                           const float* dout, const float* W, const float* bias, int relu, float* out);

#ifdef __cplusplus
}
#endif

#endif /* MOONS_GPU_H */
