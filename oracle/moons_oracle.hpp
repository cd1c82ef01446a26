// moons_oracle.hpp -- CPU restatement of the MOONS time-step hot path.
//
// TEST INFRASTRUCTURE ONLY.  This is the parity oracle for the CUDA product
// in moons_b200/: it restates, routine by routine and on the reference's own
// array layout (Fortran column-major, 1-based, one ghost layer), the Fortran
// code it cites.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline may load it; the product never links or calls it.
//
// Parity status: the reference is Fortran and no Fortran compiler is
// installed next to this code, so this restatement cannot be run side by side
// with the reference.  It is pinned by the reference's own verification routines
// restated as tests (operator identities, Poisson residual drop, SPD
// symmetry, analytic profiles); per-field parity with a Fortran build is
// therefore "unpinned" beyond those pins.
//
// All loops use 1-based indices exactly as the cited Fortran does.
#pragma once
#include <array>
#include <functional>
#include <cmath>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace mo {

// Host threads of the oracle (CPU baseline): loops are cut into a fixed
// number of chunks whatever the thread count, and reductions add the chunk
// sums in chunk order, so results do not depend on the number of threads.
// MOONS_ORACLE_THREADS sets the count (default: all hardware threads).
int oracle_threads();
void set_oracle_threads(int n);
void par_chunks(long n, const std::function<void(long, long)>& fn);

using Vec = std::vector<double>;

// 1-based vector: element i lives at v[i]; v[0] unused.
struct V1 {
  Vec v;
  int n = 0;
  void init(int n_) { n = n_; v.assign(n_ + 1, 0.0); }
  double& operator()(int i) { return v[i]; }
  double operator()(int i) const { return v[i]; }
};

struct Tri {  // sparse tri-diagonal stencil (L,D,U) 1-based
  V1 L, D, U;
};

// coordinates (HW/grid/coordinates_extend.f90)
struct Coord {
  int sn = 0, sc = 0;
  V1 hn, hc, dhn, dhc;
  Tri stagCC2N, stagN2CC, colCC[2], colN[2], theta;
  void init(const double* hn_in, int sn_in);
};

struct Grid {
  Coord c[3];
};

// data location helpers: loc[d]=1 when the data is node-located along d
std::array<int, 3> dl_eye(int dl);
inline bool N_along(int dl, int d) { return dl_eye(dl)[d - 1] == 1; }
inline bool CC_along(int dl, int d) { return dl_eye(dl)[d - 1] == 0; }

enum { BC_NONE = 0, BC_DIRICHLET = 1, BC_NEUMANN = 2, BC_PERIODIC = 3, BC_ROBIN = 4 };

struct BCs {
  bool defined = false;
  int type[7] = {0};
  int prescribed[7] = {0};
  double value[7] = {0};
  double c_w[7] = {0};
  int order[7] = {0};
  double dh[7] = {0};
  double nhat[7] = {0};
  bool all_neumann = false;
  bool many_cell[4] = {false};
};

struct SF {
  int dl = 0;
  int s[4] = {0, 0, 0, 0};  // s[1..3]
  Vec f;
  std::shared_ptr<BCs> bc;  // shared like the reference's copied BCs
  double vol = 0;           // SF%vol (volume_SF)
  void init(const Grid& g, int dl_);
  double& operator()(int i, int j, int k) {
    return f[(size_t)(i - 1) + (size_t)s[1] * ((size_t)(j - 1) + (size_t)s[2] * (size_t)(k - 1))];
  }
  double operator()(int i, int j, int k) const {
    return f[(size_t)(i - 1) + (size_t)s[1] * ((size_t)(j - 1) + (size_t)s[2] * (size_t)(k - 1))];
  }
  size_t n() const { return f.size(); }
  bool has_bcs() const { return bc && bc->defined; }
};

using VF = std::array<SF*, 3>;

// ---- setup
void set_bcs(SF& u, const Grid& g, const int type[6], const int prescribed[6],
             const double value[6], const double c_w[6], const int order[6]);

// ---- pointwise / aux
void assign(SF& a, double v);
void assign(SF& a, const SF& b);
void add(SF& a, const SF& b);
void subtract(SF& a, const SF& b);
void multiply(SF& a, const SF& b);
void multiply(SF& a, double c);
void add_product(SF& a, const SF& b, double c);   // a = a + b*c
void product_add(SF& a, double c, const SF& b);   // a = a*c + b
double sum_pad(const SF& a, int pad);
void volume(SF& u, const Grid& g);
void assign_ghost_XPeriodic(SF& u, double v, const SF* with_bcs);
void assign_ghost_N_XPeriodic(SF& u, double v, const SF* with_bcs);
void assign_wall_Dirichlet(SF& u, double v, const SF* with_bcs);
void multiply_wall_Neumann(SF& u, double v, const SF* with_bcs);
void assign_wall_Periodic_single(SF& u, double v, const SF* with_bcs);
void assign_ghost_dir(SF& u, double v, int dir);   // assign_ghost_{x,y,z}min_max

// ---- BCs
void apply_BCs(SF& u);
void apply_BCs_implicit(SF& u);

// ---- discrete operators
void del(SF& out, const SF& in, const Grid& g, int n, int dir, int pad, int gen);
void grad(SF& gx, SF& gy, SF& gz, const SF& u, const Grid& g);
void div(SF& out, const SF& ux, const SF& uy, const SF& uz, const Grid& g);
void curl_comp(SF& out, const SF& u, const SF& v, const SF& w, const Grid& g, int dir);
void curl(SF& ox, SF& oy, SF& oz, const SF& ux, const SF& uy, const SF& uz, const Grid& g);
void lap_centered(SF& out, const SF& u, const Grid& g);        // SF any location
void lap_uniform_coeff(SF& out, const SF& u, const Grid& g);   // lapUniformCoeff_SF
void lap_var(SF& out, const SF& u, const SF& kx, const SF& ky, const SF& kz, const Grid& g);
void interp(SF& out, const SF& in, const Grid& g, int dir);

// ---- PCG
enum { OP_LAP_UNIFORM = 1, OP_LAP_PROPS = 2, OP_IND_DIFFUSION = 3, OP_MOM_DIFFUSION = 4, OP_NRG_DIFFUSION = 5 };
enum { PREC_IDENTITY = 0, PREC_LAP = 1, PREC_MOM = 2, PREC_IND = 3 };

struct ISP {
  int iter_max = 5;
  double tol_rel = 1e-6, tol_abs = 1e-13;
  int n_skip_check_res = 1;
  int iter_total = 0, iter_per_call = 0;
  bool exit_loop[4] = {false, false, false, false};
};

struct SolveInfo {
  int iterations = 0;
  double res0 = 0, res = 0, rel = 0;
  int exit_reason = 0;
  int nan = 0;
};

struct PCG {
  const Grid* g = nullptr;
  int op = 0, prec = 0, nc = 1;
  double coeff = 0;  // MFP%coeff_implicit_time_split
  std::vector<SF> p, x_BC, r, Ax, vol, z, Minv, tempx, k, tempk;
  void init(const Grid& g, int op, int prec, int nc, SF* const* x, SF* const* xbc,
            SF* const* kin, double coeff_implicit);
  void update_MFP(double c, bool update_prec);
  void compute_prec();
  void apply_operator(std::vector<SF>& Ax, std::vector<SF>& x, bool explicit_only);
  SolveInfo solve(SF* const* x, SF* const* b, ISP& isp);
};

}  // namespace mo
