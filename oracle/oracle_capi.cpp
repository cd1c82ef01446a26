// oracle_capi.cpp -- C entry points of the CPU oracle, for the tests'
// ctypes harness.  TEST INFRASTRUCTURE ONLY (see moons_oracle.hpp).
// The entry points mirror the product C-ABI in include/moons_gpu.h one for
// one, with the prefix "or_", so a parity test drives both the same way.
#include <cstring>
#include <string>

#include "../include/moons_gpu.h"
#include "moons_oracle.hpp"

namespace {
struct OMesh {
  mo::Grid g;
};
struct OSF {
  mo::SF f;
  const mo::Grid* g;
};
struct OPCG {
  mo::PCG s;
  mo::ISP isp;
};
thread_local std::string g_err;
int fail(const std::string& m) {
  g_err = m;
  return MOONS_ERR_ARG;
}
}  // namespace

#define OR_TRY(body)                       \
  try {                                    \
    body;                                  \
    return MOONS_OK;                       \
  } catch (const std::exception& e) {      \
    return fail(e.what());                 \
  }

extern "C" {

// host threads the oracle's loops use (MOONS_ORACLE_THREADS or all)
int or_threads() { return mo::oracle_threads(); }

const char* or_last_error(void) { return g_err.c_str(); }

void* or_mesh_create(const double* hx, int sx, const double* hy, int sy, const double* hz, int sz) {
  try {
    auto* m = new OMesh();
    m->g.c[0].init(hx, sx);
    m->g.c[1].init(hy, sy);
    m->g.c[2].init(hz, sz);
    return m;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void or_mesh_destroy(void* m) { delete (OMesh*)m; }

void* or_sf_create(void* mesh, int dl) {
  try {
    auto* s = new OSF();
    s->g = &((OMesh*)mesh)->g;
    s->f.init(*s->g, dl);
    return s;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void or_sf_destroy(void* s) { delete (OSF*)s; }
int or_sf_shape(void* s, int* out) {
  auto* f = (OSF*)s;
  for (int d = 0; d < 3; d++) out[d] = f->f.s[d + 1];
  return MOONS_OK;
}
int or_sf_upload(void* s, const double* h, long long n) {
  auto* f = (OSF*)s;
  if ((size_t)n != f->f.n()) return fail("size mismatch");
  std::memcpy(f->f.f.data(), h, n * sizeof(double));
  return MOONS_OK;
}
int or_sf_download(void* s, double* h, long long n) {
  auto* f = (OSF*)s;
  if ((size_t)n != f->f.n()) return fail("size mismatch");
  std::memcpy(h, f->f.f.data(), n * sizeof(double));
  return MOONS_OK;
}
int or_sf_set_bcs(void* s, const moons_bc_spec* b) {
  auto* f = (OSF*)s;
  OR_TRY(mo::set_bcs(f->f, *f->g, b->type, b->prescribed, b->value, b->c_w, b->order);
         f->f.bc->all_neumann = b->all_neumann != 0;)
}
int or_apply_bcs(void* s) { OR_TRY(mo::apply_BCs(((OSF*)s)->f)) }
int or_apply_bcs_implicit(void* s) { OR_TRY(mo::apply_BCs_implicit(((OSF*)s)->f)) }

#define F(p) (((OSF*)(p))->f)
#define G(p) (*((OSF*)(p))->g)
int or_del(void* out, void* in, int n, int dir, int pad, int gen) {
  OR_TRY(mo::del(F(out), F(in), G(out), n, dir, pad, gen))
}
int or_grad(void* gx, void* gy, void* gz, void* u) { OR_TRY(mo::grad(F(gx), F(gy), F(gz), F(u), G(u))) }
int or_div(void* o, void* ux, void* uy, void* uz) { OR_TRY(mo::div(F(o), F(ux), F(uy), F(uz), G(o))) }
int or_curl(void* ox, void* oy, void* oz, void* ux, void* uy, void* uz) {
  OR_TRY(mo::curl(F(ox), F(oy), F(oz), F(ux), F(uy), F(uz), G(ox)))
}
int or_lap_centered(void* o, void* u) { OR_TRY(mo::lap_centered(F(o), F(u), G(o))) }
int or_lap_uniform_coeff(void* o, void* u) { OR_TRY(mo::lap_uniform_coeff(F(o), F(u), G(o))) }
int or_lap_var(void* o, void* u, void* kx, void* ky, void* kz) {
  OR_TRY(mo::lap_var(F(o), F(u), F(kx), F(ky), F(kz), G(o)))
}
int or_interp(void* o, void* i, int dir) { OR_TRY(mo::interp(F(o), F(i), G(o), dir)) }

void* or_pcg_create(int op, int prec, int nc, void** x, void** xbc, void** k, double coeff_implicit) {
  try {
    auto* p = new OPCG();
    mo::SF* xs[3];
    mo::SF* xb[3];
    mo::SF* ks[3] = {nullptr, nullptr, nullptr};
    for (int c = 0; c < nc; c++) {
      xs[c] = &F(x[c]);
      xb[c] = &F(xbc[c]);
    }
    if (k)
      for (int c = 0; c < 3; c++) ks[c] = k[c] ? &F(k[c]) : nullptr;
    p->s.init(G(x[0]), op, prec, nc, xs, xb, ks, coeff_implicit);
    return p;
  } catch (const std::exception& e) {
    g_err = e.what();
    return nullptr;
  }
}
void or_pcg_destroy(void* p) { delete (OPCG*)p; }
int or_pcg_update_mfp(void* p, double c, int upd) { OR_TRY(((OPCG*)p)->s.update_MFP(c, upd != 0)) }
// operator_explicit of the solver (matrix_free_operators.f90), out = A x
int or_pcg_apply_op(void* p, void** out, void** x) {
  auto* s = (OPCG*)p;
  try {
    std::vector<mo::SF> A, xs;
    for (int c = 0; c < s->s.nc; c++) {
      A.push_back(F(out[c]));
      xs.push_back(F(x[c]));
    }
    s->s.apply_operator(A, xs, true);
    for (int c = 0; c < s->s.nc; c++) F(out[c]).f = A[c].f;
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}
// clean_div (clean_divergence.f90:37-59) with the solver p
int or_clean_div(void* p, void** X, void** Xs, void* phi, double scale, void** tF, void* tCC, const moons_isp* isp,
                 moons_solve_info* info);
int or_pcg_solve(void* p, void** x, void** b, const moons_isp* isp, moons_solve_info* info) {
  auto* s = (OPCG*)p;
  try {
    s->isp.iter_max = isp->iter_max;
    s->isp.tol_rel = isp->tol_rel;
    s->isp.tol_abs = isp->tol_abs;
    s->isp.n_skip_check_res = isp->n_skip_check_res;
    mo::SF* xs[3];
    mo::SF* bs[3];
    for (int c = 0; c < s->s.nc; c++) {
      xs[c] = &F(x[c]);
      bs[c] = &F(b[c]);
    }
    mo::SolveInfo r = s->s.solve(xs, bs, s->isp);
    if (info) {
      info->iterations = r.iterations;
      info->res0 = r.res0;
      info->res = r.res;
      info->rel = r.rel;
      info->exit_reason = r.exit_reason;
      info->ms = 0;
    }
    return r.nan ? MOONS_ERR_NAN : MOONS_OK;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}
int or_clean_div(void* p, void** X, void** Xs, void* phi, double scale, void** tF, void* tCC, const moons_isp* isp,
                 moons_solve_info* info) {
  try {
    mo::SF& tc = F(tCC);
    // div(temp_CC, Xstar); multiply(temp_CC, scale)
    mo::div(tc, F(Xs[0]), F(Xs[1]), F(Xs[2]), G(tCC));
    mo::multiply(tc, scale);
    void* xp[1] = {phi};
    void* bp[1] = {tCC};
    const int r = or_pcg_solve(p, xp, bp, isp, info);
    if (r) return r;
    // grad(temp_F, phi); multiply(temp_F, 1/scale); subtract(X, Xstar, temp_F); apply_BCs(X)
    mo::grad(F(tF[0]), F(tF[1]), F(tF[2]), F(phi), G(phi));
    for (int k = 0; k < 3; k++) {
      mo::multiply(F(tF[k]), 1.0 / scale);
      mo::SF& x = F(X[k]);
      const mo::SF& xs = F(Xs[k]);
      const mo::SF& t = F(tF[k]);
      for (size_t i = 0; i < x.f.size(); i++) x.f[i] = xs.f[i] - t.f[i];
      mo::apply_BCs(x);
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(e.what());
  }
}
}
