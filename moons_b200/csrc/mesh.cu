// mesh.cu -- mesh, field and operator entry points of the C-ABI.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>

#include "coeffs.hpp"
#include "kernels.cuh"
#include "runtime.cuh"

namespace mg {

static thread_local std::string g_err;
long long g_launch_count = 0;
void set_error(const std::string& m) { g_err = m; }
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string("CUDA error ") + cudaGetErrorString(e) + " in " + what;
  return MOONS_ERR_CUDA;
}
static int arg_fail(const std::string& m) {
  g_err = m;
  return MOONS_ERR_ARG;
}

using host::HostCoord;
using host::build_coord;

DF make_df(moons_mesh* m, int dl, double** storage) {
  DF f{};
  f.dl = dl;
  int b = dl_bits(dl);
  f.s0 = (b & 1) ? m->sn[0] : m->sn[0] - 1;
  f.s1 = (b & 2) ? m->sn[1] : m->sn[1] - 1;
  f.s2 = (b & 4) ? m->sn[2] : m->sn[2] - 1;
  f.f = storage ? *storage : nullptr;
  return f;
}
int dl_after_diff(int dl, int dir) { return dl_from_bits(dl_bits(dl) ^ (1 << (dir - 1))); }

// ---- launch helpers -------------------------------------------------------
int launch_del(moons_mesh* m, DF out, DF in, int n, int dir, int pad, int gen) {
  bool fc = !n_along(in.dl, dir), oc = !n_along(out.dl, dir);
  int diffType = (fc && oc) ? 1 : (!fc && !oc) ? 2 : (fc && !oc) ? 3 : 4;
  for (int d = 1; d <= 3; d++)
    if (d != dir && in.s(d) != out.s(d)) return arg_fail("del: transverse shapes differ");
  if (diffType >= 3 && (in.s(dir) - out.s(dir) != (diffType == 3 ? -1 : 1)))
    return arg_fail("del: staggered extents do not match the data locations");
  if (diffType <= 2 && in.s(dir) != out.s(dir)) return arg_fail("del: collocated extents differ");
  if (n < 1 || n > 2) return arg_fail("del: n must be 1 or 2");
  MG_LAUNCH(k_del, nblocks(out.n()), kBlock, m->stream, out, in, m->dg.c[dir - 1], dir, diffType, n, pad, gen);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
int launch_pw(moons_mesh* m, int op, DF a, const DF* b, double c) {
  MG_LAUNCH(k_pw, nblocks(a.n()), kBlock, m->stream, op, a.f, b ? b->f : nullptr, c, a.n());
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
int launch_bcs(moons_mesh* m, DF u, const DBC& bc, bool implicit) {
  if (!bc.defined) return MOONS_OK;
  for (int o = 1; o <= 6; o++) {
    int f = bc.order[o];
    int d = (f + 1) / 2;
    int np = (d == 1 ? u.s1 * u.s2 : (d == 2 ? u.s0 * u.s2 : u.s0 * u.s1));
    MG_LAUNCH(k_bc_face, nblocks(np), kBlock, m->stream, u, bc, f, implicit ? 1 : 0);
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
int launch_plane(moons_mesh* m, DF u, int d, int idx, double v, int mode) {
  int np = (d == 1 ? u.s1 * u.s2 : (d == 2 ? u.s0 * u.s2 : u.s0 * u.s1));
  MG_LAUNCH(k_plane, nblocks(np), kBlock, m->stream, u, d, idx, v, mode);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
int launch_lap_centered(moons_mesh* m, DF out, DF u, int ghost_zero, int scale_mode, double coeff) {
  if (out.dl != u.dl) return arg_fail("lap_centered: data locations differ");
  MG_LAUNCH(k_lap_centered, nblocks(out.n()), kBlock, m->stream, out, u, m->dg, ghost_zero, scale_mode, coeff);
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}
int launch_interp(moons_mesh* m, DF out, DF in, int dir) {
  if (n_along(out.dl, dir) && !n_along(in.dl, dir)) {
    MG_LAUNCH(k_interp_c2n, nblocks(out.n()), kBlock, m->stream, out, in, m->dg.c[dir - 1], dir);
    int a = dir == 1 ? 2 : 1, b = dir == 3 ? 2 : 3;
    MG_LAUNCH(k_extrap, nblocks(out.s(a) * out.s(b)), kBlock, m->stream, out, in, dir);
  } else if (!n_along(out.dl, dir) && n_along(in.dl, dir)) {
    MG_LAUNCH(k_interp_n2c, nblocks(out.n()), kBlock, m->stream, out, in, dir);
  } else {
    return arg_fail("interp: bad data locations");
  }
  MG_CUDA(cudaGetLastError());
  return MOONS_OK;
}

// ---- masks (block_field_extend.f90:232-375) -------------------------------
int ghost_zero_bits(const DBC* w) {
  int bits = 0;
  for (int f = 1; f <= 6; f++) {
    bool apply = (w && w->defined) ? (w->type[f] != MOONS_BC_PERIODIC) : true;
    if (apply) bits |= 1 << (f - 1);
  }
  return bits;
}
int dirichlet_wall_bits(const DBC* w, int dl) {
  int bits = 0;
  for (int f = 1; f <= 6; f++) {
    int d = (f + 1) / 2;
    if (!n_along(dl, d)) continue;
    bool apply = (w && w->defined) ? (w->type[f] == MOONS_BC_DIRICHLET) : true;
    if (apply) bits |= 1 << (f - 1);
  }
  return bits;
}
int mask_ghost_XPeriodic(moons_mesh* m, DF u, const DBC* w) {
  int bits = ghost_zero_bits(w);
  for (int f = 1; f <= 6; f++)
    if (bits & (1 << (f - 1))) {
      int d = (f + 1) / 2;
      int r = launch_plane(m, u, d, (f & 1) ? 1 : u.s(d), 0.0, 0);
      if (r) return r;
    }
  return MOONS_OK;
}
int mask_ghost_N_XPeriodic(moons_mesh* m, DF u, const DBC* w, int dlw) {
  if (!(w && w->defined)) return MOONS_OK;
  for (int f = 1; f <= 6; f++) {
    int d = (f + 1) / 2;
    if (w->type[f] != MOONS_BC_PERIODIC && n_along(dlw, d)) {
      int r = launch_plane(m, u, d, (f & 1) ? 1 : u.s(d), 0.0, 0);
      if (r) return r;
    }
  }
  return MOONS_OK;
}
int mask_wall_Dirichlet(moons_mesh* m, DF u, const DBC* w, int dlw, double v) {
  int bits = dirichlet_wall_bits(w, dlw);
  for (int f = 1; f <= 6; f++)
    if (bits & (1 << (f - 1))) {
      int d = (f + 1) / 2;
      int r = launch_plane(m, u, d, (f & 1) ? 2 : u.s(d) - 1, v, 0);
      if (r) return r;
    }
  return MOONS_OK;
}
int mask_wall_Neumann(moons_mesh* m, DF u, const DBC* w, int dlw, double v) {
  for (int f = 1; f <= 6; f++) {
    int d = (f + 1) / 2;
    if (!n_along(dlw, d)) continue;
    bool apply = (w && w->defined) ? (w->type[f] == MOONS_BC_NEUMANN) : true;
    if (apply) {
      int r = launch_plane(m, u, d, (f & 1) ? 2 : u.s(d) - 1, v, 1);
      if (r) return r;
    }
  }
  return MOONS_OK;
}
int mask_wall_Periodic_single(moons_mesh* m, DF u, const DBC* w, int dlw, double v) {
  if (!(w && w->defined)) return MOONS_OK;
  for (int d = 1; d <= 3; d++) {
    bool L = n_along(dlw, d) && w->type[2 * d - 1] == MOONS_BC_PERIODIC && w->type[2 * d] == MOONS_BC_PERIODIC &&
             u.s(d) > 4;
    if (L) {
      int r = launch_plane(m, u, d, u.s(d) - 1, v, 0);
      if (r) return r;
    }
  }
  return MOONS_OK;
}

}  // namespace mg

using namespace mg;

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

const char* moons_last_error(void) { return g_err.c_str(); }

long long moons_kernel_launches(void) { return g_launch_count; }

int moons_mesh_create(moons_mesh** out, const double* hx, int sx, const double* hy, int sy, const double* hz,
                      int sz, int device) {
  if (!out || !hx || !hy || !hz) return arg_fail("moons_mesh_create: null pointer");
  if (sx < 4 || sy < 4 || sz < 4) return arg_fail("moons_mesh_create: need at least 4 nodes per axis");
  // kernels index points with 32-bit integers and put z on gridDim.y
  if ((double)sx * sy * sz >= 2147483647.0 || sz > 65535) {
    g_err = "moons_mesh_create: mesh beyond 2^31 points or 65535 z-nodes";
    return MOONS_ERR_LIMIT;
  }
  auto* m = new moons_mesh();
  int dev = device;
  if (dev < 0) {
    if (cudaGetDevice(&dev) != cudaSuccess) {
      delete m;
      return arg_fail("moons_mesh_create: no CUDA device");
    }
  }
  m->device = dev;
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    delete m;
    return cuda_fail(e, "cudaSetDevice");
  }
  e = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    delete m;
    return cuda_fail(e, "cudaStreamCreate");
  }
  const double* hs[3] = {hx, hy, hz};
  int ss[3] = {sx, sy, sz};
  for (int d = 0; d < 3; d++) {
    m->sn[d] = ss[d];
    m->hn[d].assign(hs[d], hs[d] + ss[d]);
    HostCoord c = build_coord(hs[d], ss[d]);
    DCoord& dc = m->dg.c[d];
    dc.sn = c.sn;
    dc.sc = c.sc;
    auto up = [&](const std::vector<double>& v) -> const double* {
      void* p = nullptr;
      if (cudaMalloc(&p, v.size() * sizeof(double)) != cudaSuccess) return nullptr;
      cudaMemcpy(p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice);
      m->allocs.push_back(p);
      return (const double*)p;
    };
    dc.hn = up(c.hn); dc.hc = up(c.hc); dc.dhn = up(c.dhn); dc.dhc = up(c.dhc);
    dc.cc2nD = up(c.cc2nD); dc.cc2nU = up(c.cc2nU); dc.n2ccD = up(c.n2ccD); dc.n2ccU = up(c.n2ccU);
    dc.thD = up(c.thD); dc.thU = up(c.thU);
    dc.diagC = up(c.diagC); dc.diagN = up(c.diagN);
    for (int o = 0; o < 2; o++) {
      dc.colCC_L[o] = up(c.colCC_L[o]); dc.colCC_D[o] = up(c.colCC_D[o]); dc.colCC_U[o] = up(c.colCC_U[o]);
      dc.colN_L[o] = up(c.colN_L[o]); dc.colN_D[o] = up(c.colN_D[o]); dc.colN_U[o] = up(c.colN_U[o]);
    }
    if (!dc.hn || !dc.thU || !dc.colN_U[1] || !dc.diagN) {
      moons_mesh_destroy(m);
      g_err = "moons_mesh_create: device allocation failed";
      return MOONS_ERR_NOMEM;
    }
  }
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(double) * kRedBlocks * moons_mesh::kSlots) != cudaSuccess) goto nomem;
  m->allocs.push_back(p);
  m->d_partial = (double*)p;
  if (cudaMalloc(&p, sizeof(unsigned) * moons_mesh::kSlots) != cudaSuccess) goto nomem;
  m->allocs.push_back(p);
  m->d_ticket = (unsigned*)p;
  cudaMemset(m->d_ticket, 0, sizeof(unsigned) * moons_mesh::kSlots);
  if (cudaMalloc(&p, sizeof(double) * moons_mesh::kSlots) != cudaSuccess) goto nomem;
  m->allocs.push_back(p);
  m->d_scal = (double*)p;
  if (cudaMallocHost(&p, sizeof(double) * moons_mesh::kSlots) != cudaSuccess) goto nomem;
  m->h_scal = (double*)p;
  *out = m;
  return MOONS_OK;
nomem:
  moons_mesh_destroy(m);
  g_err = "moons_mesh_create: device allocation failed";
  return MOONS_ERR_NOMEM;
}

int moons_mesh_destroy(moons_mesh* m) {
  if (!m) return MOONS_OK;
  mesh_unref(m);
  return MOONS_OK;
}

}  // extern "C"

namespace mg {
void mesh_ref(moons_mesh* m) { m->refs++; }
void mesh_unref(moons_mesh* m) {
  if (--m->refs > 0) return;
  cudaSetDevice(m->device);
  if (m->stream) cudaStreamSynchronize(m->stream);
  for (void* p : m->allocs) cudaFree(p);
  if (m->h_scal) cudaFreeHost(m->h_scal);
  if (m->stream) cudaStreamDestroy(m->stream);
  delete m;
}
}  // namespace mg

extern "C" {

int moons_mesh_sync(moons_mesh* m) {
  if (!m) return arg_fail("null mesh");
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_sf_create(moons_mesh* m, int dl, moons_sf** out) {
  if (!m || !out) return arg_fail("moons_sf_create: null pointer");
  if (dl < 0 || dl > 7) return arg_fail("moons_sf_create: bad data location");
  auto* s = new moons_sf();
  s->m = m;
  mesh_ref(m);
  s->f = make_df(m, dl, nullptr);
  cudaSetDevice(m->device);
  if (cudaMalloc(&s->f.f, s->f.n() * sizeof(double)) != cudaSuccess) {
    delete s;
    mesh_unref(m);
    g_err = "moons_sf_create: device allocation failed";
    return MOONS_ERR_NOMEM;
  }
  cudaMemsetAsync(s->f.f, 0, s->f.n() * sizeof(double), m->stream);
  *out = s;
  return MOONS_OK;
}
int moons_sf_destroy(moons_sf* s) {
  if (!s) return MOONS_OK;
  cudaSetDevice(s->m->device);
  cudaStreamSynchronize(s->m->stream);
  if (s->owns) cudaFree(s->f.f);
  moons_mesh* m = s->m;
  delete s;
  mesh_unref(m);
  return MOONS_OK;
}
int moons_sf_shape(const moons_sf* s, int out[3]) {
  if (!s || !out) return arg_fail("moons_sf_shape: null pointer");
  out[0] = s->f.s0;
  out[1] = s->f.s1;
  out[2] = s->f.s2;
  return MOONS_OK;
}
int moons_sf_upload(moons_sf* s, const double* h, long long n) {
  if (!s || !h) return arg_fail("moons_sf_upload: null pointer");
  if ((size_t)n != s->f.n()) {
    g_err = "moons_sf_upload: size does not match the field extents";
    return MOONS_ERR_SHAPE;
  }
  MG_CUDA(cudaMemcpyAsync(s->f.f, h, n * sizeof(double), cudaMemcpyHostToDevice, s->m->stream));
  MG_CUDA(cudaStreamSynchronize(s->m->stream));
  return MOONS_OK;
}
int moons_sf_download(const moons_sf* s, double* h, long long n) {
  if (!s || !h) return arg_fail("moons_sf_download: null pointer");
  if ((size_t)n != s->f.n()) {
    g_err = "moons_sf_download: size does not match the field extents";
    return MOONS_ERR_SHAPE;
  }
  MG_CUDA(cudaMemcpyAsync(h, s->f.f, n * sizeof(double), cudaMemcpyDeviceToHost, s->m->stream));
  MG_CUDA(cudaStreamSynchronize(s->m->stream));
  return MOONS_OK;
}
int moons_sf_fill(moons_sf* s, double v) {
  if (!s) return arg_fail("moons_sf_fill: null pointer");
  int r = launch_pw(s->m, PW_FILL, s->f, nullptr, v);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(s->m->stream));
  return MOONS_OK;
}
int moons_sf_set_bcs(moons_sf* s, const moons_bc_spec* b) {
  if (!s || !b) return arg_fail("moons_sf_set_bcs: null pointer");
  DBC bc{};
  bc.defined = 1;
  int seen = 0;
  for (int f = 1; f <= 6; f++) {
    if (b->type[f - 1] < MOONS_BC_DIRICHLET || b->type[f - 1] > MOONS_BC_ROBIN)
      return arg_fail("moons_sf_set_bcs: bad BC type");
    bc.type[f] = b->type[f - 1];
    bc.prescribed[f] = b->prescribed[f - 1];
    bc.value[f] = b->value[f - 1];
    bc.c_w[f] = b->c_w[f - 1];
    int o = b->order[f - 1];
    if (o < 1 || o > 6 || (seen & (1 << o))) return arg_fail("moons_sf_set_bcs: order must permute 1..6");
    seen |= 1 << o;
    bc.order[f] = o;
    int d = (f + 1) / 2;
    const auto& hn = s->m->hn[d - 1];
    int sn = s->m->sn[d - 1];
    bc.dh[f] = (f & 1) ? (hn[1] - hn[0]) : (hn[sn - 1] - hn[sn - 2]);
    bc.nhat[f] = (f & 1) ? -1.0 : 1.0;
    if (bc.type[f] == MOONS_BC_ROBIN && bc.c_w[f] == 0.0) return arg_fail("moons_sf_set_bcs: Robin needs c_w != 0");
  }
  s->bc = bc;
  s->all_neumann = b->all_neumann;
  return MOONS_OK;
}

int moons_apply_bcs(moons_sf* s) {
  if (!s) return arg_fail("null field");
  int r = launch_bcs(s->m, s->f, s->bc, false);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(s->m->stream));
  return MOONS_OK;
}
int moons_apply_bcs_implicit(moons_sf* s) {
  if (!s) return arg_fail("null field");
  int r = launch_bcs(s->m, s->f, s->bc, true);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(s->m->stream));
  return MOONS_OK;
}

int moons_del(moons_sf* out, const moons_sf* in, int n, int dir, int pad, int gen) {
  if (!out || !in) return arg_fail("moons_del: null field");
  if (dir < 1 || dir > 3 || gen < 1 || gen > 3 || pad < 0) return arg_fail("moons_del: bad dir/gen/pad");
  int r = launch_del(out->m, out->f, in->f, n, dir, pad, gen);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(out->m->stream));
  return MOONS_OK;
}

int moons_grad(moons_sf* gx, moons_sf* gy, moons_sf* gz, const moons_sf* u) {
  if (!gx || !gy || !gz || !u) return arg_fail("moons_grad: null field");
  moons_mesh* m = u->m;
  int r;
  if ((r = launch_del(m, gx->f, u->f, 1, 1, 0, 1))) return r;
  if ((r = launch_del(m, gy->f, u->f, 1, 2, 0, 1))) return r;
  if ((r = launch_del(m, gz->f, u->f, 1, 3, 0, 1))) return r;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_div(moons_sf* o, const moons_sf* ux, const moons_sf* uy, const moons_sf* uz) {
  if (!o || !ux || !uy || !uz) return arg_fail("moons_div: null field");
  moons_mesh* m = o->m;
  int r;
  if ((r = launch_del(m, o->f, ux->f, 1, 1, 0, 1))) return r;
  if ((r = launch_del(m, o->f, uy->f, 1, 2, 0, 2))) return r;
  if ((r = launch_del(m, o->f, uz->f, 1, 3, 0, 2))) return r;
  if ((r = mask_ghost_XPeriodic(m, o->f, o->bc.defined ? &o->bc : nullptr))) return r;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_curl(moons_sf* ox, moons_sf* oy, moons_sf* oz, const moons_sf* ux, const moons_sf* uy,
               const moons_sf* uz) {
  if (!ox || !oy || !oz || !ux || !uy || !uz) return arg_fail("moons_curl: null field");
  moons_mesh* m = ox->m;
  int r;
  // curl_SF (ops_discrete.f90:184-202)
  if ((r = launch_del(m, ox->f, uz->f, 1, 2, 0, 1))) return r;
  if ((r = launch_del(m, ox->f, uy->f, 1, 3, 0, 3))) return r;
  if ((r = launch_del(m, oy->f, ux->f, 1, 3, 0, 1))) return r;
  if ((r = launch_del(m, oy->f, uz->f, 1, 1, 0, 3))) return r;
  if ((r = launch_del(m, oz->f, uy->f, 1, 1, 0, 1))) return r;
  if ((r = launch_del(m, oz->f, ux->f, 1, 2, 0, 3))) return r;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_lap_centered(moons_sf* o, const moons_sf* u) {
  if (!o || !u) return arg_fail("moons_lap_centered: null field");
  int gz = (u->f.dl == MOONS_CC) ? ghost_zero_bits(o->bc.defined ? &o->bc : nullptr) : 0;
  int r = launch_lap_centered(o->m, o->f, u->f, gz, 0, 0.0);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(o->m->stream));
  return MOONS_OK;
}

int moons_lap_var(moons_sf* o, const moons_sf* u, const moons_sf* kx, const moons_sf* ky, const moons_sf* kz) {
  if (!o || !u || !kx || !ky || !kz) return arg_fail("moons_lap_var: null field");
  moons_mesh* m = o->m;
  // lapVarCoeff_VF: grad(tempk,u); multiply(tempk,k); div(lapU,tempk)
  double* tmp[3] = {nullptr, nullptr, nullptr};
  DF t[3];
  int r = MOONS_OK;
  for (int d = 0; d < 3; d++) {
    t[d] = make_df(m, dl_after_diff(u->f.dl, d + 1), nullptr);
    if (cudaMallocAsync((void**)&tmp[d], t[d].n() * sizeof(double), m->stream) != cudaSuccess) {
      r = MOONS_ERR_NOMEM;
      break;
    }
    t[d].f = tmp[d];
  }
  if (!r) {
    const moons_sf* ks[3] = {kx, ky, kz};
    for (int d = 0; d < 3 && !r; d++) r = launch_del(m, t[d], u->f, 1, d + 1, 0, 1);
    for (int d = 0; d < 3 && !r; d++) r = launch_pw(m, PW_MUL, t[d], &ks[d]->f, 0.0);
    if (!r) r = launch_del(m, o->f, t[0], 1, 1, 0, 1);
    if (!r) r = launch_del(m, o->f, t[1], 1, 2, 0, 2);
    if (!r) r = launch_del(m, o->f, t[2], 1, 3, 0, 2);
    if (!r) r = mask_ghost_XPeriodic(m, o->f, o->bc.defined ? &o->bc : nullptr);
  }
  for (int d = 0; d < 3; d++)
    if (tmp[d]) cudaFreeAsync(tmp[d], m->stream);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}

int moons_interp(moons_sf* o, const moons_sf* i, int dir) {
  if (!o || !i) return arg_fail("moons_interp: null field");
  if (dir < 1 || dir > 3) return arg_fail("moons_interp: bad dir");
  int r = launch_interp(o->m, o->f, i->f, dir);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(o->m->stream));
  return MOONS_OK;
}

}  // extern "C"
