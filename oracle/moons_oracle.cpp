#include <tuple>
#include <map>
#include <cstdlib>
#include <condition_variable>
#include <mutex>
#include <thread>
// moons_oracle.cpp -- CPU restatement of the MOONS hot path (TEST ORACLE).
// See moons_oracle.hpp for scope and parity status.  Citations are paths
// inside the reference project; HW = code/handwritten.
#include "moons_oracle.hpp"

#include <algorithm>
#include <cstring>
#include <functional>

namespace mo {

// ---------------------------------------------------------------------------
// fixed-chunk thread pool (CPU baseline only; see moons_oracle.hpp)
// ---------------------------------------------------------------------------
namespace {
constexpr long kChunks = 64;
thread_local bool t_in_par = false;  // a loop nested in a parallel loop runs serially
struct Pool {
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::vector<std::thread> workers;
  const std::function<void(long, long, int)>* job = nullptr;
  long n = 0, next = 0, finished = 0;
  unsigned gen = 0;
  bool quit = false;
  int nthreads = 0;
  void run_chunks() {
    for (;;) {
      long c;
      {
        std::lock_guard<std::mutex> l(mu);
        if (next >= kChunks) return;
        c = next++;
      }
      const long b = n * c / kChunks, e = n * (c + 1) / kChunks;
      if (b < e) {
        t_in_par = true;
        (*job)(b, e, (int)c);
        t_in_par = false;
      }
      std::lock_guard<std::mutex> l(mu);
      if (++finished == kChunks) done_cv.notify_all();
    }
  }
  void start(int t) {
    nthreads = t;
    for (int w = 1; w < t; w++)
      workers.emplace_back([this] {
        unsigned seen = 0;
        for (;;) {
          {
            std::unique_lock<std::mutex> l(mu);
            cv.wait(l, [&] { return quit || gen != seen; });
            if (quit) return;
            seen = gen;
          }
          run_chunks();
        }
      });
  }
  ~Pool() {
    {
      std::lock_guard<std::mutex> l(mu);
      quit = true;
    }
    cv.notify_all();
    for (auto& w : workers) w.join();
  }
};
Pool* g_pool = nullptr;
int g_threads = 0;
std::mutex g_pool_mu;
}  // namespace

int oracle_threads() {
  if (g_threads > 0) return g_threads;
  const char* e = getenv("MOONS_ORACLE_THREADS");
  int n = e ? atoi(e) : (int)std::thread::hardware_concurrency();
  return std::max(1, n);
}
void set_oracle_threads(int n) {
  std::lock_guard<std::mutex> l(g_pool_mu);
  delete g_pool;
  g_pool = nullptr;
  g_threads = std::max(1, n);
}
// fn(begin, end, chunk) over the kChunks fixed chunks of [0, n); serial
// below `min_parallel` units
void par_chunks_i(long n, long min_parallel, const std::function<void(long, long, int)>& fn) {
  const int t = oracle_threads();
  if (t <= 1 || n < min_parallel || t_in_par) {
    for (long c = 0; c < kChunks; c++) {
      const long b = n * c / kChunks, e = n * (c + 1) / kChunks;
      if (b < e) fn(b, e, (int)c);
    }
    return;
  }
  std::lock_guard<std::mutex> l(g_pool_mu);  // one parallel loop at a time
  if (!g_pool || g_pool->nthreads != t) {
    delete g_pool;
    g_pool = new Pool();
    g_pool->start(t);
  }
  Pool& P = *g_pool;
  {
    std::lock_guard<std::mutex> lk(P.mu);
    P.job = &fn;
    P.n = n;
    P.next = 0;
    P.finished = 0;
    P.gen++;
  }
  P.cv.notify_all();
  P.run_chunks();
  std::unique_lock<std::mutex> lk(P.mu);
  P.done_cv.wait(lk, [&] { return P.finished == kChunks; });
  P.job = nullptr;
}
void par_chunks(long n, const std::function<void(long, long)>& fn) {
  par_chunks_i(n, 4096, [&](long b, long e, int) { fn(b, e); });
}
// sum of f(b, e) over the fixed chunks of [0, n), added in chunk order
static double par_sum(long n, long min_parallel, const std::function<double(long, long)>& f) {
  std::vector<double> part(kChunks, 0.0);
  par_chunks_i(n, min_parallel, [&](long b, long e, int c) { part[c] = f(b, e); });
  double s = 0.0;
  for (double v : part) s += v;
  return s;
}


// ---------------------------------------------------------------------------
// coordinates: HW/grid/coordinates_extend.f90:78-173 (init_c),
// :506-523 (init_stencils_c); HW/grid/derivative_stencils.f90:31-217;
// HW/grid/interpolation_stencils.f90:12-35
// ---------------------------------------------------------------------------
static void staggered(Tri& T, const V1& dh, int s) {
  // staggered_CC2N / staggered_N2CC: D = -1/dh, U = +1/dh, size s-1
  T.D.init(s - 1);
  T.U.init(s - 1);
  T.L.init(1);
  for (int i = 1; i <= s - 1; i++) {
    T.D(i) = -(1.0 / dh(i));
    T.U(i) = 1.0 / dh(i);
  }
}

static void collocated_2(Tri& T, const V1& dh, int s, bool cc) {
  // collocated_CC_2 (cc) / collocated_Node_2, derivative_stencils.f90:110-217
  T.L.init(std::max(s - 2, 1));
  T.D.init(std::max(s - 2, 1));
  T.U.init(std::max(s - 2, 1));
  if (cc ? (s <= 2) : (s <= 3)) return;
  int i;
  if (cc) {
    i = 2;
    T.L(1) = 2.0 / ((0.5 * dh(i - 1)) * ((0.5 * dh(i - 1)) + dh(i)));
    T.D(1) = -2.0 / ((0.5 * dh(i - 1)) * dh(i));
    T.U(1) = 2.0 / (dh(i) * ((0.5 * dh(i - 1)) + dh(i)));
    for (i = 3; i <= s - 2; i++) {
      T.L(i - 1) = 2.0 / (dh(i - 1) * (dh(i - 1) + dh(i)));
      T.D(i - 1) = -(2.0 / (dh(i - 1) * dh(i)));
      T.U(i - 1) = 2.0 / (dh(i) * (dh(i - 1) + dh(i)));
    }
    i = s - 1;
    T.L(s - 2) = 2.0 / (dh(i - 1) * (dh(i - 1) + (0.5 * dh(i))));
    T.D(s - 2) = -2.0 / (dh(i - 1) * (0.5 * dh(i)));
    T.U(s - 2) = 2.0 / ((0.5 * dh(i)) * (dh(i - 1) + (0.5 * dh(i))));
  } else {
    i = 2;
    T.L(1) = 2.0 / (dh(i) * (dh(i + 1) + dh(i)));
    T.D(1) = -2.0 / (dh(i + 1) * dh(i));
    T.U(1) = 2.0 / (dh(i + 1) * (dh(i + 1) + dh(i)));
    for (i = 3; i <= s - 2; i++) {
      T.L(i - 1) = 2.0 / (dh(i - 1) * (dh(i - 1) + dh(i)));
      T.D(i - 1) = -2.0 / (dh(i - 1) * dh(i));
      T.U(i - 1) = 2.0 / (dh(i) * (dh(i - 1) + dh(i)));
    }
    i = s - 1;
    T.L(s - 2) = 2.0 / (dh(i - 2) * (dh(i - 1) + dh(i - 2)));
    T.D(s - 2) = -2.0 / (dh(i - 1) * dh(i - 2));
    T.U(s - 2) = 2.0 / (dh(i - 1) * (dh(i - 1) + dh(i - 2)));
  }
}

static void collocated_1(Tri& T, const V1& dh, int s, bool cc) {
  // collocated_CC_1 / collocated_Node_1, derivative_stencils.f90:79-180
  T.L.init(std::max(s - 2, 1));
  T.D.init(std::max(s - 2, 1));
  T.U.init(std::max(s - 2, 1));
  if (cc ? (s <= 2) : (s <= 3)) return;
  int i;
  if (cc) {
    i = 2;
    double a = 0.5 * dh(i - 1);
    T.L(1) = (-(dh(i)) / (a * (a + dh(i))));
    T.D(1) = ((-a + dh(i)) / (a * dh(i)));
    T.U(1) = (a / (dh(i) * (a + dh(i))));
    for (i = 3; i <= s - 2; i++) {
      T.L(i - 1) = (-dh(i) / (dh(i - 1) * (dh(i - 1) + dh(i))));
      T.D(i - 1) = ((-dh(i - 1) + dh(i)) / (dh(i - 1) * dh(i)));
      T.U(i - 1) = (dh(i - 1) / (dh(i) * (dh(i - 1) + dh(i))));
    }
    i = s - 1;
    double b = 0.5 * dh(i);
    T.L(s - 2) = (-b / (dh(i - 1) * (dh(i - 1) + b)));
    T.D(s - 2) = ((-dh(i - 1) + b) / (dh(i - 1) * b));
    T.U(s - 2) = (dh(i - 1) / (b * (dh(i - 1) + b)));
  } else {
    i = 2;
    T.L(1) = -(dh(i + 1) + 2.0 * dh(i)) / (dh(i) * (dh(i + 1) + dh(i)));
    T.D(1) = (dh(i + 1) + dh(i)) / (dh(i + 1) * dh(i));
    T.U(1) = -dh(i) / (dh(i + 1) * (dh(i + 1) + dh(i)));
    for (i = 3; i <= s - 2; i++) {
      T.L(i - 1) = -((dh(i) / (dh(i - 1) * (dh(i - 1) + dh(i)))));
      T.D(i - 1) = (((-dh(i - 1) + dh(i)) / (dh(i - 1) * dh(i))));
      T.U(i - 1) = ((dh(i - 1) / (dh(i) * (dh(i - 1) + dh(i)))));
    }
    i = s - 1;
    T.L(s - 2) = dh(i - 1) / (dh(i - 2) * (dh(i - 1) + dh(i - 2)));
    T.D(s - 2) = -(dh(i - 1) + dh(i - 2)) / (dh(i - 1) * dh(i - 2));
    T.U(s - 2) = (2.0 * dh(i - 1) + dh(i - 2)) / (dh(i - 1) * (dh(i - 1) + dh(i - 2)));
  }
}

void Coord::init(const double* h, int sn_in) {
  if (sn_in < 3) throw std::runtime_error("coordinates need >= 3 nodes (typical init)");
  sn = sn_in;
  hn.init(sn);
  for (int i = 1; i <= sn; i++) hn(i) = h[i - 1];
  dhn.init(sn - 1);
  for (int i = 1; i <= sn - 1; i++) dhn(i) = hn(i + 1) - hn(i);
  sc = sn - 1;
  hc.init(sc);
  for (int i = 1; i <= sn - 1; i++) hc(i) = (hn(i + 1) + hn(i)) / 2.0;
  dhc.init(sc - 1);
  for (int i = 1; i <= sc - 1; i++) dhc(i) = hc(i + 1) - hc(i);
  // interpolation_stencil: D = (hn(i+1)-hc(i))/(hc(i+1)-hc(i)), U = 1-D
  theta.D.init(sc - 1);
  theta.U.init(sc - 1);
  theta.L.init(1);
  for (int i = 1; i <= sc - 1; i++) {
    theta.D(i) = (hn(i + 1) - hc(i)) / (hc(i + 1) - hc(i));
    theta.U(i) = 1.0 - theta.D(i);
  }
  staggered(stagCC2N, dhc, sc);
  staggered(stagN2CC, dhn, sn);
  collocated_1(colCC[0], dhc, sc, true);
  collocated_2(colCC[1], dhc, sc, true);
  collocated_1(colN[0], dhn, sn, false);
  collocated_2(colN[1], dhn, sn, false);
}

// data_location: N_eye
std::array<int, 3> dl_eye(int dl) {
  switch (dl) {
    case 0: return {0, 0, 0};
    case 1: return {1, 0, 0};
    case 2: return {0, 1, 0};
    case 3: return {0, 0, 1};
    case 4: return {0, 1, 1};
    case 5: return {1, 0, 1};
    case 6: return {1, 1, 0};
    case 7: return {1, 1, 1};
  }
  throw std::runtime_error("bad data location");
}

void SF::init(const Grid& g, int dl_) {
  dl = dl_;
  auto e = dl_eye(dl);
  for (int d = 0; d < 3; d++) s[d + 1] = e[d] ? g.c[d].sn : g.c[d].sc;
  f.assign((size_t)s[1] * s[2] * s[3], 0.0);
}

// ---------------------------------------------------------------------------
// BC setup: boundary_conditions_extend.f90:120-340; face_SD_extend.f90:37-84
// (dh(face) = width of the cell next to the boundary; nhat = -1,+1)
// ---------------------------------------------------------------------------
void set_bcs(SF& u, const Grid& g, const int type[6], const int prescribed[6],
             const double value[6], const double c_w[6], const int order[6]) {
  auto b = std::make_shared<BCs>();
  b->defined = true;
  bool alln = true;
  for (int f = 1; f <= 6; f++) {
    b->type[f] = type[f - 1];
    b->prescribed[f] = prescribed ? prescribed[f - 1] : 0;
    b->value[f] = value ? value[f - 1] : 0.0;
    b->c_w[f] = c_w ? c_w[f - 1] : 0.0;
    b->order[f] = order ? order[f - 1] : f;
    int d = (f + 1) / 2;
    const Coord& c = g.c[d - 1];
    b->dh[f] = (f % 2 == 1) ? c.dhn(1) : c.dhn(c.sn - 1);
    b->nhat[f] = (f % 2 == 1) ? -1.0 : 1.0;
    if (type[f - 1] != BC_NEUMANN) alln = false;
  }
  b->all_neumann = alln;
  // block_field_extend.f90:340-346 many_cell
  for (int d = 1; d <= 3; d++) {
    bool L1 = N_along(u.dl, d), L2 = CC_along(u.dl, d);
    b->many_cell[d] = (L1 && u.s[d] > 4) || (L2 && u.s[d] > 3);
  }
  u.bc = b;
}

// ---------------------------------------------------------------------------
// pointwise ops (HW/grid_field/GF_3D/*)
// ---------------------------------------------------------------------------
void assign(SF& a, double v) { std::fill(a.f.begin(), a.f.end(), v); }
void assign(SF& a, const SF& b) {
  if (a.f.size() != b.f.size()) {
    a.f = b.f;
    return;
  }
  par_chunks((long)a.n(), [&](long s, long e) { std::copy(b.f.begin() + s, b.f.begin() + e, a.f.begin() + s); });
}
void add(SF& a, const SF& b) {
  par_chunks((long)a.n(), [&](long s, long e) {
    for (long i = s; i < e; i++) a.f[i] += b.f[i];
  });
}
void subtract(SF& a, const SF& b) {
  par_chunks((long)a.n(), [&](long s, long e) {
    for (long i = s; i < e; i++) a.f[i] -= b.f[i];
  });
}
void multiply(SF& a, const SF& b) {
  par_chunks((long)a.n(), [&](long s, long e) {
    for (long i = s; i < e; i++) a.f[i] *= b.f[i];
  });
}
void multiply(SF& a, double c) {
  par_chunks((long)a.n(), [&](long s, long e) {
    for (long i = s; i < e; i++) a.f[i] *= c;
  });
}
void add_product(SF& a, const SF& b, double c) {  // GF_add_product.f90:13-30
  par_chunks((long)a.n(), [&](long s, long e) {
    for (long i = s; i < e; i++) a.f[i] = a.f[i] + b.f[i] * c;
  });
}
void product_add(SF& a, double c, const SF& b) {  // GF_product_add.f90:14-30
  par_chunks((long)a.n(), [&](long s, long e) {
    for (long i = s; i < e; i++) a.f[i] = a.f[i] * c + b.f[i];
  });
}
// sum_GF_pad (GF_aux.f90:140-160, _PARALLELIZE_GF_ branch: 1+pad..s-pad);
// plane sums added in k order (fixed chunks of planes)
double sum_pad(const SF& a, int pad) {
  const int k0 = 1 + pad, nk = a.s[3] - 2 * pad;
  return par_sum(std::max(nk, 0), 8, [&](long b, long e) {
    double m = 0;
    for (int k = k0 + (int)b; k < k0 + (int)e; k++)
      for (int j = 1 + pad; j <= a.s[2] - pad; j++)
        for (int i = 1 + pad; i <= a.s[1] - pad; i++) m += a(i, j, k);
    return m;
  });
}

// volume_DL_GF (GF_distributions.f90:61-88) + volume_SF (SF_extend.f90:571-581)
void volume(SF& u, const Grid& g) {
  assign(u, 0.0);
  auto e = dl_eye(u.dl);
  const V1* dh[3];
  for (int d = 0; d < 3; d++) dh[d] = e[d] ? &g.c[d].dhc : &g.c[d].dhn;
  for (int k = 2; k <= u.s[3] - 1; k++)
    for (int j = 2; j <= u.s[2] - 1; j++)
      for (int i = 2; i <= u.s[1] - 1; i++)
        u(i, j, k) = (*dh[0])(i - e[0]) * (*dh[1])(j - e[1]) * (*dh[2])(k - e[2]);
  double s = 0;
  for (double v : u.f) s += v;
  u.vol = s;
}

// plane helpers
static void plane_op(SF& u, int dir, int idx, double v, bool mul) {
  int a = dir == 1 ? 2 : 1, b = dir == 3 ? 2 : 3;
  int ia[4];
  for (int y = 1; y <= u.s[b]; y++)
    for (int x = 1; x <= u.s[a]; x++) {
      ia[dir] = idx;
      ia[a] = x;
      ia[b] = y;
      double& r = u(ia[1], ia[2], ia[3]);
      r = mul ? r * v : v;
    }
}
static inline int face_dir(int f) { return (f + 1) / 2; }
static inline bool is_min(int f) { return f % 2 == 1; }

// assign_ghost_XPeriodic (block_field_extend.f90:232-276, :832-870)
void assign_ghost_XPeriodic(SF& u, double v, const SF* w) {
  const SF& o = w ? *w : u;
  for (int f = 1; f <= 6; f++) {
    int d = face_dir(f);
    bool apply = o.has_bcs() ? (o.bc->type[f] != BC_PERIODIC) : true;
    if (apply) plane_op(u, d, is_min(f) ? 1 : u.s[d], v, false);
  }
}
// assign_ghost_N_XPeriodic: only defined when BCs are defined
void assign_ghost_N_XPeriodic(SF& u, double v, const SF* w) {
  const SF& o = w ? *w : u;
  if (!o.has_bcs()) return;
  for (int f = 1; f <= 6; f++) {
    int d = face_dir(f);
    if (o.bc->type[f] != BC_PERIODIC && N_along(o.dl, d))
      plane_op(u, d, is_min(f) ? 1 : u.s[d], v, false);
  }
}
// assign_wall_Dirichlet (block_field_extend.f90:278-310)
void assign_wall_Dirichlet(SF& u, double v, const SF* w) {
  const SF& o = w ? *w : u;
  for (int f = 1; f <= 6; f++) {
    int d = face_dir(f);
    if (!N_along(o.dl, d)) continue;
    bool apply = o.has_bcs() ? (o.bc->type[f] == BC_DIRICHLET) : true;
    if (apply) plane_op(u, d, is_min(f) ? 2 : u.s[d] - 1, v, false);
  }
}
// multiply_wall_Neumann (block_field_extend.f90:350-375)
void multiply_wall_Neumann(SF& u, double v, const SF* w) {
  const SF& o = w ? *w : u;
  for (int f = 1; f <= 6; f++) {
    int d = face_dir(f);
    if (!N_along(o.dl, d)) continue;
    bool apply = o.has_bcs() ? (o.bc->type[f] == BC_NEUMANN) : true;
    if (apply) plane_op(u, d, is_min(f) ? 2 : u.s[d] - 1, v, true);
  }
}
// assign_wall_Periodic_single (block_field_extend.f90:312-338)
void assign_wall_Periodic_single(SF& u, double v, const SF* w) {
  const SF& o = w ? *w : u;
  if (!o.has_bcs()) return;
  for (int d = 1; d <= 3; d++) {
    bool L = N_along(o.dl, d) && o.bc->type[2 * d - 1] == BC_PERIODIC &&
             o.bc->type[2 * d] == BC_PERIODIC && o.s[d] > 4;
    if (L) plane_op(u, d, u.s[d] - 1, v, false);
  }
}
void assign_ghost_dir(SF& u, double v, int dir) {
  plane_op(u, dir, 1, v, false);
  plane_op(u, dir, u.s[dir], v, false);
}

// ---------------------------------------------------------------------------
// BCs: HW/BCs/apply/apply_BCs.f90:31-64, HW/BCs/direct/apply_BCs_faces_raw.f90,
// HW/BCs/direct/apply_BCs_faces_bridge.f90 (index sets from
// HW/sub_domain/face_SD_extend.f90:37-84); implicit: HW/BCs/implicit/*
// ---------------------------------------------------------------------------
struct FaceIdx {
  int G, B, I, Iopp, Gp, Ip;  // plane indices along the face direction
};
static FaceIdx face_idx(const SF& u, int f) {
  int d = face_dir(f), s = u.s[d];
  bool mn = is_min(f);
  FaceIdx r{};
  if (CC_along(u.dl, d)) {
    r.G = mn ? 1 : s;
    r.I = mn ? 2 : s - 1;
    r.Iopp = mn ? s - 1 : 2;  // I_OPP(face) = I(opp face)
    r.B = 0;
    r.Gp = r.G;
    r.Ip = r.Iopp;
  } else {
    r.G = mn ? 1 : s;
    r.B = mn ? 2 : s - 1;
    r.I = mn ? 3 : s - 2;
    r.Iopp = mn ? s - 2 : 3;
    // periodic N: many-cell max face uses boundary planes (face_SD_extend.f90:72-79)
    bool many = s > 4;
    if (!mn && many) {
      r.Gp = s - 1;
      r.Ip = 2;
    } else {
      r.Gp = r.G;
      r.Ip = r.Iopp;
    }
  }
  return r;
}

template <class F>
static void plane_loop(SF& u, int d, F&& fn) {
  int a = d == 1 ? 2 : 1, b = d == 3 ? 2 : 3;
  for (int y = 1; y <= u.s[b]; y++)
    for (int x = 1; x <= u.s[a]; x++) fn(a, b, x, y);
}

static void apply_face(SF& u, int f, bool implicit) {
  const BCs& bc = *u.bc;
  int d = face_dir(f);
  int t = bc.type[f];
  bool N = N_along(u.dl, d);
  FaceIdx ix = face_idx(u, f);
  double b = implicit ? 0.0 : bc.value[f];
  double dh = bc.dh[f], nhat = bc.nhat[f], cw = bc.c_w[f];
  bool pres = bc.prescribed[f] != 0;
  auto at = [&](int a, int bb, int x, int y, int p) -> double& {
    int ia[4];
    ia[d] = p;
    ia[a] = x;
    ia[bb] = y;
    return u(ia[1], ia[2], ia[3]);
  };
  plane_loop(u, d, [&](int a, int bb, int x, int y) {
    switch (t) {
      case BC_DIRICHLET:
        if (!N) {  // Dirichlet_C: ug = 2b - ui ; implicit: ug = -ui
          at(a, bb, x, y, ix.G) = implicit ? -at(a, bb, x, y, ix.I) : 2.0 * b - at(a, bb, x, y, ix.I);
        } else {   // Dirichlet_N: ub = b; ug = 2ub - ui ; implicit: ub = 0; ug = -ui
          if (implicit) {
            at(a, bb, x, y, ix.B) = 0.0;
            at(a, bb, x, y, ix.G) = -at(a, bb, x, y, ix.I);
          } else {
            at(a, bb, x, y, ix.B) = b;
            at(a, bb, x, y, ix.G) = 2.0 * at(a, bb, x, y, ix.B) - at(a, bb, x, y, ix.I);
          }
        }
        break;
      case BC_NEUMANN:
        if (implicit) {
          at(a, bb, x, y, ix.G) = at(a, bb, x, y, ix.I);
        } else if (!N) {  // ug = ui + b*dh*nhat
          at(a, bb, x, y, ix.G) = at(a, bb, x, y, ix.I) + b * (dh * nhat);
        } else {          // ug = ui + 2*b*dh*nhat
          at(a, bb, x, y, ix.G) = at(a, bb, x, y, ix.I) + 2.0 * b * (dh * nhat);
        }
        break;
      case BC_PERIODIC:
        if (!N) {
          if (pres && !implicit) at(a, bb, x, y, ix.G) = b;  // Periodic_C_prescribed
          else at(a, bb, x, y, ix.G) = at(a, bb, x, y, ix.Iopp);
        } else {
          if (pres && !implicit) at(a, bb, x, y, ix.G) = b;  // Periodic_N_prescribed (G)
          else at(a, bb, x, y, ix.Gp) = at(a, bb, x, y, ix.Ip);
        }
        break;
      case BC_ROBIN:
        if (!N) {  // Robin_C: coeff_1 = (2 c_w nhat/dh - 1)/(2 c_w nhat/dh + 1), coeff_2 = 0
          double c1 = (2.0 * cw * nhat / dh - 1.0) / (2.0 * cw * nhat / dh + 1.0);
          at(a, bb, x, y, ix.G) = at(a, bb, x, y, ix.I) * c1 + (implicit ? 0.0 : b * 0.0);
        } else {   // Robin_N: ug = ui + ub*(-2 dh/c_w nhat) + b*(2 dh/c_w nhat)
          if (implicit) {
            double c1 = -2.0 * dh * nhat / cw;
            at(a, bb, x, y, ix.G) = at(a, bb, x, y, ix.I) + at(a, bb, x, y, ix.B) * c1;
          } else {
            double c1 = -2.0 * dh / cw * nhat, c2 = 2.0 * dh / cw * nhat;
            at(a, bb, x, y, ix.G) = at(a, bb, x, y, ix.I) + at(a, bb, x, y, ix.B) * c1 + b * c2;
          }
        }
        break;
      default: break;
    }
  });
}

void apply_BCs(SF& u) {
  if (!u.has_bcs()) return;
  for (int o = 1; o <= 6; o++) apply_face(u, u.bc->order[o], false);
}
void apply_BCs_implicit(SF& u) {
  if (!u.has_bcs()) return;
  for (int o = 1; o <= 6; o++) apply_face(u, u.bc->order[o], true);
}

// ---------------------------------------------------------------------------
// del: HW/ops/ops_del.f90:59-288 with the pencil stencils of
// HW/stencils/stencils.f90:47-206
// ---------------------------------------------------------------------------
static void pencil_ops(SF& out, const SF& in, int dir, int pad,
                       const std::function<void(std::vector<double>&, const std::vector<double>&)>& op) {
  int a = dir == 1 ? 2 : 1, b = dir == 3 ? 2 : 3;
  int sin_ = in.s[dir], sout = out.s[dir];
  // loops over the input's transverse extents (diff_stag/diff_col use f%s);
  // pencils are independent, so they are cut into chunks of y
  const int y0 = 1 + pad, ny = in.s[b] - 2 * pad;
  par_chunks_i(std::max(ny, 0), 8, [&](long cb, long ce, int) {
  std::vector<double> pin(sin_ + 1), pout(sout + 1);
  for (int y = y0 + (int)cb; y < y0 + (int)ce; y++) {
    for (int x = 1 + pad; x <= in.s[a] - pad; x++) {
      int ia[4];
      ia[a] = x;
      ia[b] = y;
      for (int t = 1; t <= sin_; t++) {
        ia[dir] = t;
        pin[t] = in(ia[1], ia[2], ia[3]);
      }
      for (int t = 1; t <= sout; t++) {
        ia[dir] = t;
        pout[t] = out(ia[1], ia[2], ia[3]);
      }
      op(pout, pin);
      for (int t = 1; t <= sout; t++) {
        ia[dir] = t;
        out(ia[1], ia[2], ia[3]) = pout[t];
      }
    }
  }
  });
}

void del(SF& out, const SF& in, const Grid& g, int n, int dir, int pad, int gen) {
  const Coord& c = g.c[dir - 1];
  bool fc = CC_along(in.dl, dir), oc = CC_along(out.dl, dir);
  int diffType;
  if (fc && oc) diffType = 1;
  else if (!fc && !oc) diffType = 2;
  else if (fc && !oc) diffType = 3;
  else diffType = 4;
  double sgn = (gen == 3) ? -1.0 : 1.0;
  if (diffType >= 3) {
    const Tri& T = diffType == 3 ? c.stagCC2N : c.stagN2CC;
    int gt = diffType == 3 ? 1 : 0;
    pencil_ops(out, in, dir, pad, [&](std::vector<double>& d, const std::vector<double>& f) {
      int s = (int)f.size() - 1, sd = (int)d.size() - 1;
      d[1] = 0.0;
      d[sd] = 0.0;
      for (int i = 1; i <= s - 1; i++) {
        double v = f[i] * T.D(i) + f[i + 1] * T.U(i);
        if (gen == 1) d[i + gt] = v;
        else if (gen == 2) d[i + gt] = d[i + gt] + v;
        else d[i + gt] = d[i + gt] - v;
      }
    });
  } else {
    const Tri& T = diffType == 1 ? c.colCC[n - 1] : c.colN[n - 1];
    bool cc = diffType == 1;
    int pad1 = 0, pad2 = 0;
    pencil_ops(out, in, dir, pad, [&](std::vector<double>& d, const std::vector<double>& f) {
      int s = (int)f.size() - 1;
      auto put = [&](int i, double v) {
        if (gen == 1) d[i] = v;
        else d[i] = d[i] + sgn * v;
      };
      for (int i = 3; i <= s - 2; i++)
        put(i, f[i - 1] * T.L(i - 1) + f[i] * T.D(i - 1) + f[i + 1] * T.U(i - 1));
      if (cc) {
        put(2, 0.5 * (f[1] + f[2]) * T.L(1) * (1.0 - pad1) + f[1] * T.L(1) * pad1 + f[2] * T.D(1) +
                   f[3] * T.U(1));
        put(s - 1, f[s - 2] * T.L(s - 2) + f[s - 1] * T.D(s - 2) +
                       0.5 * (f[s - 1] + f[s]) * T.U(s - 2) * (1.0 - pad2) + f[s] * T.U(s - 2) * pad2);
      } else {
        put(2, f[2 - pad1] * T.L(1) + f[3 - pad1] * T.D(1) + f[4 - pad1] * T.U(1));
        put(s - 1, f[s - 3 + pad2] * T.L(s - 2) + f[s - 2 + pad2] * T.D(s - 2) +
                       f[s - 1 + pad2] * T.U(s - 2));
      }
      d[1] = 0.0;
      d[s] = 0.0;
    });
  }
  if (gen == 1 && pad > 0) {  // ops_del.f90:215-229
    for (int t = 1; t <= 3; t++)
      if (t != dir) assign_ghost_dir(out, 0.0, t);
  }
}

// grad_SF (ops_discrete.f90:173-182)
void grad(SF& gx, SF& gy, SF& gz, const SF& u, const Grid& g) {
  del(gx, u, g, 1, 1, 0, 1);
  del(gy, u, g, 1, 2, 0, 1);
  del(gz, u, g, 1, 3, 0, 1);
}
// div_SF (ops_discrete.f90:158-171)
void div(SF& out, const SF& ux, const SF& uy, const SF& uz, const Grid& g) {
  del(out, ux, g, 1, 1, 0, 1);
  del(out, uy, g, 1, 2, 0, 2);
  del(out, uz, g, 1, 3, 0, 2);
  assign_ghost_XPeriodic(out, 0.0, nullptr);
}
// curl_SF (ops_discrete.f90:184-202)
void curl_comp(SF& o, const SF& u, const SF& v, const SF& w, const Grid& g, int dir) {
  switch (dir) {
    case 1: del(o, w, g, 1, 2, 0, 1); del(o, v, g, 1, 3, 0, 3); break;
    case 2: del(o, u, g, 1, 3, 0, 1); del(o, w, g, 1, 1, 0, 3); break;
    case 3: del(o, v, g, 1, 1, 0, 1); del(o, u, g, 1, 2, 0, 3); break;
  }
}
void curl(SF& ox, SF& oy, SF& oz, const SF& ux, const SF& uy, const SF& uz, const Grid& g) {
  curl_comp(ox, ux, uy, uz, g, 1);
  curl_comp(oy, ux, uy, uz, g, 2);
  curl_comp(oz, ux, uy, uz, g, 3);
}

static int dl_after_diff(int dl, int dir) {  // flip location along dir
  auto e = dl_eye(dl);
  e[dir - 1] ^= 1;
  for (int d = 0; d < 8; d++)
    if (dl_eye(d) == e) return d;
  return -1;
}

// lap_centered_SF_new (ops_discrete.f90:124-132) for CC data;
// lap_centered_SF_given_both (:112-122) for staggered data (what
// lap_centered_VF_new applies per component).  Both are div(grad) through
// staggered temporaries; div_SF's ghost zeroing applies only to the SF_new
// (CC) form.
// operator temporaries kept between calls (every entry that the second
// pass reads was written by the first, a del "assign", in the same call)
static SF& temp_sf(const Grid& g, int dl, int slot) {
  static thread_local std::map<std::tuple<const Grid*, int, int>, SF> cache;
  SF& t = cache[std::make_tuple(&g, dl, slot)];
  auto e = dl_eye(dl);
  bool same = !t.f.empty() && t.dl == dl;
  for (int d = 0; d < 3 && same; d++) same = t.s[d + 1] == (e[d] ? g.c[d].sn : g.c[d].sc);
  if (!same) t.init(g, dl);
  return t;
}

void lap_centered(SF& out, const SF& u, const Grid& g) {
  SF& t0 = temp_sf(g, dl_after_diff(u.dl, 1), 1);
  SF& t1 = temp_sf(g, dl_after_diff(u.dl, 2), 2);
  SF& t2 = temp_sf(g, dl_after_diff(u.dl, 3), 3);
  if (u.dl == 0) {
    grad(t0, t1, t2, u, g);
    div(out, t0, t1, t2, g);
  } else {
    del(t0, u, g, 1, 1, 0, 1);
    del(out, t0, g, 1, 1, 0, 1);
    del(t1, u, g, 1, 2, 0, 1);
    del(out, t1, g, 1, 2, 0, 2);
    del(t2, u, g, 1, 3, 0, 1);
    del(out, t2, g, 1, 3, 0, 2);
  }
}
// lapUniformCoeff_SF (ops_discrete.f90:101-110)
void lap_uniform_coeff(SF& out, const SF& u, const Grid& g) {
  del(out, u, g, 2, 1, 0, 1);
  del(out, u, g, 2, 2, 0, 2);
  del(out, u, g, 2, 3, 0, 2);
}
// lapVarCoeff_VF (ops_discrete.f90:275-285)
void lap_var(SF& out, const SF& u, const SF& kx, const SF& ky, const SF& kz, const Grid& g) {
  SF& t0 = temp_sf(g, dl_after_diff(u.dl, 1), 4);
  SF& t1 = temp_sf(g, dl_after_diff(u.dl, 2), 5);
  SF& t2 = temp_sf(g, dl_after_diff(u.dl, 3), 6);
  grad(t0, t1, t2, u, g);
  multiply(t0, kx);
  multiply(t1, ky);
  multiply(t2, kz);
  div(out, t0, t1, t2, g);
}

// interpO2_SF (ops_interp.f90:190-220) -> interp_C2N_GF / interp_N2C_GF
// (HW/grid_field/GF_interp/GF_interp.f90:19-76) + extrap_staggered_GF
// (GF_extrap.f90:17-46)
void interp(SF& N, const SF& C, const Grid& g, int dir) {
  int e[4] = {0, 0, 0, 0};
  e[dir] = 1;
  if (N_along(N.dl, dir) && CC_along(C.dl, dir)) {
    const Coord& c = g.c[dir - 1];
    for (int k = 1; k <= C.s[3] - e[3]; k++)
      for (int j = 1; j <= C.s[2] - e[2]; j++)
        for (int i = 1; i <= C.s[1] - e[1]; i++) {
          int t = i * e[1] + j * e[2] + k * e[3];
          N(i + e[1], j + e[2], k + e[3]) =
              C(i + e[1], j + e[2], k + e[3]) * c.theta.D(t) + C(i, j, k) * c.theta.U(t);
        }
    // extrapolation of the two end planes
    int a = dir == 1 ? 2 : 1, b = dir == 3 ? 2 : 3;
    for (int y = 1; y <= N.s[b]; y++)
      for (int x = 1; x <= N.s[a]; x++) {
        int in_[4], ic[4];
        in_[a] = ic[a] = x;
        in_[b] = ic[b] = y;
        in_[dir] = 2;
        double n2 = N(in_[1], in_[2], in_[3]);
        ic[dir] = 1;
        in_[dir] = 1;
        N(in_[1], in_[2], in_[3]) = 2.0 * C(ic[1], ic[2], ic[3]) - n2;
        in_[dir] = N.s[dir] - 1;
        double nm = N(in_[1], in_[2], in_[3]);
        ic[dir] = C.s[dir];
        in_[dir] = N.s[dir];
        N(in_[1], in_[2], in_[3]) = 2.0 * C(ic[1], ic[2], ic[3]) - nm;
      }
  } else if (CC_along(N.dl, dir) && N_along(C.dl, dir)) {
    // here N is the CC output and C the node input (names kept from the caller)
    SF& out = N;
    const SF& in = C;
    for (int k = 1; k <= in.s[3] - e[3]; k++)
      for (int j = 1; j <= in.s[2] - e[2]; j++)
        for (int i = 1; i <= in.s[1] - e[1]; i++)
          out(i, j, k) = 0.5 * (in(i, j, k) + in(i + e[1], j + e[2], k + e[3]));
  } else {
    throw std::runtime_error("bad DLs in interp");
  }
}

// ---------------------------------------------------------------------------
// PCG: HW/PCG/PCG_solver_extend.f90:51-291,
//      HW/solvers/PCG/PCG_solver_algorithm.f90:37-179,
//      HW/solvers/PCG/PCG_aux.f90:30-107,
//      HW/solvers/matrix_free_operators.f90, HW/solvers/preconditioners/*,
//      HW/grid_field/GF_diagonals.f90
// ---------------------------------------------------------------------------
static SF like(const Grid& g, const SF& x) {
  SF t;
  t.init(g, x.dl);
  return t;
}

void PCG::init(const Grid& g_, int op_, int prec_, int nc_, SF* const* x, SF* const* xbc,
               SF* const* kin, double coeff_implicit) {
  g = &g_;
  op = op_;
  prec = prec_;
  nc = nc_;
  p.clear(); x_BC.clear(); r.clear(); Ax.clear(); vol.clear(); z.clear(); Minv.clear(); tempx.clear();
  k.clear(); tempk.clear();
  for (int c = 0; c < nc; c++) {
    tempx.push_back(like(*g, *x[c]));       // no BCs
    SF pp = like(*g, *x[c]);
    pp.bc = x[c]->bc;                       // init(PCG%p,x) copies BCs
    p.push_back(pp);
    SF xb = like(*g, *xbc[c]);
    xb.bc = xbc[c]->bc;
    x_BC.push_back(xb);
    r.push_back(like(*g, *x[c]));
    Ax.push_back(like(*g, *x[c]));
    SF v = like(*g, *x[c]);
    volume(v, *g);
    vol.push_back(v);
    z.push_back(like(*g, *x[c]));
    Minv.push_back(like(*g, *x[c]));
  }
  int nk = (op == OP_LAP_PROPS || op == OP_IND_DIFFUSION || op == OP_NRG_DIFFUSION) ? 3 : 0;
  for (int c = 0; c < nk; c++) {
    k.push_back(*kin[c]);
    SF t = like(*g, *kin[c]);
    tempk.push_back(t);
  }
  coeff = coeff_implicit;
  compute_prec();  // PCG%prec(PCG%Minv,m,k,MFP%coeff_implicit,PCG%tempx)
}

void PCG::update_MFP(double c, bool update_prec) {
  coeff = c;
  if (update_prec) compute_prec();
}

// laplacian_diagonal (GF_diagonals.f90:15-35)
static void lap_diag(SF& d, const Grid& g) {
  assign(d, 0.0);
  auto e = dl_eye(d.dl);
  const Coord *cx = &g.c[0], *cy = &g.c[1], *cz = &g.c[2];
  int px = e[0], py = e[1], pz = e[2];
  for (int k = 2; k <= d.s[3] - 1; k++)
    for (int j = 2; j <= d.s[2] - 1; j++)
      for (int i = 2; i <= d.s[1] - 1; i++)
        d(i, j, k) = cx->stagN2CC.D(i) * cx->stagCC2N.U(i - 1) + cx->stagN2CC.U(i - px) * cx->stagCC2N.D(i - px) +
                     cy->stagN2CC.D(j) * cy->stagCC2N.U(j - 1) + cy->stagN2CC.U(j - py) * cy->stagCC2N.D(j - py) +
                     cz->stagN2CC.D(k) * cz->stagCC2N.U(k - 1) + cz->stagN2CC.U(k - pz) * cz->stagCC2N.D(k - pz);
}
// curl_curl_diagonal (GF_diagonals.f90:37-71)
static void curl_curl_diag(SF& dx, SF& dy, SF& dz, const Grid& g, const SF& sx, const SF& sy, const SF& sz) {
  assign(dx, 0.0);
  assign(dy, 0.0);
  assign(dz, 0.0);
  const Coord &c1 = g.c[0], &c2 = g.c[1], &c3 = g.c[2];
  for (int k = 2; k <= dx.s[3] - 1; k++)
    for (int j = 2; j <= dx.s[2] - 1; j++)
      for (int i = 2; i <= dx.s[1] - 1; i++)
        dx(i, j, k) = -c2.stagN2CC.D(j) * sz(i, j, k) * c2.stagCC2N.U(j - 1) -
                      c2.stagN2CC.U(j) * sz(i, j + 1, k) * c2.stagCC2N.D(j) -
                      c3.stagN2CC.D(k) * sy(i, j, k) * c3.stagCC2N.U(k - 1) -
                      c3.stagN2CC.U(k) * sy(i, j, k + 1) * c3.stagCC2N.D(k);
  for (int k = 2; k <= dy.s[3] - 1; k++)
    for (int j = 2; j <= dy.s[2] - 1; j++)
      for (int i = 2; i <= dy.s[1] - 1; i++)
        dy(i, j, k) = -c1.stagN2CC.D(i) * sz(i, j, k) * c1.stagCC2N.U(i - 1) -
                      c1.stagN2CC.U(i) * sz(i + 1, j, k) * c1.stagCC2N.D(i) -
                      c3.stagN2CC.D(k) * sx(i, j, k) * c3.stagCC2N.U(k - 1) -
                      c3.stagN2CC.U(k) * sx(i, j, k + 1) * c3.stagCC2N.D(k);
  for (int k = 2; k <= dz.s[3] - 1; k++)
    for (int j = 2; j <= dz.s[2] - 1; j++)
      for (int i = 2; i <= dz.s[1] - 1; i++)
        dz(i, j, k) = -c1.stagN2CC.D(i) * sy(i, j, k) * c1.stagCC2N.U(i - 1) -
                      c1.stagN2CC.U(i) * sy(i + 1, j, k) * c1.stagCC2N.D(i) -
                      c2.stagN2CC.D(j) * sx(i, j, k) * c2.stagCC2N.U(j - 1) -
                      c2.stagN2CC.U(j) * sx(i, j + 1, k) * c2.stagCC2N.D(j);
}

void PCG::compute_prec() {
  // preconditioners.f90:27-129; Minv has no BCs, so assign_ghost_XPeriodic
  // zeroes all six ghost planes.
  if (prec == PREC_IDENTITY) {
    for (auto& m : Minv) assign(m, 1.0);
    return;
  }
  if (prec == PREC_IND) {
    curl_curl_diag(Minv[0], Minv[1], Minv[2], *g, k[0], k[1], k[2]);
  }
  for (int c = 0; c < nc; c++) {
    SF& M = Minv[c];
    SF tv = like(*g, M);
    if (prec == PREC_LAP) {
      lap_diag(M, *g);
    } else if (prec == PREC_MOM) {
      assign(M, 0.0);
      lap_diag(M, *g);
      multiply(M, coeff);
      for (auto& v : M.f) v += 1.0;
    } else if (prec == PREC_IND) {
      multiply(M, coeff);
      for (auto& v : M.f) v += 1.0;
    }
    volume(tv, *g);
    multiply(M, tv);
    for (auto& v : M.f) v = 1.0 / v;
    assign_ghost_XPeriodic(M, 0.0, nullptr);
  }
}

// operator_explicit (matrix_free_operators.f90) on component fields
void PCG::apply_operator(std::vector<SF>& A, std::vector<SF>& x, bool explicit_only) {
  if (!explicit_only)
    for (auto& xc : x) apply_BCs_implicit(xc);
  switch (op) {
    case OP_LAP_UNIFORM:
      for (int c = 0; c < nc; c++) lap_centered(A[c], x[c], *g);
      break;
    case OP_LAP_PROPS:
      lap_var(A[0], x[0], k[0], k[1], k[2], *g);
      break;
    case OP_NRG_DIFFUSION:
      // nrg_diffusion_explicit (matrix_free_operators.f90:148-162):
      // grad(tempk,x); multiply(tempk,k); div(Ax,tempk); multiply(Ax,coeff); add(Ax,x)
      lap_var(A[0], x[0], k[0], k[1], k[2], *g);
      multiply(A[0], coeff);
      add(A[0], x[0]);
      break;
    case OP_MOM_DIFFUSION:
      for (int c = 0; c < nc; c++) {
        lap_centered(A[c], x[c], *g);
        multiply(A[c], coeff);
        add(A[c], x[c]);
      }
      break;
    case OP_IND_DIFFUSION: {
      // curl(tempk%x,x); multiply(tempk%x,k%x); curl(Ax,tempk%x)
      curl(tempk[0], tempk[1], tempk[2], x[0], x[1], x[2], *g);
      for (int c = 0; c < 3; c++) multiply(tempk[c], k[c]);
      curl(A[0], A[1], A[2], tempk[0], tempk[1], tempk[2], *g);
      for (int c = 0; c < 3; c++) {
        multiply(A[c], coeff);
        add(A[c], x[c]);
      }
    } break;
  }
}

static double dotp(const std::vector<SF>& A, const std::vector<SF>& B, SF* const* x, std::vector<SF>& tmp) {
  // dot_product_SF/VF (ops_aux.f90:199-216)
  double d = 0;
  for (size_t c = 0; c < A.size(); c++) {
    if (tmp[c].f.size() != A[c].f.size()) tmp[c].f = A[c].f;
    par_chunks((long)A[c].n(), [&](long s, long e) {
      for (long i = s; i < e; i++) tmp[c].f[i] = A[c].f[i] * B[c].f[i];
    });
    assign_wall_Dirichlet(tmp[c], 0.0, x[c]);
    d += sum_pad(tmp[c], 1);
  }
  return d;
}

SolveInfo PCG::solve(SF* const* x, SF* const* b, ISP& isp) {
  SolveInfo info;
  std::vector<SF> xs;
  for (int c = 0; c < nc; c++) xs.push_back(*x[c]);
  // ---- modify_RHS (PCG_aux.f90:30-79)
  for (int c = 0; c < nc; c++) assign(r[c], *b[c]);
  if (nc == 1 && x[0]->bc && x[0]->bc->all_neumann) {
    // subtract_phys_mean_vol_SF (ops_aux.f90:146-157)
    SF t = like(*g, r[0]);
    t.f = r[0].f;
    multiply(t, vol[0]);
    double meanU = sum_pad(t, 1) / vol[0].vol;
    for (auto& v : r[0].f) v -= meanU;
    assign_ghost_XPeriodic(r[0], 0.0, nullptr);
  }
  // compute_Ax_BC (PCG_aux.f90:81-107)
  for (int c = 0; c < nc; c++) {
    assign(x_BC[c], 0.0);
    apply_BCs(x_BC[c]);
    assign_ghost_N_XPeriodic(x_BC[c], 0.0, nullptr);
  }
  apply_operator(tempx, x_BC, true);
  for (int c = 0; c < nc; c++) {
    assign_ghost_XPeriodic(tempx[c], 0.0, x[c]);
    subtract(r[c], tempx[c]);
  }
  apply_operator(Ax, xs, false);
  for (int c = 0; c < nc; c++) {
    subtract(r[c], Ax[c]);
    multiply(r[c], vol[c]);
    if (r[c].dl != 0) {
      assign_wall_Periodic_single(r[c], 0.0, &x_BC[c]);
      assign_wall_Dirichlet(r[c], 0.0, &x_BC[c]);
      multiply_wall_Neumann(r[c], 0.5, &x_BC[c]);
    }
  }
  // ---- PCG_solver_algorithm.f90:56-106
  double l2 = 0;
  for (int c = 0; c < nc; c++)
    for (double v : r[c].f) l2 += v * v;
  double res0 = std::sqrt(l2);
  isp.iter_per_call = 0;
  info.res0 = res0;
  if (std::isnan(res0)) info.nan = 1;
  for (int c = 0; c < nc; c++) {
    assign(z[c], Minv[c]);
    multiply(z[c], r[c]);
    assign(p[c], z[c]);
  }
  SF* xp[3] = {x[0], nc > 1 ? x[1] : nullptr, nc > 1 ? x[2] : nullptr};
  double rhok = dotp(r, z, xp, tempx);
  double res = std::sqrt(std::fabs(rhok));
  auto update_exit = [&](double rs) {
    isp.exit_loop[1] = rs / res0 < isp.tol_rel;
    isp.exit_loop[2] = rs < isp.tol_abs;
    isp.exit_loop[3] = isp.iter_per_call >= isp.iter_max;
  };
  update_exit(res);
  // copy xs back into x before the loop: the operator applied implicit BCs
  for (int c = 0; c < nc; c++) *x[c] = xs[c];
  if (!isp.exit_loop[2]) {
    for (int it = 1; it <= isp.iter_max; it++) {
      apply_operator(Ax, p, false);
      for (int c = 0; c < nc; c++) {
        multiply_wall_Neumann(Ax[c], 0.5, &x_BC[c]);
        assign_wall_Dirichlet(Ax[c], 0.0, &x_BC[c]);
        assign_wall_Periodic_single(Ax[c], 0.0, &x_BC[c]);
        multiply(Ax[c], vol[c]);
      }
      double alpha = rhok / dotp(p, Ax, xp, tempx);
      for (int c = 0; c < nc; c++) {
        add_product(*x[c], p[c], alpha);
        apply_BCs(*x[c]);
      }
      isp.iter_total++;
      isp.iter_per_call++;
      for (int c = 0; c < nc; c++) add_product(r[c], Ax[c], -alpha);
      if (isp.iter_per_call % isp.n_skip_check_res == 0) {
        res = std::sqrt(std::fabs(dotp(r, r, xp, tempx)));
        update_exit(res);
        if (isp.exit_loop[1] || isp.exit_loop[2] || isp.exit_loop[3]) break;
      }
      for (int c = 0; c < nc; c++) {
        assign(z[c], Minv[c]);
        multiply(z[c], r[c]);
      }
      double rhokp1 = dotp(z, r, xp, tempx);
      for (int c = 0; c < nc; c++) product_add(p[c], rhokp1 / rhok, z[c]);
      rhok = rhokp1;
      isp.exit_loop[3] = isp.iter_per_call >= isp.iter_max;
    }
  } else {
    for (int c = 0; c < nc; c++) apply_BCs(*x[c]);
    isp.iter_total++;
    isp.iter_per_call++;
  }
  info.iterations = isp.iter_per_call;
  info.res = res;
  info.rel = (res0 == 0.0) ? res : res / res0;
  info.exit_reason = isp.exit_loop[1] ? 1 : isp.exit_loop[2] ? 2 : isp.exit_loop[3] ? 3 : 0;
  if (std::isnan(res)) info.nan = 1;
  return info;
}

}  // namespace mo
