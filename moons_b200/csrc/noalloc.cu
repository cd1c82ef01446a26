// noalloc.cu -- moons_lap_var_noalloc: the sigma-weighted Laplacian
// div(k grad u) (lapVarCoeff_VF, ops_discrete.f90:275-285) without any
// device allocation.
//
// moons_lap_var needs three face-located temporaries (k * grad u along each
// axis) and takes them from the stream-ordered allocator on every call.
// Some callers cannot allocate at that point: a host whose own pool already
// holds the free device memory (a PyTorch caching allocator, or a Fortran
// code that sized its arrays to fill HBM) gets an out-of-memory error for a
// few megabytes, and a host that keeps allocator traffic out of a timed loop
// does not want the pool to grow or shrink there.  This variant takes the
// temporaries from one file-scope device array instead, so the only device
// memory it touches is the caller's fields and that array.
//
// Limits and rules (also in include/moons_gpu.h):
//  * each temporary holds at most kNoallocMaxPoints doubles; a field whose
//    face temporaries would be larger is rejected with MOONS_ERR_LIMIT;
//  * the first call on a device looks up the array's address on that device
//    (cudaGetSymbolAddress, with that device made current for the lookup and
//    the caller's current device restored after it) and keeps it; make that
//    first call before any stream capture;
//  * every call synchronizes the mesh's stream before it returns;
//  * nothing in the array needs an initial value: the gradient pass writes
//    every element that the divergence pass reads;
//  * the array is shared by all callers on a device, so calls that overlap in
//    time (several host threads, or several streams) race on it.
#include <mutex>

#include "runtime.cuh"

using namespace mg;

namespace {

constexpr long long kNoallocMaxPoints = MOONS_LAP_VAR_NOALLOC_MAX_POINTS;  // per temporary (1 MiB of FP64)
constexpr int kNoallocMaxDevices = 64;

// three face temporaries, 3 MiB in all
static __device__ __align__(256) double g_lap_var_scratch[3 * kNoallocMaxPoints];

std::mutex g_noalloc_mutex;
double* g_noalloc_base[kNoallocMaxDevices] = {};

// device address of the scratch array on `dev` (looked up once per device)
int noalloc_scratch(int dev, double** out) {
  if (dev < 0 || dev >= kNoallocMaxDevices) {
    mg::set_error("moons_lap_var_noalloc: device index out of range");
    return MOONS_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_base[dev]) {
    int prev = -1;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) return mg::cuda_fail(e, "cudaGetDevice");
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) return mg::cuda_fail(e, "cudaSetDevice");
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lap_var_scratch);
    const cudaError_t e2 = cudaSetDevice(prev);  // the caller's current device stays current
    if (e != cudaSuccess) return mg::cuda_fail(e, "cudaGetSymbolAddress(g_lap_var_scratch)");
    if (e2 != cudaSuccess) return mg::cuda_fail(e2, "cudaSetDevice (restore)");
    g_noalloc_base[dev] = static_cast<double*>(p);
  }
  *out = g_noalloc_base[dev];
  return MOONS_OK;
}

}  // namespace

extern "C" int moons_lap_var_noalloc(moons_sf* o, const moons_sf* u, const moons_sf* kx, const moons_sf* ky,
                                     const moons_sf* kz) {
  if (!o || !u || !kx || !ky || !kz) {
    mg::set_error("moons_lap_var_noalloc: null field");
    return MOONS_ERR_ARG;
  }
  moons_mesh* m = o->m;
  DF t[3];
  for (int d = 0; d < 3; d++) {
    t[d] = make_df(m, dl_after_diff(u->f.dl, d + 1), nullptr);
    if ((long long)t[d].n() > kNoallocMaxPoints) {
      mg::set_error("moons_lap_var_noalloc: field too large for the built-in scratch (" + std::to_string(t[d].n()) +
                    " points per face temporary, at most " + std::to_string(kNoallocMaxPoints) +
                    "); use moons_lap_var");
      return MOONS_ERR_LIMIT;
    }
  }
  double* base = nullptr;
  int r = noalloc_scratch(m->device, &base);
  if (r) return r;
  for (int d = 0; d < 3; d++) t[d].f = base + (size_t)d * (size_t)kNoallocMaxPoints;
  // lapVarCoeff_VF: grad(tempk,u); multiply(tempk,k); div(lapU,tempk)
  const moons_sf* ks[3] = {kx, ky, kz};
  for (int d = 0; d < 3 && !r; d++) r = launch_del(m, t[d], u->f, 1, d + 1, 0, 1);
  for (int d = 0; d < 3 && !r; d++) r = launch_pw(m, PW_MUL, t[d], &ks[d]->f, 0.0);
  if (!r) r = launch_del(m, o->f, t[0], 1, 1, 0, 1);
  if (!r) r = launch_del(m, o->f, t[1], 1, 2, 0, 2);
  if (!r) r = launch_del(m, o->f, t[2], 1, 3, 0, 2);
  if (!r) r = mask_ghost_XPeriodic(m, o->f, o->bc.defined ? &o->bc : nullptr);
  if (r) return r;
  MG_CUDA(cudaStreamSynchronize(m->stream));
  return MOONS_OK;
}
