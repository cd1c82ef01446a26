// persist.cuh -- the whole PCG loop (PCG_solver_algorithm.f90:69-96) as ONE
// persistent, cooperatively launched kernel.
//
// The three steps of an iteration are the column routines of lean.cuh; what
// separates them is a grid barrier instead of a kernel boundary:
//   A  Ap = op(p) (+ mask, vol) and the block partial of p.Ap   -> barrier
//   B  x += alpha p; r -= alpha Ap; partials of r.r and z.r     -> barrier
//   C  p' = beta p + Minv r with p's implicit BC values          -> barrier
// (the curl-curl operator needs one more barrier inside A, between the edge
// field sigma*curl(p) and its curl).  Every block sums all block partials in
// the same fixed order after a barrier, so alpha, beta and the exit test are
// formed identically -- and deterministically -- in every block without a
// serial "last block" step, and the loop ends in all blocks at the same
// iteration.  The launch is cooperative, so all blocks are resident; each
// barrier wait is bounded in time and raises an error flag (which ends the
// loop in every block) instead of waiting forever.
#pragma once
#include "lean.cuh"

namespace mg {

struct GridSync {
  unsigned count;  // blocks arrived at the current barrier
  unsigned gen;    // barrier generation
  int err;         // a wait gave up
  int pad;
};

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s per wait

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// grid-wide barrier; false when any wait gave up (then every block leaves)
__device__ __forceinline__ bool grid_sync(GridSync* gs, unsigned& gen) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();  // release this block's writes
    const unsigned arrived = atomicAdd(&gs->count, 1u);
    if (arrived == gridDim.x - 1) {
      atomicExch(&gs->count, 0u);
      __threadfence();
      atomicExch(&gs->gen, gen + 1u);
    } else {
      const unsigned long long t0 = global_ns();
      unsigned spins = 0;
      while (ld_acquire(&gs->gen) == gen) {
        if ((++spins & 63u) == 0 && global_ns() - t0 > kBarrierTimeoutNs) {
          atomicExch(&gs->err, 1);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();  // acquire the other blocks' writes
    if (*(volatile int*)&gs->err) ok = 0;
    s_ok = ok;
  }
  __syncthreads();
  gen++;
  return s_ok != 0;
}

// sum of n block partials, same order in every block; valid in all threads
__device__ __forceinline__ double all_sum(const double* part, unsigned n) {
  __shared__ double s_tot;
  double v = 0.0;
  for (unsigned t = threadIdx.x; t < n; t += blockDim.x) v += __ldcg(part + t);
  v = block_sum(v);
  if (threadIdx.x == 0) s_tot = v;
  __syncthreads();
  v = s_tot;
  __syncthreads();
  return v;
}

constexpr int kKCB = 8;  // planes per thread in the pointwise steps B and C

struct PersistArgs {
  FComp X, P0, P1, R, Ap, M;
  DGrid g;
  FBC b0, b1, b2;
  DF k0, k1, k2;     // LAP_PROPS face coefficients / IND edge sigma
  DF E0, E1, E2;     // IND: edge work field
  double coeff;
  int mm;            // Minv mode (0 stored, 1 Lap, 2 mom)
  unsigned npb, nkc;   // plane blocks and k chunks (kKC planes) of the unknown's grid
  unsigned nkcB;       // k chunks of kKCB planes
  unsigned npbE, nkcE; // same for the IND edge field
  PcgScalars* S;
  double* part;      // 3 x gridDim.x block partials
  GridSync* gs;
};

// one work item of each step, component C known at compile time (no
// run-time indexing of the kernel's parameter structs)
template <int OP, int C>
__device__ __forceinline__ double step_a(const PersistArgs& a, int cur, unsigned pb, int k0) {
  const DF& A = a.Ap.f[C];
  const int k1 = min(k0 + kKC - 1, A.s2);
  const FBC& b = C == 0 ? a.b0 : (C == 1 ? a.b1 : a.b2);
  const DF p = cur ? a.P1.f[C] : a.P0.f[C];
  if (OP == 3) {
    // curl_c(E): C=0 (E_z, E_y), C=1 (E_x, E_z), C=2 (E_y, E_x)
    const DF& Ea = C == 0 ? a.E2 : (C == 1 ? a.E0 : a.E1);
    const DF& Eb = C == 0 ? a.E1 : (C == 1 ? a.E2 : a.E0);
    return curl_ap_column<C>(A, p, b, Ea, Eb, a.g, a.coeff, pb, k0, k1);
  }
  return lap_column<OP>(A, p, b, a.g, a.k0, a.k1, a.k2, a.coeff, pb, k0, k1);
}
template <int L>
__device__ __forceinline__ void step_e(const PersistArgs& a, int cur, unsigned pb, int k0) {
  // E_l = sig_l curl_l(p): l=0 (p_z, p_y), l=1 (p_x, p_z), l=2 (p_y, p_x)
  const DF& E = L == 0 ? a.E0 : (L == 1 ? a.E1 : a.E2);
  const DF& sg = L == 0 ? a.k0 : (L == 1 ? a.k1 : a.k2);
  constexpr int ca = L == 0 ? 2 : (L == 1 ? 0 : 1);
  constexpr int cb = L == 0 ? 1 : (L == 1 ? 2 : 0);
  const DF pa = cur ? a.P1.f[ca] : a.P0.f[ca];
  const DF pbf = cur ? a.P1.f[cb] : a.P0.f[cb];
  curl_sig_column<L>(E, pa, pbf, sg, a.g, pb, k0, min(k0 + kKC - 1, E.s2));
}
template <int C>
__device__ __forceinline__ void step_b(const PersistArgs& a, int cur, double alpha, unsigned pb, int k0, double& arr,
                                       double& azr) {
  const FBC& b = C == 0 ? a.b0 : (C == 1 ? a.b1 : a.b2);
  const DF& x = a.X.f[C];
  const DF p = cur ? a.P1.f[C] : a.P0.f[C];
  update_column<kKCB>(x, p, a.R.f[C], a.Ap.f[C], a.M.f[C], b, a.g, a.mm, a.coeff, alpha, pb, k0,
                      min(k0 + kKCB - 1, x.s2), arr, azr);
}
template <int C>
__device__ __forceinline__ void step_c(const PersistArgs& a, int cur, double beta, unsigned pb, int k0) {
  const FBC& b = C == 0 ? a.b0 : (C == 1 ? a.b1 : a.b2);
  const DF p = cur ? a.P1.f[C] : a.P0.f[C];
  const DF pn = cur ? a.P0.f[C] : a.P1.f[C];
  pupd_column<kKCB>(p, pn, a.R.f[C], a.M.f[C], b, a.g, a.mm, a.coeff, beta, pb, k0, min(k0 + kKCB - 1, p.s2));
}

// OP: 0 LAP_UNIFORM, 1 LAP_PROPS, 2 MOM_DIFFUSION, 3 IND_DIFFUSION
template <int OP>
__global__ void __launch_bounds__(kLB, 2) k_pcg_persist(PersistArgs a) {
  PcgScalars* S = a.S;
  if (S->done) return;
  const int nc = a.X.nc;
  const unsigned G = gridDim.x;
  const unsigned nwork = a.npb * a.nkc * (unsigned)nc;
  const unsigned nworkE = a.npbE * a.nkcE * 3u;
  const unsigned nworkB = a.npb * a.nkcB * (unsigned)nc;
  unsigned gen = 0;
  double rhok = S->rhok;
  const double res0 = S->res0, tol_rel = S->tol_rel, tol_abs = S->tol_abs;
  const int iter_max = S->iter_max, nskip = S->nskip;
  const int iter0 = S->iter;
  int iter = iter0;
  int exit_reason = 0, nan = 0;
  double res = S->res, rr = 0.0, zr = 0.0, alpha = 0.0, beta = 0.0, pap = 0.0;
  bool sync_ok = true;
  int cur = 0;
  for (;;) {
    // ---- A: Ap = op(p), p.Ap
    if (OP == 3) {
      for (unsigned w = blockIdx.x; w < nworkE; w += G) {
        const Item it = item_of<kKC>(w, a.npbE, a.nkcE);
        if (it.c == 0) step_e<0>(a, cur, it.pb, it.k0);
        else if (it.c == 1) step_e<1>(a, cur, it.pb, it.k0);
        else step_e<2>(a, cur, it.pb, it.k0);
      }
      if (!(sync_ok = grid_sync(a.gs, gen))) break;
    }
    double acc = 0.0;
    for (unsigned w = blockIdx.x; w < nwork; w += G) {
      const Item it = item_of<kKC>(w, a.npb, a.nkc);
      if (it.c == 0) acc += step_a<OP, 0>(a, cur, it.pb, it.k0);
      else if (it.c == 1) acc += step_a<OP, 1>(a, cur, it.pb, it.k0);
      else acc += step_a<OP, 2>(a, cur, it.pb, it.k0);
    }
    {
      const double bs = block_sum(acc);
      if (threadIdx.x == 0) a.part[blockIdx.x] = bs;
    }
    if (!(sync_ok = grid_sync(a.gs, gen))) break;
    pap = all_sum(a.part, G);
    alpha = rhok / pap;
    // ---- B: x, r update, r.r and z.r
    double arr = 0.0, azr = 0.0;
    for (unsigned w = blockIdx.x; w < nworkB; w += G) {
      const Item it = item_of<kKCB>(w, a.npb, a.nkcB);
      if (it.c == 0) step_b<0>(a, cur, alpha, it.pb, it.k0, arr, azr);
      else if (it.c == 1) step_b<1>(a, cur, alpha, it.pb, it.k0, arr, azr);
      else step_b<2>(a, cur, alpha, it.pb, it.k0, arr, azr);
    }
    {
      const double s1 = block_sum(arr);
      const double s2 = block_sum(azr);
      if (threadIdx.x == 0) {
        a.part[G + blockIdx.x] = s1;
        a.part[2 * G + blockIdx.x] = s2;
      }
    }
    if (!(sync_ok = grid_sync(a.gs, gen))) break;
    rr = all_sum(a.part + G, G);
    zr = all_sum(a.part + 2 * G, G);
    // update_exit_loop (PCG_solver_algorithm.f90:84-88)
    iter += 1;
    bool stop = false;
    if (iter % nskip == 0) {
      res = sqrt(fabs(rr));
      const bool e1 = res / res0 < tol_rel;
      const bool e2 = res < tol_abs;
      const bool e3 = iter >= iter_max;
      if (e1 || e2 || e3) {
        stop = true;
        exit_reason = e1 ? 1 : (e2 ? 2 : 3);
      }
      if (isnan(res)) {
        nan = 1;
        stop = true;
      }
    }
    if (!stop) {
      beta = zr / rhok;
      rhok = zr;
      if (iter >= iter_max) {
        stop = true;
        exit_reason = 3;
      }
    }
    if (stop) break;
    // ---- C: p' = beta p + Minv r (+ implicit BC values)
    for (unsigned w = blockIdx.x; w < nworkB; w += G) {
      const Item it = item_of<kKCB>(w, a.npb, a.nkcB);
      if (it.c == 0) step_c<0>(a, cur, beta, it.pb, it.k0);
      else if (it.c == 1) step_c<1>(a, cur, beta, it.pb, it.k0);
      else step_c<2>(a, cur, beta, it.pb, it.k0);
    }
    if (!(sync_ok = grid_sync(a.gs, gen))) break;
    cur ^= 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    S->iter = iter;
    S->iter_total += iter - iter0;
    S->runs_total += 1;
    S->res = res;
    S->rr = rr;
    S->zr = zr;
    S->alpha = alpha;
    S->beta = beta;
    S->pap = pap;
    S->rhok = rhok;
    S->exit_reason = exit_reason;
    S->nan = nan;
    if (nan) S->nan_any = 1;
    S->done = 1;
    if (!sync_ok || *(volatile int*)&a.gs->err) S->sync_err = 1;
  }
}

}  // namespace mg
