// lean_cc.cuh -- the operator step (K1) of the PCG iteration for one
// cell-centred unknown (pressure, cleaning or electric potential,
// temperature): Lap_uniform_SF, Lap_nonuniform_props and nrg_diffusion
// (matrix_free_operators.f90:35-62, 92-118, 148-174) with the volume
// weighting of PCG_solver_algorithm.f90:72-75, and the block partials of
// p.Ap that give alpha.
//
// Layout of the work: a block owns a 32 x 16 tile of interior (i,j) columns
// (eight compute warps of two consecutive tile rows each, lanes along x) and
// marches a chunk of interior planes k.  The planes of p it reads stream
// through a ring of shared-memory stages that a ninth (producer) warp fills
// with bulk copies (cp.async.bulk, one per staged row: the tile's rows and
// one halo row on each side), so a block keeps up to eight planes in flight
// without holding them in registers.  Full/empty mbarriers pair each stage
// between the producer and the compute warps; no block-wide barrier sits in
// the loop.  The z neighbours roll through registers, the y neighbours of a
// warp's inner rows are its own rows' values, the rest come from the staged
// rows.
//
// Ghost values: the reference reads p after apply_BCs_implicit.  For a
// cell-centred unknown every ghost value an interior stencil reads lies on
// exactly one ghost plane and is fac * p(src) with src the adjacent interior
// cell (Dirichlet fac -1, Neumann 1, Robin rc), the interior cell at the far
// end (periodic), or the stored ghost itself when no BC is defined.  This
// kernel forms those values from the interior, so the iteration needs no BC
// fill of p, and it never writes Ap's ghost points (the solve clears Ap once
// before the loop; the update kernel reads them as zeros).
#pragma once
#include <cuda.h>

#include "lean.cuh"
#include "tc.cuh"

namespace mg {

constexpr int kCTX = 32;                 // tile columns along x (lanes)
constexpr int kCW = 8;                   // compute warps per block
constexpr int kCRW = 2;                  // consecutive tile rows per compute warp
constexpr int kCTY = kCW * kCRW;         // tile rows along y
constexpr int kCRows = kCTY + 2;         // staged rows per plane
constexpr int kCRS = kCTX + 4;           // row stride (doubles): 34 values + alignment shift, 16-byte multiple
constexpr int kCStages = 8;              // planes in the ring
constexpr int kCStagesF = 6;             // planes in the ring when p and z are staged
constexpr int kCStage = ((kCRows * kCRS + 15) / 16) * 16;  // doubles per stage (128-byte multiple)
constexpr int kCWaitCode = 101;          // wait_err code of a stage wait that ran out
constexpr int kCThreads = (kCW + 1) * 32;  // compute warps and one producer warp
// dynamic shared memory: 128 bytes of alignment slack, the ring, then 8
// doubles of z coefficients per plane of the block's chunk
inline size_t cc_smem(int klen, bool fz) {
  const size_t ring = fz ? (size_t)kCStagesF * 2 * kCStage : (size_t)kCStages * kCStage;
  return 128 + (ring + 8 * (size_t)klen) * sizeof(double);
}

// ghost rule at one face of a CC axis: kind 0 stored value, 1 fac * adjacent
// interior cell, 2 the interior cell at the far end (periodic)
struct CGhost {
  int kind;
  double fac;
};
MG_HD CGhost cghost(const FBC& b, int face) {
  CGhost g{0, 1.0};
  if (!b.defined) return g;
  const int t = b.type[face];
  if (t == MOONS_BC_DIRICHLET) {
    g.kind = 1;
    g.fac = -1.0;
  } else if (t == MOONS_BC_NEUMANN) {
    g.kind = 1;
  } else if (t == MOONS_BC_ROBIN) {
    g.kind = 1;
    g.fac = b.rc[face];
  } else if (t == MOONS_BC_PERIODIC) {
    g.kind = 2;
  }
  return g;
}

// tiles of the interior of a CC field (kCTX x kCTY columns): along x and in all
MG_HD int cc_tiles_x(const DF& a) { return (a.s0 - 2 + kCTX - 1) / kCTX; }
MG_HD int cc_tiles(const DF& a) { return cc_tiles_x(a) * ((a.s1 - 2 + kCTY - 1) / kCTY); }

// EVEN: s0 is even (every staged row starts on an even element).  TM: the
// stages are filled by one tiled tensor load (TMA) per plane through `tmap`
// (a 3-D map of p with a 36 x 18 x 1 box; needs EVEN) instead of one bulk
// copy per row.
// FZ (fused iteration): the operator acts on p' = beta p + z, formed here
// from the staged p and z (z = Minv r, stored by the update kernel), and p'
// is written to pn -- the p update of the previous iteration folded into
// this kernel (PCG_solver_algorithm.f90:93-96, then :70-76); the previous
// iteration's x += alpha p (:78-79), with the staged p, is applied here too.
template <int MODE, bool EVEN, bool TM, bool FZ>
__global__ void __launch_bounds__(kCThreads, (MODE == 0 && !FZ) ? 3 : 2)
    k_cc_lap(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap tmapz, DF A, DF p, DF z,
             DF pn, DF x, DGrid g, FBC b, DF kx, DF ky, DF kz, double coeff, int klen, PcgScalars* S, double* partial,
             unsigned* ticket) {
  constexpr int NST = FZ ? kCStagesF : kCStages;  // stages in the ring
  constexpr int SST = (FZ ? 2 : 1) * kCStage;     // doubles per stage (p, then z)
  extern __shared__ __align__(16) double smem_raw[];
  // NST stages of kCRows x kCRS doubles per staged array, 128-byte aligned (tensor loads)
  double* ring = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) unsigned long long full[kCStages], empty[kCStages];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ntx = cc_tiles_x(A);
  const int i0 = 2 + (int)(blockIdx.x % (unsigned)ntx) * kCTX, j0 = 2 + (int)(blockIdx.x / (unsigned)ntx) * kCTY;
  const int kb = 2 + (int)blockIdx.y * klen, ke = min(A.s2 - 1, kb + klen - 1);
  const bool work = kb <= ke;  // uniform per block
  double* zt = ring + NST * SST;
  // ---- set-up that reads nothing the preceding kernel writes: it runs
  // while that kernel drains (programmatic dependent launch)
  if (work) {
    if (threadIdx.x == 0) {
      for (int s = 0; s < NST; s++) {
        tc::mbar_init(tc::smem_u32(&full[s]), 1);
        tc::mbar_init(tc::smem_u32(&empty[s]), kCW);  // one arrival per compute warp
      }
      tc::fence_mbar_init();
    }
    // the z coefficients of the block's planes, once: a1 a2 b1 b2 o1 o2 dhn
    for (int t = threadIdx.x; t < (ke - kb + 1) * 8; t += blockDim.x) {
      const int k = kb + t / 8, f = t % 8;
      const DCoord& c = g.c[2];
      if (MODE == 0) {  // folded: czm czp cz0 vz
        const Ax6 Z = axis_coef(c, false, k);
        zt[t] = f == 0 ? Z.a1 * Z.o1 : f == 1 ? Z.b2 * Z.o2 : f == 2 ? Z.a2 * Z.o1 + Z.b1 * Z.o2 : f == 3 ? c.dhn[k] : 0.0;
      } else {
        zt[t] = f == 0 ? c.cc2nD[k - 1] : f == 1 ? c.cc2nU[k - 1] : f == 2 ? c.cc2nD[k] : f == 3 ? c.cc2nU[k]
                : f == 4 ? c.n2ccD[k] : f == 5 ? c.n2ccU[k] : f == 6 ? c.dhn[k] : 0.0;
      }
    }
  }
  __syncthreads();
  pdl_enter();
  if (S->done) return;
  double acc = 0.0;
  if (work) {
    const unsigned s0 = (unsigned)A.s0, sxy = (unsigned)A.s0 * (unsigned)A.s1;
    const int nq = ke - kb + 3;                       // staged planes kb-1 .. ke+1
    const int nrows = min(kCRows, A.s1 - j0 + 2);     // staged rows j0-1 .. min(j0+kCTY, s1)
    if (w == kCW) {
      // ---- producer warp: row r of plane kb-1+q -> stage q % kCStages.  A
      // row copy is kCRS doubles from the even element at or below (i0-1, jr,
      // k); it ends at most 33 doubles past the field (internal fields are
      // padded for it).
      bool live = true;
      int issued = 0;
      for (int q = 0; q < nq; q++) {
        const int st = q % NST;
        if (q >= NST && live)
          live = tc::mbar_wait_sleep(tc::smem_u32(&empty[st]), (uint32_t)(((q / NST) - 1) & 1), &S->wait_err,
                                     kCWaitCode);
        if (!live) break;
        const int k = kb - 1 + q;
        const uint32_t bar = tc::smem_u32(&full[st]);
        if (TM) {
          // one box per staged array: columns i0-1 .. i0+34, rows j0-1 ..
          // j0+16 of plane k (0-based x = i0-2, even), zero fill past the field
          if (lane == 0) {
            tc::mbar_expect_tx(bar, (uint32_t)((FZ ? 2 : 1) * kCRows * kCRS * 8));
            tc::tma_load_3d(tc::smem_u32(ring + st * SST), &tmap, i0 - 2, j0 - 2, k - 1, bar);
            if (FZ) tc::tma_load_3d(tc::smem_u32(ring + st * SST + kCStage), &tmapz, i0 - 2, j0 - 2, k - 1, bar);
          }
        } else {
          if (lane == 0) tc::mbar_expect_tx(bar, (uint32_t)((FZ ? 2 : 1) * nrows) * (uint32_t)(kCRS * 8));
          __syncwarp();
          for (int r = lane; r < nrows; r += 32) {
            const unsigned e0 = (unsigned)(k - 1) * sxy + (unsigned)(j0 - 2 + r) * s0 + (unsigned)(i0 - 2);
            tc::bulk_g2s(tc::smem_u32(ring + st * SST + r * kCRS), p.f + (e0 & ~1u), kCRS * 8, bar);
            if (FZ) tc::bulk_g2s(tc::smem_u32(ring + st * SST + kCStage + r * kCRS), z.f + (e0 & ~1u), kCRS * 8, bar);
          }
        }
        issued = q + 1;
      }
      // no copy may land in this block's shared memory after it exits: wait
      // (bounded) for the last copy issued into each stage
      if (lane == 0)
        for (int q = max(0, issued - NST); q < issued; q++)
          tc::mbar_wait(tc::smem_u32(&full[q % NST]), (uint32_t)((q / NST) & 1), &S->wait_err, kCWaitCode);
    } else {
      // ---- compute warps: warp w owns tile rows jw .. jw+kCRW-1, lane the column
      const int i = i0 + lane, jw = j0 + w * kCRW;
      const bool coli = i <= A.s0 - 1;
      bool act[kCRW];
#pragma unroll
      for (int r = 0; r < kCRW; r++) act[r] = coli && jw + r <= A.s1 - 1;
      // block touches a ghost plane along x or y: the ghost rules apply
      const bool edge = i0 == 2 || i0 + kCTX - 1 >= A.s0 - 1 || j0 == 2 || j0 + kCTY - 1 >= A.s1 - 1;
      // per-axis coefficients.  MODE 0: the two-gradient composition
      // (pm*a1 + p0*a2)*o1 + (p0*b1 + pp*b2)*o2 folded to cm*pm + c0*p0 + cp*pp
      // (the same operator; rounding differs from the unfolded form at the
      // last bit).  MODE 1/3 keep the unfolded form: the face coefficients
      // sit between the two differences.
      Ax6 X{};
      Ax6 Y[kCRW];
      double vxy[kCRW], c0xy[kCRW], cym[kCRW], cyp[kCRW];
      if (coli) X = axis_coef(g.c[0], false, i);
      const double cxm = X.a1 * X.o1, cxp = X.b2 * X.o2, cx0 = X.a2 * X.o1 + X.b1 * X.o2;
#pragma unroll
      for (int r = 0; r < kCRW; r++) {
        Y[r] = act[r] ? axis_coef(g.c[1], false, jw + r) : Ax6{};
        vxy[r] = act[r] ? g.c[0].dhn[i] * g.c[1].dhn[jw + r] : 0.0;
        c0xy[r] = cx0 + (Y[r].a2 * Y[r].o1 + Y[r].b1 * Y[r].o2);
        cym[r] = Y[r].a1 * Y[r].o1;
        cyp[r] = Y[r].b2 * Y[r].o2;
      }
      // staged offset of this column in row jr: (jr - j0 + 1) * kCRS + oc +
      // shift, shift = element parity of the row's first staged column (0 on
      // meshes with an even s0)
      const int oc = i - i0 + 1;
      const unsigned odd0 = s0 & 1u, oddxy = sxy & 1u;
      auto roff = [&](int jr, unsigned ak) -> int {
        if (EVEN) return (jr - j0 + 1) * kCRS + oc;
        return (jr - j0 + 1) * kCRS + oc + (int)(ak ^ (((unsigned)(jr - 1) & 1u) & odd0));
      };
      bool ok = true;
      auto wait_q = [&](int q) {
        if (ok)
          ok = tc::mbar_wait_sleep(tc::smem_u32(&full[q % NST]), (uint32_t)((q / NST) & 1), &S->wait_err,
                                   kCWaitCode);
      };
      auto release = [&](int q) {
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(tc::smem_u32(&empty[q % NST]));
      };
      // the operand at a staged offset: p, or (FZ) p' = beta p + z
      const double beta = FZ ? S->beta : 0.0;
      const double alpha_prev = FZ ? S->alpha : 0.0;  // the previous iteration's alpha (x update)
      auto sv = [&](int off) -> double {
        if (FZ) return ring[off] * beta + ring[off + kCStage];
        return ring[off];
      };
      // the operand at an interior point read from global memory (periodic ghost sources)
      auto gv = [&](int ii, int jj, int kk) -> double {
        if (FZ) return p(ii, jj, kk) * beta + z(ii, jj, kk);
        return p(ii, jj, kk);
      };
      // planes kb-1 (pm) and kb (p0)
      wait_q(0);
      wait_q(1);
      double pm[kCRW], p0[kCRW];
      {
        const unsigned a0 = ((unsigned)(kb - 2) & 1u) & oddxy, a1 = ((unsigned)(kb - 1) & 1u) & oddxy;
        const int s1b = (1 % NST) * SST;
#pragma unroll
        for (int r = 0; r < kCRW; r++) {
          p0[r] = sv(s1b + roff(jw + r, a1));
          pm[r] = sv(roff(jw + r, a0));
          if (kb - 1 == 1) {  // plane 1 is the ghost plane
            const CGhost gzm = cghost(b, 5);
            if (gzm.kind == 1) pm[r] = gzm.fac * p0[r];
            else if (gzm.kind == 2 && act[r]) pm[r] = gv(i, jw + r, A.s2 - 1);
          }
        }
      }
      release(0);
      const size_t o0 = coli ? A.at(i, min(jw, A.s1), kb) : 0;  // (i, jw, kb): + r*s0 per row, + sxy per plane
      double* out = A.f + o0;
      double* outp = FZ ? pn.f + o0 : nullptr;
      double* xo = FZ ? x.f + o0 : nullptr;
      double xv[kCRW];  // x of this plane, loaded one plane ahead
      if (FZ) {
#pragma unroll
        for (int r = 0; r < kCRW; r++) xv[r] = act[r] ? xo[r * (int)s0] : 0.0;
      }
#pragma unroll 1  // one plane per trip: unrolled by 2 it held more live values (93.9 -> 88.3 us per
                   // iteration on the over-L2 mesh when unrolling was dropped)
      for (int k = kb; k <= ke; k++, out += sxy, outp += FZ ? sxy : 0, xo += FZ ? sxy : 0) {
        const int qk = k - kb + 1;
        double xn[kCRW];
        if (FZ) {
#pragma unroll
          for (int r = 0; r < kCRW; r++) xn[r] = (act[r] && k < ke) ? xo[sxy + r * (int)s0] : 0.0;
        }
        wait_q(qk + 1);
        const int sk = (qk % NST) * SST, sn = ((qk + 1) % NST) * SST;
        const unsigned ak = ((unsigned)(k - 1) & 1u) & oddxy, an = ((unsigned)k & 1u) & oddxy;
        double pp[kCRW], xm[kCRW], xp[kCRW];
#pragma unroll
        for (int r = 0; r < kCRW; r++) {
          pp[r] = sv(sn + roff(jw + r, an));
          const int c0 = sk + roff(jw + r, ak);
          xm[r] = sv(c0 - 1);
          xp[r] = sv(c0 + 1);
        }
        const double ylo = sv(sk + roff(jw - 1, ak)), yhi = sv(sk + roff(jw + kCRW, ak));
        if (k + 1 == A.s2) {  // plane s2 is the ghost plane
          const CGhost gzp = cghost(b, 6);
#pragma unroll
          for (int r = 0; r < kCRW; r++)
            if (gzp.kind == 1) pp[r] = gzp.fac * p0[r];
            else if (gzp.kind == 2 && act[r]) pp[r] = gv(i, jw + r, 2);
        }
        const double* zk = zt + (k - kb) * 8;
        Ax6 Z{};
        double czm = 0.0, czp = 0.0, cz0 = 0.0, vz;
        if (MODE == 0) {
          czm = zk[0];
          czp = zk[1];
          cz0 = zk[2];
          vz = zk[3];
        } else {
          Z = Ax6{zk[0], zk[1], zk[2], zk[3], zk[4], zk[5]};
          vz = zk[6];
        }
#pragma unroll
        for (int r = 0; r < kCRW; r++) {
          const int j = jw + r;
          double ym = r == 0 ? ylo : p0[r - 1];
          double yp = r == kCRW - 1 ? yhi : p0[r + 1];
          double xmr = xm[r], xpr = xp[r];
          if (edge && act[r]) {
            if (i == 2) {
              const CGhost gh = cghost(b, 1);
              if (gh.kind) xmr = gh.kind == 1 ? gh.fac * p0[r] : gv(A.s0 - 1, j, k);
            }
            if (i == A.s0 - 1) {
              const CGhost gh = cghost(b, 2);
              if (gh.kind) xpr = gh.kind == 1 ? gh.fac * p0[r] : gv(2, j, k);
            }
            if (j == 2) {
              const CGhost gh = cghost(b, 3);
              if (gh.kind) ym = gh.kind == 1 ? gh.fac * p0[r] : gv(i, A.s1 - 1, k);
            }
            if (j == A.s1 - 1) {
              const CGhost gh = cghost(b, 4);
              if (gh.kind) yp = gh.kind == 1 ? gh.fac * p0[r] : gv(i, 2, k);
            }
          }
          const double c = p0[r];
          double v;
          if constexpr (MODE == 0) {
            v = ((cxm * xmr + cxp * xpr) + (cym[r] * ym + cyp[r] * yp)) + ((czm * pm[r] + czp * pp[r]) + (c0xy[r] + cz0) * c);
          } else {
            double gl = xmr * X.a1 + c * X.a2, gr = c * X.b1 + xpr * X.b2;
            if (act[r]) {
              gl = gl * kx(i, j, k);
              gr = gr * kx(i + 1, j, k);
            }
            v = gl * X.o1 + gr * X.o2;
            gl = ym * Y[r].a1 + c * Y[r].a2;
            gr = c * Y[r].b1 + yp * Y[r].b2;
            if (act[r]) {
              gl = gl * ky(i, j, k);
              gr = gr * ky(i, j + 1, k);
            }
            v = v + (gl * Y[r].o1 + gr * Y[r].o2);
            gl = pm[r] * Z.a1 + c * Z.a2;
            gr = c * Z.b1 + pp[r] * Z.b2;
            if (act[r]) {
              gl = gl * kz(i, j, k);
              gr = gr * kz(i, j, k + 1);
            }
            v = v + (gl * Z.o1 + gr * Z.o2);
            if (MODE == 3) {
              v = v * coeff;
              v = v + c;
            }
          }
          v = v * (vxy[r] * vz);
          if (act[r]) {
            out[r * (int)s0] = v;
            if (FZ) {
              outp[r * (int)s0] = c;
              xo[r * (int)s0] = xv[r] + ring[sk + roff(j, ak)] * alpha_prev;  // x += alpha p (staged p)
            }
            acc += c * v;
          }
        }
#pragma unroll
        for (int r = 0; r < kCRW; r++) {
          pm[r] = p0[r];
          p0[r] = pp[r];
          if (FZ) xv[r] = xn[r];
        }
        release(qk);  // this warp is done with plane k's stage
      }
    }
  }
  finish_alpha(acc, S, partial, ticket);
}

// the CC operator kernel's grid: tiles x plane chunks, one resident wave;
// klen = planes per chunk
inline dim3 cc_lap_grid(const DF& a, int nsm, const void* kern, bool fz, int& klen) {
  // occupancy with the largest z table (one chunk), then the chunking
  const int tiles = cc_tiles(a);
  const int nk = a.s2 - 2;
  int occ = 0;
  cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cc_smem(nk, fz));
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, kCThreads, cc_smem(nk, fz));
  int chunks = std::max(1, std::min(nk, (std::max(occ, 1) * std::max(nsm, 1)) / std::max(tiles, 1)));
  klen = (nk + chunks - 1) / chunks;
  chunks = (nk + klen - 1) / klen;
  return dim3((unsigned)tiles, (unsigned)chunks, 1);
}

// the 3-D tensor map of a CC field for the staged operator's tensor loads
// (box 36 x 18 x 1 of FP64; rows must be a 16-byte multiple: even s0)
inline bool cc_tensor_map(CUtensorMap* out, const DF& a) {
  using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  static EncodeFn fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !f)
      return false;
    fn = reinterpret_cast<EncodeFn>(f);
  }
  if ((a.s0 & 1) || (reinterpret_cast<uintptr_t>(a.f) & 15)) return false;
  const cuuint64_t dims[3] = {(cuuint64_t)a.s0, (cuuint64_t)a.s1, (cuuint64_t)a.s2};
  const cuuint64_t strides[2] = {(cuuint64_t)a.s0 * 8, (cuuint64_t)a.s0 * a.s1 * 8};
  const cuuint32_t box[3] = {(cuuint32_t)kCRS, (cuuint32_t)kCRows, 1u};
  const cuuint32_t es[3] = {1u, 1u, 1u};
  return fn(out, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, a.f, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

}  // namespace mg
