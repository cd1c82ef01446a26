// unet.cuh -- kernels of the learned preconditioner: a 3-D U-Net whose 3x3x3
// convolutions run as implicit GEMMs on the 5th-generation tensor cores
// (tcgen05.mma, BF16 operands staged in shared memory by bulk TMA copies,
// FP32 accumulators in tensor memory), plus the memory-bound pieces around
// them (input packing, pooling, upsampling, the 1x1 head, loss, Adam).
//
// Activation layout ("UT"): BF16, channels blocked by 8, each 8-channel group
// a padded 3-D grid with one zero ghost layer per side, x fastest:
//   element (c, x, y, z) at  base + (c/8)*GS*8 + (G + z*PS + y*Xp + x)*8 + c%8
// with Xp = X+2, Yp = Y+2, PS = Xp*(Y+1) + max(Xp, 128) (>= Xp*Yp: each plane
// ends in at least 128 zero voxels, so a 128-voxel tile that starts in the
// interior rows never reaches the next plane's data) and G = 256 guard voxels
// before and after each group.  The ghost layer, the plane tails and the
// guards are zero and stay zero: kernels write interior voxels only.  The
// padded (x, y) position of a voxel within its plane, p = y*Xp + x, is the GEMM
// row index: a convolution tap (dx, dy) shifts p by (dy-1)*Xp + (dx-1), i.e.
// shifts the operand's start address by 16 bytes per voxel.
#pragma once
#include <cuda_bf16.h>

#include <cstdint>

#include "tc.cuh"

namespace un {

typedef __nv_bfloat16 bf16;

constexpr int kGuard = 256;   // guard voxels per side of a channel group
constexpr int kTile = 128;    // GEMM rows (voxel positions) per CTA
constexpr int kConvThreads = 128;

// error codes written to the device error word
enum { kErrFull = 1, kErrEmpty = 2, kErrDone = 3 };

struct Geo {
  int X, Y, Z;      // interior cells
  int Xp, Yp;       // X+2, Y+2
  int PS;           // plane stride (voxels)
  long long GS;     // channel-group stride (voxels), guards included
  __host__ __device__ static Geo make(int X, int Y, int Z) {
    Geo g;
    g.X = X; g.Y = Y; g.Z = Z;
    g.Xp = X + 2; g.Yp = Y + 2;
    g.PS = g.Xp * (Y + 1) + (g.Xp > kTile ? g.Xp : kTile);
    g.GS = 2LL * kGuard + (long long)(Z + 2) * g.PS;
    return g;
  }
  __host__ __device__ int tiles_per_plane() const { return (Y * Xp + kTile - 1) / kTile; }
  // voxel offset (in voxels) of padded (x, y, z) inside a group, guard included
  __host__ __device__ long long vox(int x, int y, int z) const {
    return kGuard + (long long)z * PS + (long long)y * Xp + x;
  }
};

__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 r;
  __nv_bfloat162 h;
  h = __floats2bfloat162_rn(v[0], v[1]); r.x = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[2], v[3]); r.y = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[4], v[5]); r.z = *reinterpret_cast<uint32_t*>(&h);
  h = __floats2bfloat162_rn(v[6], v[7]); r.w = *reinterpret_cast<uint32_t*>(&h);
  return r;
}
__device__ __forceinline__ void unpack8(uint4 r, float* v) {
  const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
  for (int i = 0; i < 4; i++) {
    __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
    float2 f = __bfloat1622float2(h);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}

// ---------------------------------------------------------------------------
// 3x3x3 convolution, zero padding, as an implicit GEMM on tcgen05.
//
// CTA = 128 consecutive positions p0..p0+127 of one plane z (p0 = Xp + 128*t):
// GEMM rows.  N = output channels (16..256, multiple of 16).  K runs over
// (dz, 16-channel chunk j, tap dy, tap dx): for each (dz, j) the CTA stages
//  * A: the input span of plane z+dz-1, positions [p0-Xp-1, p0+128+Xp+1),
//    as two K-major planes (channels 16j..16j+7 and 16j+8..16j+15), each
//    L = 128 + 2*(Xp+1) rows of 16 bytes;
//  * B: the packed weights of the 9 (dy, dx) taps, [2][9][N][8] BF16,
// with one bulk copy per plane, and issues 9 MMAs (M=128, N, K=16) whose A
// start is the span shifted by dy*Xp + dx rows.  A pipeline of S stages
// (mbarriers for full / free) overlaps the copies of chunk c+S-1 with the
// MMAs of chunk c.  One thread issues copies and MMAs; all four warps read
// the accumulator back (tcgen05.ld) for the epilogue.
//
// Inputs may be two tensors (channel concatenation): groups [0, cgA) come
// from inA, [cgA, cgA+cgB) from inB.  An odd group count leaves the second
// half of the last chunk without data: its weights are zero, and the staged
// buffers are cleared at the start so that what the MMA multiplies by those
// zeros is finite.
//
// Epilogue modes:
//  kRelu  : out = max(acc + bias, 0)                       (forward)
//  kLinear: out = acc (* [mask > 0] when a mask is given)   (backward data)
// Outputs: groups [0, ocgA) to outA, the rest to outB (same geometry).  With
// head_w set (N == 16), also y = head_b + sum_c head_w[c]*out_c is written as
// FP32 to y32 and, when z64 is set, zscale[0]*y as FP64, both in the
// (X+2)(Y+2)(Z+2) cell-centred layout of a grid_field.
// ---------------------------------------------------------------------------
enum { kRelu = 0, kLinear = 1 };

struct ConvArgs {
  Geo g;
  const bf16* inA; const bf16* inB; int cgA, cgB;
  const bf16* wt;        // [3][nk][2][9][N][8]
  const float* bias;     // [N] (kRelu)
  int N, nk, S;          // out channels, 16-channel chunks, pipeline stages
  int L;                 // span rows
  int mode;
  bf16* outA; bf16* outB; int ocgA;
  const bf16* maskA; const bf16* maskB;   // kLinear: zero where mask <= 0
  const float* head_w; const float* head_b; float* y32; double* z64; const double* zscale;
  int* err;
  const int* skip;       // nonzero *skip: return at once (the enclosing solve is done)
};

__host__ __device__ inline int conv_stage_bytes(int L, int N) {
  int b = 2 * L * 16 + 2 * 9 * N * 16;
  return (b + 127) & ~127;
}

// epilogue of one 128-position tile: thread m (warp m/32 reads TMEM lanes
// 32*(m/32) ..) takes row m of the accumulator at TMEM column `tcol`:
// bias + ReLU (kRelu) or mask (kLinear), BF16 stores to the interior voxels,
// and the fused 1x1 head when requested.  Warp-collective (tcgen05.ld).
__device__ __forceinline__ void conv_epilogue(const ConvArgs& a, uint32_t tcol, int m, int z, int p0, bool done) {
  const Geo& g = a.g;
  const int N = a.N;
  const int warp = m >> 5;
  const int p = p0 + m;
  const int yy = p / g.Xp, xx = p - yy * g.Xp;
  const bool valid = done && xx >= 1 && xx <= g.X && yy >= 1 && yy <= g.Y;
  const long long vo = kGuard + (long long)z * g.PS + p;   // voxel offset in a group
  const long long gsE = g.GS * 8;
  float hy = 0.f;
  for (int c0 = 0; c0 < N; c0 += 16) {
    float v[16];
    tc::tmem_ld16(tcol + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
    if (!done) continue;
    if (a.mode == kRelu) {
#pragma unroll
      for (int i = 0; i < 16; i++) v[i] = fmaxf(v[i] + a.bias[c0 + i], 0.f);
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
      const int cg = c0 / 8 + h;
      const bool inA = cg < a.ocgA;
      const long long off = (inA ? cg : cg - a.ocgA) * gsE + vo * 8;
      if (a.mode == kLinear) {
        const bf16* mk = inA ? a.maskA : a.maskB;
        if (mk && valid) {
          float mv[8];
          unpack8(*reinterpret_cast<const uint4*>(mk + off), mv);
#pragma unroll
          for (int i = 0; i < 8; i++) v[8 * h + i] = mv[i] > 0.f ? v[8 * h + i] : 0.f;
        }
      }
      if (valid) {
        bf16* dst = (inA ? a.outA : a.outB) + off;
        *reinterpret_cast<uint4*>(dst) = pack8(v + 8 * h);
      }
    }
    if (a.head_w) {
      // the head sees the stored (BF16-rounded) activations
#pragma unroll
      for (int i = 0; i < 16; i++) hy += a.head_w[c0 + i] * __bfloat162float(__float2bfloat16_rn(v[i]));
    }
  }
  if (a.head_w && valid) {
    const float yv = hy + a.head_b[0];
    const long long ci = (long long)xx + (long long)g.Xp * (yy + (long long)g.Yp * z);
    if (a.y32) a.y32[ci] = yv;
    if (a.z64) a.z64[ci] = a.zscale[0] * (double)yv;
  }
}

__global__ void __launch_bounds__(kConvThreads) k_conv3(ConvArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar_full[8];
  __shared__ __align__(8) uint64_t bar_empty[8];
  __shared__ __align__(8) uint64_t bar_done;
  __shared__ uint32_t tmem_slot;

  if (a.skip && *a.skip) return;
  const int tid = threadIdx.x, warp = tid >> 5;
  const Geo& g = a.g;
  const int z = blockIdx.y + 1;
  const int p0 = g.Xp + kTile * blockIdx.x;
  const int N = a.N, S = a.S, L = a.L;
  const int SB = conv_stage_bytes(L, N);
  const int nchunk = 3 * a.nk;
  const int cgT = a.cgA + a.cgB;
  const uint32_t sbase = tc::smem_u32(smem);
  const uint32_t ncols = N <= 32 ? 32 : (N <= 64 ? 64 : (N <= 128 ? 128 : 256));

  if (cgT & 1) {  // finite contents under the zero weights of the missing half
    uint4 zero = make_uint4(0, 0, 0, 0);
    uint4* s4 = reinterpret_cast<uint4*>(smem);
    for (int i = tid; i < S * SB / 16; i += kConvThreads) s4[i] = zero;
    tc::fence_proxy_async_smem();
  }
  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      tc::mbar_init(tc::smem_u32(&bar_full[s]), 1);
      tc::mbar_init(tc::smem_u32(&bar_empty[s]), 1);
    }
    tc::mbar_init(tc::smem_u32(&bar_done), 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_u32(&tmem_slot), ncols);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;

  bool ok = true;
  if (tid == 0) {
    const long long gsE = g.GS * 8;  // group stride in elements
    auto issue = [&](int c) {
      const int s = c % S;
      const int dz = c / a.nk, j = c % a.nk;
      const uint32_t st = sbase + s * SB;
      const uint32_t bar = tc::smem_u32(&bar_full[s]);
      const int halves = (2 * j + 1 < cgT) ? 2 : 1;
      const uint32_t abytes = (uint32_t)L * 16;
      const uint32_t bbytes = 2u * 9u * (uint32_t)N * 16u;
      tc::mbar_expect_tx(bar, halves * abytes + bbytes);
      const long long v0 = kGuard + (long long)(z + dz - 1) * g.PS + p0 - g.Xp - 1;
      for (int h = 0; h < halves; h++) {
        const int cg = 2 * j + h;
        const bf16* src = cg < a.cgA ? a.inA + cg * gsE : a.inB + (cg - a.cgA) * gsE;
        tc::bulk_g2s(st + h * abytes, src + v0 * 8, abytes, bar);
      }
      tc::bulk_g2s(st + 2 * abytes, a.wt + (long long)c * 2 * 9 * N * 8, bbytes, bar);
    };
    const int pro = nchunk < S ? nchunk : S;
    for (int c = 0; c < pro; c++) issue(c);
    int issued = pro, c = 0;
    const uint32_t idesc = tc::idesc_bf16(kTile, N);
    const uint32_t lboA = (uint32_t)L * 16, lboB = 9u * (uint32_t)N * 16u;
    for (; c < nchunk && ok; c++) {
      const int s = c % S;
      ok = tc::mbar_wait(tc::smem_u32(&bar_full[s]), (c / S) & 1, a.err, kErrFull);
      if (!ok) break;
      tc::tc_fence_after();
      const uint32_t st = sbase + s * SB;
      const uint32_t sB = st + 2 * lboA;
#pragma unroll 1
      for (int t = 0; t < 9; t++) {
        const int dy = t / 3, dx = t % 3;
        const uint64_t ad = tc::sdesc(st + (uint32_t)(dy * g.Xp + dx) * 16u, lboA, 128);
        const uint64_t bd = tc::sdesc(sB + (uint32_t)t * (uint32_t)N * 16u, lboB, 128);
        tc::mma_bf16(tmem, ad, bd, idesc, (c > 0 || t > 0) ? 1u : 0u);
      }
      tc::mma_commit(tc::smem_u32(&bar_empty[s]));
      // refill the stage of the previous chunk once its MMAs are done
      if (c >= 1 && c - 1 + S < nchunk) {
        const int sp = (c - 1) % S;
        ok = tc::mbar_wait(tc::smem_u32(&bar_empty[sp]), ((c - 1) / S) & 1, a.err, kErrEmpty);
        if (ok) issue(issued++);
      }
    }
    if (!ok) {  // gave up: let the copies already in flight land first
      for (int q = c; q < issued; q++) tc::mbar_wait(tc::smem_u32(&bar_full[q % S]), (q / S) & 1, nullptr, 0);
    }
    tc::mma_commit(tc::smem_u32(&bar_done));
  }
  __syncwarp();
  // every thread waits for the accumulator (thread 0 committed it even when
  // it gave up early, so the phase completes once the issued MMAs retire)
  const bool done = __syncthreads_and(tc::mbar_wait_sleep(tc::smem_u32(&bar_done), 0, a.err, kErrDone)) != 0;
  tc::tc_fence_after();

  conv_epilogue(a, tmem, tid, z, p0, done);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// Weight gradient on tcgen05: dW[co][ci][tap] = sum over interior voxels v of
// dOut[v][co] * in[v + shift(tap)][ci].  GEMM with M = 128 rows = (shift s,
// input group, channel) triples, N = co, K = voxel positions; both operands
// MN-major straight from the activation layout (8 channels x 16 bytes per
// voxel, consecutive voxels 16 bytes apart).
//
// A CTA owns nsh (dz, dy) shifts x ncg input groups (nsh*ncg <= 16 planes of
// 130 rows: positions p0 + (dy-1)*Xp - 1 + [0,130) of plane z+dz-1) and a
// range of (plane, tile) work items; per item it stages those planes and the
// dOut tile (N/8 planes of 128 rows) and issues 3 (dx) x 8 (K=16 steps) MMAs
// into three accumulators D_dx (TMEM columns dx*N .. dx*N+N-1).  Planes
// beyond nsh*ncg are never loaded and feed only rows that are discarded.
// The CTA adds its partial sums to the FP32 gradient with atomics (the
// summation order across CTAs is not fixed).
// ---------------------------------------------------------------------------
constexpr int kWRows = 130;

struct WgradArgs {
  Geo g;
  const bf16* inA; const bf16* inB; int cgA, cgB;
  const bf16* dout; int N;
  int nsh, ncg;          // shifts per CTA (1, 3 or 9), input groups per CTA
  int items, per_cta;    // work items (planes x tiles) and items per CTA
  int S;
  float* dW; int cin;    // [co][cin][27]
  int* err;
};

// one stage: the nreal staged input planes, then the dOut tile; the rows of
// the 16 - nreal padded plane groups read past them (into the dOut tile or
// the next stage), and past the last stage into wgrad_tail_bytes of padding
__host__ __device__ inline int wgrad_stage_bytes(int N, int nreal) {
  return (nreal * kWRows * 16 + N * 256 + 127) & ~127;
}
__host__ __device__ inline int wgrad_tail_bytes(int N, int nreal) {
  const int t = 16 * kWRows * 16 - wgrad_stage_bytes(N, nreal);
  return t > 0 ? ((t + 127) & ~127) : 0;
}

__global__ void __launch_bounds__(kConvThreads) k_wgrad(WgradArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar_full[4];
  __shared__ __align__(8) uint64_t bar_empty[4];
  __shared__ __align__(8) uint64_t bar_done;
  __shared__ uint32_t tmem_slot;

  const int tid = threadIdx.x, warp = tid >> 5;
  const Geo& g = a.g;
  const int N = a.N, S = a.S;
  const int sg = blockIdx.x, ct = blockIdx.y;
  const int it0 = blockIdx.z * a.per_cta;
  const int it1 = min(a.items, it0 + a.per_cta);
  const int nit = it1 > it0 ? it1 - it0 : 0;
  const int cg0 = ct * a.ncg;
  const int cgT = a.cgA + a.cgB;
  const int ncg = min(a.ncg, cgT - cg0);
  const int NR = a.nsh * a.ncg;                // staged planes per stage
  const int SB = wgrad_stage_bytes(N, NR);
  const int APL = kWRows * 16;                 // bytes per staged input plane
  const uint32_t sbase = tc::smem_u32(smem);
  const int cols = 3 * N;
  const uint32_t ncols = cols <= 32 ? 32 : (cols <= 64 ? 64 : (cols <= 128 ? 128 : (cols <= 256 ? 256 : 512)));
  const int tpp = g.tiles_per_plane();

  if (tid == 0) {
    for (int s = 0; s < S; s++) {
      tc::mbar_init(tc::smem_u32(&bar_full[s]), 1);
      tc::mbar_init(tc::smem_u32(&bar_empty[s]), 1);
    }
    tc::mbar_init(tc::smem_u32(&bar_done), 1);
    tc::fence_mbar_init();
  }
  if (warp == 0) {
    tc::tmem_alloc(tc::smem_u32(&tmem_slot), ncols);
    tc::tmem_relinquish();
  }
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (tid == 0 && nit > 0) {
    const long long gsE = g.GS * 8;
    auto issue = [&](int q) {
      const int s = q % S;
      const int item = it0 + q;
      const int z = item / tpp + 1, t = item % tpp;
      const int p0 = g.Xp + kTile * t;
      const uint32_t st = sbase + s * SB;
      const uint32_t bar = tc::smem_u32(&bar_full[s]);
      tc::mbar_expect_tx(bar, (uint32_t)(a.nsh * ncg * APL + N * 256));
      for (int sh = 0; sh < a.nsh; sh++) {
        const int shg = sg * a.nsh + sh;
        const int dz = shg / 3, dy = shg % 3;
        const long long v0 = kGuard + (long long)(z + dz - 1) * g.PS + p0 + (dy - 1) * g.Xp - 1;
        for (int c = 0; c < ncg; c++) {
          const int cg = cg0 + c;
          const bf16* src = cg < a.cgA ? a.inA + cg * gsE : a.inB + (cg - a.cgA) * gsE;
          tc::bulk_g2s(st + (sh * ncg + c) * APL, src + v0 * 8, APL, bar);
        }
      }
      const long long vo = kGuard + (long long)z * g.PS + p0;
      for (int c = 0; c < N / 8; c++)
        tc::bulk_g2s(st + NR * APL + c * 2048, a.dout + c * gsE + vo * 8, 2048, bar);
    };
    const int pro = nit < S ? nit : S;
    for (int q = 0; q < pro; q++) issue(q);
    int issued = pro, q = 0;
    bool ok = true;
    const uint32_t idesc = tc::idesc_bf16(kTile, N, 1, 1);
    for (; q < nit && ok; q++) {
      const int s = q % S;
      ok = tc::mbar_wait(tc::smem_u32(&bar_full[s]), (q / S) & 1, a.err, kErrFull);
      if (!ok) break;
      tc::tc_fence_after();
      const uint32_t st = sbase + s * SB;
      const uint32_t sB = st + NR * APL;
#pragma unroll 1
      for (int dx = 0; dx < 3; dx++) {
#pragma unroll 1
        for (int kk = 0; kk < 8; kk++) {
          const uint64_t ad = tc::sdesc(st + (uint32_t)(dx + 16 * kk) * 16u, 128, (uint32_t)APL);
          const uint64_t bd = tc::sdesc(sB + (uint32_t)(16 * kk) * 16u, 128, 2048);
          tc::mma_bf16(tmem + (uint32_t)(dx * N), ad, bd, idesc, (q > 0 || kk > 0) ? 1u : 0u);
        }
      }
      tc::mma_commit(tc::smem_u32(&bar_empty[s]));
      if (q >= 1 && q - 1 + S < nit) {
        const int sp = (q - 1) % S;
        ok = tc::mbar_wait(tc::smem_u32(&bar_empty[sp]), ((q - 1) / S) & 1, a.err, kErrEmpty);
        if (ok) issue(issued++);
      }
    }
    if (!ok) {
      for (int r = q; r < issued; r++) tc::mbar_wait(tc::smem_u32(&bar_full[r % S]), (r / S) & 1, nullptr, 0);
    }
    tc::mma_commit(tc::smem_u32(&bar_done));
  }
  __syncwarp();
  bool done = true;
  if (nit > 0) done = tc::mbar_wait_sleep(tc::smem_u32(&bar_done), 0, a.err, kErrDone);
  done = __syncthreads_and(done) != 0 && nit > 0;
  tc::tc_fence_after();

  // row m: plane gA = m/8 (shift m/8/ncg, group m/8%ncg), channel m%8
  const int m = tid;
  const int gA = m >> 3;
  const bool row_ok = done && gA < a.nsh * ncg;
  const int sh = row_ok ? gA / ncg : 0, c = row_ok ? gA % ncg : 0;
  const int shg = sg * a.nsh + sh;
  const int ci = (cg0 + c) * 8 + (m & 7);
  const int tapb = (shg / 3) * 9 + (shg % 3) * 3;
  if (nit > 0) {
    for (int dx = 0; dx < 3; dx++) {
      for (int c0 = 0; c0 < N; c0 += 16) {
        float v[16];
        tc::tmem_ld16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(dx * N + c0), v);
        if (row_ok && ci < a.cin) {
#pragma unroll
          for (int i = 0; i < 16; i++) atomicAdd(&a.dW[((long long)(c0 + i) * a.cin + ci) * 27 + tapb + dx], v[i]);
        }
      }
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, ncols);
}

// ---------------------------------------------------------------------------
// Memory-bound kernels (one thread per interior voxel, 16-byte accesses)
// ---------------------------------------------------------------------------

// packed GEMM weights from the FP32 master W[co][ci][27]
//  fwd: P[dz][j][h][t9][n][e] = W[n][16j+8h+e][dz*9+t9]            (n < cout)
//  bwd: P[dz][j][h][t9][n][e] = W[16j+8h+e][n][26-(dz*9+t9)]        (n < cin)
__global__ void k_pack_w(const float* W, int cin, int cout, int bwd, bf16* P) {
  const int kin = bwd ? cout : cin, nout = bwd ? cin : cout;
  const int nk = (kin + 15) / 16;
  const long long total = 3LL * nk * 2 * 9 * nout * 8;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int e = r % 8; r /= 8;
    const int n = r % nout; r /= nout;
    const int t9 = r % 9; r /= 9;
    const int h = r % 2; r /= 2;
    const int j = r % nk; r /= nk;
    const int dz = (int)r;
    const int k = 16 * j + 8 * h + e;
    float v = 0.f;
    if (k < kin) {
      const int tap = dz * 9 + t9;
      v = bwd ? W[((long long)k * cin + n) * 27 + 26 - tap] : W[((long long)n * cin + k) * 27 + tap];
    }
    P[i] = __float2bfloat16_rn(v);
  }
}

__device__ __forceinline__ bool interior_of(const Geo& g, long long i, int& x, int& y, int& z) {
  x = (int)(i % g.X) + 1;
  long long r = i / g.X;
  y = (int)(r % g.Y) + 1;
  z = (int)(r / g.Y) + 1;
  return z <= g.Z;
}

// input tensor (one group): ch0 = r / rms(r), ch1 = feature, ch2..7 = 0;
// r and feat in the (X+2)(Y+2)(Z+2) cell-centred layout
__global__ void k_pack_in(Geo g, const double* r, const float* feat, const double* scal, bf16* in, const int* skip) {
  if (skip && *skip) return;
  const double sinv = scal[1];
  const long long n = (long long)g.X * g.Y * g.Z;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    interior_of(g, i, x, y, z);
    const long long c = x + (long long)g.Xp * (y + (long long)g.Yp * z);
    float v[8] = {(float)(r[c] * sinv), feat ? feat[c] : 0.f, 0, 0, 0, 0, 0, 0};
    *reinterpret_cast<uint4*>(in + g.vox(x, y, z) * 8) = pack8(v);
  }
}

// per-cell feature of a face-coefficient operator: log10(mean of the six
// face values) / 3, cell-centred layout (kx, ky, kz face fields of the mesh)
__global__ void k_feat_faces(Geo g, const double* kx, const double* ky, const double* kz, float* feat) {
  const long long n = (long long)g.X * g.Y * g.Z;
  const long long sx = g.X + 2, sy = g.Y + 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    interior_of(g, i, x, y, z);
    // face arrays: Fx (sx+1, sy, sz), Fy (sx, sy+1, sz), Fz (sx, sy, sz+1)
    const double a = kx[x + (sx + 1) * (y + sy * (long long)z)] + kx[x + 1 + (sx + 1) * (y + sy * (long long)z)];
    const double b = ky[x + sx * (y + (sy + 1) * (long long)z)] + ky[x + sx * (y + 1 + (sy + 1) * (long long)z)];
    const double c = kz[x + sx * (y + sy * (long long)z)] + kz[x + sx * (y + sy * (long long)(z + 1))];
    const double mean = (a + b + c) / 6.0;
    feat[x + sx * (y + sy * (long long)z)] = mean > 0.0 ? (float)(log10(mean) / 3.0) : 0.f;
  }
}

// 2x2x2 average: out (coarse geometry gc) from in (fine geometry gf)
__global__ void k_pool(Geo gf, Geo gc, int ncg, const bf16* in, bf16* out, const int* skip) {
  if (skip && *skip) return;
  const long long n = (long long)gc.X * gc.Y * gc.Z * ncg;
  const long long nv = (long long)gc.X * gc.Y * gc.Z;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int cg = (int)(i / nv);
    int x, y, z;
    interior_of(gc, i % nv, x, y, z);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const bf16* src = in + cg * gf.GS * 8;
    for (int k = 0; k < 8; k++) {
      float v[8];
      unpack8(*reinterpret_cast<const uint4*>(src + gf.vox(2 * x - 1 + (k & 1), 2 * y - 1 + ((k >> 1) & 1), 2 * z - 1 + (k >> 2)) * 8), v);
#pragma unroll
      for (int e = 0; e < 8; e++) acc[e] += v[e];
    }
#pragma unroll
    for (int e = 0; e < 8; e++) acc[e] *= 0.125f;
    *reinterpret_cast<uint4*>(out + cg * gc.GS * 8 + gc.vox(x, y, z) * 8) = pack8(acc);
  }
}

// nearest-neighbour x2: out (fine) from in (coarse)
__global__ void k_up(Geo gc, Geo gf, int ncg, const bf16* in, bf16* out, const int* skip) {
  if (skip && *skip) return;
  const long long nv = (long long)gf.X * gf.Y * gf.Z;
  const long long n = nv * ncg;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int cg = (int)(i / nv);
    int x, y, z;
    interior_of(gf, i % nv, x, y, z);
    *reinterpret_cast<uint4*>(out + cg * gf.GS * 8 + gf.vox(x, y, z) * 8) =
        *reinterpret_cast<const uint4*>(in + cg * gc.GS * 8 + gc.vox((x + 1) >> 1, (y + 1) >> 1, (z + 1) >> 1) * 8);
  }
}

// backward of pool + skip: d (fine, in place) = (d + dp[parent] / 8) * [act > 0]
__global__ void k_pool_bwd(Geo gf, Geo gc, int ncg, bf16* d, const bf16* dp, const bf16* act) {
  const long long nv = (long long)gf.X * gf.Y * gf.Z;
  const long long n = nv * ncg;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int cg = (int)(i / nv);
    int x, y, z;
    interior_of(gf, i % nv, x, y, z);
    const long long of = cg * gf.GS * 8 + gf.vox(x, y, z) * 8;
    float a[8], b[8], m[8];
    unpack8(*reinterpret_cast<const uint4*>(d + of), a);
    unpack8(*reinterpret_cast<const uint4*>(dp + cg * gc.GS * 8 + gc.vox((x + 1) >> 1, (y + 1) >> 1, (z + 1) >> 1) * 8), b);
    unpack8(*reinterpret_cast<const uint4*>(act + of), m);
#pragma unroll
    for (int e = 0; e < 8; e++) a[e] = m[e] > 0.f ? a[e] + 0.125f * b[e] : 0.f;
    *reinterpret_cast<uint4*>(d + of) = pack8(a);
  }
}

// backward of upsampling: dc (coarse) = sum of the 8 children of du * [act > 0]
__global__ void k_up_bwd(Geo gf, Geo gc, int ncg, const bf16* du, const bf16* act, bf16* dc) {
  const long long nv = (long long)gc.X * gc.Y * gc.Z;
  const long long n = nv * ncg;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int cg = (int)(i / nv);
    int x, y, z;
    interior_of(gc, i % nv, x, y, z);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const bf16* src = du + cg * gf.GS * 8;
    for (int k = 0; k < 8; k++) {
      float v[8];
      unpack8(*reinterpret_cast<const uint4*>(src + gf.vox(2 * x - 1 + (k & 1), 2 * y - 1 + ((k >> 1) & 1), 2 * z - 1 + (k >> 2)) * 8), v);
#pragma unroll
      for (int e = 0; e < 8; e++) acc[e] += v[e];
    }
    const long long oc = cg * gc.GS * 8 + gc.vox(x, y, z) * 8;
    float m[8];
    unpack8(*reinterpret_cast<const uint4*>(act + oc), m);
#pragma unroll
    for (int e = 0; e < 8; e++) acc[e] = m[e] > 0.f ? acc[e] : 0.f;
    *reinterpret_cast<uint4*>(dc + oc) = pack8(acc);
  }
}

// ---- deterministic reductions: fixed grid, block partials, ordered sum ----
constexpr int kURedBlocks = 296;
constexpr int kURedThreads = 256;

template <int K>
__device__ __forceinline__ void block_sums(float (&v)[K], float* out /* K values of this block */) {
  __shared__ float sh[K][kURedThreads / 32];
#pragma unroll
  for (int k = 0; k < K; k++) {
    float x = v[k];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sh[k][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    float x = 0.f;
    for (int w = 0; w < kURedThreads / 32; w++) x += sh[threadIdx.x][w];
    out[threadIdx.x] = x;
  }
  __syncthreads();
}

// sum of squares of r over the interior, in FP64: partial[b]
__global__ void __launch_bounds__(kURedThreads) k_sumsq_cc(Geo g, const double* r, double* partial, const int* skip) {
  if (skip && *skip) return;
  const long long n = (long long)g.X * g.Y * g.Z;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    interior_of(g, i, x, y, z);
    const double v = r[x + (long long)g.Xp * (y + (long long)g.Yp * z)];
    acc += v * v;
  }
  __shared__ double sh[kURedThreads / 32];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < kURedThreads / 32; w++) s += sh[w];
    partial[blockIdx.x] = s;
  }
}

// scal[0] = rms(r), scal[1] = 1/rms, scal[2] = out_scale * rms  (0 when r == 0)
__global__ void k_scale_fin(const double* partial, int nb, long long n, double out_scale, double* scal,
                            const int* skip) {
  if (threadIdx.x != 0 || (skip && *skip)) return;
  double s = 0.0;
  for (int b = 0; b < nb; b++) s += partial[b];
  const double rms = sqrt(s / (double)n);
  scal[0] = rms;
  scal[1] = rms > 0.0 ? 1.0 / rms : 0.0;
  scal[2] = out_scale * rms;
}

// bias gradient: partial[b][c] = sum over the block's voxels of d[c]
__global__ void __launch_bounds__(kURedThreads) k_bias_grad(Geo g, int ncg, const bf16* d, float* partial) {
  const long long nv = (long long)g.X * g.Y * g.Z;
  const int C = ncg * 8;
  for (int cg = 0; cg < ncg; cg++) {
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nv; i += (long long)gridDim.x * blockDim.x) {
      int x, y, z;
      interior_of(g, i, x, y, z);
      float v[8];
      unpack8(*reinterpret_cast<const uint4*>(d + cg * g.GS * 8 + g.vox(x, y, z) * 8), v);
#pragma unroll
      for (int e = 0; e < 8; e++) acc[e] += v[e];
    }
    block_sums<8>(acc, partial + (long long)blockIdx.x * C + cg * 8);
  }
}

// out[c] = sum_b partial[b][c] (+ out[c] when accumulate)
__global__ void k_sum_partials(const float* partial, int nb, int C, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= C) return;
  float s = 0.f;
  for (int b = 0; b < nb; b++) s += partial[(long long)b * C + c];
  out[c] = s;
}

// target t = e / scale (FP32 cell-centred layout) and partial sums of t^2
__global__ void __launch_bounds__(kURedThreads) k_target(Geo g, const double* e, const double* scal, float* t,
                                                        float* partial) {
  const long long n = (long long)g.X * g.Y * g.Z;
  const double inv = scal[2] > 0.0 ? 1.0 / scal[2] : 0.0;
  float acc[1] = {0.f};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y, z;
    interior_of(g, i, x, y, z);
    const long long c = x + (long long)g.Xp * (y + (long long)g.Yp * z);
    const float v = (float)(e[c] * inv);
    t[c] = v;
    acc[0] += v * v;
  }
  block_sums<1>(acc, partial + blockIdx.x);
}

// partial sums per block of y.t and y.y (cosine loss)
__global__ void __launch_bounds__(kURedThreads) k_yt(Geo g, const float* y, const float* t, float* partial) {
  const long long n = (long long)g.X * g.Y * g.Z;
  float acc[2] = {0.f, 0.f};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y_, z;
    interior_of(g, i, x, y_, z);
    const long long c = x + (long long)g.Xp * (y_ + (long long)g.Yp * z);
    acc[0] += y[c] * t[c];
    acc[1] += y[c] * y[c];
  }
  block_sums<2>(acc, partial + (long long)blockIdx.x * 2);
}

// FP64 partial sums per block for the energy-norm loss, with A the solver's
// (negative definite, volume-weighted) operator, s = out_scale rms(r) the
// scale of the target t = e / s (so A t = r / s):
//   [0] a = -y.(A t) = -y.r / s,  [1] E = -t.(A t) = -e.r / s^2
// (these sums cancel heavily where the coefficients are large: FP64)
__global__ void __launch_bounds__(kURedThreads) k_energy_sums(Geo g, const float* y, const double* e,
                                                             const double* r, const double* scal, double* partial) {
  const long long n = (long long)g.X * g.Y * g.Z;
  const double tinv = scal[2] > 0.0 ? 1.0 / scal[2] : 0.0;
  double a0 = 0.0, a1 = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y_, z;
    interior_of(g, i, x, y_, z);
    const long long c = x + (long long)g.Xp * (y_ + (long long)g.Yp * z);
    const double at = r[c] * tinv;
    a0 -= (double)y[c] * at;
    a1 -= e[c] * tinv * at;
  }
  __shared__ double sh[2][kURedThreads / 32];
  for (int o = 16; o > 0; o >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, o);
    a1 += __shfl_down_sync(0xffffffffu, a1, o);
  }
  if ((threadIdx.x & 31) == 0) {
    sh[0][threadIdx.x >> 5] = a0;
    sh[1][threadIdx.x >> 5] = a1;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double s = 0.0;
    for (int w = 0; w < kURedThreads / 32; w++) s += sh[threadIdx.x][w];
    partial[(long long)blockIdx.x * 2 + threadIdx.x] = s;
  }
}

// out = (a, B, E) as FP32 from the FP64 partials: pa[b][2] = (a, E) and
// pb[b] = y.(A y) (B = -y.(A y))
__global__ void k_energy_fin(const double* pa, const double* pb, int nb, float* out) {
  if (threadIdx.x != 0) return;
  double a = 0.0, E = 0.0, yay = 0.0;
  for (int b = 0; b < nb; b++) {
    a += pa[2 * b];
    E += pa[2 * b + 1];
    yay += pb[b];
  }
  out[0] = (float)a;
  out[1] = (float)(-yay);
  out[2] = (float)E;
}

// the loss and the head backward.
//  kind 0 (relative L2):  L = sum (y - t)^2 / T2,  dL/dy = 2 (y - t) / T2
//  kind 1 (cosine, invariant to a positive scale of y: flexible CG is
//    invariant to a rescaling of z at every iteration, so only the direction
//    counts; the sign is kept):
//    L = 1 - y.t / (|y| |t|),  dL/dy = -t / (|y| |t|) + (y.t) y / (|y|^3 |t|)
//  kind 2 (cosine in the energy norm of -A, the norm CG minimises; A e = r,
//    t = e / s, A t = r / s):
//    L = 1 - a / sqrt(B E) with a = -y.(A t), B = -y.(A y), E = -t.(A t),
//    dL/dy = (A t) / sqrt(B E) - a (A y) / (B^1.5 sqrt(E))
// then dh[c] = head_w[c] * dL/dy * [h_c > 0] (dPre of the last conv);
// partial sums per block: [0] (y-t)^2, [1] dL/dy, [2..17] dL/dy * h_c
struct LossArgs {
  Geo g;
  const float* y; const float* t; const float* T2p;
  int kind;
  const float* sums;     // kind 1: y.t, y.y; kind 2: a, B, E
  const float* ay;       // kind 2: A y
  const double* r; const double* scal;   // kind 2: r and s (scal[2])
  const bf16* h; const float* head_w; bf16* dh;
  float* partial;
};

__global__ void __launch_bounds__(kURedThreads) k_loss_head(LossArgs a) {
  const Geo& g = a.g;
  const long long n = (long long)g.X * g.Y * g.Z;
  const float T2 = a.T2p[0] > 0.f ? a.T2p[0] : 1.f;
  float ca = 0.f, cb = 0.f;  // dL/dy = ca * (t or rh) + cb * (y or Ay)
  if (a.kind == 1) {
    const float yt = a.sums[0], yy = a.sums[1] > 0.f ? a.sums[1] : 1.f;
    const float ny = sqrtf(yy), nt = sqrtf(T2);
    ca = -1.f / (ny * nt);
    cb = yt / (yy * ny * nt);
  } else if (a.kind == 2) {
    const float aa = a.sums[0], B = a.sums[1] > 0.f ? a.sums[1] : 1.f, E = a.sums[2] > 0.f ? a.sums[2] : 1.f;
    const float sBE = sqrtf(B * E);
    ca = 1.f / sBE;
    cb = -aa / (B * sqrtf(B) * sqrtf(E));
  }
  const double tinv = (a.kind == 2 && a.scal[2] > 0.0) ? 1.0 / a.scal[2] : 0.0;
  float acc[18];
#pragma unroll
  for (int k = 0; k < 18; k++) acc[k] = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    int x, y_, z;
    interior_of(g, i, x, y_, z);
    const long long c = x + (long long)g.Xp * (y_ + (long long)g.Yp * z);
    const float d = a.y[c] - a.t[c];
    float dy;
    if (a.kind == 1) dy = ca * a.t[c] + cb * a.y[c];
    else if (a.kind == 2) dy = ca * (float)(a.r[c] * tinv) + cb * a.ay[c];
    else dy = 2.f * d / T2;
    acc[0] += d * d;
    acc[1] += dy;
    const long long vo = g.vox(x, y_, z) * 8;
#pragma unroll
    for (int cg = 0; cg < 2; cg++) {
      float hv[8], o[8];
      unpack8(*reinterpret_cast<const uint4*>(a.h + cg * g.GS * 8 + vo), hv);
#pragma unroll
      for (int e = 0; e < 8; e++) {
        acc[2 + 8 * cg + e] += dy * hv[e];
        o[e] = hv[e] > 0.f ? a.head_w[8 * cg + e] * dy : 0.f;
      }
      *reinterpret_cast<uint4*>(a.dh + cg * g.GS * 8 + vo) = pack8(o);
    }
  }
  block_sums<18>(acc, a.partial + (long long)blockIdx.x * 18);
}

// Adam (decoupled from the layout: one flat FP32 parameter array)
__global__ void k_adam(float* w, const float* gr, float* m, float* v, long long n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = gr[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  }
}

}  // namespace un
