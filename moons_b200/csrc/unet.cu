// unet.cu -- the learned preconditioner: a 3-D U-Net (4 levels, channels
// 16/32/64/128, 3x3x3 convolutions, BF16 activations and weights, FP32
// accumulation on tcgen05) that maps a residual r (and a per-cell feature of
// the operator's coefficients) to a correction z ~ A^-1 r, trained on the GPU
// by its own forward, backward and Adam kernels.
//
// No reference counterpart: the reference's preconditioners are the Jacobi
// family of code/handwritten/solvers/preconditioners/preconditioners.f90:55-129;
// this object is an additional preconditioner selected behind the same
// PCG entry points (flexible CG, see pcg.cu).
//
// Network (input 2 channels in one 8-channel group: r / rms(r), feature):
//   enc0a 8->16, enc0b 16->16 | pool | enc1a 16->32, enc1b 32->32 | pool |
//   enc2a 32->64, enc2b 64->64 | pool | enc3a 64->128, enc3b 128->128 |
//   up | dec2a (128+64)->64, dec2b 64->64 | up | dec1a (64+32)->32, dec1b |
//   up | dec0a (32+16)->16, dec0b 16->16 | head 1x1 16->1 (linear)
// every 3x3x3 convolution followed by bias and ReLU; pool = 2x2x2 mean,
// up = nearest x2.  Output z = out_scale * rms(r) * y.
//
// Parameters: one flat FP32 array, per convolution W[co][ci][dz][dy][dx]
// then b[co], in the layer order above, then head w[16], head b.
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "runtime.cuh"
#include "unet.cuh"

using namespace un;

struct MGHier;
namespace mg {
int mg_apply_fine_f32(MGHier* h, const float* in, float* out, cudaStream_t st);
int mg_energy_fine_f64(MGHier* h, const float* y, double* partial, int nblocks, cudaStream_t st);
bool mg_is_mixed(const MGHier* h);
MGHier* pcg_mg_hier(moons_pcg* s);
moons_mesh* pcg_mesh(moons_pcg* s);
}  // namespace mg

namespace {

enum {
  T_IN, T_E0A, T_E0, T_P1, T_E1A, T_E1, T_P2, T_E2A, T_E2, T_P3, T_E3A, T_E3,
  T_U2, T_D2A, T_D2, T_U1, T_D1A, T_D1, T_U0, T_D0A, T_D0, T_COUNT
};
// level and channels of each activation tensor
const int kTLvl[T_COUNT] = {0, 0, 0, 1, 1, 1, 2, 2, 2, 3, 3, 3, 2, 2, 2, 1, 1, 1, 0, 0, 0};
const int kTC[T_COUNT] = {8, 16, 16, 16, 32, 32, 32, 64, 64, 64, 128, 128, 128, 64, 64, 64, 32, 32, 32, 16, 16};

struct LayerDef {
  int inA, inB, out;  // tensors (inB = -1: single input)
};
// convolution layers in parameter order
const LayerDef kLayers[] = {
    {T_IN, -1, T_E0A},  {T_E0A, -1, T_E0},  {T_P1, -1, T_E1A}, {T_E1A, -1, T_E1}, {T_P2, -1, T_E2A},
    {T_E2A, -1, T_E2},  {T_P3, -1, T_E3A},  {T_E3A, -1, T_E3}, {T_U2, T_E2, T_D2A}, {T_D2A, -1, T_D2},
    {T_U1, T_E1, T_D1A}, {T_D1A, -1, T_D1}, {T_U0, T_E0, T_D0A}, {T_D0A, -1, T_D0}};
constexpr int kNL = sizeof(kLayers) / sizeof(kLayers[0]);

int launch_err(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return mg::cuda_fail(e, what);
  ++mg::g_launch_count;
  return MOONS_OK;
}

// largest dynamic shared memory a kernel may request on this device
template <class K>
int allow_max_smem(K kernel, int device) {
  int optin = 0;
  MG_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
  cudaFuncAttributes fa{};
  MG_CUDA(cudaFuncGetAttributes(&fa, kernel));
  MG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
  return MOONS_OK;
}

bool g_attr_done[64] = {};

// raise the dynamic shared memory limit of the tcgen05 kernels (once per
// device, outside any stream capture)
int ensure_attrs(int device) {
  if (g_attr_done[device & 63]) return MOONS_OK;
  if (int e = allow_max_smem(k_conv3, device)) return e;
  if (int e = allow_max_smem(k_wgrad, device)) return e;
  g_attr_done[device & 63] = true;
  return MOONS_OK;
}

unsigned ew_grid(long long n, int nsm) {
  long long b = (n + 255) / 256;
  long long cap = (long long)nsm * 8;
  return (unsigned)std::max<long long>(1, std::min(b, cap));
}

struct Layer {
  int cin, cout, lvl;
  long long wofs, bofs;     // offsets in the flat parameter array
  bf16* wf = nullptr;       // packed forward weights
  bf16* wb = nullptr;       // packed transposed weights (backward data)
};

}  // namespace

struct moons_unet {
  moons_mesh* m = nullptr;
  int device = 0, nsm = 148;
  cudaStream_t stream = nullptr;
  Geo geo[4];
  std::vector<void*> allocs;
  bf16* t[T_COUNT] = {};   // activations
  bf16* d[T_COUNT] = {};   // gradients w.r.t. activations (pre-activation where masked)
  Layer L[kNL];
  long long nparams = 0;
  float *params = nullptr, *grads = nullptr, *am = nullptr, *av = nullptr;
  long long head_ofs = 0;
  float* feat = nullptr;      // per-cell feature, cell-centred layout
  float* y32 = nullptr;       // network output, cell-centred layout
  float* t32 = nullptr;       // training target, cell-centred layout
  double* scal = nullptr;     // [0] rms(r), [1] 1/rms, [2] out_scale*rms
  double* dpart = nullptr;    // kURedBlocks
  float* fpart = nullptr;     // kURedBlocks * 256
  float* fred = nullptr;      // reduced scalars (loss, T2, ...)
  int* err = nullptr;
  double out_scale = 1.0;
  int adam_t = 0;
  long long ncell = 0;
  bool packed = false;
  int loss_kind = 1;          // 0 relative L2, 1 cosine, 2 energy-norm cosine
  MGHier* op = nullptr;       // kind 2: the solver operator (FP32 finest multigrid level)
  float* ay32 = nullptr;      // kind 2: A y, cell-centred layout
};

namespace {

template <class T>
T* dalloc(moons_unet* u, size_t n, bool zero = true) {
  void* p = nullptr;
  if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(T)) != cudaSuccess) return nullptr;
  u->allocs.push_back(p);
  if (zero) cudaMemset(p, 0, std::max<size_t>(1, n) * sizeof(T));
  return static_cast<T*>(p);
}

size_t tensor_elems(const Geo& g, int C) { return (size_t)(C / 8) * (size_t)g.GS * 8; }

int check_err(moons_unet* u) {
  int h = 0;
  MG_CUDA(cudaMemcpyAsync(&h, u->err, sizeof(int), cudaMemcpyDeviceToHost, u->stream));
  MG_CUDA(cudaStreamSynchronize(u->stream));
  if (h) {
    mg::set_error("U-Net kernel wait timed out (code " + std::to_string(h) + ")");
    cudaMemsetAsync(u->err, 0, sizeof(int), u->stream);
    return MOONS_ERR_CUDA;
  }
  return MOONS_OK;
}

// ---- convolution launch --------------------------------------------------
struct ConvOut {
  bf16* outA; bf16* outB; int ocgA;
  const bf16* maskA; const bf16* maskB;
  const float* head_w; const float* head_b; float* y32; double* z64; const double* zscale;
  const int* skip;
};

int launch_conv(moons_unet* u, int lvl, const bf16* inA, int cgA, const bf16* inB, int cgB, const bf16* wt,
                const float* bias, int N, int mode, const ConvOut& o) {
  const Geo& g = u->geo[lvl];
  ConvArgs a{};
  a.g = g;
  a.inA = inA; a.inB = inB; a.cgA = cgA; a.cgB = cgB;
  a.wt = wt; a.bias = bias; a.N = N;
  a.nk = (cgA + cgB + 1) / 2;
  a.L = kTile + 2 * (g.Xp + 1);
  const int SB = conv_stage_bytes(a.L, N);
  const int nchunk = 3 * a.nk;
  // large grids (many waves): two stages, so that more CTAs fit per SM (the
  // latency of each CTA's load -> MMA -> epilogue chain is hidden by other
  // CTAs; measured 25% faster at full resolution); small grids: deeper
  // pipelines within each CTA
  const long long ctas = (long long)g.tiles_per_plane() * g.Z;
  int S = ctas >= 8LL * u->nsm ? 2 : std::max(2, std::min(4, (200 * 1024) / SB));
  S = std::min(S, nchunk);
  a.S = S;
  a.mode = mode;
  a.outA = o.outA; a.outB = o.outB; a.ocgA = o.ocgA;
  a.maskA = o.maskA; a.maskB = o.maskB;
  a.head_w = o.head_w; a.head_b = o.head_b; a.y32 = o.y32; a.z64 = o.z64; a.zscale = o.zscale;
  a.err = u->err;
  a.skip = o.skip;
  if (N % 16 || N < 16 || N > 256) {
    mg::set_error("U-Net convolution: output channels must be a multiple of 16 in [16, 256]");
    return MOONS_ERR_ARG;
  }
  const int smem = S * SB;
  if (int e = ensure_attrs(u->device)) return e;
  dim3 grid(g.tiles_per_plane(), g.Z);
  k_conv3<<<grid, kConvThreads, smem, u->stream>>>(a);
  return launch_err("k_conv3");
}

int launch_wgrad(moons_unet* u, int lvl, const bf16* inA, int cgA, const bf16* inB, int cgB, const bf16* dout, int N,
                 float* dW, int cin) {
  const Geo& g = u->geo[lvl];
  WgradArgs a{};
  a.g = g;
  a.inA = inA; a.inB = inB; a.cgA = cgA; a.cgB = cgB;
  a.dout = dout; a.N = N;
  const int cgT = cgA + cgB;
  a.ncg = std::min(16, cgT);
  a.nsh = a.ncg == 1 ? 9 : (3 * a.ncg <= 16 ? 3 : 1);
  const int nsg = 9 / a.nsh;
  const int nct = (cgT + a.ncg - 1) / a.ncg;
  a.items = g.Z * g.tiles_per_plane();
  const int NR = a.nsh * a.ncg;
  const int SB = wgrad_stage_bytes(N, NR), tail = wgrad_tail_bytes(N, NR);
  a.S = std::max(2, std::min(4, (160 * 1024 - tail) / SB));
  const int smem = a.S * SB + tail;
  if (int e = ensure_attrs(u->device)) return e;
  // enough CTAs for every SM's resident slots (shared memory and TMEM)
  int occ = 0;
  MG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_wgrad, kConvThreads, smem));
  const int cols = 3 * N <= 32 ? 32 : (3 * N <= 64 ? 64 : (3 * N <= 128 ? 128 : (3 * N <= 256 ? 256 : 512)));
  occ = std::max(1, std::min(occ, 512 / cols));
  int chunks = std::max(1, std::min(a.items, (2 * occ * u->nsm) / std::max(1, nsg * nct)));
  a.per_cta = (a.items + chunks - 1) / chunks;
  chunks = (a.items + a.per_cta - 1) / a.per_cta;
  a.dW = dW; a.cin = cin;
  a.err = u->err;
  dim3 grid(nsg, nct, chunks);
  k_wgrad<<<grid, kConvThreads, smem, u->stream>>>(a);
  return launch_err("k_wgrad");
}

int pack_weights(moons_unet* u) {
  for (int l = 0; l < kNL; l++) {
    Layer& y = u->L[l];
    k_pack_w<<<ew_grid(3LL * 2 * 9 * 8 * 16 * 256, u->nsm), 256, 0, u->stream>>>(u->params + y.wofs, y.cin, y.cout, 0,
                                                                                y.wf);
    int r = launch_err("k_pack_w");
    if (r) return r;
    if (y.wb) {
      k_pack_w<<<ew_grid(3LL * 2 * 9 * 8 * 16 * 256, u->nsm), 256, 0, u->stream>>>(u->params + y.wofs, y.cin, y.cout,
                                                                                  1, y.wb);
      r = launch_err("k_pack_w");
      if (r) return r;
    }
  }
  u->packed = true;
  return MOONS_OK;
}

// rms of r (FP64 cell-centred) -> u->scal
int scale_of(moons_unet* u, const double* r, const int* skip) {
  const Geo& g = u->geo[0];
  k_sumsq_cc<<<kURedBlocks, kURedThreads, 0, u->stream>>>(g, r, u->dpart, skip);
  int e = launch_err("k_sumsq_cc");
  if (e) return e;
  k_scale_fin<<<1, 32, 0, u->stream>>>(u->dpart, kURedBlocks, u->ncell, u->out_scale, u->scal, skip);
  return launch_err("k_scale_fin");
}

// forward pass from r; z64 (optional) receives out_scale*rms(r)*y; every
// kernel returns at once while *skip (optional device flag) is nonzero
int forward(moons_unet* u, const double* r, double* z64, const int* skip = nullptr) {
  if (!u->packed) {
    int e = pack_weights(u);
    if (e) return e;
  }
  int e = scale_of(u, r, skip);
  if (e) return e;
  const Geo& g0 = u->geo[0];
  k_pack_in<<<ew_grid(u->ncell, u->nsm), 256, 0, u->stream>>>(g0, r, u->feat, u->scal, u->t[T_IN], skip);
  if ((e = launch_err("k_pack_in"))) return e;
  for (int l = 0; l < kNL; l++) {
    const LayerDef& D = kLayers[l];
    Layer& y = u->L[l];
    // pooled / upsampled inputs are produced just before their consumer
    if (D.inA == T_P1 || D.inA == T_P2 || D.inA == T_P3) {
      const int src = D.inA == T_P1 ? T_E0 : (D.inA == T_P2 ? T_E1 : T_E2);
      const int lf = kTLvl[src];
      const long long n = (long long)u->geo[lf + 1].X * u->geo[lf + 1].Y * u->geo[lf + 1].Z * (kTC[src] / 8);
      k_pool<<<ew_grid(n, u->nsm), 256, 0, u->stream>>>(u->geo[lf], u->geo[lf + 1], kTC[src] / 8, u->t[src],
                                                         u->t[D.inA], skip);
      if ((e = launch_err("k_pool"))) return e;
    }
    if (D.inA == T_U2 || D.inA == T_U1 || D.inA == T_U0) {
      const int src = D.inA == T_U2 ? T_E3 : (D.inA == T_U1 ? T_D2 : T_D1);
      const int lc = kTLvl[src];
      const long long n = (long long)u->geo[lc - 1].X * u->geo[lc - 1].Y * u->geo[lc - 1].Z * (kTC[src] / 8);
      k_up<<<ew_grid(n, u->nsm), 256, 0, u->stream>>>(u->geo[lc], u->geo[lc - 1], kTC[src] / 8, u->t[src],
                                                       u->t[D.inA], skip);
      if ((e = launch_err("k_up"))) return e;
    }
    ConvOut o{};
    o.outA = u->t[D.out];
    o.ocgA = kTC[D.out] / 8;
    o.skip = skip;
    if (l == kNL - 1) {
      o.head_w = u->params + u->head_ofs;
      o.head_b = u->params + u->head_ofs + 16;
      o.y32 = u->y32;
      o.z64 = z64;
      o.zscale = u->scal + 2;
    }
    e = launch_conv(u, y.lvl, u->t[D.inA], kTC[D.inA] / 8, D.inB >= 0 ? u->t[D.inB] : nullptr,
                    D.inB >= 0 ? kTC[D.inB] / 8 : 0, y.wf, u->params + y.bofs, y.cout, kRelu, o);
    if (e) return e;
  }
  return MOONS_OK;
}

int bias_grad(moons_unet* u, int lvl, const bf16* dpre, int C, float* out) {
  k_bias_grad<<<kURedBlocks, kURedThreads, 0, u->stream>>>(u->geo[lvl], C / 8, dpre, u->fpart);
  int e = launch_err("k_bias_grad");
  if (e) return e;
  k_sum_partials<<<(C + 127) / 128, 128, 0, u->stream>>>(u->fpart, kURedBlocks, C, out);
  return launch_err("k_sum_partials");
}

// forward + backward for one (r, e) pair: grads (flat) and fred[0] = loss
int forward_backward(moons_unet* u, const double* r, const double* ecorr) {
  if (u->loss_kind == 2 && !u->op) {
    mg::set_error("U-Net energy-norm loss: no operator (moons_unet_set_operator)");
    return MOONS_ERR_STATE;
  }
  int e = forward(u, r, nullptr);
  if (e) return e;
  const Geo& g0 = u->geo[0];
  // target and its energy
  k_target<<<kURedBlocks, kURedThreads, 0, u->stream>>>(g0, ecorr, u->scal, u->t32, u->fpart);
  if ((e = launch_err("k_target"))) return e;
  k_sum_partials<<<1, 32, 0, u->stream>>>(u->fpart, kURedBlocks, 1, u->fred + 1);
  if ((e = launch_err("k_sum_partials"))) return e;
  MG_CUDA(cudaMemsetAsync(u->grads, 0, u->nparams * sizeof(float), u->stream));
  // cosine losses: their global sums first (fred[20..22])
  if (u->loss_kind == 1) {
    k_yt<<<kURedBlocks, kURedThreads, 0, u->stream>>>(g0, u->y32, u->t32, u->fpart);
    if ((e = launch_err("k_yt"))) return e;
    k_sum_partials<<<1, 32, 0, u->stream>>>(u->fpart, kURedBlocks, 2, u->fred + 20);
    if ((e = launch_err("k_sum_partials"))) return e;
  } else if (u->loss_kind == 2) {
    if ((e = mg::mg_apply_fine_f32(u->op, u->y32, u->ay32, u->stream))) return e;
    if ((e = mg::mg_energy_fine_f64(u->op, u->y32, u->dpart + 2 * kURedBlocks, kURedBlocks, u->stream))) return e;
    k_energy_sums<<<kURedBlocks, kURedThreads, 0, u->stream>>>(g0, u->y32, ecorr, r, u->scal, u->dpart);
    if ((e = launch_err("k_energy_sums"))) return e;
    k_energy_fin<<<1, 32, 0, u->stream>>>(u->dpart, u->dpart + 2 * kURedBlocks, kURedBlocks, u->fred + 20);
    if ((e = launch_err("k_energy_fin"))) return e;
  }
  // loss + head backward -> d[T_D0] (dPre of dec0b)
  LossArgs la{};
  la.g = g0;
  la.y = u->y32; la.t = u->t32; la.T2p = u->fred + 1;
  la.kind = u->loss_kind;
  la.sums = u->fred + 20;
  la.ay = u->ay32; la.r = r; la.scal = u->scal;
  la.h = u->t[T_D0]; la.head_w = u->params + u->head_ofs; la.dh = u->d[T_D0];
  la.partial = u->fpart;
  k_loss_head<<<kURedBlocks, kURedThreads, 0, u->stream>>>(la);
  if ((e = launch_err("k_loss_head"))) return e;
  k_sum_partials<<<1, 32, 0, u->stream>>>(u->fpart, kURedBlocks, 18, u->fred + 2);
  if ((e = launch_err("k_sum_partials"))) return e;

  for (int l = kNL - 1; l >= 0; l--) {
    const LayerDef& D = kLayers[l];
    Layer& y = u->L[l];
    const bf16* dpre = u->d[D.out];
    const int cgA = kTC[D.inA] / 8, cgB = D.inB >= 0 ? kTC[D.inB] / 8 : 0;
    // weight and bias gradients
    e = launch_wgrad(u, y.lvl, u->t[D.inA], cgA, D.inB >= 0 ? u->t[D.inB] : nullptr, cgB, dpre, y.cout,
                     u->grads + y.wofs, y.cin);
    if (e) return e;
    if ((e = bias_grad(u, y.lvl, dpre, y.cout, u->grads + y.bofs))) return e;
    if (l == 0) break;  // no gradient w.r.t. the input
    // gradient w.r.t. the inputs (transposed convolution)
    ConvOut o{};
    const bool single_consumer = (D.inB < 0) && (D.inA == T_E0A || D.inA == T_E1A || D.inA == T_E2A ||
                                                 D.inA == T_E3A || D.inA == T_D2A || D.inA == T_D1A ||
                                                 D.inA == T_D0A);
    o.outA = u->d[D.inA];
    o.ocgA = cgA;
    o.outB = D.inB >= 0 ? u->d[D.inB] : nullptr;
    o.maskA = single_consumer ? u->t[D.inA] : nullptr;
    e = launch_conv(u, y.lvl, dpre, y.cout / 8, nullptr, 0, y.wb, nullptr, y.cin, kLinear, o);
    if (e) return e;
    // pooled input: d[P] -> add into d[E] (skip gradient already there) and mask
    if (D.inA == T_P1 || D.inA == T_P2 || D.inA == T_P3) {
      const int src = D.inA == T_P1 ? T_E0 : (D.inA == T_P2 ? T_E1 : T_E2);
      const int lf = kTLvl[src];
      const long long n = (long long)u->geo[lf].X * u->geo[lf].Y * u->geo[lf].Z * (kTC[src] / 8);
      k_pool_bwd<<<ew_grid(n, u->nsm), 256, 0, u->stream>>>(u->geo[lf], u->geo[lf + 1], kTC[src] / 8, u->d[src],
                                                             u->d[D.inA], u->t[src]);
      if ((e = launch_err("k_pool_bwd"))) return e;
    }
    // upsampled input: d[U] -> d[source] (children summed) and mask
    if (D.inA == T_U2 || D.inA == T_U1 || D.inA == T_U0) {
      const int src = D.inA == T_U2 ? T_E3 : (D.inA == T_U1 ? T_D2 : T_D1);
      const int lc = kTLvl[src];
      const long long n = (long long)u->geo[lc].X * u->geo[lc].Y * u->geo[lc].Z * (kTC[src] / 8);
      k_up_bwd<<<ew_grid(n, u->nsm), 256, 0, u->stream>>>(u->geo[lc - 1], u->geo[lc], kTC[src] / 8, u->d[D.inA],
                                                           u->t[src], u->d[src]);
      if ((e = launch_err("k_up_bwd"))) return e;
    }
  }
  // head gradients: fred[4..19] = sum dy*h_c, fred[3] = sum dy
  MG_CUDA(cudaMemcpyAsync(u->grads + u->head_ofs, u->fred + 4, 16 * sizeof(float), cudaMemcpyDeviceToDevice,
                          u->stream));
  MG_CUDA(cudaMemcpyAsync(u->grads + u->head_ofs + 16, u->fred + 3, sizeof(float), cudaMemcpyDeviceToDevice,
                          u->stream));
  return MOONS_OK;
}

// the loss of the last forward_backward (syncs)
int read_loss(moons_unet* u, float* loss) {
  float h[23];  // [1] |t|^2, [2] |y-t|^2, [20..22] the cosine sums
  MG_CUDA(cudaMemcpyAsync(h, u->fred, 23 * sizeof(float), cudaMemcpyDeviceToHost, u->stream));
  if (int e = check_err(u)) return e;
  const float T2 = h[1] > 0.f ? h[1] : 1.f;
  if (!loss) return MOONS_OK;
  if (u->loss_kind == 1) {
    const float yy = h[21] > 0.f ? h[21] : 1.f;
    *loss = 1.f - h[20] / sqrtf(yy * T2);
  } else if (u->loss_kind == 2) {
    const float B = h[21] > 0.f ? h[21] : 1.f, E = h[22] > 0.f ? h[22] : 1.f;
    *loss = 1.f - h[20] / sqrtf(B * E);
  } else {
    *loss = h[2] / T2;
  }
  return MOONS_OK;
}

int unet_fail_arg(const char* m) {
  mg::set_error(m);
  return MOONS_ERR_ARG;
}

bool cc_field_ok(const moons_unet* u, const moons_sf* f) {
  if (!f || f->m != u->m || f->f.dl != MOONS_CC) return false;
  return f->f.s0 == u->geo[0].Xp && f->f.s1 == u->geo[0].Yp && f->f.s2 == u->geo[0].Z + 2;
}

}  // namespace

namespace mg {
// the preconditioner apply for flexible CG: z = M(r) on the mesh stream,
// skipped while *skip is nonzero (graph-capturable once prepared)
int unet_apply_dev(moons_unet* u, double* z, const double* r, const int* skip) { return forward(u, r, z, skip); }
// pack the weights and set kernel attributes outside any stream capture
int unet_prepare(moons_unet* u) {
  int e = MOONS_OK;
  if (!u->packed) e = pack_weights(u);
  if (!e) e = ensure_attrs(u->device);
  if (!e) e = check_err(u);
  return e;
}
int unet_check(moons_unet* u) { return check_err(u); }
moons_mesh* unet_mesh(moons_unet* u) { return u->m; }
}  // namespace mg

extern "C" {

int moons_unet_create(moons_mesh* m, unsigned long long seed, moons_unet** out) {
  if (!m || !out) return unet_fail_arg("moons_unet_create: null argument");
  const int X = m->sn[0] - 2 - 1, Y = m->sn[1] - 2 - 1, Z = m->sn[2] - 2 - 1;  // node counts -> interior cells
  if (X < 8 || Y < 8 || Z < 8 || X % 8 || Y % 8 || Z % 8)
    return unet_fail_arg("moons_unet_create: interior cell counts must be multiples of 8 (three 2x poolings)");
  auto* u = new moons_unet();
  u->m = m;
  u->device = m->device;
  u->stream = m->stream;
  MG_CUDA(cudaSetDevice(u->device));
  cudaDeviceGetAttribute(&u->nsm, cudaDevAttrMultiProcessorCount, u->device);
  for (int l = 0; l < 4; l++) u->geo[l] = Geo::make(X >> l, Y >> l, Z >> l);
  u->ncell = (long long)X * Y * Z;
  bool okm = true;
  for (int i = 0; i < T_COUNT; i++) {
    u->t[i] = dalloc<bf16>(u, tensor_elems(u->geo[kTLvl[i]], kTC[i]));
    u->d[i] = i == T_IN ? nullptr : dalloc<bf16>(u, tensor_elems(u->geo[kTLvl[i]], kTC[i]));
    okm = okm && u->t[i] && (i == T_IN || u->d[i]);
  }
  // parameters
  long long ofs = 0;
  for (int l = 0; l < kNL; l++) {
    Layer& y = u->L[l];
    const LayerDef& D = kLayers[l];
    y.cin = kTC[D.inA] + (D.inB >= 0 ? kTC[D.inB] : 0);
    y.cout = kTC[D.out];
    y.lvl = kTLvl[D.out];
    y.wofs = ofs;
    ofs += (long long)y.cout * y.cin * 27;
    y.bofs = ofs;
    ofs += y.cout;
  }
  u->head_ofs = ofs;
  ofs += 17;
  u->nparams = ofs;
  u->params = dalloc<float>(u, ofs);
  u->grads = dalloc<float>(u, ofs);
  u->am = dalloc<float>(u, ofs);
  u->av = dalloc<float>(u, ofs);
  for (int l = 0; l < kNL; l++) {
    Layer& y = u->L[l];
    const size_t nf = 3ull * ((y.cin + 15) / 16) * 2 * 9 * y.cout * 8;
    const size_t nb = 3ull * ((y.cout + 15) / 16) * 2 * 9 * y.cin * 8;
    y.wf = dalloc<bf16>(u, nf, false);
    y.wb = l == 0 ? nullptr : dalloc<bf16>(u, nb, false);
    okm = okm && y.wf && (l == 0 || y.wb);
  }
  const size_t ncc = (size_t)u->geo[0].Xp * u->geo[0].Yp * (Z + 2);
  u->feat = dalloc<float>(u, ncc);
  u->y32 = dalloc<float>(u, ncc);
  u->t32 = dalloc<float>(u, ncc);
  u->ay32 = dalloc<float>(u, ncc);
  u->scal = dalloc<double>(u, 4);
  u->dpart = dalloc<double>(u, 3 * kURedBlocks);
  u->fpart = dalloc<float>(u, (size_t)kURedBlocks * 256);
  u->fred = dalloc<float>(u, 64);
  u->err = dalloc<int>(u, 1);
  okm = okm && u->params && u->grads && u->am && u->av && u->feat && u->y32 && u->t32 && u->ay32 && u->scal && u->dpart &&
        u->fpart && u->fred && u->err;
  if (!okm) {
    for (void* p : u->allocs) cudaFree(p);
    delete u;
    mg::set_error("moons_unet_create: device allocation failed");
    return MOONS_ERR_NOMEM;
  }
  // He-uniform initialisation (fan-in), zero biases; head small
  std::vector<float> h(ofs, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < kNL; l++) {
    Layer& y = u->L[l];
    const int fan_real = (l == 0 ? 2 : y.cin) * 27;
    const float lim = std::sqrt(6.0f / fan_real);
    std::uniform_real_distribution<float> U(-lim, lim);
    for (long long i = 0; i < (long long)y.cout * y.cin * 27; i++) {
      const int ci = (int)((i / 27) % y.cin);
      h[y.wofs + i] = (l == 0 && ci >= 2) ? 0.f : U(rng);
    }
  }
  {
    std::uniform_real_distribution<float> U(-0.25f, 0.25f);
    for (int c = 0; c < 16; c++) h[u->head_ofs + c] = U(rng);
  }
  MG_CUDA(cudaMemcpy(u->params, h.data(), ofs * sizeof(float), cudaMemcpyHostToDevice));
  MG_CUDA(cudaDeviceSynchronize());
  mg::mesh_ref(m);
  *out = u;
  return MOONS_OK;
}

int moons_unet_destroy(moons_unet* u) {
  if (!u) return MOONS_OK;
  cudaSetDevice(u->device);
  cudaStreamSynchronize(u->stream);
  for (void* p : u->allocs) cudaFree(p);
  moons_mesh* m = u->m;
  delete u;
  mg::mesh_unref(m);
  return MOONS_OK;
}

int moons_unet_nparams(const moons_unet* u, long long* n) {
  if (!u || !n) return unet_fail_arg("moons_unet_nparams: null argument");
  *n = u->nparams;
  return MOONS_OK;
}

int moons_unet_get_params(moons_unet* u, float* host, long long n) {
  if (!u || !host || n != u->nparams) return unet_fail_arg("moons_unet_get_params: bad argument");
  MG_CUDA(cudaMemcpyAsync(host, u->params, n * sizeof(float), cudaMemcpyDeviceToHost, u->stream));
  MG_CUDA(cudaStreamSynchronize(u->stream));
  return MOONS_OK;
}

int moons_unet_set_params(moons_unet* u, const float* host, long long n) {
  if (!u || !host || n != u->nparams) return unet_fail_arg("moons_unet_set_params: bad argument");
  MG_CUDA(cudaMemcpyAsync(u->params, host, n * sizeof(float), cudaMemcpyHostToDevice, u->stream));
  MG_CUDA(cudaMemsetAsync(u->am, 0, n * sizeof(float), u->stream));
  MG_CUDA(cudaMemsetAsync(u->av, 0, n * sizeof(float), u->stream));
  u->adam_t = 0;
  u->packed = false;
  MG_CUDA(cudaStreamSynchronize(u->stream));
  return MOONS_OK;
}

int moons_unet_set_loss(moons_unet* u, int kind) {
  if (!u || kind < 0 || kind > 2) return unet_fail_arg("moons_unet_set_loss: kind must be 0, 1 or 2");
  u->loss_kind = kind;
  return MOONS_OK;
}

int moons_unet_set_operator(moons_unet* u, moons_pcg* s) {
  if (!u || !s) return unet_fail_arg("moons_unet_set_operator: null argument");
  MGHier* h = mg::pcg_mg_hier(s);
  if (!h || !mg::mg_is_mixed(h) || mg::pcg_mesh(s) != u->m)
    return unet_fail_arg("moons_unet_set_operator: needs a MOONS_PREC_MG_MIXED or MOONS_PREC_UNET solver on the "
                         "net's mesh");
  u->op = h;
  return MOONS_OK;
}

int moons_unet_set_out_scale(moons_unet* u, double c) {
  if (!u || !(c > 0.0)) return unet_fail_arg("moons_unet_set_out_scale: bad argument");
  u->out_scale = c;
  return MOONS_OK;
}

int moons_unet_get_out_scale(const moons_unet* u, double* c) {
  if (!u || !c) return unet_fail_arg("moons_unet_get_out_scale: null argument");
  *c = u->out_scale;
  return MOONS_OK;
}

int moons_unet_set_feature(moons_unet* u, const float* host, long long n) {
  if (!u) return unet_fail_arg("moons_unet_set_feature: null net");
  const long long ncc = (long long)u->geo[0].Xp * u->geo[0].Yp * (u->geo[0].Z + 2);
  if (!host || n != ncc) return unet_fail_arg("moons_unet_set_feature: expects one value per cell (ghosts included)");
  MG_CUDA(cudaMemcpyAsync(u->feat, host, n * sizeof(float), cudaMemcpyHostToDevice, u->stream));
  MG_CUDA(cudaStreamSynchronize(u->stream));
  return MOONS_OK;
}

int moons_unet_set_coeff(moons_unet* u, const moons_sf* kx, const moons_sf* ky, const moons_sf* kz) {
  if (!u || !kx || !ky || !kz) return unet_fail_arg("moons_unet_set_coeff: null argument");
  const Geo& g = u->geo[0];
  if (kx->m != u->m || ky->m != u->m || kz->m != u->m || kx->f.dl != MOONS_FX || ky->f.dl != MOONS_FY ||
      kz->f.dl != MOONS_FZ)
    return unet_fail_arg("moons_unet_set_coeff: kx, ky, kz must be x, y, z face fields of the net's mesh");
  k_feat_faces<<<ew_grid(u->ncell, u->nsm), 256, 0, u->stream>>>(g, kx->f.f, ky->f.f, kz->f.f, u->feat);
  int e = launch_err("k_feat_faces");
  if (e) return e;
  return check_err(u);
}

int moons_unet_apply(moons_unet* u, moons_sf* z, const moons_sf* r) {
  if (!u || !cc_field_ok(u, z) || !cc_field_ok(u, r))
    return unet_fail_arg("moons_unet_apply: z and r must be cell-centred fields of the net's mesh");
  MG_CUDA(cudaMemsetAsync(z->f.f, 0, z->f.n() * sizeof(double), u->stream));
  int e = forward(u, r->f.f, z->f.f);
  if (e) return e;
  return check_err(u);
}

int moons_unet_loss_grad(moons_unet* u, const moons_sf* r, const moons_sf* ecorr, float* loss, float* grads_host,
                         long long n) {
  if (!u || !cc_field_ok(u, r) || !cc_field_ok(u, ecorr))
    return unet_fail_arg("moons_unet_loss_grad: r and e must be cell-centred fields of the net's mesh");
  if (grads_host && n != u->nparams) return unet_fail_arg("moons_unet_loss_grad: gradient size mismatch");
  int e = forward_backward(u, r->f.f, ecorr->f.f);
  if (e) return e;
  if (grads_host)
    MG_CUDA(cudaMemcpyAsync(grads_host, u->grads, n * sizeof(float), cudaMemcpyDeviceToHost, u->stream));
  return read_loss(u, loss);
}

int moons_unet_train_step(moons_unet* u, const moons_sf* r, const moons_sf* ecorr, float lr, float* loss) {
  if (!u || !cc_field_ok(u, r) || !cc_field_ok(u, ecorr))
    return unet_fail_arg("moons_unet_train_step: r and e must be cell-centred fields of the net's mesh");
  int e = forward_backward(u, r->f.f, ecorr->f.f);
  if (e) return e;
  u->adam_t++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f / (1.f - std::pow(b1, (float)u->adam_t));
  const float c2 = 1.f / (1.f - std::pow(b2, (float)u->adam_t));
  k_adam<<<ew_grid(u->nparams, u->nsm), 256, 0, u->stream>>>(u->params, u->grads, u->am, u->av, u->nparams, lr, b1,
                                                              b2, 1e-8f, c1, c2);
  if ((e = launch_err("k_adam"))) return e;
  if ((e = pack_weights(u))) return e;
  if (loss) return read_loss(u, loss);
  return MOONS_OK;
}

// ---- kernel self-checks: one layer on host data ----------------------------
// Host tensors are [C][Z][Y][X] FP32 (interior only); they are rounded to BF16
// on upload, as the network stores them.
static int upload_tensor(const Geo& g, int C, const float* h, bf16* d) {
  std::vector<bf16> buf(tensor_elems(g, C), __float2bfloat16(0.f));
  for (int c = 0; c < C; c++)
    for (int z = 1; z <= g.Z; z++)
      for (int y = 1; y <= g.Y; y++)
        for (int x = 1; x <= g.X; x++)
          buf[(size_t)(c / 8) * g.GS * 8 + g.vox(x, y, z) * 8 + c % 8] =
              __float2bfloat16(h[(((size_t)c * g.Z + z - 1) * g.Y + y - 1) * g.X + x - 1]);
  MG_CUDA(cudaMemcpy(d, buf.data(), buf.size() * sizeof(bf16), cudaMemcpyHostToDevice));
  return MOONS_OK;
}
static int download_tensor(const Geo& g, int C, const bf16* d, float* h) {
  std::vector<bf16> buf(tensor_elems(g, C));
  MG_CUDA(cudaMemcpy(buf.data(), d, buf.size() * sizeof(bf16), cudaMemcpyDeviceToHost));
  for (int c = 0; c < C; c++)
    for (int z = 1; z <= g.Z; z++)
      for (int y = 1; y <= g.Y; y++)
        for (int x = 1; x <= g.X; x++)
          h[(((size_t)c * g.Z + z - 1) * g.Y + y - 1) * g.X + x - 1] =
              __bfloat162float(buf[(size_t)(c / 8) * g.GS * 8 + g.vox(x, y, z) * 8 + c % 8]);
  return MOONS_OK;
}

// op 0: out = conv(in) (+ bias, ReLU when relu);  op 1: out = conv^T(in) (the
// gradient w.r.t. the input of a layer with weights W[cout][cin][27]);  op 2:
// dW = weight gradient of that layer for input `in` (cin channels) and output
// gradient `dout` (cout channels), FP32.
int moons_unet_layer_check(int op, int X, int Y, int Z, int cinA, int cinB, int cout, const float* in,
                           const float* dout, const float* W, const float* bias, int relu, float* out) {
  if (X < 1 || Y < 1 || Z < 1 || cinA % 8 || cinB % 8 || cout % 8 || cinA < 8 || cout < 16)
    return unet_fail_arg("moons_unet_layer_check: bad sizes");
  moons_unet u;
  MG_CUDA(cudaGetDevice(&u.device));
  cudaDeviceGetAttribute(&u.nsm, cudaDevAttrMultiProcessorCount, u.device);
  MG_CUDA(cudaStreamCreate(&u.stream));
  u.geo[0] = Geo::make(X, Y, Z);
  const Geo& g = u.geo[0];
  const int cin = cinA + cinB;
  int e = MOONS_OK;
  bf16 *tA = dalloc<bf16>(&u, tensor_elems(g, cinA)), *tB = cinB ? dalloc<bf16>(&u, tensor_elems(g, cinB)) : nullptr;
  bf16* to = dalloc<bf16>(&u, tensor_elems(g, std::max(cin, cout)));
  bf16* td = dalloc<bf16>(&u, tensor_elems(g, cout));
  float* dW = dalloc<float>(&u, (size_t)cout * cin * 27 + cout);
  float* db = dalloc<float>(&u, std::max(cin, cout));
  bf16* wp = dalloc<bf16>(&u, 3ull * ((std::max(cin, cout) + 15) / 16) * 2 * 9 * std::max(cin, cout) * 8);
  u.err = dalloc<int>(&u, 1);
  u.fpart = dalloc<float>(&u, (size_t)kURedBlocks * 256);
  if (!tA || (cinB && !tB) || !to || !td || !dW || !db || !wp || !u.err || !u.fpart) e = MOONS_ERR_NOMEM;
  if (!e && op != 2 && !W) e = unet_fail_arg("moons_unet_layer_check: ops 0 and 1 need weights");
  if (!e && W) MG_CUDA(cudaMemcpy(dW, W, (size_t)cout * cin * 27 * sizeof(float), cudaMemcpyHostToDevice));
  if (!e && bias) MG_CUDA(cudaMemcpy(db, bias, cout * sizeof(float), cudaMemcpyHostToDevice));
  if (!e && op == 0) {
    std::vector<float> hA((size_t)cinA * X * Y * Z), hB((size_t)cinB * X * Y * Z);
    std::memcpy(hA.data(), in, hA.size() * sizeof(float));
    if (cinB) std::memcpy(hB.data(), in + hA.size(), hB.size() * sizeof(float));
    e = upload_tensor(g, cinA, hA.data(), tA);
    if (!e && cinB) e = upload_tensor(g, cinB, hB.data(), tB);
    if (!e) {
      k_pack_w<<<ew_grid(1 << 20, u.nsm), 256, 0, u.stream>>>(dW, cin, cout, 0, wp);
      e = launch_err("k_pack_w");
    }
    ConvOut o{};
    o.outA = to;
    o.ocgA = cout / 8;
    if (!e) e = launch_conv(&u, 0, tA, cinA / 8, tB, cinB / 8, wp, db, cout, relu ? kRelu : kLinear, o);
    if (!e) e = check_err(&u);
    if (!e) e = download_tensor(g, cout, to, out);
  } else if (!e && op == 1) {
    e = upload_tensor(g, cout, dout, td);
    if (!e) {
      k_pack_w<<<ew_grid(1 << 20, u.nsm), 256, 0, u.stream>>>(dW, cin, cout, 1, wp);
      e = launch_err("k_pack_w");
    }
    ConvOut o{};
    o.outA = to;
    o.ocgA = cin / 8;
    if (!e) e = launch_conv(&u, 0, td, cout / 8, nullptr, 0, wp, nullptr, cin, kLinear, o);
    if (!e) e = check_err(&u);
    if (!e) e = download_tensor(g, cin, to, out);
  } else if (!e && op == 2) {
    std::vector<float> hA((size_t)cinA * X * Y * Z), hB((size_t)cinB * X * Y * Z);
    std::memcpy(hA.data(), in, hA.size() * sizeof(float));
    if (cinB) std::memcpy(hB.data(), in + hA.size(), hB.size() * sizeof(float));
    e = upload_tensor(g, cinA, hA.data(), tA);
    if (!e && cinB) e = upload_tensor(g, cinB, hB.data(), tB);
    if (!e) e = upload_tensor(g, cout, dout, td);
    if (!e) {
      cudaMemsetAsync(dW, 0, (size_t)cout * cin * 27 * sizeof(float), u.stream);
      e = launch_wgrad(&u, 0, tA, cinA / 8, tB, cinB / 8, td, cout, dW, cin);
    }
    if (!e) e = bias_grad(&u, 0, td, cout, dW + (size_t)cout * cin * 27);
    if (!e) e = check_err(&u);
    if (!e) MG_CUDA(cudaMemcpy(out, dW, ((size_t)cout * cin * 27 + cout) * sizeof(float), cudaMemcpyDeviceToHost));
  } else if (!e) {
    e = unet_fail_arg("moons_unet_layer_check: op must be 0, 1 or 2");
  }
  cudaStreamSynchronize(u.stream);
  for (void* p : u.allocs) cudaFree(p);
  cudaStreamDestroy(u.stream);
  return e;
}

}  // extern "C"
