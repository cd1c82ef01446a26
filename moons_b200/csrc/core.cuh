// core.cuh -- device data model of the MOONS hot path on B200.
//
// A field lives in HBM exactly as the reference's grid_field array
// f(sx,sy,sz): column-major, x fastest, one ghost layer per side, FP64
// (GEN/grid_field/grid_field.f90:39-43).  Kernels address it with 1-based
// (i,j,k) so the stencil formulas read like the Fortran they restate.
// 1-D coefficient arrays are stored 1-based too (element 0 unused).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/moons_gpu.h"

#define MG_HD __host__ __device__ __forceinline__

namespace mg {

// ---- 1-D coordinates and stencil coefficients of one axis --------------
// (HW/grid/coordinates_extend.f90:78-173,506-523)
struct DCoord {
  int sn, sc;
  const double *hn, *hc, *dhn, *dhc;
  const double *cc2nD, *cc2nU;  // stagCC2N, size sc-1
  const double *n2ccD, *n2ccU;  // stagN2CC, size sn-1
  const double *colCC_L[2], *colCC_D[2], *colCC_U[2];  // size sc-2
  const double *colN_L[2], *colN_D[2], *colN_U[2];     // size sn-2
  const double *thD, *thU;      // interpolation theta, size sc-1
  // this axis' share of laplacian_diagonal (GF_diagonals.f90:15-35) for data
  // CC along the axis (diagC, index 2..sc-1) and node-located (diagN, 2..sn-1)
  const double *diagC, *diagN;
};
struct DGrid {
  DCoord c[3];
};

// ---- a field as kernels see it -----------------------------------------
struct DF {
  double* f;
  int s0, s1, s2;  // extents x,y,z
  int dl;          // data location (MOONS_CC ...)
  __host__ __device__ int s(int d) const { return d == 1 ? s0 : (d == 2 ? s1 : s2); }
  __host__ __device__ size_t n() const { return (size_t)s0 * s1 * s2; }
  // fields hold < 2^31 points (moons_mesh_create checks), so the offset is
  // formed in 32-bit arithmetic
  MG_HD size_t at(int i, int j, int k) const {
    return (size_t)((unsigned)(i - 1) + (unsigned)s0 * ((unsigned)(j - 1) + (unsigned)s1 * (unsigned)(k - 1)));
  }
  MG_HD double& operator()(int i, int j, int k) const { return f[at(i, j, k)]; }
};

// node-location eye of a data location: bit d-1 set when N along d
__host__ __device__ inline int dl_bits(int dl) {
  switch (dl) {
    case MOONS_CC: return 0;
    case MOONS_FX: return 1;
    case MOONS_FY: return 2;
    case MOONS_FZ: return 4;
    case MOONS_EX: return 6;
    case MOONS_EY: return 5;
    case MOONS_EZ: return 3;
    default: return 7;
  }
}
__host__ __device__ inline bool n_along(int dl, int d) { return (dl_bits(dl) >> (d - 1)) & 1; }
__host__ inline int dl_from_bits(int b) {
  for (int d = 0; d < 8; d++)
    if (dl_bits(d) == b) return d;
  return -1;
}

// ---- BCs of one field as kernels see them ------------------------------
struct DBC {
  int defined;
  int type[7];
  int prescribed[7];
  double value[7];
  double c_w[7];
  double dh[7];
  double nhat[7];
  int order[7];
};

// ---- error plumbing ----------------------------------------------------
void set_error(const std::string& m);
int cuda_fail(cudaError_t e, const char* what);
#define MG_CUDA(call)                                   \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return mg::cuda_fail(e_, #call); \
  } while (0)

// every kernel launch of the library goes through MG_LAUNCH, which counts it
extern long long g_launch_count;
#define MG_LAUNCH(K, GRID, BLOCK, STREAM, ...)            \
  do {                                                    \
    K<<<(GRID), (BLOCK), 0, (STREAM)>>>(__VA_ARGS__);     \
    ++mg::g_launch_count;                                 \
  } while (0)

// the same, launched with programmatic stream serialisation (programmatic
// dependent launch; the kernel must call griddepcontrol.wait before reading
// what its predecessor wrote); returns from the caller on a launch error
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ++g_launch_count;
  return cudaLaunchKernelEx(&cfg, k, args...);
}
#define MG_LAUNCH_PDL(K, GRID, BLOCK, STREAM, ...)                                             \
  do {                                                                                         \
    cudaError_t e_ = mg::launch_pdl(K, dim3(GRID), dim3(BLOCK), (STREAM), __VA_ARGS__);        \
    if (e_ != cudaSuccess) return mg::cuda_fail(e_, #K);                                       \
  } while (0)
// the same with dynamic shared memory
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl_smem(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                                   Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  ++g_launch_count;
  return cudaLaunchKernelEx(&cfg, k, args...);
}
#define MG_LAUNCH_PDL_SMEM(K, GRID, BLOCK, SMEM, STREAM, ...)                                  \
  do {                                                                                         \
    cudaError_t e_ = mg::launch_pdl_smem(K, dim3(GRID), dim3(BLOCK), (SMEM), (STREAM), __VA_ARGS__); \
    if (e_ != cudaSuccess) return mg::cuda_fail(e_, #K);                                       \
  } while (0)

constexpr int kBlock = 256;
inline unsigned nblocks(size_t n, int bs = kBlock) { return (unsigned)((n + bs - 1) / bs); }

// index -> (i,j,k) 1-based
// (fields are < 2^32 points: 32-bit division only)
__device__ __forceinline__ void ijk_of(size_t idx, const DF& a, int& i, int& j, int& k) {
  unsigned u = (unsigned)idx, s0 = (unsigned)a.s0, s1 = (unsigned)a.s1;
  unsigned q = u / s0;
  i = (int)(u - q * s0) + 1;
  unsigned kk = q / s1;
  j = (int)(q - kk * s1) + 1;
  k = (int)kk + 1;
}
MG_HD int pick(int d, int i, int j, int k) { return d == 1 ? i : (d == 2 ? j : k); }

}  // namespace mg
