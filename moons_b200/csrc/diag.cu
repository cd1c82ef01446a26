// diag.cu -- moons_debug_bounded_wait: a self-test of the bounded in-kernel
// waits (no reference counterpart).
//
// Every wait of the library's kernels on an mbarrier (the staged PCG operator,
// the tensor-core convolutions) is bounded by a wall-clock limit; a wait that
// runs out records a site code in a device word, the kernel winds down, and
// the host returns MOONS_ERR_CUDA naming the site, with the CUDA context still
// usable.  This entry point runs that path on purpose without any fault: one
// thread initialises an mbarrier that expects one arrival, nothing arrives
// and no copy targets it, and the thread waits with the given limit.
#include "runtime.cuh"
#include "tc.cuh"

namespace mg {

constexpr int kDiagWaitCode = 900;

__global__ void k_diag_wait(int* err, unsigned long long limit_ns) {
  __shared__ __align__(8) unsigned long long bar;
  if (threadIdx.x != 0) return;
  const uint32_t b = tc::smem_u32(&bar);
  tc::mbar_init(b, 1);
  tc::fence_mbar_init();
  // parity 0: the barrier's first phase, which needs the one arrival that
  // never comes
  tc::mbar_wait(b, 0u, err, kDiagWaitCode, limit_ns);
}

}  // namespace mg

using namespace mg;

extern "C" int moons_debug_bounded_wait(unsigned long long limit_ns) {
  if (limit_ns == 0 || limit_ns > tc::kWaitLimitNs) {
    set_error("moons_debug_bounded_wait: limit must be in (0, 1 s]");
    return MOONS_ERR_ARG;
  }
  int* d = nullptr;
  MG_CUDA(cudaMalloc(&d, sizeof(int)));
  cudaMemset(d, 0, sizeof(int));
  k_diag_wait<<<1, 32>>>(d, limit_ns);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return cuda_fail(e, "moons_debug_bounded_wait");
  if (h) {
    set_error("bounded wait ran out (site " + std::to_string(h) + ")");
    return MOONS_ERR_CUDA;
  }
  return MOONS_OK;
}
