// mi_selftest.cu -- the bounded-wait mechanism of the caking kernels, exercised on its own.
//
// Every wait in the library's kernels is an mbarrier poll with an iteration limit; when the
// limit runs out the kernel records MI_E_TIMEOUT in a status word the host reads, and
// returns.  mi_selftest_wait runs one such wait on a barrier that nothing completes (or, with
// `arrive`, on one that its own thread completed first), so a test can show that a lost wait
// ends as an error status with the context still usable -- without faulting or hanging a GPU.
#include <stdint.h>

#include "mi_internal.h"

namespace mi {

__global__ void k_wait_selftest(uint32_t polls, int arrive, int *status) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  if (arrive) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
  uint32_t done = 0;
  for (uint32_t it = 0; it < polls && !done; ++it)
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(0u)
        : "memory");
  *status = done ? MI_OK : MI_E_TIMEOUT;
}

}  // namespace mi

using namespace mi;

extern "C" int mi_selftest_wait(uint32_t polls, int arrive, int device, int *status) {
  if (!status) return set_error(MI_E_ARG, "mi_selftest_wait: null status");
  int prev = 0;
  cudaGetDevice(&prev);
  if (cudaSetDevice(device) != cudaSuccess) return set_error(MI_E_ARG, "mi_selftest_wait: bad device %d", device);
  int *d = nullptr;
  int rc = MI_OK;
  cudaError_t e = cudaMalloc((void **)&d, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(d, 0x7f, sizeof(int));
  if (e == cudaSuccess) {
    k_wait_selftest<<<1, 32>>>(polls, arrive, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(status, d, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) rc = cuda_error(e, "mi_selftest_wait", __FILE__, __LINE__);
  cudaFree(d);
  cudaSetDevice(prev);
  return rc;
}
