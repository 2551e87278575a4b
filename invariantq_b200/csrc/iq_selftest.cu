// iq_selftest.cu -- a check of the tile kernel's failure path that faults
// nothing: a CTA waits, with the tile kernel's own bounded wait, on an
// mbarrier phase that nothing completes (its one expected arrival never
// comes).  The wait must give up after `limit_ns`, raise the CTA's abort flag,
// set the status word and let the kernel return normally, so the context stays
// usable.
#include <cuda_runtime.h>

#include "../../include/invariantq_b200.h"
#include "iq_tile.cuh"

namespace iqb {

namespace {

__global__ void selftest_wait_kernel(int* __restrict__ status, uint64_t limit_ns, unsigned long long* __restrict__ waited) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ volatile int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);   // one arrival expected; none is made
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();
  const uint64_t t0 = global_ns();
  const bool ok = bounded_wait(&bar, 0, &abort_flag, status, DEV_WAIT_LOADED, limit_ns);
  __syncthreads();
  if (threadIdx.x == 0) *waited = ok ? 0ull : (unsigned long long)(global_ns() - t0);
}

}  // namespace
}  // namespace iqb

extern "C" int iq_selftest_bounded_wait(double limit_ms, double* waited_ms) {
  using namespace iqb;
  if (!(limit_ms > 0.0) || limit_ms > 1000.0) {
    record_error(1, "iq_selftest_bounded_wait: limit_ms must be in (0, 1000]");
    return -1;
  }
  int* d_status = nullptr;
  unsigned long long* d_waited = nullptr;
  cudaStream_t st = nullptr;
  int status = -1;
  unsigned long long waited = 0;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&d_status, sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&d_waited, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_status, 0, sizeof(int), st);
  if (e == cudaSuccess) {
    selftest_wait_kernel<<<1, 128, 0, st>>>(d_status, (uint64_t)(limit_ms * 1e6), d_waited);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&waited, d_waited, sizeof(waited), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (d_status) cudaFree(d_status);
  if (d_waited) cudaFree(d_waited);
  if (st) cudaStreamDestroy(st);
  if (e != cudaSuccess) {
    record_error(2, cudaGetErrorString(e));
    return -1;
  }
  count_launches(1);
  if (waited_ms) *waited_ms = (double)waited * 1e-6;
  return status;
}
