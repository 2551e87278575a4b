// iq_noalloc.cu -- <Z_q> of every qubit for amplitudes the caller already holds
// in device memory, without allocating anything.
//
// Who needs this: code that cannot call cudaMalloc at the point where it wants
// the expectation values -- for example a host whose device memory is already
// fully committed (a 33-qubit state vector alone takes 128 GiB of the GPU), or
// one running inside another framework that owns all free device memory through
// its own caching pool, where an extra allocation would fail or fragment that
// pool.  Such a caller hands over its amplitude buffer and an output buffer and
// this entry point uses only memory that exists from the moment the library is
// loaded.
//
// The reduction is the two-kernel one behind iq_statevector_expval_z_all
// (launch_zsums in iq_kernels.cu); its partial sums go to `g_noalloc_scratch`,
// a fixed file-scope device array instead of a per-handle buffer.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/invariantq_b200.h"
#include "iq_kernels.h"

namespace {

// Largest qubit count the scratch array is sized for (the state-vector limit of
// this library); 592 partial blocks x (34 + 1) sums + the 35 final sums.
constexpr int kNoAllocMaxQubits = IQ_NOALLOC_MAX_QUBITS;
constexpr size_t kNoAllocScratchDoubles = (size_t)iqb::kRedBlocks * (kNoAllocMaxQubits + 1) + (kNoAllocMaxQubits + 1);

// Every GPU that loads the library holds this array (about 166 KB) until the
// process exits.  All calls on a device share it.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

__global__ void z_from_sums_kernel(const double* __restrict__ sums, int n, double* __restrict__ out) {
  for (int q = threadIdx.x; q < n; q += blockDim.x) out[q] = sums[0] - 2.0 * sums[1 + q];
}

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_scratch_ptr[kMaxDevices] = {nullptr};

int fail(int code, const char* msg) {
  iqb::record_error(code, msg);   // reported through iq_last_error
  return -1;
}

}  // namespace

extern "C" {

int iq_statevector_expval_z_all_noalloc(const void* d_amps, size_t num_qubits, double* d_out, void* stream) {
  if (!d_amps || !d_out) return fail(1, "expval_z_all_noalloc: null pointer");
  if (num_qubits < 1 || num_qubits > (size_t)kNoAllocMaxQubits) {
    char m[160];
    snprintf(m, sizeof(m), "expval_z_all_noalloc: %zu qubits is outside 1..%d, the size its fixed scratch array holds",
             num_qubits, kNoAllocMaxQubits);
    return fail(1, m);
  }
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, d_amps) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
    cudaGetLastError();
    return fail(1, "expval_z_all_noalloc: the amplitudes are not in device memory");
  }
  const int dev = attr.device;
  if (dev < 0 || dev >= kMaxDevices) return fail(1, "expval_z_all_noalloc: device index out of range");
  if (cudaSetDevice(dev) != cudaSuccess) return fail(2, "expval_z_all_noalloc: cudaSetDevice failed");
  double* scratch;
  {
    // one-time set-up per device, with that device current: the device address
    // of the file-scope scratch array (a host-side name is not a device address)
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p) {
        char m[160];
        snprintf(m, sizeof(m), "expval_z_all_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return fail(2, m);
      }
      g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    scratch = g_scratch_ptr[dev];
  }
  const int n = (int)num_qubits;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* partials = scratch;
  double* sums = scratch + (size_t)iqb::kRedBlocks * (n + 1);
  // every partial and sum slot read below is written earlier in this same call,
  // so nothing left over from a previous call is used
  if (iqb::launch_zsums(static_cast<const double2*>(d_amps), n, partials, sums, st) != cudaSuccess)
    return fail(2, "expval_z_all_noalloc: reduction launch failed");
  z_from_sums_kernel<<<1, 64, 0, st>>>(sums, n, d_out);
  if (cudaGetLastError() != cudaSuccess) return fail(2, "expval_z_all_noalloc: launch failed");
  return 0;
}

}  // extern "C"
