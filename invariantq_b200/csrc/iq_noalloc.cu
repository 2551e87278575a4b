// iq_noalloc.cu -- <Z_q> of every qubit for amplitudes the caller already holds
// in device memory, without allocating anything.
//
// Who needs this: code that cannot call cudaMalloc at the point where it wants
// the expectation values -- for example a host whose device memory is already
// fully committed (a 33-qubit state vector alone takes 128 GiB of the GPU), or
// one running inside another framework that owns all free device memory through
// its own caching pool, where an extra allocation would fail or fragment that
// pool.  Such a caller hands over its amplitude buffer and an output buffer, and
// this entry point works in a fixed array that is part of the library's device
// code.
//
// The first call on a device does a one-time set-up with that device current:
// it loads this file's kernels and the two reduction kernels (under CUDA's lazy
// module loading, the default, code is loaded into device memory at first use)
// and looks up the device address of the scratch array.  That first call is the
// only one that may need device memory (for code, not data), so make it before
// the device memory is committed, and before any stream capture.  Later calls
// use only what that set-up loaded.
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
// Device address of g_noalloc_scratch per device, looked up once.  A
// cudaDeviceReset ends the context the address belongs to; the set-up is not
// repeated after one.
double* g_scratch_ptr[kMaxDevices] = {nullptr};

int fail(int code, const char* msg) {
  iqb::record_error(code, msg);   // reported through iq_last_error
  return -1;
}

// Puts the caller's current device back on every return path.
struct DeviceRestore {
  int prev = -1;
  DeviceRestore() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      cudaGetLastError();
    }
  }
  ~DeviceRestore() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// One-time set-up on the current device `dev`: load the kernels this entry
// point launches and look up the scratch array's device address.
int setup_device(int dev, double** out) {
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_scratch_ptr[dev]) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, z_from_sums_kernel);
    if (e == cudaSuccess) e = iqb::preload_zsums();
    if (e != cudaSuccess) {
      cudaGetLastError();
      char m[192];
      snprintf(m, sizeof(m), "expval_z_all_noalloc: loading its kernels failed: %s", cudaGetErrorString(e));
      return fail(2, m);
    }
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      cudaGetLastError();
      char m[192];
      snprintf(m, sizeof(m), "expval_z_all_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return fail(2, m);
    }
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_ptr[dev];
  return 0;
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
  if (cudaPointerGetAttributes(&attr, d_amps) != cudaSuccess ||
      (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)) {
    cudaGetLastError();
    return fail(1, "expval_z_all_noalloc: the amplitudes are not device or managed memory");
  }
  const int dev = attr.device;
  if (dev < 0 || dev >= kMaxDevices) return fail(1, "expval_z_all_noalloc: device index out of range");
  DeviceRestore restore;
  if (cudaSetDevice(dev) != cudaSuccess) {
    cudaGetLastError();
    return fail(2, "expval_z_all_noalloc: cudaSetDevice failed");
  }
  double* scratch = nullptr;
  if (setup_device(dev, &scratch) != 0) return -1;
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
