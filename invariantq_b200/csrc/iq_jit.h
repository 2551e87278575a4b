// iq_jit.h -- tile-pass kernels specialised per pass at run time.
//
// The interpreting kernel (iq_tile.cuh) reads each stage's register slots,
// lane bits and operations from the pass descriptor and dispatches on them at
// run time; every operation then writes a second register array and the
// compiler cannot schedule across operations.  For a pass whose descriptor is
// known ahead of its launches (a recorded program, or a flush whose structure
// repeats), iq_jit.cpp writes the pass's stages out as straight-line CUDA --
// slot offsets as constants, monomial operations as renamings of values,
// matrix entries read from the kernel's parameter space -- and compiles it
// with NVRTC for sm_100a.  The tile pipeline (TMA loads and stores, bounded
// waits) is the same code as the interpreting kernel's (iq_pipe.cuh), and
// every operation uses the same arithmetic expression, so both kernels give
// the same amplitudes.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "iq_kernels.h"

namespace iqb {

struct JitKernel;

// Kernels for several passes: looked up in the in-memory cache, then in the
// cubin cache directory (IQ_JIT_CACHE; default ~/.cache/invariantq_b200/jit,
// "off" disables it), and compiled with NVRTC otherwise -- distinct sources in
// parallel.  out[i] is null for a pass that is not specialised.  Returns false
// (with `err`) when NVRTC or the driver entry points are unavailable or a
// compile fails.
// min_blocks: resident CTAs per SM the kernels are compiled for (the launch's
// TileLaunch::ctas_per_sm).
// threads: CTA size of the kernels (128, 256; 0 = by register slots).
// set_mode: the shared-memory form (passes over parameter sets, adjoint steps;
// launched with jit_launch_sets).
// narrow (with set_mode): kernels for complex64 arrays (jit_launch_narrow).
bool jit_prepare(const std::vector<const PassDesc*>& passes, std::vector<const JitKernel*>& out, std::string& err,
                 int min_blocks, int threads, bool set_mode = false, bool narrow = false);

// Kernels already compiled for these passes (null where none); with
// queue_missing, the missing ones are queued for compilation on background
// threads, so a later plan with the same structure finds them.
void jit_lookup(const std::vector<const PassDesc*>& passes, std::vector<const JitKernel*>& out, bool queue_missing,
                int min_blocks, int threads, bool set_mode = false);

// Wait (at most timeout_s) until the background compilations have finished.
bool jit_wait(double timeout_s);

// Launch a specialised pass.  host_mats: the pass's matrix block on the host
// (d.mat_elems complex values), copied into the launch's parameters.
cudaError_t jit_launch(const JitKernel* k, const CUtensorMap& tm, const PassDesc& d, const double2* host_mats,
                       int* dev_status, const TileLaunch& tl, int num_sms, cudaStream_t st);

// Launch a specialised pass of the shared-memory form with the interpreting
// kernel's arguments (device matrix pool, gradient partials).
cudaError_t jit_launch_sets(const JitKernel* k, const CUtensorMap& tm, const PassDesc& d, const double2* dev_mats,
                            int* dev_status, const TileLaunch& tl, int num_sms, cudaStream_t st,
                            double* grad_partials);

// Launch a complex64 pass (jit_prepare with narrow): `state` is the float2
// array (set s at state + s * 2^nbits, or the gap layout of PassDesc::gap),
// dev_mats the device matrix pool, grad_partials as for jit_launch_sets.
cudaError_t jit_launch_narrow(const JitKernel* k, const PassDesc& d, const double2* dev_mats, void* state,
                              const TileLaunch& tl, int num_sms, cudaStream_t st, double* grad_partials);

// Kernels compiled and cubins loaded from the cache directory so far.
void jit_counters(uint64_t* compiled, uint64_t* loaded_from_disk);

}  // namespace iqb
