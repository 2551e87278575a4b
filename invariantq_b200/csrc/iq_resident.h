// iq_resident.h -- the persistent executor for small circuits in a gradient
// batch (iq_resident.cu): every (circuit, parameter set) whose [psi | lambda]
// pair fits one CTA's shared memory is a work item of one persistent launch.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "iq_kernels.h"
#include "iq_plan.h"

namespace iqb {

// Largest qubit count whose psi and lambda (2 x 16 B x 2^n) live in shared memory.
constexpr int kResidentMaxQubits = 12;
// Most parameters (gradient accumulators in shared memory) of a resident circuit.
constexpr int kResidentMaxParams = 4096;

struct ResidentJob {
  int n = 0;
  const std::vector<AnsatzOp>* ops = nullptr;
  int nparams = 0;
  size_t nsets = 0;
  const double* params = nullptr;         // nsets x nparams, row-major (host)
  const HamTerms* groups = nullptr;       // Pauli terms grouped by X part
  const std::vector<uint64_t>* zmask = nullptr;
  const std::vector<double2>* coef = nullptr;
  double* energy_out = nullptr;           // nsets (host)
  double* grad_out = nullptr;             // nsets x nparams (host)
};

// Run every set of every job on device `dev` in one persistent launch,
// replayed from a CUDA graph captured the first time a batch of this structure
// (qubit counts, gates, Hamiltonian terms, set counts) is seen; results are in
// the jobs' host outputs on return.  Returns false with `err` on failure.
bool resident_run(int dev, const std::vector<ResidentJob>& jobs, std::string& err, double* host_ms = nullptr);

// Frees every cached plan (graphs, device and pinned buffers).
void resident_release();

}  // namespace iqb
