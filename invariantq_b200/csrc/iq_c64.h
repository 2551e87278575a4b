// iq_c64.h -- launchers of the complex64 adjoint-gradient kernels (iq_c64.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "iq_kernels.h"

namespace iqb {

constexpr int kC64MaxRunOps = 8;   // one-qubit gates per run (longer runs are split)
constexpr int kC64Blocks = 592;    // fixed grid: the partials' row length (4 x 148 SMs)

struct C64Mat { double m[8]; };    // 2x2 row-major, re/im interleaved

struct C64Op {
  int gen;          // rotation exp(-i t P / 2) with P = X (0), Y (1), Z (2); -1: fixed gate
  int term;         // gradient term of a rotation
  double c, s;      // cos(t / 2), sin(t / 2)
  double inv[8];    // fixed gate: its inverse (2x2, re/im interleaved)
};

struct C64Run {     // one-qubit gates on qubit q, in forward order
  int q;
  int nops;
  C64Op ops[kC64MaxRunOps];
};

cudaError_t c64_set_basis(float2* s, int n, cudaStream_t st);
cudaError_t c64_apply1q(float2* s, int n, int q, const C64Mat& m, cudaStream_t st);
cudaError_t c64_cz(float2* s, int n, int a, int b, cudaStream_t st);
cudaError_t c64_cx(float2* s, int n, int control, int target, cudaStream_t st);
// backward walk of a run on psi and lambda; partials[term * kC64Blocks + block]
cudaError_t c64_grad_run(float2* psi, float2* lam, int n, const C64Run& run, double* partials, cudaStream_t st);
// lambda = H psi; partials[block] = block sums of Re <psi|lambda>
cudaError_t c64_hamiltonian(const float2* psi, int n, const HamTerms& h, const uint64_t* zmask, const double2* coef,
                            float2* lam, double* partials, cudaStream_t st);

}  // namespace iqb
