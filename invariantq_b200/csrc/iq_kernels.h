// iq_kernels.h -- launchers for the sm_100a kernels in iq_kernels.cu.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "iq_plan.h"

namespace iqb {

struct TileLaunch {
  int nbuf;                // shared-memory tile buffers per CTA (pipeline depth)
  int ctas_per_sm;         // resident CTAs per SM the grid is sized for
  int consumers;           // threads per CTA (128)
};

// Encode the pass tensor map for `state` (2^nbits complex128).
int encode_pass_tmap(CUtensorMap* tm, void* state, int nbits, const PassDesc& d, char* err, size_t errlen);

// Launch one tile pass.  `mats` is the device copy of the flush's matrix pool.
// grad_partials: [gradient term][CTA] partial sums of the pass's OP_GRAD2 terms (or null)
cudaError_t launch_tile_pass(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status,
                             const TileLaunch& tl, int num_sms, cudaStream_t st, double* grad_partials = nullptr);
// dynamic shared memory of a pass: tile buffers, matrix block, gradient accumulators
size_t tile_pass_smem_bytes(int M, int R, int nbuf, uint32_t mat_elems, uint32_t ngrad);
// one launcher per kernel instantiation (iq_tile_r3.cu, iq_tile_r4.cu, iq_tile_r5.cu)
cudaError_t launch_tile_r3(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status, int nbuf,
                           unsigned grid, size_t smem, cudaStream_t st, double* grad_partials);
cudaError_t launch_tile_r4(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status, int nbuf,
                           unsigned grid, size_t smem, cudaStream_t st, double* grad_partials);
cudaError_t launch_tile_r5(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status, int nbuf,
                           unsigned grid, size_t smem, cudaStream_t st, double* grad_partials);
// grid size the tile pass uses for `d` (the stride of its gradient partials)
unsigned tile_pass_grid(const PassDesc& d, const TileLaunch& tl, int num_sms);

// Simple path: one operation straight in global memory (k = 1..5, LSB-first bits).
struct SimpleOp {
  int k;
  int q[kMaxK];
  uint32_t mat;            // dense 2^k x 2^k row-major matrix in `mats`
};
cudaError_t launch_simple_op(double2* s, int nbits, const SimpleOp& op, const double2* mats, cudaStream_t st);

// ---- reductions (deterministic: fixed grid, partials summed in order) ----
constexpr int kRedBlocks = 592;    // 4 * 148 SMs
constexpr int kRedThreads = 256;
// sum |s_i|^2 over i with (i & mask) == val
cudaError_t launch_sumsq_masked(const double2* s, uint64_t dim, uint64_t mask, uint64_t val, double* partials,
                                double* out, cudaStream_t st);
// sum Re rho_ii (rho is dim x dim row-major) over i with (i & mask) == val
cudaError_t launch_diag_sum(const double2* rho, uint64_t dim, uint64_t mask, uint64_t val, double* partials,
                            double* out, cudaStream_t st);
// sum over the diagonal of -p log2 p, p = max(0, Re rho_ii), p > 1e-14
cudaError_t launch_diag_entropy(const double2* rho, uint64_t dim, double* partials, double* out, cudaStream_t st);
// <psi| P |psi> core sum: sum_i [skip if |a_i|^2 < thresh] (-1)^popc(i & zmask) conj(a_{i^xmask}) a_i
cudaError_t launch_pauli_sum(const double2* s, uint64_t dim, uint64_t xmask, uint64_t zmask, double thresh,
                             double2* partials, double2* out, cudaStream_t st);
// out[0] = sum |a|^2, out[1 + b] = sum over i with bit b set of |a_i|^2, b < nbits
cudaError_t launch_zsums(const double2* s, int nbits, double* partials, double* out, cudaStream_t st);
// Loads the two kernels of launch_zsums on the current device now (under lazy
// module loading they would otherwise load, and take device memory for their
// code, at their first launch).
cudaError_t preload_zsums();
size_t zsums_partials_doubles(int nbits);

// ---- elementwise ----
cudaError_t launch_collapse(double2* s, uint64_t dim, uint64_t mask, uint64_t val, double factor, cudaStream_t st);
// rho[r][c] *= factor if bits(r) and bits(c) at mask both equal val, else 0
cudaError_t launch_dm_collapse(double2* rho, int n, uint64_t mask, uint64_t val, double factor, cudaStream_t st);
cudaError_t launch_set_basis(double2* s, uint64_t dim, cudaStream_t st);   // s = e_0
// nsets arrays of dim amplitudes (dim a power of two) laid end to end, each set to e_0
cudaError_t launch_set_basis_sets(double2* s, uint64_t dim, int nsets, cudaStream_t st);
cudaError_t launch_split(const double2* s, uint64_t count, double* re, double* im, cudaStream_t st);
// Copy the half of the 2^nbits amplitudes with index bit `bit` == val to buf
// (unpack = false) or back from buf (unpack = true), in increasing index order.
cudaError_t launch_half_copy(double2* s, int nbits, int bit, int val, double2* buf, bool unpack, cudaStream_t st);
cudaError_t launch_probs(const double2* s, uint64_t count, double* p, cudaStream_t st);

// ---- sampling ----
// block sums of |a|^2 over blocks of 2^bbits amplitudes
cudaError_t launch_block_sums(const double2* s, uint64_t dim, int bbits, double* out, cudaStream_t st);
// for each shot: within block blk[k], the first index whose running sum (starting at base[k])
// reaches target[k]; falls back to the block's last index
cudaError_t launch_block_search(const double2* s, int bbits, const uint64_t* blk, const double* base,
                                const double* target, uint64_t* out, int shots, cudaStream_t st);

// ---- reduced density matrix for entropy ----
// rho_A[r][c] = sum_env a[idx(r,env)] conj(a[idx(c,env)]), keep[] LSB-first (k <= 12)
cudaError_t launch_partial_trace(const double2* s, int nbits, const int* keep, int k, double2* out, cudaStream_t st);

// ---- adjoint gradients ----
// Pauli terms grouped by their X part: group g covers terms [first[g], first[g+1]).
constexpr int kMaxHamGroups = 64;
struct HamTerms {
  int ngroups;
  uint64_t xmask[kMaxHamGroups];
  int first[kMaxHamGroups + 1];
};
// For each of nsets states psi_s = psi + s * pstride (2^n amplitudes):
// lambda_s = H psi_s written to lam + s * lstride (when lam is not null), and
// energy[s] = Re <psi_s|H|psi_s>.  partials: nsets * kRedBlocks.
cudaError_t launch_hamiltonian_joint(const double2* psi, uint64_t pstride, int n, int nsets, const HamTerms& h,
                                     const uint64_t* zmask, const double2* coef, double2* lam, uint64_t lstride,
                                     double* partials, double* energy, cudaStream_t st);
// nsets joint arrays [psi | lambda | zero padding] of jdim amplitudes end to
// end: psi halves (2^n amplitudes) set to e_0, padding above 2^(n+1) zeroed.
cudaError_t launch_init_joint(double2* s, int n, uint64_t jdim, int nsets, cudaStream_t st);
// The same two with complex64 (float2) storage; products and sums in FP64.
cudaError_t launch_hamiltonian_c64(const float2* psi, uint64_t pstride, int n, int nsets, const HamTerms& h,
                                   const uint64_t* zmask, const double2* coef, float2* lam, uint64_t lstride,
                                   double* partials, double* energy, cudaStream_t st);
cudaError_t launch_init_joint_c64(float2* s, int n, uint64_t jdim, int nsets, cudaStream_t st);
cudaError_t launch_row_sums(const double* in, int rows, int cols, double* out, cudaStream_t st);

// Eigenvalues (ascending) of the reduced state on the kept qubits keep[0..k) of
// the 2^nbits state psi, computed on the device (iq_entropy.cu); k is at most
// reduced_spectrum_max_bits() and below nbits.  Synchronises `st`.
int reduced_spectrum_max_bits();
cudaError_t reduced_spectrum(const double2* psi, int nbits, const int* keep, int k, std::vector<double>& eig,
                             cudaStream_t st);

// Measurement shots on the device (iq_sampling.cu): `shots` outcome indices
// of the 2^nbits state into d_out, with the reference's random numbers
// (mt19937_64 seeded with `seed`, uniform_real_distribution(0, 1)) and its
// lower_bound rule.  work: sample_work_bytes(nbits, shots) bytes of device memory.
size_t sample_work_bytes(int nbits, uint64_t shots);
cudaError_t sample_on_device(const double2* s, int nbits, uint64_t shots, uint64_t seed, void* work, uint64_t* d_out,
                             cudaStream_t st);
// `count` uniform draws of the mt19937_64 stream seeded with `seed` (one CTA).
cudaError_t launch_mt64_uniform(uint64_t seed, uint64_t count, double* out, cudaStream_t st);
// Sorted distinct outcomes of d_shots and their counts (d_nuniq: how many).
// work: count_work_bytes(shots) bytes.
size_t count_work_bytes(uint64_t shots);
cudaError_t count_outcomes(const uint64_t* d_shots, uint64_t shots, void* work, uint64_t* d_vals, uint64_t* d_cnts,
                           uint64_t* d_nuniq, cudaStream_t st);

// Record an error for iq_last_error (defined in iq_runtime.cu).
void record_error(int code, const char* msg);
// Add to the iq_kernel_launches counter (defined in iq_runtime.cu).
void count_launches(uint64_t n);

}  // namespace iqb
