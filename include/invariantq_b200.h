/*
 * invariantq_b200.h -- C ABI of libinvariantq.so, the B200 (sm_100a) CUDA
 * implementation of InvariantQ's state-vector and density-matrix core.
 *
 * Part 1 repeats, symbol for symbol and with the same signatures, the
 * reference's C ABI (core/include/c_api.h:10-65) that its ctypes binding
 * (invariantq/core/binding.py:54-299) binds at import time, so this library
 * drops in under the unmodified binding.  Each declaration names the reference
 * function it replaces.  Part 2 adds entry points the reference does not have.
 *
 * Conventions (as the reference): qubit q is bit q of the amplitude index;
 * matrices are row-major with split real/imaginary double arrays; a 2-qubit
 * matrix's local index has q0 as its most significant bit; a fused k-qubit
 * matrix (k >= 3) has qubits[b] as local index bit b.  A density matrix is
 * row-major rho[r * 2^n + c].
 *
 * Execution model: amplitudes live in GPU memory.  Gate and channel calls are
 * queued on the handle and applied in fused tile passes when a result is read
 * (or the queue is long); every call that returns data to the host waits for
 * the GPU first, so the host-visible behaviour is that of the reference's
 * synchronous calls.  Calls on one handle must not overlap; distinct handles
 * are independent.
 *
 * Errors: where the reference throws through extern "C" (and so terminates the
 * process) this library records a message (iq_last_error) and returns: void
 * calls become no-ops, int calls return -1, double calls return NaN, create
 * returns NULL.  NULL pointer arguments are silent no-ops returning 0, as in the
 * reference (core/src/api.cpp).
 */
#ifndef INVARIANTQ_B200_H
#define INVARIANTQ_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ===================== Part 1: the reference ABI (core/include/c_api.h) ===================== */

/* -- state vector (c_api.h:11-24; implementations core/src/api.cpp:14-112) -- */
void* iq_statevector_create(size_t num_qubits);                                   /* api.cpp:14-20  */
void  iq_statevector_free(void* sv);                                              /* api.cpp:22-24  */
void  iq_statevector_reset(void* sv);                                             /* api.cpp:26-28  */
void  iq_statevector_apply_1q(void* sv, size_t target, const double* u_real,
                              const double* u_imag);                              /* api.cpp:30-37, statevector.cpp:26-47 */
void  iq_statevector_apply_2q(void* sv, size_t q0, size_t q1, const double* u_real,
                              const double* u_imag);                              /* api.cpp:39-46, statevector.cpp:49-87 */
void  iq_statevector_apply_fused(void* sv, const size_t* qubits, size_t k,
                                 const double* u_real, const double* u_imag);     /* api.cpp:48-57, statevector.cpp:89-152; k <= 5 here (reference: 4) */
int   iq_statevector_measure(void* sv, size_t target, double rand_val);           /* api.cpp:59-62, statevector.cpp:190-195 */
void  iq_statevector_reset_qubit(void* sv, size_t target, double rand_val);       /* api.cpp:64-67, statevector.cpp:197-204 */
double iq_statevector_measure_prob(void* sv, size_t target, int outcome);         /* api.cpp:69-72, statevector.cpp:154-169 */
void  iq_statevector_get_amplitudes(void* sv, double* real_out, double* imag_out);/* api.cpp:74-83  */
void  iq_statevector_get_probabilities(void* sv, double* probs_out);              /* api.cpp:85-90, statevector.cpp:226-233 */
void  iq_statevector_sample(void* sv, size_t num_shots, uint64_t seed,
                            uint64_t* results_out);                               /* api.cpp:92-97, statevector.cpp:235-256 */
double iq_statevector_entropy(void* sv, const size_t* qubits, size_t num_subsys_qubits); /* api.cpp:99-103, statevector.cpp:293-410 */
void  iq_statevector_expval_pauli(void* sv, const char* pauli_str, const size_t* qubits,
                                  size_t len, double* val_real, double* val_imag);/* api.cpp:105-112, statevector.cpp:258-291 */

/* -- density matrix (c_api.h:27-38; api.cpp:116-192) -- */
void* iq_density_matrix_create(size_t num_qubits);                                /* api.cpp:116-122 */
void  iq_density_matrix_free(void* dm);                                           /* api.cpp:124-126 */
void  iq_density_matrix_reset(void* dm);                                          /* api.cpp:128-130 */
void  iq_density_matrix_apply_1q_unitary(void* dm, size_t target, const double* u_real,
                                         const double* u_imag);                   /* api.cpp:132-137, density_matrix.cpp:18-67 */
void  iq_density_matrix_apply_2q_unitary(void* dm, size_t q0, size_t q1, const double* u_real,
                                         const double* u_imag);                   /* api.cpp:139-144, density_matrix.cpp:69-145 */
void  iq_density_matrix_apply_kraus_1q(void* dm, size_t target, size_t num_kraus,
                                       const double* k_real, const double* k_imag);/* api.cpp:146-155, density_matrix.cpp:147-163 */
void  iq_density_matrix_get_elements(void* dm, double* real_out, double* imag_out);/* api.cpp:157-167 */
double iq_density_matrix_trace(void* dm);                                         /* api.cpp:169-172, density_matrix.cpp:193-199 */
double iq_density_matrix_purity(void* dm);                                        /* api.cpp:174-177, density_matrix.cpp:201-208 */
double iq_density_matrix_entropy(void* dm);                                       /* api.cpp:179-182, density_matrix.cpp:310-380 */
int   iq_density_matrix_measure(void* dm, size_t target, double rand_val);        /* api.cpp:184-187, density_matrix.cpp:218-256 */
void  iq_density_matrix_reset_qubit(void* dm, size_t target);                     /* api.cpp:189-192, density_matrix.cpp:258-269 */

/* -- stabilizer (c_api.h:41-55) and MPS (c_api.h:58-65).  Not GPU paths: these
 * forward to a CPU core named by the environment variable IQ_CPU_CORE_LIB (a
 * build of the reference's core/ library) when it is set; otherwise create
 * returns NULL with an error message and the other calls are no-ops. -- */
void* iq_stabilizer_create(size_t num_qubits);
void  iq_stabilizer_free(void* stab);
void  iq_stabilizer_reset(void* stab);
void  iq_stabilizer_reset_qubit(void* stab, size_t a, double rand_val);
void  iq_stabilizer_apply_h(void* stab, size_t a);
void  iq_stabilizer_apply_s(void* stab, size_t a);
void  iq_stabilizer_apply_sdg(void* stab, size_t a);
void  iq_stabilizer_apply_cnot(void* stab, size_t a, size_t b);
void  iq_stabilizer_apply_cz(void* stab, size_t a, size_t b);
void  iq_stabilizer_apply_swap(void* stab, size_t a, size_t b);
void  iq_stabilizer_apply_x(void* stab, size_t a);
void  iq_stabilizer_apply_y(void* stab, size_t a);
void  iq_stabilizer_apply_z(void* stab, size_t a);
int   iq_stabilizer_measure(void* stab, size_t a, double rand_val);
void  iq_stabilizer_to_string(void* stab, char* buffer, size_t max_len);
void* iq_mps_create(size_t num_qubits, size_t max_bond_dim, double cutoff);
void  iq_mps_free(void* mps);
void  iq_mps_reset(void* mps);
void  iq_mps_apply_1q(void* mps, size_t target, const double* u_real, const double* u_imag);
void  iq_mps_apply_2q(void* mps, size_t q0, size_t q1, const double* u_real, const double* u_imag);
double iq_mps_entropy(void* mps, size_t bond_idx);
void  iq_mps_to_statevector(void* mps, double* real_out, double* imag_out);
int   iq_mps_measure(void* mps, size_t target, double rand_val);

/* ===================== Part 2: additions (no counterpart in the reference) ===================== */

/* Last error recorded on the calling thread: returns its code (0 = none) and
 * copies the message (NUL-terminated, truncated to len). */
int  iq_last_error(char* buf, size_t len);
void iq_clear_error(void);
const char* iq_version(void);
/* Kernels this library has launched since it was loaded (all handles). */
uint64_t iq_kernel_launches(void);

/* Apply every queued operation now (asynchronous) / and wait for it. 0 = ok. */
int iq_statevector_flush(void* sv);
int iq_statevector_sync(void* sv);
/* sum_i |a_i|^2 (the reference's unexported StateVector::norm_squared, statevector.cpp:206-213). */
double iq_statevector_norm(void* sv);
/* <Z_q> for every qubit q = 0..n-1 in one pass. 0 = ok. */
int iq_statevector_expval_z_all(void* sv, double* out);
/* sum_t coeff[t] <P_t> for nterms Pauli strings, each n characters long
 * (character q acts on qubit q; 'I','X','Y','Z'), exact sums. 0 = ok. */
int iq_statevector_expval_pauli_sum(void* sv, size_t nterms, const double* coeffs, const char* paulis,
                                    double* val_real, double* val_imag);
/* Overwrite the amplitudes from split host arrays (2^n each). 0 = ok. */
int iq_statevector_set_amplitudes(void* sv, const double* real_in, const double* imag_in);
/* Device address of the amplitude array (complex128, 2^n), after a flush; the
 * handle's stream (cudaStream_t) for ordering work against it. */
void* iq_statevector_device_ptr(void* sv);
void* iq_statevector_stream(void* sv);
/* The half of the amplitudes whose index bit `bit` equals `value` (0 or 1), in
 * increasing index order, copied to (pack) or from (unpack) a device buffer of
 * 2^(n-1) complex128; queued gates are applied first and the copy has finished
 * when the call returns.  The exchange step of a state vector sharded across
 * GPUs by its top qubits (a global qubit swapped with a local one moves one
 * such half to the partner rank).  No counterpart in the reference.  0 = ok. */
/* Measurement shots as sorted distinct outcomes and their counts, computed on
 * the device (the same shots as iq_statevector_sample with this seed; the
 * counts dictionary the reference's driver builds in Python,
 * invariantq/simulator/statevector.py:105-114).  values_out and counts_out
 * hold up to num_shots entries; *num_unique receives how many were written.
 * At most 2^30 shots.  No counterpart in the reference ABI.  0 = ok. */
int iq_statevector_sample_counts(void* sv, size_t num_shots, uint64_t seed, uint64_t* values_out,
                                 uint64_t* counts_out, size_t* num_unique);
/* `count` draws of std::uniform_real_distribution<double>(0, 1) over
 * std::mt19937_64 seeded with `seed`, generated on the current device (the
 * stream iq_statevector_sample uses).  0 = ok. */
int iq_mt64_uniform(uint64_t seed, size_t count, double* out);
int iq_statevector_pack_half(void* sv, size_t bit, int value, void* d_dst);
int iq_statevector_unpack_half(void* sv, size_t bit, int value, const void* d_src);
size_t iq_statevector_num_qubits(void* sv);

/* Tuning / diagnostics for either handle kind ("inject_status" = code: set the
 * handle's device status word, as a timed-out tile pass would).  Keys: "tile_bits", "chunk_bits",
 * "reg_slots" (register slots R = 3, 4, 5 per tile-pass thread: 2^R amplitudes
 * each; raised to the widest fused block), "max_stages", "budget", "nbuf",
 * "ctas_per_sm", "eager", "fuse", "flush_ops", "profile", "jit" (tile passes
 * run by kernels generated for each pass's structure and compiled with NVRTC:
 * 0 off; 1, the default, compiles a recorded program's kernels at record_end
 * and lets flushes use kernels already compiled for their structure, queuing
 * the missing ones for compilation on background threads, for arrays of at
 * least 2^18 amplitudes; 2 compiles before every first launch, any size),
 * "plan_style" (0: follow "jit"; 1: plan for the interpreting kernel, fusing
 * one-qubit gates into two-qubit blocks; 2: plan for specialised kernels,
 * leaving CX/CZ/SWAP apart and normalising dense one-qubit gates), "normalize"
 * (1: normalised one-qubit gates in plans of style 2).  Plans of style 2 run
 * 4 CTAs per SM with one tile buffer unless those options (or IQ_CTAS_PER_SM,
 * IQ_NBUF) are set; get_option reports the values the handle's next plan
 * uses.  "chunk_bits" 3 with "budget" 160 plans fewer, fuller passes: a
 * faster circuit at a lower bandwidth per pass.
 * 0 = ok, -1 = unknown key or bad value. */
int iq_handle_set_option(void* h, const char* key, double value);
double iq_handle_get_option(void* h, const char* key);
/* Counters: out[0] passes, [1] operations applied, [2] algorithmic bytes moved by
 * passes, [3] kernel launches, [4] flushes, [5] tile-pass launches, [6] bytes of
 * operation matrices copied host->device by flushes, [7] tile passes run by a
 * specialised kernel.  Returns the number of values written. */
int iq_handle_stats(void* h, double* out, size_t n);
/* Specialised pass kernels of the process: out[0] compiled with NVRTC, [1]
 * loaded from the cubin cache directory (IQ_JIT_CACHE, default
 * ~/.cache/invariantq_b200/jit, "off" = none); `note` gets why the last
 * compilation attempt failed ("" if none).  Returns the values written. */
int iq_jit_info(double* out, size_t n, char* note, size_t note_len);
/* Wait up to timeout_s for background compilations to finish: 0 = idle. */
int iq_jit_wait(double timeout_s);
/* Recorded programs: operations issued between record_begin and record_end are
 * planned once into tile passes whose matrices and descriptors stay on the
 * device; program_run launches them on the handle's stream (any number of
 * times, on the handle's current amplitudes).  program_info: out[0] passes,
 * [1] operations, [2] matrix bytes, [3] planned arithmetic cost.
 * program_pass_info: pass i's out[0] operations, [1] planned arithmetic cost
 * (real multiply-adds per amplitude), [2] register stages, [3] tile bits M,
 * [4] chunk bits c, [5] tiles; returns the count written, 0 past the end. */
int   iq_handle_record_begin(void* h);
void* iq_handle_record_end(void* h);
int   iq_handle_program_run(void* h, void* prog);
int   iq_program_info(void* prog, double* out, size_t n);
int   iq_program_pass_info(void* prog, size_t i, double* out, size_t n);
void  iq_program_free(void* prog);
/* With option "profile" = 1 every tile pass is bracketed by CUDA events; this
 * returns up to max per-pass durations in ms (oldest first) and clears them. */
int iq_handle_profile_read(void* h, double* ms_out, size_t max);

/* <Z_q> for q = 0..num_qubits-1 of a complex128 amplitude array the caller
 * holds in device memory (d_amps, 2^num_qubits elements), written to the
 * caller's device array d_out (num_qubits doubles), launched on `stream`
 * (a cudaStream_t; results are ready when the stream reaches them).  No
 * counterpart in the reference.  It allocates no memory of any kind: it is for
 * callers that cannot call cudaMalloc where they need the result -- a host
 * whose device memory is already committed (a 33-qubit state fills 128 GiB) or
 * code running inside another framework that owns the free device memory.  Its
 * reduction scratch is a fixed array in the library (about 166 KB per GPU,
 * held until the process exits), so num_qubits is limited to
 * IQ_NOALLOC_MAX_QUBITS and larger sizes are rejected with an error.  d_amps
 * may be device or managed memory; the call runs on the device that holds it
 * and leaves the caller's current device as it found it.  The first call on
 * each device does a one-time set-up: it loads the call's kernels (with CUDA's
 * default lazy module loading, code is loaded into device memory at first use)
 * and looks up the scratch array's device address.  Make that first call before
 * the device memory is committed and before any stream capture; later calls
 * take no device memory.  A cudaDeviceReset invalidates the set-up (the looked-up
 * address belongs to the context it ends).  All calls on one device share the
 * array, so calls that overlap on the GPU (different streams, no ordering
 * between them) race and must be avoided.  Returns 0, or -1 with iq_last_error
 * set. */
#define IQ_NOALLOC_MAX_QUBITS 34
int iq_statevector_expval_z_all_noalloc(const void* d_amps, size_t num_qubits, double* d_out, void* stream);

/* ---- Adjoint-method gradients (no counterpart in the reference; the energy
 * they differentiate is the TFIM expectation of invariantq/algorithms/vqe.py:44-79).
 *
 * A parametrised circuit on num_qubits qubits, starting from |0...0>: gate i
 * has kind kinds[i] (IQ_GATE_*), qubit q0[i] (control q0, target q1 for CX;
 * the two qubits of CZ) and, for the rotation kinds, first parameter index
 * param_index[i].  RX/RY/RZ(t) = exp(-i t P / 2); P(l) = diag(1, e^{i l});
 * U3 reads parameters p, p+1, p+2 as (theta, phi, lambda) with the
 * reference's U3 matrix.  H = sum_t coeffs[t] P_t with P_t the num_qubits
 * characters paulis[t * num_qubits .. +num_qubits) ('I','X','Y','Z';
 * character q acts on qubit q).  Outputs: energy <psi|H|psi> and dE/dparam
 * for every parameter (parameters read by several gates sum their terms). */
#define IQ_GATE_RX 1
#define IQ_GATE_RY 2
#define IQ_GATE_RZ 3
#define IQ_GATE_U3 4
#define IQ_GATE_P  5
#define IQ_GATE_CZ 6
#define IQ_GATE_CX 7
#define IQ_GATE_H  8
#define IQ_GATE_X  9
#define IQ_GATE_SX 10

typedef struct iq_adjoint_circuit {
  size_t num_qubits;
  size_t num_ops;
  const int* kinds;
  const int* q0;
  const int* q1;
  const int* param_index;
  size_t num_params;        /* parameters per set (columns of params) */
  size_t num_sets;          /* parameter sets evaluated for this circuit */
  const double* params;     /* num_sets x num_params, row-major */
  size_t num_terms;
  const double* coeffs;     /* num_terms */
  const char* paulis;       /* num_terms x num_qubits */
  double* energy_out;       /* num_sets */
  double* grad_out;         /* num_sets x num_params (unused by iq_ansatz_energy) */
} iq_adjoint_circuit;

/* One circuit, one parameter set.  Returns 0, or -1 with iq_last_error set. */
int iq_adjoint_gradient(size_t num_qubits, size_t num_ops, const int* kinds, const int* q0, const int* q1,
                        const int* param_index, size_t num_params, const double* params, size_t num_terms,
                        const double* coeffs, const char* paulis, double* energy_out, double* grad_out);
/* The same gradient with the states stored as complex64 (8 B per amplitude,
 * half the memory and traffic of complex128): every gate and Hamiltonian
 * product is computed in FP64 from the loaded amplitudes, values are rounded
 * to complex64 where they are stored (the array, and the shared-memory tile
 * between register stages), every sum (gradient terms, energy) is
 * accumulated in FP64.  One
 * parameter set; two state buffers (psi and lambda, 8 B x 2^n each).  The
 * result differs from iq_adjoint_gradient by the complex64 rounding of the
 * states (~1e-7 relative at 30 qubits, 16 layers). */
int iq_adjoint_gradient_c64(size_t num_qubits, size_t num_ops, const int* kinds, const int* q0, const int* q1,
                            const int* param_index, size_t num_params, const double* params, size_t num_terms,
                            const double* coeffs, const char* paulis, double* energy_out, double* grad_out);
/* Every parameter set of every circuit, run concurrently on num_streams CUDA
 * streams (<= 0: IQ_ADJOINT_STREAMS or 8), each with its own device workspace;
 * the parameter sets of one circuit run together, through the same tile-pass
 * launches, in groups that fit IQ_ADJOINT_JOB_BYTES (4 GiB) of states.  Fewer
 * streams when the workspaces would not fit in device memory.  Workspaces are
 * kept for later calls unless they hold more than 8 GiB of device memory.
 * Returns 0, or -1 with iq_last_error set. */
int iq_adjoint_gradient_batch(const iq_adjoint_circuit* circuits, size_t num_circuits, int num_streams);
/* Free the device and pinned host memory the adjoint calls keep between calls;
 * returns the number of workspaces freed. */
int iq_adjoint_release(void);
/* Energies only (grad_out unused): the forward circuit and <psi|H|psi> for each
 * parameter set of one circuit, one set after another on one stream -- the
 * plain path a parameter-shift gradient evaluates 2 x num_params times. */
int iq_ansatz_energy(const iq_adjoint_circuit* circuit);
/* Counters of the calling thread's last adjoint / energy call: out[0] jobs,
 * [1] forward passes, [2] backward passes, [3] kernel launches, [4] algorithmic
 * HBM bytes of the passes, [5] host preparation ms (summed over workers),
 * [6] wall ms, [7] streams used, [8] passes run by specialised kernels
 * (IQ_ADJOINT_JIT, default 1), [9] parameter sets run by the persistent
 * shared-memory executor (circuits of at most IQ_RESIDENT_MAX_QUBITS = 12
 * qubits: one launch for all of them, fed from a device-side queue of
 * (circuit, set) items and replayed from a captured CUDA graph).  Returns the
 * number of counters (10). */
int iq_adjoint_stats(double* out, size_t n);

/* Failure-path check (no counterpart in the reference): one CTA waits, with
 * the tile kernel's bounded wait, on an mbarrier phase that never completes.
 * The wait gives up after limit_ms (at most 1000), sets the status word and the
 * kernel returns, leaving the GPU context usable.  Returns the status the
 * kernel set (1: a tile load timed out) and the time it waited in *waited_ms;
 * -1 on a CUDA error.  Handles report the same status word on their next
 * synchronising call (option "inject_status" sets it, for tests). */
int iq_selftest_bounded_wait(double limit_ms, double* waited_ms);

/* Density-matrix additions. */
int iq_density_matrix_flush(void* dm);
/* Kraus channel on two qubits: num_kraus 4x4 matrices, q0 = most significant
 * local bit (the reference declares DensityMatrix::apply_kraus for this,
 * density_matrix.cpp:165-191, but does not export it). */
void iq_density_matrix_apply_kraus_2q(void* dm, size_t q0, size_t q1, size_t num_kraus,
                                      const double* k_real, const double* k_imag);
/* rho_ii for i = 0..2^n-1. */
void iq_density_matrix_get_diagonal(void* dm, double* out);
/* P(qubit target = outcome) = sum of matching diagonal entries. */
double iq_density_matrix_measure_prob(void* dm, size_t target, int outcome);
void* iq_density_matrix_device_ptr(void* dm);

#ifdef __cplusplus
}
#endif
#endif /* INVARIANTQ_B200_H */
