// iq_plan.h -- the contract between the host gate scheduler (iq_sched.cpp) and
// the device tile-pass kernel (iq_kernels.cu).
//
// A *pass* streams the whole amplitude array through shared memory once (one
// read + one write of 16 B per amplitude).  The array is cut into tiles of 2^M
// amplitudes: a tile holds every combination of M "tile-local" index bits for
// one fixed value of all other bits.  Tile-local bit j < c is physical bit j
// (a contiguous chunk of 2^c amplitudes); tile-local bit c + i is physical bit
// H[i] (H ascending).  Inside the tile the pass runs a list of *stages*; in a
// stage each thread holds 2^R amplitudes in registers (the R "register slots"
// S[0..R-1] are tile-local bits), eight consecutive lanes (an octet) span three
// more "lane" bits, and the remaining "thread" bits enumerate the octets.  A
// stage applies its operations to the registers (lane-bit operations use warp
// shuffles inside the octet) and writes the registers back.
//
// All operation matrices use one convention: for an operation on qubit list
// q[0..k-1], bit i of the 2^k local row/column index is qubit q[i] (LSB-first).
// The C ABI's 2-qubit calls (q0 = most significant) are converted to this form
// before they reach the scheduler.
#pragma once
#if defined(__CUDACC_RTC__)
// runtime-compiled kernels (NVRTC): no system headers
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
#else
#include <stdint.h>
#include <stddef.h>
#endif

#if defined(__CUDACC__)
#define IQ_HD __host__ __device__ __forceinline__
#else
#define IQ_HD inline
#endif

namespace iqb {

constexpr int kMaxTileBits = 13;   // 2^13 amplitudes * 16 B = 128 KiB of shared memory
constexpr int kLaneBits = 3;       // octet = 8 lanes
constexpr int kMaxStages = 24;
constexpr int kMaxPassOps = 160;
constexpr int kMaxK = 5;           // widest dense block the kernels apply
constexpr int kSmemMatElems = 1024; // per-pass matrix block kept in shared memory (16 KiB)
constexpr int kMaxPassGrads = 64;   // gradient terms accumulated by one pass

// Error codes a kernel can raise in the per-handle device status word.
enum DevErr : int {
  DEV_OK = 0,
  DEV_WAIT_LOADED = 1,     // a tile load did not complete in the wait limit
  DEV_WAIT_COMPUTED = 2,   // the producer waited too long for the consumers
};

// Threads per tile-pass CTA for R register slots: R = 3 (8 amplitudes per
// thread, <= 128 registers) runs 256 threads so a 2^11 tile is still one row
// set per stage and twice the warps are resident; R = 4, 5 run 128.
constexpr int tile_pass_threads(int R) { return R == 3 ? 256 : 128; }

enum OpKind : uint8_t {
  OP_NONE = 0,
  OP_D1R = 1,   // dense 2x2, register slot a
  OP_D1L = 2,   // dense 2x2, lane bit a
  OP_D2R = 3,   // dense 4x4, register slots a (matrix bit 0) and b (matrix bit 1)
  OP_DKR = 4,   // dense 2^k x 2^k, register slots 0..k-1 (matrix bit i = slot i); ends its stage
  OP_M1R = 5,   // monomial 2x2 (permutation + phases), register slot a
  OP_M1L = 6,   // monomial 2x2, lane bit a
  OP_M2R = 7,   // monomial 4x4, register slots a (bit 0) and b (bit 1)
  OP_GRAD2 = 8, // adjoint step on slots a (psi/lambda select bit) and b (qubit bit): add
                // Im<lambda|P|psi> (P = X, Y, Z for `perm` = 0, 1, 2) to gradient term
                // `gidx`, then apply the 2x2 matrix at `mat` to the qubit for both halves; the
                // matrix is the inverse rotation exp(+i t P / 2), or a multiple of it, read
                // through its structure (entries 0, 1, 3) in the form `flags` names:
                // GRAD_PLAIN, GRAD_TAN, GRAD_COT (X, Y) or GRAD_PHASE (Z)
  OP_N1R = 9,   // one-qubit 2x2 on register slot a whose row-0 entry in column `perm`
                // (0 or 1) is exactly 1: that product is skipped (6 instead of 8 FMAs per
                // amplitude); the matrix is stored whole, so a lane placement runs it as OP_D1L
  OP_R1R = 10,  // real rotation on register slot a, normalised (2 FMAs per amplitude): perm 0:
                // [[1, -t], [t, 1]] with t = Re m[2]; perm 1: [[u, -1], [1, u]] with u = Re m[0];
                // stored whole, so a lane placement runs it as OP_D1L
  OP_R1L = 11,  // the same rotation on lane bit a: each lane combines its own amplitude with its
                // partner's (warp shuffle): 2 FMAs per amplitude in the tan form
  OP_X2R = 12,  // 4x4 on register slots a (bit 0) and b (bit 1) whose only nonzero entries are
                // the corners (0,0), (0,3), (3,0), (3,3) and the middle (1,1), (2,2) -- the shape
                // of the superoperators of depolarizing, amplitude / phase damping and thermal
                // relaxation channels and of their products; stored whole (16 entries); flags
                // bit 0: the corners are real, bit 1: the middle is real (3 to 6 FMAs per
                // amplitude)
};

// SchedOp::xpat bits (0: not OP_X2R's shape)
constexpr uint8_t XPAT_SHAPE = 1;
constexpr uint8_t XPAT_CORNERS_REAL = 2;
constexpr uint8_t XPAT_MIDDLE_REAL = 4;

// flags
constexpr uint8_t OPF_UNIT_PHASE = 1;  // monomial whose phases are all exactly 1
constexpr uint8_t OPF_REAL = 2;        // OP_D1R / OP_D1L whose entries are real (4 FMAs per amplitude, not 8)

// Forms of an adjoint step's inverse rotation (OP_GRAD2 flags).  The step may
// apply a multiple of the inverse: a unit phase common to psi and lambda
// leaves every later Im<lambda|P|psi> unchanged; a real factor k scales
// every later term by k^2, which the host divides out (ansatz_backward's
// grad_scale).
enum GradForm : uint8_t {
  GRAD_PLAIN = 0,   // [[c, i s], [i s, c]] (X), [[c, s], [-s, c]] (Y), diag(u0, u3) (Z)
  GRAD_TAN = 1,     // X, Y divided by c: [[1, i t], [i t, 1]], [[1, t], [-t, 1]] (t = Im / Re m[1])
  GRAD_COT = 2,     // X, Y divided by s: [[u, i], [i, u]], [[u, 1], [-1, u]] (u = Re m[0])
  GRAD_PHASE = 1,   // Z divided by its row-0 phase: diag(1, u3)
};

struct OpDesc {          // 16 bytes
  uint8_t kind;
  uint8_t a, b, k;
  uint8_t perm;          // monomial: row r reads column (perm >> (2r)) & 3 (1q: bit 0 = swap)
  uint8_t flags;
  uint8_t urows;         // monomial: bit r set = row r's phase is exactly 1 (its product is skipped)
  uint8_t pad1;
  uint32_t mat;          // offset (complex elements) into the flush's matrix buffer
  uint32_t gidx;         // OP_GRAD2: the pass's local gradient index (global term: PassDesc::grad_term)
};

struct StageDesc {       // 28 bytes
  uint8_t S[kMaxK];      // register slot -> tile-local bit
  uint8_t lane[kLaneBits];
  uint8_t nt;            // number of thread bits
  uint8_t tb[kMaxTileBits];
  uint16_t op0, op1;     // operation range [op0, op1)
  uint16_t pad;
};

struct PassDesc {
  uint8_t M, c, R, nstages;
  uint8_t nH, nbox;
  // gap != 0: tile addresses carry a zero at address bit `gap` (above every
  // bit the pass touches), so the pass runs over the lower half of each
  // 2^(gap + 1)-amplitude block -- e.g. the psi half of a [psi | lambda] array.
  uint8_t gap;
  uint8_t pad1;
  uint8_t H[kMaxTileBits + 3];   // physical bit of tile-local bit c + i (ascending)
  uint64_t ntiles;
  uint32_t nops, pad2;
  uint32_t mat_base;             // this pass's matrix block in the flush's matrix pool
  uint32_t mat_elems;            // complex elements in the block (ops' `mat` are relative to it)
  uint32_t grad_base;            // unused (0)
  uint32_t ngrad;                // OP_GRAD2 steps in the pass (<= kMaxPassGrads)
  uint32_t grad_term[kMaxPassGrads];   // global gradient term of local index i
  // Several arrays of 2^nbits amplitudes laid end to end ("sets", e.g. one per
  // parameter set of a circuit), all run through the same planned operations
  // with their own matrices: ntiles counts the tiles of every set, set s owns
  // tiles [s << set_shift, (s + 1) << set_shift), its matrix block starts
  // set_mat_stride complex elements after set s - 1's, and its gradient terms
  // are rows s * grad_stride + term of the partials.  nsets 0 or 1: one array.
  uint32_t nsets;
  uint32_t set_shift;
  uint32_t set_mat_stride;
  uint32_t grad_stride;
  StageDesc st[kMaxStages];
  OpDesc ops[kMaxPassOps];
};

// One queued gate / channel as the scheduler sees it.
struct SchedOp {
  uint8_t k;             // 1..5
  uint8_t q[kMaxK];      // index bits, LSB-first matrix convention
  uint8_t mono;          // 1 = monomial matrix (perm + phases)
  uint8_t perm;          // monomial permutation (see OpDesc)
  uint8_t unit;          // monomial with unit phases
  uint32_t mat;          // complex offset of the 2^k x 2^k row-major matrix (dense) or 2^k phases (monomial)
  uint32_t dense;        // complex offset of the dense 2^k x 2^k matrix (always present)
  uint8_t norm;          // k = 1 dense, normalised: row-0 entry in column norm - 1 is exactly 1 (0: not)
  uint8_t rot;           // k = 1 real rotation, normalised: 1 = tan form, 2 = cot form (0: not);
                         // adjoint step: its inverse rotation's form (OpDesc::flags of OP_GRAD2)
  uint8_t urows;         // monomial: bit r = row r's phase is exactly 1
  uint8_t grad;          // 1: adjoint step (k = 2; q[0] = select bit, q[1] = qubit bit; 2x2 matrix)
  uint8_t xpat;          // k = 2 dense matrix of OP_X2R's shape: XPAT_* bits (0: not)
  uint8_t realm;         // k = 1 dense matrix with real entries (OPF_REAL)
  uint8_t gen;           // adjoint step generator: 0 = X, 1 = Y, 2 = Z
  uint32_t gidx;         // adjoint step gradient term index (increasing in queue order)
  // factor the operation multiplies the scale of a scaled backward sweep by
  // (stored amplitudes = true amplitudes / scale; 0 means 1): a scaled
  // adjoint step's divisor, or 1 / f for a scalar operation multiplying by f
  double smul;
};

struct SchedParams {
  int nbits;             // index bits of the array (SV: n, DM: 2n)
  int M;                 // tile bits
  int c;                 // contiguous chunk bits (>= 3)
  int R;                 // register slots per thread (3, 4 or 5)
  int max_stages;        // stages per pass (each costs one shared-memory round trip)
  double budget;         // max arithmetic cost per pass (real FMAs per amplitude)
  double grad_cost = 6.0;    // cost of an adjoint step: a structured rotation on both halves (4) plus its products
};

// A planned pass.  desc.ops[].mat are offsets into the caller's op matrix pool
// (SchedOp::mat), so the pool uploaded once per flush serves every pass.
#if !defined(__CUDACC_RTC__)
}  // namespace iqb
#include <vector>
namespace iqb {
struct PassPlan {
  PassDesc desc;
  int nsrc;              // number of scheduled ops
  double cost;           // planned arithmetic cost per amplitude
  std::vector<uint32_t> src;   // index of desc.ops[i]'s operation in the scheduled list
};
#endif

// Cost (real multiply-adds per amplitude) of applying an operation in a pass.
double op_cost(const SchedOp& op);

// ---- tile addressing, shared by the kernel and the CPU emulator in tests/ ----

// Amplitude index of element 0 of tile t: t's bits are spread over the
// non-tile bit positions (all bits except [0, c) and H).
IQ_HD uint64_t tile_base(uint64_t t, const PassDesc& P) {
  uint64_t x = t << P.c;
  for (int i = 0; i < P.nH; ++i) {
    const int h = P.H[i];
    x = ((x >> h) << (h + 1)) | (x & ((1ULL << h) - 1));
  }
  if (P.gap) x = ((x >> P.gap) << (P.gap + 1)) | (x & ((1ULL << P.gap) - 1));
  return x;
}

// Offset of TMA issue j inside a tile: issue j covers the tile bits H[nbox..].
IQ_HD uint64_t issue_offset(int j, const PassDesc& P) {
  uint64_t off = 0;
  const int nb = P.nH - P.nbox;
  for (int i = 0; i < nb; ++i)
    if ((j >> i) & 1) off |= 1ULL << P.H[P.nbox + i];
  return off;
}

// Shared-memory slot of tile-local amplitude j: the 128-byte TMA swizzle XORs
// bits 0..2 of the 16-byte unit index with bits 3..5.  The map is linear over
// XOR, so slot(a ^ b) = slot(a) ^ slot(b) for any two indices.
IQ_HD uint32_t swz(uint32_t j) { return j ^ ((j >> 3) & 7u); }

// 5-D view of the array used by the pass tensor map (dimension 0 innermost,
// counted in doubles; strides in bytes for dimensions 1..4).  The bits of the
// amplitude index are cut at the first two tile bits H[0], H[1]:
//   dim0 = 8 amplitudes (128 B, the swizzle span), dim1 = bits [3, H0),
//   dim2 = bit H0, dim3 = bits (H0, H1), dim4 = bits [H1, nbits).
// The box takes 2^(c-3) rows of dim1 (the rest of the 2^c chunk) and both
// values of H0 and H1, so one copy moves 2^(c + nbox) amplitudes; the other
// tile bits are enumerated by issues.
IQ_HD void pass_tmap_layout(const PassDesc& d, int nbits, uint64_t gd[5], uint64_t gs[4], uint32_t box[5]) {
  if (d.gap) nbits = d.gap + 1;   // the map covers the whole 2^(gap + 1) block of each array
  const int c = d.c;
  const uint64_t E = 16;
  const uint64_t top = (1ull << nbits) * E;
  gd[0] = 16;
  gs[0] = 8 * E;
  box[0] = 16;
  box[1] = 1u << (c - 3);
  const uint64_t sets = d.nsets > 1 ? d.nsets : 1;   // sets extend the top dimension
  if (d.nbox == 2) {
    const int h0 = d.H[0], h1 = d.H[1];
    gd[1] = 1ull << (h0 - 3); gd[2] = 2; gd[3] = 1ull << (h1 - h0 - 1); gd[4] = (1ull << (nbits - h1)) * sets;
    gs[1] = (1ull << h0) * E; gs[2] = (1ull << (h0 + 1)) * E; gs[3] = (1ull << h1) * E;
    box[2] = 2; box[3] = 1; box[4] = 2;
  } else if (d.nbox == 1) {
    const int h0 = d.H[0];
    gd[1] = 1ull << (h0 - 3); gd[2] = (1ull << (nbits - h0)) * sets; gd[3] = 1; gd[4] = 1;
    gs[1] = (1ull << h0) * E; gs[2] = top; gs[3] = top;
    box[2] = 2; box[3] = 1; box[4] = 1;
  } else {
    gd[1] = (1ull << (nbits - 3)) * sets; gd[2] = 1; gd[3] = 1; gd[4] = 1;
    gs[1] = top; gs[2] = top; gs[3] = top;
    box[2] = 1; box[3] = 1; box[4] = 1;
  }
}

// Tensor-map coordinates (dims 1..4) of the copy whose first amplitude is A
// (A has zeros in bits [0, c) and at the box bits).
IQ_HD void chunk_coords(uint64_t A, const PassDesc& P, int& c1, int& c2, int& c3, int& c4) {
  if (P.nbox == 2) {
    const int h0 = P.H[0], h1 = P.H[1];
    c1 = (int)((A >> 3) & ((1ULL << (h0 - 3)) - 1));
    c2 = 0;
    c3 = (int)((A >> (h0 + 1)) & ((1ULL << (h1 - h0 - 1)) - 1));
    c4 = (int)(A >> h1);
  } else if (P.nbox == 1) {
    const int h0 = P.H[0];
    c1 = (int)((A >> 3) & ((1ULL << (h0 - 3)) - 1));
    c2 = (int)(A >> h0);
    c3 = 0;
    c4 = 0;
  } else {
    c1 = (int)(A >> 3);
    c2 = c3 = c4 = 0;
  }
}

// Tensor-map coordinates of tile t's first copy, computed from t directly
// (equal to chunk_coords(tile_base(t, P), P)).  The tile index's bits fill the
// non-tile bit positions in order; cut at H[0] and H[1] they give: the low
// n1 = H0 - c bits -> dim 1 (above the chunk's 2^(c-3) rows), the next
// n3 = H1 - H0 - 1 bits -> dim 3, the rest -> the top dimension with the
// higher tile bits as zero gaps.  Built once per thread; 32-bit arithmetic.
struct TileCoordMap {
  int nbox;
  int n1, sh1;            // dim 1: (t & ((1 << n1) - 1)) << sh1
  int n3;                 // dim 3 (nbox 2): (t >> n1) & ((1 << n3) - 1)
  int shhi;               // top-dimension bits start at t >> shhi
  int ngap;
  uint8_t gap[kMaxTileBits + 1];   // ascending zero positions in the top coordinate
  int gap1;               // nbox 0: zero position in dim 1 (-1: none)
};

IQ_HD void tile_coord_map(const PassDesc& P, TileCoordMap& m) {
  m.nbox = P.nbox;
  m.ngap = 0;
  m.gap1 = -1;
  if (P.nbox == 0) {       // the chunk alone: dim 1 = A >> 3 = t << (c - 3)
    m.n1 = 31; m.sh1 = P.c - 3; m.n3 = 0; m.shhi = 31;
    if (P.gap) m.gap1 = P.gap - 3;
    return;
  }
  const int h0 = P.H[0];
  m.n1 = h0 - P.c;
  m.sh1 = P.c - 3;
  const int lo = (P.nbox == 2) ? P.H[1] : h0;   // the top dimension starts at this bit
  m.n3 = (P.nbox == 2) ? P.H[1] - h0 - 1 : 0;
  m.shhi = m.n1 + m.n3;
  m.gap[m.ngap++] = 0;                          // bit `lo` itself is a tile bit
  for (int i = P.nbox; i < P.nH; ++i) m.gap[m.ngap++] = (uint8_t)(P.H[i] - lo);
  if (P.gap) m.gap[m.ngap++] = (uint8_t)(P.gap - lo);   // above every tile bit: last
}

IQ_HD void tile_coords(uint32_t t, const TileCoordMap& m, int& c1, int& c2, int& c3, int& c4) {
  c1 = (int)((m.n1 >= 31 ? t : (t & ((1u << m.n1) - 1u))) << m.sh1);
  c2 = c3 = c4 = 0;
  if (m.nbox == 0) {
    if (m.gap1 >= 0) {
      const uint32_t u = (uint32_t)c1;
      c1 = (int)(((u >> m.gap1) << (m.gap1 + 1)) | (u & ((1u << m.gap1) - 1u)));
    }
    return;
  }
  uint32_t x = m.shhi >= 32 ? 0u : (t >> m.shhi);
  for (int i = 0; i < kMaxTileBits + 1; ++i)
    if (i < m.ngap) {
      const int g = m.gap[i];
      x = ((x >> g) << (g + 1)) | (x & ((1u << g) - 1u));
    }
  if (m.nbox == 2) {
    c3 = (int)((t >> m.n1) & ((1u << m.n3) - 1u));
    c4 = (int)x;
  } else {
    c2 = (int)x;
  }
}

}  // namespace iqb

#if defined(__cplusplus) && !defined(__CUDACC_RTC__)
#include <string>
#include <vector>
namespace iqb {
int plan_passes(const SchedParams& p, const std::vector<SchedOp>& ops, std::vector<PassPlan>& out,
                std::string& err);
// Source of the tile kernel specialised to pass `d` (iq_jitgen.cpp): stage
// layout, operations and matrix offsets fixed; tile bits, tile count and
// matrix values stay launch parameters.  Returns "" and sets `err` for a pass
// that is not specialised (adjoint steps, several parameter sets).
// min_blocks: resident CTAs per SM the kernel's register budget is sized for
// (launch bounds; 2 when out of 1..4; always 1 for R = 5); threads: CTA size
// (128 or 256; otherwise tile_pass_threads(R)).
// set_mode: the form for passes over several parameter sets and adjoint steps
// (matrices staged per set in shared memory, gradient accumulators; the
// interpreting kernel's launch arguments); otherwise matrices are a kernel
// parameter block.  narrow (with set_mode): the array is complex64 (float2);
// the first stage loads from and the last stores to global memory directly,
// widening to FP64, and the stages exchange through a float2 shared tile
// (arguments: pass, matrices, state, gradient partials; launched with
// jit_launch_narrow).
std::string jit_pass_source(const PassDesc& d, std::string& err, int min_blocks = 2, int threads = 0,
                            bool set_mode = false, bool narrow = false);
// Compact byte string of everything jit_pass_source's output depends on
// (equal keys give equal sources): the kernel cache's key.
std::string jit_pass_key(const PassDesc& d, int min_blocks, int threads, bool set_mode, bool narrow = false);
struct cplx64 { double re, im; };
// Fuse runs of queued operations on at most two qubits into single 4x4 blocks
// (a two-qubit operation absorbs the open one-qubit blocks of its qubits and
// later one-qubit operations on them), appending the fused matrices to `pool`.
// Operation order per qubit is preserved.  Returns the fused list.
// With monomial_barrier, two-qubit monomials (CX, CZ, SWAP: free renamings or
// phase products in the specialised kernels) are left alone and end the
// one-qubit runs of their qubits.
std::vector<SchedOp> fuse_two_qubit_blocks(const std::vector<SchedOp>& ops, std::vector<cplx64>& pool,
                                           bool monomial_barrier = false);
// Divide every dense one-qubit operation but the last of each run of at most
// kNormSegment by the larger of its row-0 entries (marking it `norm`), and
// multiply the run's last one by the product of those divisors: a scalar
// factor commutes with every operation, so the state after the run's last
// operation is unchanged, while each normalised operation costs 6 FMAs per
// amplitude instead of 8.  Runs are bounded so the scale of the intermediate
// state stays within (1/sqrt 2)^kNormSegment of the true one.
constexpr int kNormSegment = 256;
void normalize_one_qubit_ops(std::vector<SchedOp>& ops, std::vector<cplx64>& pool);
// Factor every unitary dense one-qubit operation as diag(d0, d1) R diag(1, e1)
// with R a real rotation (normalised: 2 FMAs per amplitude) and carry each
// qubit's pending output diagonal forward: through diagonal and permutation
// operations (a two-qubit monomial takes the pending diagonals of its qubits
// and passes on whatever factors per qubit; the rest becomes a phase on its
// |11> row), into the next dense operation on the qubit (columns scaled, no
// cost).  What cannot be carried is emitted as one-qubit phase operations
// diag(1, p) (2 FMAs per amplitude).  Scalars collect into runs of at most
// kNormSegment rotations, each ended by a scalar operation.  Non-unitary
// one-qubit matrices are left dense.
void decompose_one_qubit_ops(std::vector<SchedOp>& ops, std::vector<cplx64>& pool);
// Re-pack the matrix data each pass references (absolute offsets into `pool`)
// into one contiguous block per pass: sets desc.mat_base / mat_elems and makes
// every op's `mat` relative to its pass block, which the kernel stages in
// shared memory.
void pack_pass_matrices(std::vector<PassPlan>& plans, const cplx64* pool, std::vector<cplx64>& packed);

// ---- adjoint-method gradients ----------------------------------------------
// Gate kinds of a parametrised circuit (the values of the C ABI's IQ_GATE_*).
enum GateKind : int {
  GATE_RX = 1, GATE_RY = 2, GATE_RZ = 3, GATE_U3 = 4, GATE_P = 5,   // parametrised (U3 takes 3)
  GATE_CZ = 6, GATE_CX = 7, GATE_H = 8, GATE_X = 9, GATE_SX = 10    // fixed
};
struct AnsatzOp {
  int kind;
  int q0, q1;     // q1 only for CZ / CX (CX: q0 control, q1 target)
  int param;      // index of the (first) parameter, -1 for fixed gates
};
// Validate an ansatz; returns the number of parameters it reads (max index + 1) or -1.
int ansatz_check(int n, const std::vector<AnsatzOp>& ops, std::string& err);
// Forward circuit on an n-bit state vector: ops appended to `out` (matrices to `pool`).
// phase_free: RZ (and P) as diag(1, e^{i theta}), the global phase dropped.
void ansatz_forward(int n, const std::vector<AnsatzOp>& ops, const double* params, std::vector<SchedOp>& out,
                    std::vector<cplx64>& pool, bool phase_free = false);
// Backward sweep on the joint array of n + 1 bits (bit 0 selects psi (0) or
// lambda = H psi (1), bit q + 1 is qubit q): for every gate from last to first,
// an adjoint step (gradient term + inverse rotation) per rotation angle, or the
// inverse of a fixed gate.  grad_param[t] is the parameter gradient term t adds to.
// Z steps apply the phase-free form (GRAD_PHASE: no scale).  With `scaled`,
// X and Y steps apply the tan or cot form, dividing by the larger of |c| and
// |s|, and grad_scale[t] is the factor term t's accumulated value must be
// multiplied by (the square of the product of the divisors applied before
// it; 1 without `scaled`); a scalar operation restores the true scale
// whenever that product leaves [2^-64, 2^64].  The forms then depend on the
// angles, so `scaled` suits a parameter set that shares its plans with no other.
void ansatz_backward(int n, const std::vector<AnsatzOp>& ops, const double* params, std::vector<SchedOp>& out,
                     std::vector<cplx64>& pool, std::vector<int>& grad_param, int select_bit = 0,
                     bool scaled = false, std::vector<double>* grad_scale = nullptr);
// One parameter set's operation lists as the adjoint executor runs them.
// single_set: the forward goes through decompose_one_qubit_ops and
// normalize_one_qubit_ops (two-qubit monomials kept apart) and the backward
// is `scaled` -- structures that depend on the angles, for a set whose plans
// serve no other set; otherwise (fuse) runs of one- and two-qubit gates are
// fused into 4x4 blocks, a structure every set of the circuit shares.
struct AdjointOps {
  std::vector<SchedOp> fw, bw;
  std::vector<cplx64> fpool, bpool;
  std::vector<int> grad_param;
  std::vector<double> grad_scale;
};
void adjoint_ops(int n, const std::vector<AnsatzOp>& ops, const double* params, bool backward, bool fuse,
                 bool single_set, AdjointOps& j);
// The scale factors of a backward sweep's gradient terms in the order the
// operations run: the planner moves adjoint steps on different qubits past
// each other, so the scale each term sees is the product of the factors
// (SchedOp::smul) of the operations that run before it.  `plans` are the
// passes planned from `ops` (null: the operations run in list order); scale
// receives, per gradient term, the square of the scale it is accumulated at.
void exec_grad_scales(const std::vector<PassPlan>* plans, const std::vector<SchedOp>& ops, std::vector<double>& scale);
// Classify a 2^k x 2^k row-major matrix (interleaved re/im doubles): returns 1
// and fills perm/phases/unit if every row and column holds exactly one nonzero.
int classify_monomial(const double* m, int k, uint8_t* perm, double* phases, uint8_t* unit);
// OP_X2R's shape for a 4x4 row-major matrix (interleaved re/im doubles):
// 0 = not that shape, else XPAT_SHAPE plus XPAT_CORNERS_REAL / XPAT_MIDDLE_REAL.
int classify_xpattern(const double* m);
}  // namespace iqb
#endif
