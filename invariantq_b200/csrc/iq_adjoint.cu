// iq_adjoint.cu -- adjoint-method gradients of E(theta) = <psi(theta)|H|psi(theta)>
// for parametrised circuits (RX, RY, RZ, U3, P angles; H, X, SX, CZ, CX fixed
// gates), the batch executor that runs many circuits and parameter sets at
// once, and the plain forward-energy path the parameter-shift rule is built on.
//
// Method (Jones & Gacon, arXiv:2009.02823): psi = U_L..U_1 |0>, lambda = H psi;
// walking the gates backwards, each rotation exp(-i t P / 2) contributes
// dE/dt = Im <lambda|P|psi> and is then un-applied on both psi and lambda.
// Both vectors live in one joint array of 2^(n+1) amplitudes (bit 0 selects
// psi or lambda, bit q+1 is qubit q), so one tile pass un-applies a gate on
// both and reads both halves of a gradient term from the same registers
// (OP_GRAD2).  Un-applying a unitary in complex128 is exact to rounding, so
// the forward states are not stored: three state-sized buffers (psi, and the
// joint array of twice that) are all a job holds.
//
// Batch executor: one host worker thread per CUDA stream, each with its own
// device workspace sized for the largest circuit of the batch.  Workers take
// (circuit, parameter set) jobs from a shared counter, largest circuits first.
// Planning depends only on a circuit's structure, so it is done once per
// circuit (by the first worker that reaches it) and reused by every parameter
// set whose fused operation list has the same structure; a set whose angles
// change the structure (an angle that makes a fused block monomial) is
// planned on its own.  Host preparation of job j overlaps the GPU running job
// j-1 on the same stream (double-buffered pinned staging).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <map>
#include <unordered_map>
#include <vector>

#include "../../include/invariantq_b200.h"
#include "iq_c64.h"
#include "iq_jit.h"
#include "iq_kernels.h"
#include "iq_resident.h"
#include "iq_plan.h"

using namespace iqb;

namespace {

enum { E_ARG = 1, E_CUDA = 2, E_MEM = 3, E_STATE = 4, E_DEVICE = 5 };

int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return (v && *v) ? atoi(v) : dflt;
}
double env_double(const char* name, double dflt) {
  const char* v = getenv(name);
  return (v && *v) ? atof(v) : dflt;
}

struct Cfg {
  SchedParams sp{};
  TileLaunch tl{};
  int fuse = 1;
  int jit = 1;   // specialised kernels (iq_jit.cpp) for the forward and backward passes
  // complex64 states: every pass a specialised kernel that widens the loaded
  // amplitudes to FP64 and rounds to FP32 at its stage boundaries (jit_launch_narrow)
  bool c64 = false;
  // a circuit with one parameter set: forward and backward in the forms that
  // depend on its angles (fewer FP64 operations; adjoint_ops' single_set)
  bool single_forms = true;
  static Cfg from_env() {
    Cfg c;
    c.jit = env_int("IQ_ADJOINT_JIT", 1);
    // defaults: the state-vector path's specialised-kernel tile shape (2^12
    // amplitudes holding the 4 lowest index bits, 3 CTAs per SM with one tile
    // buffer each) and a budget of 200 (the adjoint autotuner's choice for the
    // batched-gradient workload)
    c.sp.M = env_int("IQ_TILE_BITS", 12);
    c.sp.c = env_int("IQ_CHUNK_BITS", 4);
    c.sp.R = std::min(5, std::max(3, env_int("IQ_SLOTS", 4)));
    c.sp.max_stages = env_int("IQ_MAX_STAGES", 8);
    c.sp.budget = env_double("IQ_ADJOINT_BUDGET", env_double("IQ_PASS_BUDGET", 200.0));
    c.sp.grad_cost = env_double("IQ_GRAD_COST", 6.0);
    c.tl.nbuf = env_int("IQ_NBUF", 1);
    c.tl.ctas_per_sm = env_int("IQ_CTAS_PER_SM", 3);
    c.tl.consumers = 128;
    c.fuse = env_int("IQ_FUSE", 1);
    c.single_forms = env_int("IQ_ADJOINT_SINGLE_FORMS", 1) != 0;
    return c;
  }
};

// -------------------------------------------------------------- Hamiltonian

// H = sum_t coeffs[t] P_t, P_t given by n characters (I, X, Y, Z; character q
// acts on qubit q), grouped by X part for the joint kernel.
struct Ham {
  HamTerms groups{};
  std::vector<uint64_t> zmask;
  std::vector<double2> coef;   // coeffs[t] * i^(number of Y)
};

bool build_ham(int n, size_t nterms, const double* coeffs, const char* paulis, Ham& h, std::string& err) {
  if (nterms == 0) { err = "the Hamiltonian has no terms"; return false; }
  std::vector<uint64_t> xs;
  std::vector<std::vector<size_t>> members;
  std::vector<uint64_t> tx(nterms), tz(nterms);
  std::vector<int> ty(nterms);
  for (size_t t = 0; t < nterms; ++t) {
    uint64_t xm = 0, zm = 0;
    int ny = 0;
    for (int q = 0; q < n; ++q) {
      const char ch = paulis[t * (size_t)n + q];
      if (ch == 'X') xm |= 1ULL << q;
      else if (ch == 'Y') { xm |= 1ULL << q; zm |= 1ULL << q; ++ny; }
      else if (ch == 'Z') zm |= 1ULL << q;
      else if (ch != 'I') { err = "Pauli strings take the characters I, X, Y, Z"; return false; }
    }
    tx[t] = xm; tz[t] = zm; ty[t] = ny;
    size_t g = 0;
    while (g < xs.size() && xs[g] != xm) ++g;
    if (g == xs.size()) {
      if ((int)xs.size() == kMaxHamGroups) { err = "more than 64 distinct X patterns in the Hamiltonian"; return false; }
      xs.push_back(xm);
      members.emplace_back();
    }
    members[g].push_back(t);
  }
  h.groups.ngroups = (int)xs.size();
  h.zmask.clear();
  h.coef.clear();
  static const double ire[4] = {1, 0, -1, 0}, iim[4] = {0, 1, 0, -1};
  for (size_t g = 0; g < xs.size(); ++g) {
    h.groups.xmask[g] = xs[g];
    h.groups.first[g] = (int)h.zmask.size();
    for (size_t t : members[g]) {
      h.zmask.push_back(tz[t]);
      const int p = ty[t] & 3;
      h.coef.push_back(make_double2(coeffs[t] * ire[p], coeffs[t] * iim[p]));
    }
  }
  h.groups.first[xs.size()] = (int)h.zmask.size();
  return true;
}

// ------------------------------------------------------------ planned shapes

// A planned operation list that depends only on the circuit's structure: the
// matrices of one parameter set are gathered into its per-pass blocks with
// `gather` (block[i] = pool[gather[i]]).
struct Shape {
  int nbits = 0;
  bool tiled = false;
  std::vector<PassPlan> plans;
  std::vector<SimpleOp> sops;
  std::vector<uint32_t> gather;
  std::vector<SchedOp> sig;
  size_t pool_size = 0;
  unsigned grid = 0;       // tile-pass grid (gradient partials row length)
  int ngrads = 0;
  std::vector<int> grad_param;
  std::vector<const JitKernel*> jit;   // specialised kernel per pass (null: interpreting kernel)
};

bool same_op(const SchedOp& a, const SchedOp& b) {
  if (a.k != b.k || a.mono != b.mono || a.perm != b.perm || a.unit != b.unit || a.mat != b.mat ||
      a.dense != b.dense || a.grad != b.grad || a.gen != b.gen || a.gidx != b.gidx || a.rot != b.rot ||
      a.norm != b.norm || a.urows != b.urows || a.xpat != b.xpat || a.realm != b.realm)
    return false;
  for (int i = 0; i < a.k; ++i)
    if (a.q[i] != b.q[i]) return false;
  return true;
}

bool matches(const Shape& s, const std::vector<SchedOp>& ops, size_t pool_size) {
  if (s.pool_size != pool_size || s.sig.size() != ops.size()) return false;
  for (size_t i = 0; i < ops.size(); ++i)
    if (!same_op(s.sig[i], ops[i])) return false;
  return true;
}

bool make_shape(const Cfg& cfg, int nbits, const std::vector<SchedOp>& fused, size_t pool_size, int num_sms,
                Shape& s, std::string& err) {
  s.nbits = nbits;
  s.sig = fused;
  s.pool_size = pool_size;
  s.tiled = nbits >= 7;
  s.gather.clear();
  if (!s.tiled) {
    for (const SchedOp& o : fused) {
      SimpleOp so{};
      so.k = o.k;
      for (int j = 0; j < o.k; ++j) so.q[j] = o.q[j];
      so.mat = (uint32_t)s.gather.size();
      const uint32_t d = 1u << o.k;
      for (uint32_t i = 0; i < d * d; ++i) s.gather.push_back(o.dense + i);
      s.sops.push_back(so);
    }
    return true;
  }
  SchedParams p = cfg.sp;
  p.nbits = nbits;
  int maxk = 1;
  for (const SchedOp& o : fused) maxk = std::max<int>(maxk, o.k);
  p.R = std::min(5, std::max(cfg.sp.R, maxk));
  if (plan_passes(p, fused, s.plans, err) < 0) return false;
  std::vector<cplx64> idx(pool_size), packed;
  for (size_t i = 0; i < pool_size; ++i) idx[i] = {(double)i, 0.0};
  pack_pass_matrices(s.plans, idx.data(), packed);
  s.gather.resize(packed.size());
  for (size_t i = 0; i < packed.size(); ++i) s.gather[i] = (uint32_t)packed[i].re;
  for (const PassPlan& pl : s.plans)
    if (pl.desc.mat_elems > (uint32_t)kSmemMatElems) {
      err = "a pass's matrices exceed the shared-memory block";
      return false;
    }
  s.grid = 0;
  for (const PassPlan& pl : s.plans) {
    const unsigned g = tile_pass_grid(pl.desc, cfg.tl, num_sms);
    if (pl.desc.ngrad) {
      if (s.grid && g != s.grid) { err = "gradient passes with different grids"; return false; }
      s.grid = g;
    }
  }
  if (cfg.jit || cfg.c64) {   // kernels specialised to the passes (shared by every circuit with the same pass structure)
    std::vector<const PassDesc*> ds;
    for (const PassPlan& pl : s.plans) ds.push_back(&pl.desc);
    std::string jerr;
    if (!jit_prepare(ds, s.jit, jerr, cfg.tl.ctas_per_sm, 0, true, cfg.c64)) s.jit.clear();
    if (cfg.c64) {
      bool all = s.jit.size() == s.plans.size();
      for (const JitKernel* k : s.jit) all = all && k;
      if (!all) {
        err = "complex64 passes need run-time compiled kernels: " + (jerr.empty() ? std::string("kernel cache full") : jerr);
        return false;
      }
    }
  }
  return true;
}

// ---------------------------------------------------------------- circuits

struct Circuit {
  int n = 0;
  std::vector<AnsatzOp> ops;
  int nparams = 0;             // columns of the parameter matrix
  size_t nsets = 0;
  const double* params = nullptr;
  Ham ham;
  double* energy_out = nullptr;
  double* grad_out = nullptr;
  // structure plans of the first parameter set, built by the first worker to reach the circuit
  std::mutex mu;
  bool planned = false;
  std::string plan_err;
  std::unique_ptr<Shape> fw, bw;
};

// fused forward / backward operation lists and matrix pools of one parameter
// set.  A circuit with a single parameter set takes the angle-dependent forms
// (rotation + phase forward, scaled adjoint steps: adjoint_ops' single_set):
// its plans serve no other set.
using JobOps = AdjointOps;

void job_ops(const Cfg& cfg, const Circuit& c, const double* theta, bool backward, JobOps& j) {
  adjoint_ops(c.n, c.ops, theta, backward, cfg.fuse != 0, cfg.single_forms && c.nsets == 1, j);
}

int joint_bits(int n) { return std::max(n + 1, 7); }

// ---------------------------------------------------------------- workspace

struct Stats {
  std::atomic<uint64_t> jobs{0}, fw_passes{0}, bw_passes{0}, launches{0}, replans{0}, jit_passes{0};
  std::atomic<uint64_t> bytes{0};           // algorithmic HBM bytes of the passes
  std::atomic<uint64_t> host_ns{0};
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  // grow to n elements; `user` (the stream that reads the buffer) is drained before the old one is freed
  // (growth doubles: allocation calls synchronise the whole device)
  bool ensure(size_t n, std::string& err, const char* what, cudaStream_t user = nullptr) {
    if (n <= cap) return true;
    if (p && user) cudaStreamSynchronize(user);
    if (p) cudaFree(p);
    n = std::max(n, 2 * cap);
    p = nullptr;
    cap = 0;
    if (cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      err = std::string("cannot allocate device memory for ") + what;
      return false;
    }
    cap = n;
    return true;
  }
  void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

template <class T>
struct HostBuf {
  T* p = nullptr;
  size_t cap = 0;
  bool ensure(size_t n, std::string& err) {
    if (n <= cap) return true;
    if (p) cudaFreeHost(p);
    n = std::max(n, 2 * cap);
    p = nullptr;
    cap = 0;
    if (cudaMallocHost(&p, std::max<size_t>(n, 1) * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      err = "cannot allocate pinned host memory";
      return false;
    }
    cap = n;
    return true;
  }
  void release() { if (p) cudaFreeHost(p); p = nullptr; cap = 0; }
};

// results of one job waiting for its stream to reach them
struct Pending {
  bool active = false;
  Circuit* c = nullptr;
  std::vector<size_t> sets;   // parameter sets in launch order (device set k = sets[k])
  std::vector<int> grad_param;
  std::vector<double> grad_scale;   // per set, ngrads factors of the scaled adjoint steps (empty: all 1)
  int ngrads = 0;
  bool grad = false;
};

struct Workspace {
  int device = 0, num_sms = 148;
  cudaStream_t stream = nullptr;
  DevBuf<double2> psi, joint, mats, coef;
  DevBuf<double> red, gpart, gsum;
  DevBuf<uint64_t> zmask;
  DevBuf<int> status;
  HostBuf<double2> hmats[2];
  HostBuf<double> hout[2];    // energies of the job's sets, then their gradient terms
  HostBuf<int> hstat[2];      // device status word
  cudaEvent_t ev[2] = {nullptr, nullptr};
  Pending pend[2];
  int slot = 0;
  std::map<std::tuple<const Shape*, uint32_t, int>, std::vector<CUtensorMap>> tmaps;   // (shape, sets, gap)
  const Circuit* ham_of = nullptr;   // circuit whose Hamiltonian tables are on the device

  // The state arrays are sized up front for the batch's largest job; matrix,
  // partial and staging buffers grow on demand (doubling, so a worker
  // reallocates a few times at the start: the largest jobs run first).
  struct Bounds {
    uint64_t psi_amps = 1, joint_amps = 1;
    size_t mats = 1, sets = 1, grads = 1;   // per job: matrix elements, sets, gradient terms x sets
  };

  // Make ready for a call on device `dev` (a workspace can come back from the
  // pool of an earlier call: pointers into that call's shapes and circuits are
  // dropped, buffers are kept when large enough).
  bool prepare(int dev, int sms, const Bounds& bd, std::string& err) {
    if (!stream) {
      device = dev;
      num_sms = sms;
      if (cudaSetDevice(dev) != cudaSuccess ||
          cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking) != cudaSuccess ||
          cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        err = "cannot create a CUDA stream or event";
        return false;
      }
    } else if (cudaSetDevice(dev) != cudaSuccess) {
      cudaGetLastError();
      err = "cudaSetDevice failed";
      return false;
    }
    tmaps.clear();
    ham_of = nullptr;
    slot = 0;
    pend[0].active = pend[1].active = false;
    if (!psi.ensure(bd.psi_amps, err, "the states", stream) ||
        !joint.ensure(bd.joint_amps, err, "the joint arrays", stream) || !status.ensure(1, err, "the status word") ||
        !red.ensure(bd.sets * (kRedBlocks + 1), err, "reduction partials", stream))
      return false;
    return cudaMemsetAsync(status.p, 0, sizeof(int), stream) == cudaSuccess;
  }

  double device_bytes() const {
    return 16.0 * ((double)psi.cap + (double)joint.cap + (double)mats.cap) +
           8.0 * ((double)red.cap + (double)gpart.cap + (double)gsum.cap);
  }

  void release() {
    if (stream) cudaStreamSynchronize(stream);
    psi.release(); joint.release(); mats.release(); coef.release(); red.release(); gpart.release(); gsum.release();
    zmask.release(); status.release();
    for (int i = 0; i < 2; ++i) {
      hmats[i].release();
      hout[i].release();
      hstat[i].release();
      if (ev[i]) cudaEventDestroy(ev[i]);
      ev[i] = nullptr;
    }
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }

  // Tensor maps of a shape's passes over `nsets` arrays at `base`.  Circuit
  // shapes live for the whole call and are cached; a job's private shape is
  // encoded into `scratch` (its address may be reused by a later shape).
  const std::vector<CUtensorMap>* maps_for(const Shape& s, double2* base, uint32_t nsets, int gap, bool cache,
                                           std::vector<CUtensorMap>& scratch, std::string& err) {
    const auto key = std::make_tuple(&s, nsets, gap);
    if (cache) {
      auto it = tmaps.find(key);
      if (it != tmaps.end()) return &it->second;
    }
    std::vector<CUtensorMap> v(s.plans.size());
    char emsg[256];
    for (size_t i = 0; i < s.plans.size(); ++i) {
      PassDesc d = s.plans[i].desc;
      d.nsets = nsets;
      d.gap = (uint8_t)gap;
      if (encode_pass_tmap(&v[i], base, s.nbits, d, emsg, sizeof(emsg)) != 0) {
        err = emsg;
        return nullptr;
      }
    }
    if (!cache) {
      scratch = std::move(v);
      return &scratch;
    }
    return &tmaps.emplace(key, std::move(v)).first->second;
  }
};

bool cuda_ok(cudaError_t e, const char* what, std::string& err) {
  if (e == cudaSuccess) return true;
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

int log2_u64(uint64_t x) {
  int r = 0;
  while ((1ULL << r) < x) ++r;
  return r;
}

// Launch a shape's passes over `nsets` arrays of 2^nbits amplitudes at `state`
// (set s's matrices at mats + s * mat_stride; gradient rows per set:
// grad_stride).  set_stride: amplitudes from one array to the next (0: the
// arrays lie end to end).  Tile passes take any stride of 2^(nbits + 1) as
// the gap bit nbits (the arrays are the lower halves of [psi | lambda] blocks).
// Returns the tile-pass grid of the launches in *grid.
bool run_shape(Workspace& w, const Cfg& cfg, const Shape& s, bool cached, double2* state, uint32_t nsets,
               const double2* mats, uint32_t mat_stride, double* gpart, uint32_t grad_stride, unsigned* grid,
               Stats& st, std::string& err, uint64_t set_stride = 0) {
  const uint64_t dim = 1ULL << s.nbits;
  const uint64_t stride = set_stride ? set_stride : dim;
  if (cfg.c64 && !s.tiled) { err = "complex64 gradients need tile passes (at least 7 qubits)"; return false; }
  int gap = 0;
  if (s.tiled && stride != dim) {
    if (stride != 2 * dim) { err = "internal: tile passes over arrays spaced other than 2^(n+1) apart"; return false; }
    gap = s.nbits;
  }
  if (!s.tiled) {
    for (uint32_t k = 0; k < nsets; ++k)
      for (const SimpleOp& so : s.sops)
        if (!cuda_ok(launch_simple_op(state + k * stride, s.nbits, so, mats + (size_t)k * mat_stride, w.stream),
                     "gate kernel", err))
          return false;
    st.launches += s.sops.size() * nsets;
    st.bytes += (uint64_t)s.sops.size() * nsets * (32ULL << s.nbits);
    return true;
  }
  if (cfg.c64) {   // complex64: direct loads and stores, no tensor maps
    for (size_t i = 0; i < s.plans.size(); ++i) {
      PassDesc d = s.plans[i].desc;
      d.gap = (uint8_t)gap;
      d.set_shift = (uint32_t)log2_u64(d.ntiles);
      d.ntiles *= nsets;
      d.nsets = nsets;
      d.set_mat_stride = mat_stride;
      d.grad_stride = grad_stride;
      if (grid) *grid = tile_pass_grid(d, cfg.tl, w.num_sms);
      if (!cuda_ok(jit_launch_narrow(s.jit[i], d, mats, state, cfg.tl, w.num_sms, w.stream, gpart),
                   "complex64 pass kernel", err))
        return false;
      ++st.jit_passes;
    }
    st.launches += s.plans.size();
    st.bytes += (uint64_t)s.plans.size() * nsets * (16ULL << s.nbits);
    return true;
  }
  std::vector<CUtensorMap> scratch;
  const std::vector<CUtensorMap>* tm = w.maps_for(s, state, nsets, gap, cached, scratch, err);
  if (!tm) return false;
  for (size_t i = 0; i < s.plans.size(); ++i) {
    PassDesc d = s.plans[i].desc;
    d.gap = (uint8_t)gap;
    d.set_shift = (uint32_t)log2_u64(d.ntiles);
    d.ntiles *= nsets;
    d.nsets = nsets;
    d.set_mat_stride = mat_stride;
    d.grad_stride = grad_stride;
    if (grid) *grid = tile_pass_grid(d, cfg.tl, w.num_sms);
    if (i < s.jit.size() && s.jit[i]) {
      if (!cuda_ok(jit_launch_sets(s.jit[i], (*tm)[i], d, mats, w.status.p, cfg.tl, w.num_sms, w.stream, gpart),
                   "specialised tile pass kernel", err))
        return false;
      ++st.jit_passes;
    } else if (!cuda_ok(launch_tile_pass((*tm)[i], d, mats, w.status.p, cfg.tl, w.num_sms, w.stream, gpart),
                        "tile pass kernel", err)) {
      return false;
    }
  }
  st.launches += s.plans.size();
  st.bytes += (uint64_t)s.plans.size() * nsets * (32ULL << s.nbits);
  return true;
}

// Finish the job that used staging slot `k`: wait for its stream, check the
// status word, write energies and gradients.
bool finish(Workspace& w, int k, std::string& err) {
  Pending& p = w.pend[k];
  if (!p.active) return true;
  p.active = false;
  if (!cuda_ok(cudaEventSynchronize(w.ev[k]), "stream sync", err)) return false;
  const double* out = w.hout[k].p;
  const int status = w.hstat[k].p[0];
  if (status != 0) {
    char m[160];
    snprintf(m, sizeof(m), "a tile pass timed out waiting for %s (status %d); the results are invalid",
             status == DEV_WAIT_LOADED ? "a tile load" : "its consumers", status);
    err = m;
    cudaMemsetAsync(w.status.p, 0, sizeof(int), w.stream);
    return false;
  }
  Circuit& c = *p.c;
  const size_t S = p.sets.size();
  for (size_t j = 0; j < S; ++j) {
    const size_t set = p.sets[j];
    if (c.energy_out) c.energy_out[set] = out[j];
    if (p.grad && c.grad_out) {
      double* g = c.grad_out + set * (size_t)c.nparams;
      for (int i = 0; i < c.nparams; ++i) g[i] = 0.0;
      const double* row = out + S + j * (size_t)p.ngrads;
      if (p.grad_scale.empty()) {
        for (int t = 0; t < p.ngrads; ++t) g[p.grad_param[t]] += row[t];
      } else {
        const double* sc = p.grad_scale.data() + j * (size_t)p.ngrads;
        for (int t = 0; t < p.ngrads; ++t) g[p.grad_param[t]] += row[t] * sc[t];
      }
    }
  }
  return true;
}

// Launch the parameter sets `sets` of circuit c together on the workspace's
// stream, all through the shapes fw / bw (their fused operation lists match
// every set's).  want_grad = false: forward and energy only.
bool launch_sets(Workspace& w, const Cfg& cfg, Circuit& c, const std::vector<size_t>& sets, std::vector<JobOps>& jo,
                 const Shape* fw, bool fw_cached, const Shape* bw, bool bw_cached, bool want_grad, Stats& st,
                 std::string& err) {
  const uint32_t S = (uint32_t)sets.size();
  const int ngrads = want_grad ? (int)jo[0].grad_param.size() : 0;
  // staging slot: wait for the job that used it last
  const int k = w.slot;
  w.slot ^= 1;
  if (!finish(w, k, err)) return false;
  const size_t nf = fw->gather.size(), nb = want_grad ? bw->gather.size() : 0;
  const size_t per = nf + nb;
  if (!w.hmats[k].ensure(per * S, err) || !w.hout[k].ensure(S + (size_t)S * ngrads, err) || !w.hstat[k].ensure(1, err))
    return false;
  double2* hm = w.hmats[k].p;
  const auto tg = std::chrono::steady_clock::now();
  for (uint32_t j = 0; j < S; ++j) {
    const JobOps& o = jo[j];
    double2* f = hm + (size_t)j * nf;
    for (size_t i = 0; i < nf; ++i) f[i] = make_double2(o.fpool[fw->gather[i]].re, o.fpool[fw->gather[i]].im);
    double2* b = hm + (size_t)S * nf + (size_t)j * nb;
    for (size_t i = 0; i < nb; ++i) b[i] = make_double2(o.bpool[bw->gather[i]].re, o.bpool[bw->gather[i]].im);
  }
  st.host_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - tg)
                    .count();
  const uint64_t dim = 1ULL << c.n;
  const int nj = joint_bits(c.n);
  const uint64_t jdim = 1ULL << nj;
  // device buffers (a buffer that grows waits for the stream's earlier work first);
  // tensor maps hold the state buffers' addresses, so they are dropped if one moves
  const double2* psi0 = w.psi.p;
  const double2* joint0 = w.joint.p;
  if (!w.mats.ensure(2 * per * S, err, "matrices", w.stream) ||
      !w.red.ensure((size_t)S * (kRedBlocks + 1), err, "reduction partials", w.stream) ||
      (!want_grad && !w.psi.ensure(dim * S, err, "the states", w.stream)))
    return false;
  const unsigned max_grid = (unsigned)w.num_sms * (unsigned)std::max(1, cfg.tl.ctas_per_sm);
  // complex64 joint arrays take half the bytes (the buffer counts complex128 units)
  const uint64_t joint_units = cfg.c64 ? (jdim * S + 1) / 2 : jdim * S;
  if (want_grad && (!w.joint.ensure(joint_units, err, "the joint arrays", w.stream) ||
                    !w.gpart.ensure((size_t)std::max(ngrads, 1) * S * max_grid, err, "gradient partials", w.stream) ||
                    !w.gsum.ensure((size_t)std::max(ngrads, 1) * S, err, "gradient sums", w.stream)))
    return false;
  if (w.psi.p != psi0 || w.joint.p != joint0) w.tmaps.clear();
  if (w.ham_of != &c) {
    if (!w.zmask.ensure(c.ham.zmask.size(), err, "Hamiltonian", w.stream) ||
        !w.coef.ensure(c.ham.coef.size(), err, "Hamiltonian", w.stream))
      return false;
    // copies from pageable memory: staged before cudaMemcpyAsync returns
    if (!cuda_ok(cudaMemcpyAsync(w.zmask.p, c.ham.zmask.data(), c.ham.zmask.size() * 8, cudaMemcpyHostToDevice, w.stream),
                 "H2D Hamiltonian", err) ||
        !cuda_ok(cudaMemcpyAsync(w.coef.p, c.ham.coef.data(), c.ham.coef.size() * 16, cudaMemcpyHostToDevice, w.stream),
                 "H2D Hamiltonian", err))
      return false;
    w.ham_of = &c;
  }
  // matrices go to the half of the device buffer this slot owns, so the copy for
  // the next job cannot overwrite matrices this job's passes still read
  double2* dm = w.mats.p + (size_t)k * (w.mats.cap / 2);
  if (!cuda_ok(cudaMemcpyAsync(dm, hm, per * S * sizeof(double2), cudaMemcpyHostToDevice, w.stream), "H2D matrices",
               err))
    return false;

  double* partials = w.red.p;
  double* energy_dev = w.red.p + (size_t)S * kRedBlocks;
  if (!want_grad) {
    // forward from |0> for every set on the state buffer, then the energies
    if (!cuda_ok(launch_set_basis_sets(w.psi.p, dim, (int)S, w.stream), "reset", err)) return false;
    if (!run_shape(w, cfg, *fw, fw_cached, w.psi.p, S, dm, (uint32_t)nf, nullptr, 0, nullptr, st, err)) return false;
    st.fw_passes += (fw->tiled ? fw->plans.size() : fw->sops.size()) * S;
    if (!cuda_ok(launch_hamiltonian_joint(w.psi.p, dim, c.n, (int)S, c.ham.groups, w.zmask.p, w.coef.p, nullptr, 0,
                                          partials, energy_dev, w.stream),
                 "energy kernel", err))
      return false;
    st.launches += 3;
    st.bytes += S * 16ULL * dim;   // read psi
  } else {
    // Each set's joint array is [psi | lambda] (select bit n; small circuits
    // zero-padded to 2^7): the forward runs on the psi half in place, lambda =
    // H psi is written to the other half, and the backward sweep runs on the
    // whole array -- two state-sized buffers per set, no copy of psi.
    float2* J64 = reinterpret_cast<float2*>(w.joint.p);   // the complex64 view (cfg.c64)
    if (cfg.c64 ? !cuda_ok(launch_init_joint_c64(J64, c.n, jdim, (int)S, w.stream), "reset", err)
                : !cuda_ok(launch_init_joint(w.joint.p, c.n, jdim, (int)S, w.stream), "reset", err))
      return false;
    if (!run_shape(w, cfg, *fw, fw_cached, w.joint.p, S, dm, (uint32_t)nf, nullptr, 0, nullptr, st, err, jdim))
      return false;
    st.fw_passes += (fw->tiled ? fw->plans.size() : fw->sops.size()) * S;
    if (cfg.c64 ? !cuda_ok(launch_hamiltonian_c64(J64, jdim, c.n, (int)S, c.ham.groups, w.zmask.p, w.coef.p, J64 + dim,
                                                  jdim, partials, energy_dev, w.stream),
                           "Hamiltonian kernel", err)
                : !cuda_ok(launch_hamiltonian_joint(w.joint.p, jdim, c.n, (int)S, c.ham.groups, w.zmask.p, w.coef.p,
                                                    w.joint.p + dim, jdim, partials, energy_dev, w.stream),
                           "Hamiltonian kernel", err))
      return false;
    unsigned grid = 0;
    // partials of the sets a CTA never reaches stay zero
    if (ngrads && !cuda_ok(cudaMemsetAsync(w.gpart.p, 0, (size_t)ngrads * S * max_grid * sizeof(double), w.stream),
                           "memset", err))
      return false;
    if (!run_shape(w, cfg, *bw, bw_cached, w.joint.p, S, dm + (size_t)S * nf, (uint32_t)nb, w.gpart.p,
                   (uint32_t)ngrads, &grid, st, err))
      return false;
    st.bw_passes += (bw->tiled ? bw->plans.size() : bw->sops.size()) * S;
    if (ngrads && grid == 0) { err = "internal: no gradient pass"; return false; }
    if (!cuda_ok(launch_row_sums(w.gpart.p, ngrads * (int)S, (int)grid, w.gsum.p, w.stream), "gradient sums", err))
      return false;
    st.launches += 6;
    st.bytes += S * (cfg.c64 ? 16ULL : 32ULL) * dim;   // read psi, write lambda
  }
  double* ho = w.hout[k].p;
  if (!cuda_ok(cudaMemcpyAsync(ho, energy_dev, S * sizeof(double), cudaMemcpyDeviceToHost, w.stream), "D2H", err) ||
      !cuda_ok(cudaMemcpyAsync(w.hstat[k].p, w.status.p, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H", err))
    return false;
  if (ngrads && !cuda_ok(cudaMemcpyAsync(ho + S, w.gsum.p, (size_t)S * ngrads * sizeof(double), cudaMemcpyDeviceToHost,
                                         w.stream),
                         "D2H", err))
    return false;
  if (!cuda_ok(cudaEventRecord(w.ev[k], w.stream), "event", err)) return false;
  Pending& p = w.pend[k];
  p.active = true;
  p.c = &c;
  p.sets = sets;
  p.grad = want_grad;
  p.ngrads = ngrads;
  p.grad_param = want_grad ? jo[0].grad_param : std::vector<int>();
  p.grad_scale.clear();
  bool unit_scales = true;
  for (uint32_t j = 0; j < S && want_grad; ++j)
    for (double f : jo[j].grad_scale) unit_scales = unit_scales && f == 1.0;
  if (!unit_scales)   // scaled adjoint steps: each term's scale in the order the backward passes run them
    for (uint32_t j = 0; j < S; ++j) {
      std::vector<double> sc;
      exec_grad_scales(bw->tiled ? &bw->plans : nullptr, jo[j].bw, sc);
      if ((int)sc.size() != ngrads) { err = "internal: gradient scales"; return false; }
      p.grad_scale.insert(p.grad_scale.end(), sc.begin(), sc.end());
    }
  st.jobs += S;
  return true;
}

// Prepare and launch the parameter sets [set0, set0 + nsets) of circuit c:
// the sets whose fused operation lists match the circuit's plans run together;
// any other set runs alone with plans of its own.
bool launch_job(Workspace& w, const Cfg& cfg, Circuit& c, size_t set0, size_t nsets, bool want_grad, Stats& st,
                std::string& err) {
  // host preparation (st.host_ns): building the operation lists, planning a
  // structure the first time, matching the sets against it and staging their
  // matrices -- CPU work only, not the CUDA calls (which may wait for the stream)
  auto since = [](std::chrono::steady_clock::time_point a) {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now() - a).count();
  };
  auto t0 = std::chrono::steady_clock::now();
  std::vector<JobOps> jo(nsets);
  for (size_t j = 0; j < nsets; ++j) job_ops(cfg, c, c.params + (set0 + j) * (size_t)c.nparams, want_grad, jo[j]);
  st.host_ns += since(t0);
  {
    std::lock_guard<std::mutex> g(c.mu);
    t0 = std::chrono::steady_clock::now();
    if (!c.planned) {
      c.planned = true;
      c.fw.reset(new Shape);
      if (!make_shape(cfg, c.n, jo[0].fw, jo[0].fpool.size(), w.num_sms, *c.fw, c.plan_err)) c.fw.reset();
      if (c.fw && want_grad) {
        c.bw.reset(new Shape);
        if (!make_shape(cfg, joint_bits(c.n), jo[0].bw, jo[0].bpool.size(), w.num_sms, *c.bw, c.plan_err)) c.bw.reset();
        else c.bw->ngrads = (int)jo[0].grad_param.size();
      }
    }
    st.host_ns += since(t0);
    if (!c.fw || (want_grad && !c.bw)) {
      err = "scheduler: " + c.plan_err;
      return false;
    }
  }
  t0 = std::chrono::steady_clock::now();
  std::vector<size_t> same, other;
  std::vector<JobOps> jsame;
  for (size_t j = 0; j < nsets; ++j) {
    const bool ok = matches(*c.fw, jo[j].fw, jo[j].fpool.size()) &&
                    (!want_grad || matches(*c.bw, jo[j].bw, jo[j].bpool.size()));
    if (ok) {
      same.push_back(set0 + j);
      jsame.push_back(std::move(jo[j]));
    } else {
      other.push_back(j);
    }
  }
  st.host_ns += since(t0);
  if (!same.empty() && !launch_sets(w, cfg, c, same, jsame, c.fw.get(), true, c.bw.get(), true, want_grad, st, err))
    return false;
  for (size_t j : other) {   // a set whose angles change the fused structure
    t0 = std::chrono::steady_clock::now();
    std::unique_ptr<Shape> own_fw(new Shape), own_bw;
    if (!make_shape(cfg, c.n, jo[j].fw, jo[j].fpool.size(), w.num_sms, *own_fw, err)) return false;
    if (want_grad) {
      own_bw.reset(new Shape);
      if (!make_shape(cfg, joint_bits(c.n), jo[j].bw, jo[j].bpool.size(), w.num_sms, *own_bw, err)) return false;
      own_bw->ngrads = (int)jo[j].grad_param.size();
    }
    st.host_ns += since(t0);
    ++st.replans;
    std::vector<JobOps> one(1);
    one[0] = std::move(jo[j]);
    if (!launch_sets(w, cfg, c, {set0 + j}, one, own_fw.get(), false, own_bw.get(), false, want_grad, st, err))
      return false;
  }
  return true;
}

int current_device(std::string& err) {
  int dev = env_int("IQ_CUDA_DEVICE", -1);
  if (dev >= 0) {
    if (cudaSetDevice(dev) != cudaSuccess) { cudaGetLastError(); err = "cudaSetDevice failed"; return -1; }
  } else if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    err = "no CUDA device";
    return -1;
  }
  int cc = 0;
  cudaDeviceGetAttribute(&cc, cudaDevAttrComputeCapabilityMajor, dev);
  if (cc < 10) { err = "this library is built for sm_100a"; return -1; }
  return dev;
}

thread_local double t_stats[10] = {0};

// Workspaces kept between calls (streams, events and buffers are costly to
// create and allocation synchronises the device).  A workspace holding more
// than kPoolKeepBytes of device memory is freed at the end of its call;
// iq_adjoint_release frees the rest.  Never freed at process exit.
constexpr double kPoolKeepBytes = 8.0 * (1ull << 30);
std::mutex g_pool_mu;
std::vector<Workspace*>* g_pool = new std::vector<Workspace*>();

Workspace* pool_take(int dev) {
  std::lock_guard<std::mutex> g(g_pool_mu);
  for (size_t i = 0; i < g_pool->size(); ++i)
    if ((*g_pool)[i]->device == dev) {
      Workspace* w = (*g_pool)[i];
      g_pool->erase(g_pool->begin() + i);
      return w;
    }
  return new Workspace();
}

void pool_give(Workspace* w, bool ok) {
  if (!ok || w->device_bytes() > kPoolKeepBytes) {
    w->release();
    delete w;
    return;
  }
  cudaStreamSynchronize(w->stream);
  std::lock_guard<std::mutex> g(g_pool_mu);
  g_pool->push_back(w);
}

// Run all jobs of `circs` (every parameter set of every circuit) on `nstreams` workers.
int run_batch(std::vector<std::unique_ptr<Circuit>>& circs, int nstreams, bool want_grad, bool c64 = false) {
  const auto t0 = std::chrono::steady_clock::now();
  std::string err;
  const int dev = current_device(err);
  if (dev < 0) { record_error(E_DEVICE, err.c_str()); return -1; }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  Cfg cfg = Cfg::from_env();
  cfg.c64 = c64;
  if (c64) {
    // complex64 passes keep a float2 tile (32 KiB at 2^12 amplitudes): four
    // CTAs fit per SM, whose extra warps hide the direct global loads (30
    // qubits: 1.99 s against 2.13 s with three)
    cfg.sp.M = env_int("IQ_C64_TILE_BITS", cfg.sp.M);
    cfg.tl.ctas_per_sm = env_int("IQ_C64_CTAS_PER_SM", 4);
  }
  // jobs: a circuit's parameter sets in groups whose joint arrays ([psi |
  // lambda], 32 B x 2^n per set) fit the per-job budget; the energy-only path
  // (the plain baseline) runs one set per job on a state buffer (16 B x 2^n)
  struct Job { Circuit* c; size_t set0, nsets; double cost; };
  std::vector<Job> jobs;
  const double job_bytes = env_double("IQ_ADJOINT_JOB_BYTES", 4.0 * (1ull << 30));
  Workspace::Bounds bd;
  // circuits whose psi and lambda fit one CTA's shared memory go to the
  // persistent executor (iq_resident.cu), all their sets in one launch
  const int res_max = (want_grad && !c64)
                          ? std::min(env_int("IQ_RESIDENT_MAX_QUBITS", kResidentMaxQubits), kResidentMaxQubits)
                          : 0;
  std::vector<ResidentJob> rjobs;
  size_t resident_sets = 0;
  for (auto& c : circs) {
    if (c->n <= res_max && c->nparams <= kResidentMaxParams && c->nsets > 0) {
      ResidentJob r;
      r.n = c->n;
      r.ops = &c->ops;
      r.nparams = c->nparams;
      r.nsets = c->nsets;
      r.params = c->params;
      r.groups = &c->ham.groups;
      r.zmask = &c->ham.zmask;
      r.coef = &c->ham.coef;
      r.energy_out = c->energy_out;
      r.grad_out = c->grad_out;
      rjobs.push_back(r);
      resident_sets += c->nsets;
      continue;
    }
    const double per_set = (c64 ? 8.0 : 16.0) * std::ldexp(1.0, joint_bits(c->n));
    const size_t group = want_grad ? (size_t)std::max(1.0, std::floor(job_bytes / per_set)) : 1;
    // per set: at most 3 rotations per gate, each at most a dense 4x4 (16
    // elements) forward and one backward; at most 3 gradient terms per gate
    const size_t nops = c->ops.size() + 1;
    for (size_t s0 = 0; s0 < c->nsets; s0 += group) {
      const size_t ns = std::min(group, c->nsets - s0);
      jobs.push_back({c.get(), s0, ns, (double)ns * std::ldexp((double)nops, c->n)});
      if (!want_grad) bd.psi_amps = std::max<uint64_t>(bd.psi_amps, (uint64_t)ns << c->n);
      if (want_grad)
        bd.joint_amps = std::max<uint64_t>(bd.joint_amps, ((uint64_t)ns << joint_bits(c->n)) >> (c64 ? 1 : 0));
      bd.mats = std::max(bd.mats, ns * 96 * nops);
      bd.sets = std::max(bd.sets, ns);
      if (want_grad) bd.grads = std::max(bd.grads, ns * 3 * nops);
    }
  }
  std::string res_err;
  bool res_ok = true;
  // the persistent launch runs beside the workers' tile passes
  std::thread res_thread;
  if (!rjobs.empty()) res_thread = std::thread([&] {
    cudaSetDevice(dev);
    res_ok = resident_run(dev, rjobs, res_err);
  });
  struct JoinRes {
    std::thread& t;
    ~JoinRes() { if (t.joinable()) t.join(); }
  } join_res{res_thread};
  // largest first
  std::stable_sort(jobs.begin(), jobs.end(), [](const Job& a, const Job& b) { return a.cost > b.cost; });
  // workers: as asked, no more than jobs, and as many workspaces as fit in 80% of free memory
  size_t freeb = 0, totalb = 0;
  cudaMemGetInfo(&freeb, &totalb);
  const int max_grid = sms * std::max(1, cfg.tl.ctas_per_sm);
  const double per = 16.0 * ((double)bd.psi_amps + (double)bd.joint_amps) + 16.0 * (double)bd.mats +
                     8.0 * (double)bd.grads * (max_grid + 2) / 3.0 + (64 << 20);
  int nw = nstreams > 0 ? nstreams : env_int("IQ_ADJOINT_STREAMS", 8);
  nw = std::min<int>(nw, (int)jobs.size());
  nw = std::min<int>(nw, std::max(1, (int)(0.8 * (double)freeb / per)));
  nw = std::max(nw, 1);

  Stats st;
  std::atomic<size_t> next{0};
  std::mutex emu;
  std::string first_err;
  auto worker = [&](int id) {
    (void)id;
    Workspace* wp = pool_take(dev);
    Workspace& w = *wp;
    std::string e;
    bool ok = w.prepare(dev, sms, bd, e);
    while (ok) {
      const size_t i = next.fetch_add(1);
      if (i >= jobs.size()) break;
      ok = launch_job(w, cfg, *jobs[i].c, jobs[i].set0, jobs[i].nsets, want_grad, st, e);
      std::lock_guard<std::mutex> g(emu);
      if (!first_err.empty()) ok = false;   // another worker failed: stop taking jobs
    }
    if (ok) ok = finish(w, 0, e) && finish(w, 1, e);
    if (!ok) {
      next.store(jobs.size());
      std::lock_guard<std::mutex> g(emu);
      if (first_err.empty()) first_err = e.empty() ? "adjoint worker failed" : e;
    }
    pool_give(wp, ok);
  };
  if (jobs.empty()) {
    nw = 0;
  } else if (nw == 1) {
    worker(0);
  } else {
    std::vector<std::thread> th;
    for (int i = 0; i < nw; ++i) th.emplace_back(worker, i);
    for (auto& t : th) t.join();
  }
  if (res_thread.joinable()) res_thread.join();
  if (!res_ok && first_err.empty()) first_err = res_err;
  cudaSetDevice(dev);
  count_launches(st.launches.load());
  const double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  t_stats[0] = (double)st.jobs.load();
  t_stats[1] = (double)st.fw_passes.load();
  t_stats[2] = (double)st.bw_passes.load();
  t_stats[3] = (double)st.launches.load();
  t_stats[4] = (double)st.bytes.load();
  t_stats[5] = (double)st.host_ns.load() * 1e-6;
  t_stats[6] = wall;
  t_stats[7] = (double)nw;
  t_stats[8] = (double)st.jit_passes.load();
  t_stats[9] = (double)resident_sets;
  (void)st.replans;
  if (!first_err.empty()) {
    record_error(first_err.find("scheduler") == 0 ? E_STATE : E_CUDA, first_err.c_str());
    return -1;
  }
  return 0;
}

bool load_circuit(const iq_adjoint_circuit& in, Circuit& c, bool want_grad, std::string& err) {
  if (in.num_qubits < 1 || in.num_qubits > 33) { err = "num_qubits must be 1..33"; return false; }
  c.n = (int)in.num_qubits;
  if (in.num_ops && (!in.kinds || !in.q0)) { err = "missing gate arrays"; return false; }
  c.ops.resize(in.num_ops);
  for (size_t i = 0; i < in.num_ops; ++i)
    c.ops[i] = {in.kinds[i], in.q0[i], in.q1 ? in.q1[i] : -1, in.param_index ? in.param_index[i] : -1};
  const int np = ansatz_check(c.n, c.ops, err);
  if (np < 0) return false;
  if ((size_t)np > in.num_params) { err = "a gate reads a parameter index >= num_params"; return false; }
  c.nparams = (int)in.num_params;
  c.nsets = in.num_sets;
  if (c.nsets && c.nparams && !in.params) { err = "missing parameters"; return false; }
  c.params = in.params;
  if (!in.coeffs || !in.paulis) { err = "missing Hamiltonian"; return false; }
  if (!build_ham(c.n, in.num_terms, in.coeffs, in.paulis, c.ham, err)) return false;
  c.energy_out = in.energy_out;
  c.grad_out = in.grad_out;
  if (c.nsets && !c.energy_out) { err = "missing energy output"; return false; }
  if (want_grad && c.nsets && c.nparams && !c.grad_out) { err = "missing gradient output"; return false; }
  return true;
}

int run_circuits(const iq_adjoint_circuit* in, size_t count, int nstreams, bool want_grad, bool c64 = false) {
  if (count && !in) { record_error(E_ARG, "null circuit array"); return -1; }
  std::vector<std::unique_ptr<Circuit>> circs;
  for (size_t i = 0; i < count; ++i) {
    std::unique_ptr<Circuit> c(new Circuit);
    std::string err;
    if (!load_circuit(in[i], *c, want_grad, err)) {
      char m[320];
      snprintf(m, sizeof(m), "circuit %zu: %s", i, err.c_str());
      record_error(E_ARG, m);
      return -1;
    }
    circs.push_back(std::move(c));
  }
  return run_batch(circs, nstreams, want_grad, c64);
}

// ------------------------------------------------------------ complex64 variant
//
// The same gradient with amplitudes stored as complex64 (float2) and FP64
// arithmetic and reductions (iq_c64.cu).  The ansatz becomes items: runs of
// one-qubit gates on one qubit (at most kC64MaxRunOps, flushed before any
// two-qubit gate on that qubit; gates on different qubits commute, so the
// circuit is unchanged) and CZ / CX gates.  Forward: one pass per item (a run
// applies its product matrix).  Backward, items in reverse: a run records each
// rotation's Im<lambda|P|psi> and un-applies it, last gate first, in one pass
// over psi and lambda.

struct C64Item {
  int kind;        // 0 = run, 1 = CZ, 2 = CX (a = control, b = target)
  int a, b;
  C64Run run;
  C64Mat fwd;      // the run's product matrix
};

void mat_rot(int gen, double c, double s, double* m) {   // exp(-i t P / 2), re/im interleaved
  for (int i = 0; i < 8; ++i) m[i] = 0.0;
  if (gen == 0) { m[0] = c; m[3] = -s; m[5] = -s; m[6] = c; }
  else if (gen == 1) { m[0] = c; m[2] = -s; m[4] = s; m[6] = c; }
  else { m[0] = c; m[1] = -s; m[6] = c; m[7] = s; }
}

void mat_mul(const double* a, const double* b, double* o) {   // o = a b
  double t[8];
  for (int r = 0; r < 2; ++r)
    for (int cc = 0; cc < 2; ++cc) {
      double re = 0.0, im = 0.0;
      for (int k = 0; k < 2; ++k) {
        const double ar = a[2 * (2 * r + k)], ai = a[2 * (2 * r + k) + 1];
        const double br = b[2 * (2 * k + cc)], bi = b[2 * (2 * k + cc) + 1];
        re += ar * br - ai * bi;
        im += ar * bi + ai * br;
      }
      t[2 * (2 * r + cc)] = re;
      t[2 * (2 * r + cc) + 1] = im;
    }
  for (int i = 0; i < 8; ++i) o[i] = t[i];
}

void mat_dagger(const double* m, double* o) {
  double t[8];
  for (int r = 0; r < 2; ++r)
    for (int cc = 0; cc < 2; ++cc) {
      t[2 * (2 * r + cc)] = m[2 * (2 * cc + r)];
      t[2 * (2 * r + cc) + 1] = -m[2 * (2 * cc + r) + 1];
    }
  for (int i = 0; i < 8; ++i) o[i] = t[i];
}

void mat_fixed(int kind, double* m) {   // H, X, SX
  for (int i = 0; i < 8; ++i) m[i] = 0.0;
  const double r = 1.0 / std::sqrt(2.0);
  if (kind == GATE_H) { m[0] = r; m[2] = r; m[4] = r; m[6] = -r; }
  else if (kind == GATE_X) { m[2] = 1.0; m[4] = 1.0; }
  else { m[0] = 0.5; m[1] = 0.5; m[2] = 0.5; m[3] = -0.5; m[4] = 0.5; m[5] = -0.5; m[6] = 0.5; m[7] = 0.5; }
}

void build_c64_items(int n, const std::vector<AnsatzOp>& ops, const double* theta, std::vector<C64Item>& items,
                     std::vector<int>& term_param) {
  std::vector<C64Item> open(n);
  for (int q = 0; q < n; ++q) {
    open[q].kind = 0;
    open[q].run.q = q;
    open[q].run.nops = 0;
  }
  auto reset = [&](int q) {
    open[q].run.nops = 0;
    double* f = open[q].fwd.m;
    for (int i = 0; i < 8; ++i) f[i] = 0.0;
    f[0] = f[6] = 1.0;
  };
  for (int q = 0; q < n; ++q) reset(q);
  auto flush = [&](int q) {
    if (open[q].run.nops) items.push_back(open[q]);
    reset(q);
  };
  auto push = [&](int q, const C64Op& o, const double* fwd) {
    if (open[q].run.nops == kC64MaxRunOps) flush(q);
    open[q].run.ops[open[q].run.nops++] = o;
    mat_mul(fwd, open[q].fwd.m, open[q].fwd.m);
  };
  auto rot = [&](int q, int gen, int par) {
    C64Op o{};
    o.gen = gen;
    o.term = (int)term_param.size();
    term_param.push_back(par);
    o.c = std::cos(0.5 * theta[par]);
    o.s = std::sin(0.5 * theta[par]);
    double f[8];
    mat_rot(gen, o.c, o.s, f);
    push(q, o, f);
  };
  for (const AnsatzOp& a : ops) {
    switch (a.kind) {
      case GATE_RX: rot(a.q0, 0, a.param); break;
      case GATE_RY: rot(a.q0, 1, a.param); break;
      case GATE_RZ: case GATE_P: rot(a.q0, 2, a.param); break;   // P = phase x Rz
      case GATE_U3:   // e^{i(phi+lambda)/2} Rz(phi) Ry(theta) Rz(lambda)
        rot(a.q0, 2, a.param + 2);
        rot(a.q0, 1, a.param);
        rot(a.q0, 2, a.param + 1);
        break;
      case GATE_H: case GATE_X: case GATE_SX: {
        C64Op o{};
        o.gen = -1;
        double f[8];
        mat_fixed(a.kind, f);
        mat_dagger(f, o.inv);
        push(a.q0, o, f);
        break;
      }
      default: {   // CZ, CX
        flush(a.q0);
        flush(a.q1);
        C64Item it{};
        it.kind = a.kind == GATE_CZ ? 1 : 2;
        it.a = a.q0;
        it.b = a.q1;
        items.push_back(it);
      }
    }
  }
  for (int q = 0; q < n; ++q) flush(q);
}

int adjoint_c64(const iq_adjoint_circuit& in) {
  Circuit c;
  std::string err;
  if (!load_circuit(in, c, true, err)) { record_error(E_ARG, err.c_str()); return -1; }
  if (in.num_sets != 1) { record_error(E_ARG, "the complex64 variant takes one parameter set"); return -1; }
  const int dev = current_device(err);
  if (dev < 0) { record_error(E_DEVICE, err.c_str()); return -1; }
  std::vector<C64Item> items;
  std::vector<int> term_param;
  build_c64_items(c.n, c.ops, c.params, items, term_param);
  const int T = (int)term_param.size();
  const uint64_t dim = 1ULL << c.n;
  float2 *psi = nullptr, *lam = nullptr;
  double *partials = nullptr, *sums = nullptr;
  uint64_t* zm = nullptr;
  double2* co = nullptr;
  cudaStream_t st = nullptr;
  uint64_t launches = 0;
  bool ok = true;
  auto check = [&](cudaError_t e, const char* what) {
    if (ok && e != cudaSuccess) {
      ok = false;
      err = std::string(what) + ": " + cudaGetErrorString(e);
    }
    return ok;
  };
  check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream");
  if (ok && (cudaMalloc(&psi, dim * sizeof(float2)) != cudaSuccess ||
             cudaMalloc(&lam, dim * sizeof(float2)) != cudaSuccess)) {
    cudaGetLastError();
    ok = false;
    err = "cannot allocate device memory for the complex64 states";
  }
  check(cudaMalloc(&partials, ((size_t)T + 1) * kC64Blocks * sizeof(double)), "cudaMalloc partials");
  check(cudaMalloc(&sums, ((size_t)T + 1) * sizeof(double)), "cudaMalloc sums");
  check(cudaMalloc(&zm, c.ham.zmask.size() * 8), "cudaMalloc Hamiltonian");
  check(cudaMalloc(&co, c.ham.coef.size() * 16), "cudaMalloc Hamiltonian");
  check(cudaMemcpyAsync(zm, c.ham.zmask.data(), c.ham.zmask.size() * 8, cudaMemcpyHostToDevice, st), "H2D");
  check(cudaMemcpyAsync(co, c.ham.coef.data(), c.ham.coef.size() * 16, cudaMemcpyHostToDevice, st), "H2D");
  check(c64_set_basis(psi, c.n, st), "reset");
  ++launches;
  for (const C64Item& it : items) {   // forward
    if (!ok) break;
    if (it.kind == 0) check(c64_apply1q(psi, c.n, it.run.q, it.fwd, st), "complex64 gate kernel");
    else if (it.kind == 1) check(c64_cz(psi, c.n, it.a, it.b, st), "complex64 CZ kernel");
    else check(c64_cx(psi, c.n, it.a, it.b, st), "complex64 CX kernel");
    ++launches;
  }
  double* hpart = partials + (size_t)T * kC64Blocks;
  check(c64_hamiltonian(psi, c.n, c.ham.groups, zm, co, lam, hpart, st), "complex64 Hamiltonian kernel");
  ++launches;
  for (size_t i = items.size(); ok && i-- > 0;) {   // backward
    const C64Item& it = items[i];
    if (it.kind == 0) {
      check(c64_grad_run(psi, lam, c.n, it.run, partials, st), "complex64 adjoint kernel");
      ++launches;
    } else {
      for (float2* s2 : {psi, lam}) {
        if (it.kind == 1) check(c64_cz(s2, c.n, it.a, it.b, st), "complex64 CZ kernel");
        else check(c64_cx(s2, c.n, it.a, it.b, st), "complex64 CX kernel");
        ++launches;
      }
    }
  }
  if (ok) check(launch_row_sums(partials, T + 1, kC64Blocks, sums, st), "sums");
  launches += 1;
  std::vector<double> h((size_t)T + 1);
  if (ok) check(cudaMemcpyAsync(h.data(), sums, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
  if (st) check(cudaStreamSynchronize(st), "stream sync");
  for (void* p : {(void*)psi, (void*)lam, (void*)partials, (void*)sums, (void*)zm, (void*)co})
    if (p) cudaFree(p);
  if (st) cudaStreamDestroy(st);
  count_launches(launches);
  if (!ok) {
    record_error(E_CUDA, err.c_str());
    return -1;
  }
  if (c.energy_out) c.energy_out[0] = h[T];
  if (c.grad_out) {
    for (int i = 0; i < c.nparams; ++i) c.grad_out[i] = 0.0;
    for (int t = 0; t < T; ++t) c.grad_out[term_param[t]] += h[t];
  }
  return 0;
}

}  // namespace

extern "C" {

int iq_adjoint_gradient(size_t num_qubits, size_t num_ops, const int* kinds, const int* q0, const int* q1,
                        const int* param_index, size_t num_params, const double* params, size_t num_terms,
                        const double* coeffs, const char* paulis, double* energy_out, double* grad_out) {
  iq_adjoint_circuit c{};
  c.num_qubits = num_qubits;
  c.num_ops = num_ops;
  c.kinds = kinds;
  c.q0 = q0;
  c.q1 = q1;
  c.param_index = param_index;
  c.num_params = num_params;
  c.num_sets = 1;
  c.params = params;
  c.num_terms = num_terms;
  c.coeffs = coeffs;
  c.paulis = paulis;
  c.energy_out = energy_out;
  c.grad_out = grad_out;
  return run_circuits(&c, 1, 1, true);
}

int iq_adjoint_gradient_c64(size_t num_qubits, size_t num_ops, const int* kinds, const int* q0, const int* q1,
                            const int* param_index, size_t num_params, const double* params, size_t num_terms,
                            const double* coeffs, const char* paulis, double* energy_out, double* grad_out) {
  iq_adjoint_circuit c{};
  c.num_qubits = num_qubits;
  c.num_ops = num_ops;
  c.kinds = kinds;
  c.q0 = q0;
  c.q1 = q1;
  c.param_index = param_index;
  c.num_params = num_params;
  c.num_sets = 1;
  c.params = params;
  c.num_terms = num_terms;
  c.coeffs = coeffs;
  c.paulis = paulis;
  c.energy_out = energy_out;
  c.grad_out = grad_out;
  // from 7 qubits: the tile-pass executor with complex64 arrays (specialised
  // kernels); below, or with IQ_C64_TILE=0, one pass per gate run (adjoint_c64)
  if (num_qubits >= 7 && env_int("IQ_C64_TILE", 1) != 0) return run_circuits(&c, 1, 1, true, true);
  return adjoint_c64(c);
}

int iq_adjoint_gradient_batch(const iq_adjoint_circuit* circuits, size_t num_circuits, int num_streams) {
  return run_circuits(circuits, num_circuits, num_streams, true);
}

int iq_ansatz_energy(const iq_adjoint_circuit* circuit) { return run_circuits(circuit, 1, 1, false); }

int iq_adjoint_release(void) {
  resident_release();
  std::vector<Workspace*> ws;
  {
    std::lock_guard<std::mutex> g(g_pool_mu);
    ws.swap(*g_pool);
  }
  for (Workspace* w : ws) {
    cudaSetDevice(w->device);
    w->release();
    delete w;
  }
  return (int)ws.size();
}

int iq_adjoint_stats(double* out, size_t n) {
  if (!out) return -1;
  for (size_t i = 0; i < n && i < 10; ++i) out[i] = t_stats[i];
  return 10;
}

}  // extern "C"
