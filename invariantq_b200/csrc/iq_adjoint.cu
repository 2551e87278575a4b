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
#include <unordered_map>
#include <vector>

#include "../../include/invariantq_b200.h"
#include "iq_kernels.h"
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
  static Cfg from_env() {
    Cfg c;
    c.sp.M = env_int("IQ_TILE_BITS", 11);
    c.sp.c = env_int("IQ_CHUNK_BITS", 5);
    c.sp.R = std::min(5, std::max(3, env_int("IQ_SLOTS", 4)));
    c.sp.max_stages = env_int("IQ_MAX_STAGES", 8);
    c.sp.budget = env_double("IQ_PASS_BUDGET", 80.0);
    c.sp.grad_cost = env_double("IQ_GRAD_COST", 6.0);
    c.tl.nbuf = env_int("IQ_NBUF", 3);
    c.tl.ctas_per_sm = env_int("IQ_CTAS_PER_SM", 2);
    c.tl.consumers = 128;
    c.fuse = env_int("IQ_FUSE", 1);
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
};

bool same_op(const SchedOp& a, const SchedOp& b) {
  if (a.k != b.k || a.mono != b.mono || a.perm != b.perm || a.unit != b.unit || a.mat != b.mat ||
      a.dense != b.dense || a.grad != b.grad || a.gen != b.gen || a.gidx != b.gidx)
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

// fused forward / backward operation lists and matrix pools of one parameter set
struct JobOps {
  std::vector<SchedOp> fw, bw;
  std::vector<cplx64> fpool, bpool;
  std::vector<int> grad_param;
};

void job_ops(const Cfg& cfg, const Circuit& c, const double* theta, bool backward, JobOps& j) {
  j.fw.clear(); j.bw.clear(); j.fpool.clear(); j.bpool.clear(); j.grad_param.clear();
  std::vector<SchedOp> raw;
  ansatz_forward(c.n, c.ops, theta, raw, j.fpool);
  j.fw = cfg.fuse ? fuse_two_qubit_blocks(raw, j.fpool) : raw;
  if (!backward) return;
  raw.clear();
  ansatz_backward(c.n, c.ops, theta, raw, j.bpool, j.grad_param);
  j.bw = cfg.fuse ? fuse_two_qubit_blocks(raw, j.bpool) : raw;
}

int joint_bits(int n) { return std::max(n + 1, 7); }

// ---------------------------------------------------------------- workspace

struct Stats {
  std::atomic<uint64_t> jobs{0}, fw_passes{0}, bw_passes{0}, launches{0}, replans{0};
  std::atomic<uint64_t> bytes{0};           // algorithmic HBM bytes of the passes
  std::atomic<uint64_t> host_ns{0};
};

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t cap = 0;
  // grow to n elements; `user` (the stream that reads the buffer) is drained before the old one is freed
  bool ensure(size_t n, std::string& err, const char* what, cudaStream_t user = nullptr) {
    if (n <= cap) return true;
    if (p && user) cudaStreamSynchronize(user);
    if (p) cudaFree(p);
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
  size_t set = 0;
  std::vector<int> grad_param;
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
  HostBuf<double> hout[2];    // energy, then the gradient terms
  HostBuf<int> hstat[2];      // device status word
  cudaEvent_t ev[2] = {nullptr, nullptr};
  Pending pend[2];
  int slot = 0;
  std::unordered_map<const Shape*, std::vector<CUtensorMap>> tmaps;
  const Circuit* ham_of = nullptr;   // circuit whose Hamiltonian tables are on the device

  bool init(int dev, int sms, int nmax, std::string& err) {
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
    if (!psi.ensure(1ULL << nmax, err, "the state") || !joint.ensure(1ULL << joint_bits(nmax), err, "the joint array") ||
        !red.ensure(kRedBlocks + 8, err, "reduction partials") || !status.ensure(1, err, "the status word"))
      return false;
    return cudaMemsetAsync(status.p, 0, sizeof(int), stream) == cudaSuccess;
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

  // Tensor maps of a shape's passes over `base`.  Circuit shapes live for the
  // whole batch and are cached by address; a job's private shape is encoded
  // into `scratch` (its address may be reused by a later shape).
  const std::vector<CUtensorMap>* maps_for(const Shape& s, double2* base, bool cache, std::vector<CUtensorMap>& scratch,
                                           std::string& err) {
    if (cache) {
      auto it = tmaps.find(&s);
      if (it != tmaps.end()) return &it->second;
    }
    std::vector<CUtensorMap> v(s.plans.size());
    char emsg[256];
    for (size_t i = 0; i < s.plans.size(); ++i)
      if (encode_pass_tmap(&v[i], base, s.nbits, s.plans[i].desc, emsg, sizeof(emsg)) != 0) {
        err = emsg;
        return nullptr;
      }
    if (!cache) {
      scratch = std::move(v);
      return &scratch;
    }
    return &tmaps.emplace(&s, std::move(v)).first->second;
  }
};

bool cuda_ok(cudaError_t e, const char* what, std::string& err) {
  if (e == cudaSuccess) return true;
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return false;
}

// launch a shape's passes on `state` (matrices at `mats`)
bool run_shape(Workspace& w, const Cfg& cfg, const Shape& s, bool cached, double2* state, const double2* mats,
               double* gpart, Stats& st, std::string& err) {
  if (!s.tiled) {
    for (const SimpleOp& so : s.sops)
      if (!cuda_ok(launch_simple_op(state, s.nbits, so, mats, w.stream), "gate kernel", err)) return false;
    st.launches += s.sops.size();
    st.bytes += (uint64_t)s.sops.size() * (32ULL << s.nbits);
    return true;
  }
  std::vector<CUtensorMap> scratch;
  const std::vector<CUtensorMap>* tm = w.maps_for(s, state, cached, scratch, err);
  if (!tm) return false;
  for (size_t i = 0; i < s.plans.size(); ++i)
    if (!cuda_ok(launch_tile_pass((*tm)[i], s.plans[i].desc, mats, w.status.p, cfg.tl, w.num_sms, w.stream, gpart),
                 "tile pass kernel", err))
      return false;
  st.launches += s.plans.size();
  st.bytes += (uint64_t)s.plans.size() * (32ULL << s.nbits);
  return true;
}

// Finish the job that used staging slot `k`: wait for its stream, check the
// status word, write energy and gradient.
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
  if (c.energy_out) c.energy_out[p.set] = out[0];
  if (p.grad && c.grad_out) {
    double* g = c.grad_out + p.set * (size_t)c.nparams;
    for (int i = 0; i < c.nparams; ++i) g[i] = 0.0;
    for (int t = 0; t < p.ngrads; ++t) g[p.grad_param[t]] += out[1 + t];
  }
  return true;
}

// Prepare and launch one job on the workspace's stream.  want_grad = false:
// forward and energy only.
bool launch_job(Workspace& w, const Cfg& cfg, Circuit& c, size_t set, bool want_grad, Stats& st, std::string& err) {
  const auto t0 = std::chrono::steady_clock::now();
  const double* theta = c.params + set * (size_t)c.nparams;
  JobOps j;
  job_ops(cfg, c, theta, want_grad, j);
  {
    std::lock_guard<std::mutex> g(c.mu);
    if (!c.planned) {
      c.planned = true;
      c.fw.reset(new Shape);
      if (!make_shape(cfg, c.n, j.fw, j.fpool.size(), w.num_sms, *c.fw, c.plan_err)) c.fw.reset();
      if (c.fw && want_grad) {
        c.bw.reset(new Shape);
        if (!make_shape(cfg, joint_bits(c.n), j.bw, j.bpool.size(), w.num_sms, *c.bw, c.plan_err)) c.bw.reset();
        else c.bw->ngrads = (int)j.grad_param.size();
      }
    }
    if (!c.fw || (want_grad && !c.bw)) {
      err = "scheduler: " + c.plan_err;
      return false;
    }
  }
  // shapes for this set (the circuit's, or private ones if the structure differs)
  std::unique_ptr<Shape> own_fw, own_bw;
  const Shape* fw = c.fw.get();
  const Shape* bw = c.bw.get();
  if (!matches(*fw, j.fw, j.fpool.size())) {
    own_fw.reset(new Shape);
    if (!make_shape(cfg, c.n, j.fw, j.fpool.size(), w.num_sms, *own_fw, err)) return false;
    fw = own_fw.get();
    ++st.replans;
  }
  if (want_grad && !matches(*bw, j.bw, j.bpool.size())) {
    own_bw.reset(new Shape);
    if (!make_shape(cfg, joint_bits(c.n), j.bw, j.bpool.size(), w.num_sms, *own_bw, err)) return false;
    own_bw->ngrads = (int)j.grad_param.size();
    bw = own_bw.get();
    ++st.replans;
  }
  const int ngrads = want_grad ? (int)j.grad_param.size() : 0;

  // staging slot: wait for the job that used it last
  const int k = w.slot;
  w.slot ^= 1;
  const auto tw = std::chrono::steady_clock::now();
  if (!finish(w, k, err)) return false;
  const auto tw1 = std::chrono::steady_clock::now();
  const size_t nf = fw->gather.size(), nb = want_grad ? bw->gather.size() : 0;
  if (!w.hmats[k].ensure(nf + nb, err) || !w.hout[k].ensure(1 + (size_t)ngrads, err) || !w.hstat[k].ensure(1, err))
    return false;
  double2* hm = w.hmats[k].p;
  for (size_t i = 0; i < nf; ++i) hm[i] = make_double2(j.fpool[fw->gather[i]].re, j.fpool[fw->gather[i]].im);
  for (size_t i = 0; i < nb; ++i) hm[nf + i] = make_double2(j.bpool[bw->gather[i]].re, j.bpool[bw->gather[i]].im);

  // device buffers (a buffer that grows waits for the stream's earlier work first)
  if (!w.mats.ensure(2 * (nf + nb), err, "matrices", w.stream)) return false;
  if (want_grad &&
      (!w.gpart.ensure((size_t)std::max(ngrads, 1) * std::max(bw->grid, 1u), err, "gradient partials", w.stream) ||
       !w.gsum.ensure((size_t)std::max(ngrads, 1), err, "gradient sums", w.stream)))
    return false;
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
  // job j+1 cannot overwrite matrices job j's passes still read
  double2* dm = w.mats.p + (size_t)k * (w.mats.cap / 2);
  if (!cuda_ok(cudaMemcpyAsync(dm, hm, (nf + nb) * sizeof(double2), cudaMemcpyHostToDevice, w.stream), "H2D matrices",
               err))
    return false;
  st.host_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                     (std::chrono::steady_clock::now() - t0) - (tw1 - tw))
                     .count();

  // forward from |0>
  const uint64_t dim = 1ULL << c.n;
  if (!cuda_ok(launch_set_basis(w.psi.p, dim, w.stream), "reset", err)) return false;
  if (!run_shape(w, cfg, *fw, !own_fw, w.psi.p, dm, nullptr, st, err)) return false;
  st.fw_passes += fw->tiled ? fw->plans.size() : fw->sops.size();
  double* energy_dev = w.red.p + kRedBlocks;
  if (!want_grad) {
    if (!cuda_ok(launch_hamiltonian_joint(w.psi.p, c.n, c.ham.groups, w.zmask.p, w.coef.p, nullptr, w.red.p,
                                          energy_dev, w.stream),
                 "energy kernel", err))
      return false;
    st.launches += 3;
  } else {
    const int nj = joint_bits(c.n);
    if (nj > c.n + 1 &&
        !cuda_ok(cudaMemsetAsync(w.joint.p + 2 * dim, 0, ((1ULL << nj) - 2 * dim) * sizeof(double2), w.stream),
                 "memset", err))
      return false;
    if (!cuda_ok(launch_hamiltonian_joint(w.psi.p, c.n, c.ham.groups, w.zmask.p, w.coef.p, w.joint.p, w.red.p,
                                          energy_dev, w.stream),
                 "Hamiltonian kernel", err))
      return false;
    if (!run_shape(w, cfg, *bw, !own_bw, w.joint.p, dm + nf, w.gpart.p, st, err)) return false;
    st.bw_passes += bw->tiled ? bw->plans.size() : bw->sops.size();
    if (!cuda_ok(launch_row_sums(w.gpart.p, ngrads, (int)bw->grid, w.gsum.p, w.stream), "gradient sums", err))
      return false;
    st.launches += 4;
  }
  st.bytes += 16ULL * dim + (want_grad ? 32ULL * dim : 0);   // read psi; write the joint array
  double* ho = w.hout[k].p;
  if (!cuda_ok(cudaMemcpyAsync(ho, energy_dev, sizeof(double), cudaMemcpyDeviceToHost, w.stream), "D2H", err) ||
      !cuda_ok(cudaMemcpyAsync(w.hstat[k].p, w.status.p, sizeof(int), cudaMemcpyDeviceToHost, w.stream), "D2H", err))
    return false;
  if (ngrads &&
      !cuda_ok(cudaMemcpyAsync(ho + 1, w.gsum.p, (size_t)ngrads * sizeof(double), cudaMemcpyDeviceToHost, w.stream),
               "D2H", err))
    return false;
  if (!cuda_ok(cudaEventRecord(w.ev[k], w.stream), "event", err)) return false;
  Pending& p = w.pend[k];
  p.active = true;
  p.c = &c;
  p.set = set;
  p.grad = want_grad;
  p.ngrads = ngrads;
  p.grad_param = std::move(j.grad_param);
  ++st.jobs;
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

thread_local double t_stats[8] = {0};

// Run all jobs of `circs` (every parameter set of every circuit) on `nstreams` workers.
int run_batch(std::vector<std::unique_ptr<Circuit>>& circs, int nstreams, bool want_grad) {
  const auto t0 = std::chrono::steady_clock::now();
  std::string err;
  const int dev = current_device(err);
  if (dev < 0) { record_error(E_DEVICE, err.c_str()); return -1; }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const Cfg cfg = Cfg::from_env();
  struct Job { Circuit* c; size_t set; double cost; };
  std::vector<Job> jobs;
  int nmax = 1;
  for (auto& c : circs) {
    nmax = std::max(nmax, c->n);
    for (size_t s = 0; s < c->nsets; ++s)
      jobs.push_back({c.get(), s, std::ldexp((double)c->ops.size() + 1.0, c->n)});
  }
  if (jobs.empty()) return 0;
  // largest first; sets of one circuit stay together so the first plans for the rest
  std::stable_sort(jobs.begin(), jobs.end(), [](const Job& a, const Job& b) { return a.cost > b.cost; });
  // workers: as asked, no more than jobs, and as many workspaces as fit in 80% of free memory
  size_t freeb = 0, totalb = 0;
  cudaMemGetInfo(&freeb, &totalb);
  const double per = 16.0 * (std::ldexp(1.0, nmax) + std::ldexp(1.0, joint_bits(nmax))) + (64 << 20);
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
    Workspace w;
    std::string e;
    bool ok = w.init(dev, sms, nmax, e);
    while (ok) {
      const size_t i = next.fetch_add(1);
      if (i >= jobs.size()) break;
      ok = launch_job(w, cfg, *jobs[i].c, jobs[i].set, want_grad, st, e);
      std::lock_guard<std::mutex> g(emu);
      if (!first_err.empty()) ok = false;   // another worker failed: stop taking jobs
    }
    if (ok) ok = finish(w, 0, e) && finish(w, 1, e);
    if (!ok) {
      next.store(jobs.size());
      std::lock_guard<std::mutex> g(emu);
      if (first_err.empty()) first_err = e.empty() ? "adjoint worker failed" : e;
    }
    w.release();
  };
  if (nw == 1) {
    worker(0);
  } else {
    std::vector<std::thread> th;
    for (int i = 0; i < nw; ++i) th.emplace_back(worker, i);
    for (auto& t : th) t.join();
  }
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

int run_circuits(const iq_adjoint_circuit* in, size_t count, int nstreams, bool want_grad) {
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
  return run_batch(circs, nstreams, want_grad);
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

int iq_adjoint_gradient_batch(const iq_adjoint_circuit* circuits, size_t num_circuits, int num_streams) {
  return run_circuits(circuits, num_circuits, num_streams, true);
}

int iq_ansatz_energy(const iq_adjoint_circuit* circuit) { return run_circuits(circuit, 1, 1, false); }

int iq_adjoint_stats(double* out, size_t n) {
  if (!out) return -1;
  for (size_t i = 0; i < n && i < 8; ++i) out[i] = t_stats[i];
  return 8;
}

}  // extern "C"
