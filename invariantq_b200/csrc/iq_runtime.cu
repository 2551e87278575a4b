// iq_runtime.cu -- handles, the lazy operation queue and the extern "C" ABI of
// libinvariantq.so (declared in include/invariantq_b200.h).
//
// Each state-vector or density-matrix handle owns one device array of complex128
// amplitudes (a density matrix is the row-major 4^n array, i.e. 2n index bits),
// one CUDA stream, and a host queue of pending operations.  Gate / channel
// calls only append to the queue; a flush plans tile passes (iq_sched.cpp) and
// launches them (iq_kernels.cu).  Any call that returns data flushes first and
// synchronises the stream before it returns.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <complex>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <mutex>
#include <random>
#include <string>
#include <vector>

#include "../../include/invariantq_b200.h"
#include "iq_jit.h"
#include "iq_kernels.h"
#include "iq_plan.h"

using namespace iqb;
using cd = std::complex<double>;

namespace {

// ------------------------------------------------------------------ errors

thread_local int t_errcode = 0;
thread_local char t_errmsg[512] = {0};
std::atomic<uint64_t> g_launches{0};

void set_error(int code, const char* fmt, ...) {
  t_errcode = code;
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(t_errmsg, sizeof(t_errmsg), fmt, ap);
  va_end(ap);
}

enum ErrCode { E_ARG = 1, E_CUDA = 2, E_MEM = 3, E_STATE = 4, E_DEVICE = 5, E_UNSUPPORTED = 6 };

const double kNaN = std::numeric_limits<double>::quiet_NaN();

bool cuda_ok(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(E_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return false;
}

int env_int(const char* name, int dflt) {
  const char* v = getenv(name);
  return v ? atoi(v) : dflt;
}
double env_double(const char* name, double dflt) {
  const char* v = getenv(name);
  return v ? atof(v) : dflt;
}

// ------------------------------------------------------ Hermitian eigenvalues
// Householder reduction of a Hermitian matrix to real tridiagonal form, then
// implicit QL iterations with Wilkinson-style shifts (eigenvalues only).

bool hermitian_eigenvalues(std::vector<cd> A, int n, std::vector<double>& w) {
  w.assign(n, 0.0);
  std::vector<double> d(n), e(n, 0.0);
  std::vector<cd> v(n), p(n);
  for (int k = 0; k + 2 < n; ++k) {
    double xn2 = 0.0;
    for (int i = k + 1; i < n; ++i) xn2 += std::norm(A[(size_t)i * n + k]);
    const double xn = std::sqrt(xn2);
    if (xn == 0.0) continue;
    const cd x0 = A[(size_t)(k + 1) * n + k];
    const cd ph = (std::abs(x0) > 0.0) ? x0 / std::abs(x0) : cd(1.0, 0.0);
    const cd alpha = -ph * xn;
    for (int i = 0; i < n; ++i) v[i] = 0.0;
    v[k + 1] = x0 - alpha;
    for (int i = k + 2; i < n; ++i) v[i] = A[(size_t)i * n + k];
    double vn2 = 0.0;
    for (int i = k + 1; i < n; ++i) vn2 += std::norm(v[i]);
    if (vn2 == 0.0) continue;
    const double vn = std::sqrt(vn2);
    for (int i = k + 1; i < n; ++i) v[i] /= vn;
    // p = A v over the trailing block (A Hermitian)
    for (int i = k; i < n; ++i) {
      cd s = 0.0;
      for (int j = k + 1; j < n; ++j) s += A[(size_t)i * n + j] * v[j];
      p[i] = s;
    }
    cd K = 0.0;
    for (int i = k + 1; i < n; ++i) K += std::conj(v[i]) * p[i];
    // w = 2 (p - K v); A <- A - v w^H - w v^H on rows/cols k..n-1
    for (int i = k; i < n; ++i) p[i] = 2.0 * (p[i] - K * v[i]);
    for (int i = k; i < n; ++i)
      for (int j = k; j < n; ++j)
        A[(size_t)i * n + j] -= v[i] * std::conj(p[j]) + p[i] * std::conj(v[j]);
  }
  for (int i = 0; i < n; ++i) d[i] = A[(size_t)i * n + i].real();
  for (int i = 0; i + 1 < n; ++i) e[i] = std::abs(A[(size_t)(i + 1) * n + i]);
  // implicit QL on (d, e)
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    int m;
    do {
      for (m = l; m + 1 < n; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= std::numeric_limits<double>::epsilon() * dd) break;
      }
      if (m != l) {
        if (++iter > 200) return false;
        double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
        double r = std::hypot(g, 1.0);
        g = d[m] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
        double s = 1.0, c = 1.0, pp = 0.0;
        int i;
        bool deflated = false;
        for (i = m - 1; i >= l; --i) {
          const double f = s * e[i], b = c * e[i];
          r = std::hypot(f, g);
          e[i + 1] = r;
          if (r == 0.0) {
            d[i + 1] -= pp;
            e[m] = 0.0;
            deflated = true;
            break;
          }
          s = f / r;
          c = g / r;
          g = d[i + 1] - pp;
          r = (d[i] - g) * s + 2.0 * c * b;
          pp = s * r;
          d[i + 1] = g + pp;
          g = c * r - b;
        }
        if (deflated) continue;
        d[l] -= pp;
        e[l] = g;
        e[m] = 0.0;
      }
    } while (m != l);
  }
  w = d;
  return true;
}

double entropy_from(const std::vector<double>& eig) {
  double s = 0.0;
  for (double l : eig)
    if (l > 1e-14) s -= l * std::log2(l);
  return s > 0.0 ? s : 0.0;
}

// why the last attempt to compile specialised pass kernels failed (the
// interpreting kernel ran those passes)
std::mutex g_jit_mu;
std::string g_jit_note;
void jit_note(const std::string& why) {
  std::lock_guard<std::mutex> lk(g_jit_mu);
  g_jit_note = why;
}

// ---------------------------------------------------------------- engine

constexpr size_t kStageBytes = 64ull << 20;   // device/host staging for readbacks

struct Engine {
  int kind = 0;            // 0 = state vector, 1 = density matrix
  int nq = 0;              // qubits
  int nbits = 0;           // index bits (SV: nq, DM: 2 nq)
  uint64_t dim = 1;
  int device = 0;
  int num_sms = 148;
  double2* d_state = nullptr;
  cudaStream_t stream = nullptr;

  std::vector<SchedOp> ops;
  std::vector<cplx64> pool;          // matrices of the queued ops (dense, plus phases of monomials)

  double2* d_pool = nullptr;
  size_t d_pool_cap = 0;
  double2* h_pool = nullptr;
  size_t h_pool_cap = 0;
  cudaEvent_t pool_ev = nullptr;
  bool pool_ev_recorded = false;

  double* d_scratch = nullptr;       // reduction partials and small results
  size_t scratch_bytes = 0;
  int* d_status = nullptr;
  double* h_small = nullptr;         // pinned small readback area
  void* d_stage = nullptr;
  void* h_stage = nullptr;

  SchedParams sp{};
  TileLaunch tl{};
  int eager = 0;
  int fuse = 1;
  int flush_ops = 4096;
  int profile = 0;
  // Specialised pass kernels (iq_jit.cpp): 0 off; 1 recorded programs are
  // compiled when recorded and flushes use kernels already compiled for their
  // structure (missing ones compile in the background), for arrays of at least
  // 2^kJitMinBits amplitudes; 2 both compiled before their first launch, any size.
  int jit = 1;
  static constexpr int kJitMinBits = 18;
  int normalize = 1;   // normalised one-qubit operations in specialised passes
  int plan_style = 0;  // 0: by the jit setting; 1: as for the interpreting kernel; 2: as for specialised kernels
  int jit_threads = 0; // CTA size of specialised kernels (0: by register slots; 128 or 256)
  // settings given explicitly (option or environment); the others take the
  // defaults of the plan style.  Specialised kernels: tiles of 2^12 amplitudes
  // holding the 4 lowest qubits, a budget of 160 FMAs per amplitude per pass,
  // 3 CTAs per SM with one tile buffer each (the fastest 30-qubit brick-wall
  // measured: 78 passes, ~627 ms, against 110 passes and ~776 ms with the
  // interpreting kernel's 11 / 5 / 120 / 4 CTAs).  Interpreting kernel: tiles of
  // 2^11 holding 5, budget 120, 2 CTAs per SM with three buffers.
  bool set_M = false, set_c = false, set_budget = false, set_nbuf = false, set_ctas = false;

  bool spec_style() const {
    return plan_style == 2 || (plan_style == 0 && jit && (jit >= 2 || nbits >= kJitMinBits) && !eager && nbits >= 7);
  }
  SchedParams plan_params(bool spec) const {
    SchedParams p = sp;
    if (spec) {
      if (!set_M) p.M = 12;
      if (!set_c) p.c = 4;
      if (!set_budget) p.budget = 160.0;
    }
    return p;
  }
  TileLaunch launch_params(bool spec) const {
    TileLaunch t = tl;
    if (spec && !set_ctas) t.ctas_per_sm = 3;
    if (spec && !set_nbuf) t.nbuf = 1;
    return t;
  }
  std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof;

  double st_passes = 0, st_ops = 0, st_bytes = 0, st_launches = 0, st_flushes = 0, st_tile = 0, st_h2d = 0;
  double st_jit = 0;                 // tile passes run by a specialised kernel
  bool recording = false;

  bool init(int kind_, size_t n) {
    kind = kind_;
    nq = (int)n;
    nbits = kind == 0 ? nq : 2 * nq;
    if ((kind == 0 && n > 34) || (kind == 1 && n > 17)) {
      set_error(E_ARG, "%s of %zu qubits exceeds the supported size", kind ? "density matrix" : "state vector", n);
      return false;
    }
    dim = 1ULL << nbits;
    device = env_int("IQ_CUDA_DEVICE", -1);
    if (device >= 0) {
      if (!cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return false;
    } else if (!cuda_ok(cudaGetDevice(&device), "cudaGetDevice")) {
      return false;
    }
    int cc = 0;
    cudaDeviceGetAttribute(&cc, cudaDevAttrComputeCapabilityMajor, device);
    if (cc < 10) {
      set_error(E_DEVICE, "device %d has compute capability %d.x; this library is built for sm_100a", device, cc);
      return false;
    }
    cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device);
    if (!cuda_ok(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
    if (cudaMalloc(&d_state, dim * sizeof(double2)) != cudaSuccess) {
      cudaGetLastError();
      set_error(E_MEM, "cannot allocate %.3f GiB of device memory for %d qubits", dim * 16.0 / (1 << 30), nq);
      d_state = nullptr;
      return false;
    }
    scratch_bytes = std::max<size_t>(zsums_partials_doubles(nbits) * 8, (size_t)kRedBlocks * 16) + 4096;
    if (!cuda_ok(cudaMalloc(&d_scratch, scratch_bytes), "cudaMalloc scratch")) return false;
    if (!cuda_ok(cudaMalloc(&d_status, sizeof(int)), "cudaMalloc status")) return false;
    if (!cuda_ok(cudaMallocHost(&h_small, 64 * 1024), "cudaMallocHost")) return false;
    if (!cuda_ok(cudaEventCreateWithFlags(&pool_ev, cudaEventDisableTiming), "cudaEventCreate")) return false;
    cudaMemsetAsync(d_status, 0, sizeof(int), stream);
    sp.nbits = nbits;
    tl.consumers = 128;
    sp.M = env_int("IQ_TILE_BITS", 11);
    sp.c = env_int("IQ_CHUNK_BITS", 5);
    sp.R = std::min(5, std::max(3, env_int("IQ_SLOTS", 4)));   // register slots (R); wider blocks raise it
    sp.max_stages = env_int("IQ_MAX_STAGES", 8);
    sp.budget = env_double("IQ_PASS_BUDGET", 120.0);
    tl.nbuf = env_int("IQ_NBUF", 3);
    tl.ctas_per_sm = env_int("IQ_CTAS_PER_SM", 2);
    set_M = getenv("IQ_TILE_BITS") != nullptr;
    set_c = getenv("IQ_CHUNK_BITS") != nullptr;
    set_budget = getenv("IQ_PASS_BUDGET") != nullptr;
    set_nbuf = getenv("IQ_NBUF") != nullptr;
    set_ctas = getenv("IQ_CTAS_PER_SM") != nullptr;
    eager = env_int("IQ_EAGER", 0);
    return reset_state();
  }

  void release() {
    if (stream) cudaStreamSynchronize(stream);
    for (auto& pe : prof) {
      cudaEventDestroy(pe.first);
      cudaEventDestroy(pe.second);
    }
    prof.clear();
    if (d_state) cudaFree(d_state);
    if (d_pool) cudaFree(d_pool);
    if (h_pool) cudaFreeHost(h_pool);
    if (d_scratch) cudaFree(d_scratch);
    if (d_status) cudaFree(d_status);
    if (h_small) cudaFreeHost(h_small);
    if (d_stage) cudaFree(d_stage);
    if (h_stage) cudaFreeHost(h_stage);
    if (pool_ev) cudaEventDestroy(pool_ev);
    if (stream) cudaStreamDestroy(stream);
    d_state = nullptr;
    stream = nullptr;
  }

  bool select() { return cuda_ok(cudaSetDevice(device), "cudaSetDevice"); }

  bool reset_state() {
    if (!recording) clear_queue();
    ++st_launches;
    ++g_launches;
    return cuda_ok(launch_set_basis(d_state, dim, stream), "reset");
  }

  bool ensure_stage() {
    if (d_stage) return true;
    if (!cuda_ok(cudaMalloc(&d_stage, kStageBytes), "cudaMalloc staging")) return false;
    if (!cuda_ok(cudaMallocHost(&h_stage, kStageBytes), "cudaMallocHost staging")) return false;
    return true;
  }

  // -------------------------------------------------------------- queue
  // Append an operation on index bits q[0..k-1] (LSB-first) with row-major
  // complex matrix m (2^k x 2^k).
  bool enqueue(int k, const int* q, const cd* m) {
    for (int i = 0; i < k; ++i) {
      if (q[i] < 0 || q[i] >= nbits) {
        set_error(E_ARG, "qubit index out of range");
        return false;
      }
      for (int j = 0; j < i; ++j)
        if (q[i] == q[j]) {
          set_error(E_ARG, "repeated qubit in a gate");
          return false;
        }
    }
    const int d = 1 << k;
    SchedOp o{};
    o.k = (uint8_t)k;
    for (int i = 0; i < k; ++i) o.q[i] = (uint8_t)q[i];
    const uint32_t dense = (uint32_t)pool.size();
    for (int i = 0; i < d * d; ++i) pool.push_back({m[i].real(), m[i].imag()});
    o.mat = dense;
    o.dense = dense;
    o.mono = 0;
    if (k <= 2) {
      double ph[8];
      uint8_t perm = 0, unit = 0;
      if (classify_monomial(reinterpret_cast<const double*>(m), k, &perm, ph, &unit)) {
        o.mono = 1;
        o.perm = perm;
        o.unit = unit;
        o.mat = (uint32_t)pool.size();
        for (int i = 0; i < d; ++i) pool.push_back({ph[2 * i], ph[2 * i + 1]});
      } else if (k == 2) {
        o.xpat = (uint8_t)classify_xpattern(reinterpret_cast<const double*>(m));
      }
    }
    ops.push_back(o);
    if (!recording && (int)ops.size() >= flush_ops) return flush();
    return true;
  }

  // copy `n` complex values to the per-handle device pool through the pinned buffer
  bool upload_pool(const double2* src, size_t n) {
    if (n == 0) return true;
    if (n > d_pool_cap) {
      if (d_pool) {
        cudaStreamSynchronize(stream);
        cudaFree(d_pool);
      }
      d_pool_cap = std::max<size_t>(n, 1 << 16);
      if (!cuda_ok(cudaMalloc(&d_pool, d_pool_cap * sizeof(double2)), "cudaMalloc matrix pool")) {
        d_pool = nullptr;
        d_pool_cap = 0;
        return false;
      }
    }
    if (n > h_pool_cap) {
      if (pool_ev_recorded) cudaEventSynchronize(pool_ev);
      if (h_pool) cudaFreeHost(h_pool);
      h_pool_cap = std::max<size_t>(n, 1 << 16);
      if (!cuda_ok(cudaMallocHost(&h_pool, h_pool_cap * sizeof(double2)), "cudaMallocHost matrix pool")) {
        h_pool = nullptr;
        h_pool_cap = 0;
        return false;
      }
    } else if (pool_ev_recorded) {
      cudaEventSynchronize(pool_ev);   // previous copy out of h_pool has finished
    }
    memcpy(h_pool, src, n * sizeof(double2));
    if (!cuda_ok(cudaMemcpyAsync(d_pool, h_pool, n * sizeof(double2), cudaMemcpyHostToDevice, stream), "H2D matrices"))
      return false;
    cudaEventRecord(pool_ev, stream);
    pool_ev_recorded = true;
    st_h2d += (double)n * sizeof(double2);
    return true;
  }

  // A planned batch of queued operations: pass descriptors + encoded tensor
  // maps (tile path) or per-op launches (simple path), with the matrix pool
  // on the device.  flush() builds a transient one over the per-handle pool
  // buffer; record_end() builds one that owns its device buffer.
  struct Program {
    bool tiled = false;
    std::vector<PassPlan> plans;
    std::vector<CUtensorMap> tmaps;
    std::vector<SimpleOp> sops;
    double2* d_mats = nullptr;   // owned when `owns` is set
    bool owns = false;
    size_t pool_elems = 0;
    int nops = 0;
    std::vector<const JitKernel*> jit;   // specialised kernel per pass (null: interpreting kernel)
    std::vector<cplx64> hmats;           // host copy of the pass matrix blocks (launch parameters)
    TileLaunch tl{};                     // launch settings of the passes
  };

  // kernels specialised to the program's passes: compiled now (recorded
  // programs, jit 2) or taken from those already compiled (flushes)
  void attach_jit(Program& pg, bool own, std::vector<cplx64>& packed) {
    if (!jit || (jit == 1 && nbits < kJitMinBits) || pg.plans.empty()) return;
    std::vector<const PassDesc*> ds;
    for (auto& pl : pg.plans) ds.push_back(&pl.desc);
    if (own || jit >= 2) {
      std::string err;
      if (!jit_prepare(ds, pg.jit, err, pg.tl.ctas_per_sm, jit_threads)) {
        jit_note(err);
        pg.jit.clear();
      }
    } else {
      jit_lookup(ds, pg.jit, true, pg.tl.ctas_per_sm, jit_threads);
    }
    bool any = false;
    for (auto* k : pg.jit) any |= k != nullptr;
    if (any) pg.hmats = std::move(packed);
    else pg.jit.clear();
  }

  bool build_program(Program& pg, bool own) {
    pg.nops = (int)ops.size();
    // passes that specialised kernels will run: two-qubit monomials stay apart
    // (renamings there) and dense one-qubit operations are normalised
    const bool spec = spec_style();
    pg.tl = launch_params(spec);
    std::vector<SchedOp> fused = fuse ? fuse_two_qubit_blocks(ops, pool, spec) : ops;
    if (spec && normalize) {
      decompose_one_qubit_ops(fused, pool);
      normalize_one_qubit_ops(fused, pool);
    }
    int maxk = 1;
    for (auto& o : fused) maxk = std::max<int>(maxk, o.k);
    pg.tiled = !eager && nbits >= 7;
    std::vector<cplx64> packed;
    const cplx64* src = pool.data();
    size_t nsrc = pool.size();
    if (!pg.tiled) {
      for (const SchedOp& o : fused) {
        SimpleOp so{};
        so.k = o.k;
        for (int j = 0; j < so.k; ++j) so.q[j] = o.q[j];
        so.mat = o.dense;
        pg.sops.push_back(so);
      }
    } else {
      SchedParams p = plan_params(spec);
      p.nbits = nbits;
      p.R = std::min(5, std::max(sp.R, maxk));
      std::string err;
      if (plan_passes(p, fused, pg.plans, err) < 0) {
        set_error(E_STATE, "scheduler: %s", err.c_str());
        return false;
      }
      pack_pass_matrices(pg.plans, pool.data(), packed);
      src = packed.data();
      nsrc = packed.size();
      pg.tmaps.resize(pg.plans.size());
      char emsg[256];
      for (size_t i = 0; i < pg.plans.size(); ++i)
        if (encode_pass_tmap(&pg.tmaps[i], d_state, nbits, pg.plans[i].desc, emsg, sizeof(emsg)) != 0) {
          set_error(E_CUDA, "%s", emsg);
          return false;
        }
    }
    pg.pool_elems = nsrc;
    if (own) {
      if (nsrc) {
        if (!cuda_ok(cudaMalloc(&pg.d_mats, nsrc * sizeof(double2)), "cudaMalloc program matrices")) return false;
        pg.owns = true;
        if (!cuda_ok(cudaMemcpy(pg.d_mats, src, nsrc * sizeof(double2), cudaMemcpyHostToDevice),
                     "H2D program matrices"))
          return false;
      }
    } else {
      if (!upload_pool(reinterpret_cast<const double2*>(src), nsrc)) return false;
      pg.d_mats = d_pool;
    }
    if (pg.tiled) attach_jit(pg, own, packed);
    return true;
  }

  bool run_program(const Program& pg) {
    if (!pg.tiled) {
      for (auto& so : pg.sops) {
        if (!cuda_ok(launch_simple_op(d_state, nbits, so, pg.d_mats, stream), "simple gate kernel")) return false;
        ++st_launches;
        ++g_launches;
        st_passes += 1;
        st_bytes += 32.0 * (double)dim;
      }
      st_ops += (double)pg.sops.size();
      return true;
    }
    for (size_t i = 0; i < pg.plans.size(); ++i) {
      cudaEvent_t e0 = nullptr, e1 = nullptr;
      if (profile) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, stream);
      }
      const PassDesc& desc = pg.plans[i].desc;
      if (i < pg.jit.size() && pg.jit[i]) {
        if (!cuda_ok(jit_launch(pg.jit[i], pg.tmaps[i], desc,
                                reinterpret_cast<const double2*>(pg.hmats.data()) + desc.mat_base, d_status, pg.tl,
                                num_sms, stream),
                     "specialised tile pass kernel"))
          return false;
        ++st_jit;
      } else if (!cuda_ok(launch_tile_pass(pg.tmaps[i], desc, pg.d_mats, d_status, pg.tl, num_sms, stream),
                          "tile pass kernel")) {
        return false;
      }
      if (profile) {
        cudaEventRecord(e1, stream);
        prof.emplace_back(e0, e1);
      }
      ++st_launches;
      ++g_launches;
      ++st_tile;
      st_passes += 1;
      st_bytes += 32.0 * (double)dim;
      st_ops += pg.plans[i].nsrc;
    }
    return true;
  }

  void clear_queue() {
    ops.clear();
    pool.clear();
  }

  bool flush() {
    if (ops.empty() || recording) return true;
    if (!select()) return false;
    ++st_flushes;
    Program pg;
    const bool ok = build_program(pg, false) && run_program(pg);
    clear_queue();
    return ok;
  }

  // flush + wait + check the device status word
  bool sync() {
    if (!flush()) return false;
    if (!cuda_ok(cudaMemcpyAsync(h_small, d_status, sizeof(int), cudaMemcpyDeviceToHost, stream), "status readback"))
      return false;
    if (!cuda_ok(cudaStreamSynchronize(stream), "stream sync")) return false;
    const int st = *reinterpret_cast<int*>(h_small);
    if (st != 0) {
      set_error(E_DEVICE, "a tile pass timed out waiting for %s (status %d); the state is invalid",
                st == DEV_WAIT_LOADED ? "a tile load" : "its consumers", st);
      cudaMemsetAsync(d_status, 0, sizeof(int), stream);
      return false;
    }
    return true;
  }

  // ------------------------------------------------------ reductions
  double* partials() { return d_scratch; }
  double* result_slot() { return reinterpret_cast<double*>(reinterpret_cast<char*>(d_scratch) + scratch_bytes - 4096); }

  bool read_doubles(const double* dsrc, size_t n, double* out) {
    if (!cuda_ok(cudaMemcpyAsync(h_small, dsrc, n * sizeof(double), cudaMemcpyDeviceToHost, stream), "D2H"))
      return false;
    if (!cuda_ok(cudaStreamSynchronize(stream), "stream sync")) return false;
    memcpy(out, h_small, n * sizeof(double));
    return true;
  }

  bool sumsq(uint64_t mask, uint64_t val, double* out) {
    if (!sync()) return false;
    g_launches += 2;
    st_launches += 2;
    if (!cuda_ok(launch_sumsq_masked(d_state, dim, mask, val, partials(), result_slot(), stream), "reduction"))
      return false;
    return read_doubles(result_slot(), 1, out);
  }

  bool diag_sum(uint64_t mask, uint64_t val, double* out) {
    if (!sync()) return false;
    const uint64_t d = 1ULL << nq;
    g_launches += 2;
    st_launches += 2;
    if (!cuda_ok(launch_diag_sum(d_state, d, mask, val, partials(), result_slot(), stream), "diagonal reduction"))
      return false;
    return read_doubles(result_slot(), 1, out);
  }

  // copy count elements produced chunk by chunk by `produce(offset, n, dst_device)`
  template <class F>
  bool chunked_readback(uint64_t count, size_t elem_bytes, int nout, double** outs, F produce) {
    if (!ensure_stage()) return false;
    const uint64_t per = kStageBytes / (elem_bytes * nout);
    for (uint64_t off = 0; off < count; off += per) {
      const uint64_t n = std::min<uint64_t>(per, count - off);
      if (!produce(off, n)) return false;
      for (int j = 0; j < nout; ++j) {
        if (!cuda_ok(cudaMemcpyAsync(h_stage, reinterpret_cast<char*>(d_stage) + (size_t)j * n * elem_bytes,
                                     n * elem_bytes, cudaMemcpyDeviceToHost, stream),
                     "D2H"))
          return false;
        if (!cuda_ok(cudaStreamSynchronize(stream), "stream sync")) return false;
        memcpy(outs[j] + off, h_stage, n * elem_bytes);
      }
    }
    return true;
  }

  bool get_split(double* re, double* im) {
    if (!sync()) return false;
    double* outs[2] = {re, im};
    return chunked_readback(dim, sizeof(double), 2, outs, [&](uint64_t off, uint64_t n) {
      double* dre = reinterpret_cast<double*>(d_stage);
      ++g_launches;
      ++st_launches;
      return cuda_ok(launch_split(d_state + off, n, dre, dre + n, stream), "split kernel");
    });
  }

  bool get_probs(double* out) {
    if (!sync()) return false;
    double* outs[1] = {out};
    return chunked_readback(dim, sizeof(double), 1, outs, [&](uint64_t off, uint64_t n) {
      ++g_launches;
      ++st_launches;
      return cuda_ok(launch_probs(d_state + off, n, reinterpret_cast<double*>(d_stage), stream), "probs kernel");
    });
  }
};

Engine* as_engine(void* h, int kind) {
  Engine* e = static_cast<Engine*>(h);
  if (e && e->kind != kind) {
    set_error(E_ARG, "handle is not a %s", kind ? "density matrix" : "state vector");
    return nullptr;
  }
  return e;
}

void load_matrix(int k, const double* re, const double* im, std::vector<cd>& m) {
  const int d = 1 << k;
  m.resize((size_t)d * d);
  for (int i = 0; i < d * d; ++i) m[i] = cd(re[i], im[i]);
}

// ---------------------------------------------- CPU core for stabilizer / MPS

struct CpuCore {
  void* lib = nullptr;
  bool tried = false;
  std::mutex mu;
  void* sym(const char* name) {
    std::lock_guard<std::mutex> g(mu);
    if (!tried) {
      tried = true;
      const char* p = getenv("IQ_CPU_CORE_LIB");
      if (p && *p) lib = dlopen(p, RTLD_NOW | RTLD_LOCAL);
    }
    return lib ? dlsym(lib, name) : nullptr;
  }
} g_cpu;

#define IQ_FORWARD(ret, name, dflt, params, args)                                             \
  ret name params {                                                                           \
    using F = ret(*) params;                                                                  \
    F f = reinterpret_cast<F>(g_cpu.sym(#name));                                              \
    if (!f) {                                                                                 \
      set_error(E_UNSUPPORTED, #name ": no CPU core loaded (set IQ_CPU_CORE_LIB to a build of " \
                               "the reference core); the GPU library provides SV/DM only");   \
      return dflt;                                                                            \
    }                                                                                         \
    return f args;                                                                            \
  }
#define IQ_FORWARD_VOID(name, params, args)                                                   \
  void name params {                                                                          \
    using F = void(*) params;                                                                 \
    F f = reinterpret_cast<F>(g_cpu.sym(#name));                                              \
    if (!f) {                                                                                 \
      set_error(E_UNSUPPORTED, #name ": no CPU core loaded (set IQ_CPU_CORE_LIB)");           \
      return;                                                                                 \
    }                                                                                         \
    f args;                                                                                   \
  }

}  // namespace

void iqb::record_error(int code, const char* msg) { set_error(code, "%s", msg); }
void iqb::count_launches(uint64_t n) { g_launches += n; }

extern "C" {

// ============================================================ errors / info

int iq_last_error(char* buf, size_t len) {
  if (buf && len) {
    strncpy(buf, t_errmsg, len - 1);
    buf[len - 1] = '\0';
  }
  return t_errcode;
}
void iq_clear_error(void) {
  t_errcode = 0;
  t_errmsg[0] = '\0';
}
const char* iq_version(void) { return "invariantq-b200 0.1 (sm_100a)"; }
uint64_t iq_kernel_launches(void) { return g_launches.load(); }

// ============================================================ state vector

void* iq_statevector_create(size_t num_qubits) {
  Engine* e = new Engine();
  if (!e->init(0, num_qubits)) {
    e->release();
    delete e;
    return nullptr;
  }
  return e;
}

void iq_statevector_free(void* sv) {
  Engine* e = as_engine(sv, 0);
  if (!e) return;
  e->select();
  e->release();
  delete e;
}

void iq_statevector_reset(void* sv) {
  Engine* e = as_engine(sv, 0);
  if (!e || !e->select()) return;
  e->reset_state();
}

void iq_statevector_apply_1q(void* sv, size_t target, const double* u_real, const double* u_imag) {
  Engine* e = as_engine(sv, 0);
  if (!e || !u_real || !u_imag) return;
  if (target >= (size_t)e->nbits) {
    set_error(E_ARG, "apply_1q: target qubit %zu out of range", target);
    return;
  }
  std::vector<cd> m;
  load_matrix(1, u_real, u_imag, m);
  const int q[1] = {(int)target};
  e->enqueue(1, q, m.data());
}

void iq_statevector_apply_2q(void* sv, size_t q0, size_t q1, const double* u_real, const double* u_imag) {
  Engine* e = as_engine(sv, 0);
  if (!e || !u_real || !u_imag) return;
  if (q0 >= (size_t)e->nbits || q1 >= (size_t)e->nbits || q0 == q1) {
    set_error(E_ARG, "apply_2q: invalid qubit indices (%zu, %zu)", q0, q1);
    return;
  }
  std::vector<cd> m;
  load_matrix(2, u_real, u_imag, m);
  const int q[2] = {(int)q1, (int)q0};   // q0 is the MSB of the local index
  e->enqueue(2, q, m.data());
}

void iq_statevector_apply_fused(void* sv, const size_t* qubits, size_t k, const double* u_real, const double* u_imag) {
  Engine* e = as_engine(sv, 0);
  if (!e || !qubits || !u_real || !u_imag) return;
  if (k == 0 || k > (size_t)kMaxK) {
    set_error(E_ARG, "apply_fused: %zu-qubit blocks are not supported (1..%d)", k, kMaxK);
    return;
  }
  for (size_t i = 0; i < k; ++i)
    if (qubits[i] >= (size_t)e->nbits) {
      set_error(E_ARG, "apply_fused: qubit %zu out of range", qubits[i]);
      return;
    }
  std::vector<cd> m;
  load_matrix((int)k, u_real, u_imag, m);
  int q[kMaxK];
  if (k == 2) {          // the reference delegates k == 2 to apply_2q: qubits[0] is the MSB
    q[0] = (int)qubits[1];
    q[1] = (int)qubits[0];
  } else {               // k == 1 and k >= 3: local index bit b <-> qubits[b]
    for (size_t i = 0; i < k; ++i) q[i] = (int)qubits[i];
  }
  e->enqueue((int)k, q, m.data());
}

double iq_statevector_measure_prob(void* sv, size_t target, int outcome) {
  Engine* e = as_engine(sv, 0);
  if (!e) return 0.0;
  if (target >= (size_t)e->nbits) {
    set_error(E_ARG, "measure_prob: target qubit out of range");
    return kNaN;
  }
  if (outcome != 0 && outcome != 1) return 0.0;
  double p = 0.0;
  if (!e->sumsq(1ULL << target, (uint64_t)outcome << target, &p)) return kNaN;
  return p;
}

static int sv_collapse(Engine* e, size_t target, int outcome) {
  double p = 0.0;
  if (!e->sumsq(1ULL << target, (uint64_t)outcome << target, &p)) return -1;
  if (p < 1e-15) {
    set_error(E_STATE, "attempted to collapse to a zero-probability state");
    return -1;
  }
  ++g_launches;
  ++e->st_launches;
  if (!cuda_ok(launch_collapse(e->d_state, e->dim, 1ULL << target, (uint64_t)outcome << target, 1.0 / std::sqrt(p),
                               e->stream),
               "collapse"))
    return -1;
  return 0;
}

int iq_statevector_measure(void* sv, size_t target, double rand_val) {
  Engine* e = as_engine(sv, 0);
  if (!e) return 0;
  if (target >= (size_t)e->nbits) {
    set_error(E_ARG, "measure: target qubit out of range");
    return -1;
  }
  double p0 = 0.0;
  if (!e->sumsq(1ULL << target, 0, &p0)) return -1;
  const int outcome = (rand_val < p0) ? 0 : 1;
  if (sv_collapse(e, target, outcome) != 0) return -1;
  return outcome;
}

void iq_statevector_reset_qubit(void* sv, size_t target, double rand_val) {
  Engine* e = as_engine(sv, 0);
  if (!e) return;
  if (target >= (size_t)e->nbits) {
    set_error(E_ARG, "reset_qubit: target qubit out of range");
    return;
  }
  const int o = iq_statevector_measure(sv, target, rand_val);
  if (o == 1) {
    const cd X[4] = {0.0, 1.0, 1.0, 0.0};
    const int q[1] = {(int)target};
    e->enqueue(1, q, X);
  }
}

void iq_statevector_get_amplitudes(void* sv, double* real_out, double* imag_out) {
  Engine* e = as_engine(sv, 0);
  if (!e || !real_out || !imag_out) return;
  e->get_split(real_out, imag_out);
}

void iq_statevector_get_probabilities(void* sv, double* probs_out) {
  Engine* e = as_engine(sv, 0);
  if (!e || !probs_out) return;
  e->get_probs(probs_out);
}

void iq_statevector_sample(void* sv, size_t num_shots, uint64_t seed, uint64_t* results_out) {
  Engine* e = as_engine(sv, 0);
  if (!e || !results_out) return;
  if (!e->sync()) return;
  if (num_shots == 0) return;
  if (num_shots > (size_t)INT32_MAX) {
    set_error(E_ARG, "sample: %zu shots exceed the supported count", num_shots);
    return;
  }
  // everything on the device (iq_sampling.cu): block sums, their prefix, the
  // mt19937_64 stream (statevector.cpp:244-245), per-shot search
  const size_t wbytes = sample_work_bytes(e->nbits, num_shots);
  void* dbuf = nullptr;
  if (!cuda_ok(cudaMallocAsync(&dbuf, wbytes + num_shots * 8 + 256, e->stream), "cudaMallocAsync sampling")) return;
  uint64_t* d_out = reinterpret_cast<uint64_t*>(static_cast<char*>(dbuf) + ((wbytes + 255) & ~(size_t)255));
  ++e->st_launches;
  cuda_ok(sample_on_device(e->d_state, e->nbits, num_shots, seed, dbuf, d_out, e->stream), "sampling") &&
      cuda_ok(cudaMemcpyAsync(results_out, d_out, num_shots * 8, cudaMemcpyDeviceToHost, e->stream), "D2H") &&
      cuda_ok(cudaStreamSynchronize(e->stream), "sync");
  cudaFreeAsync(dbuf, e->stream);
  cudaStreamSynchronize(e->stream);
}

int iq_statevector_sample_counts(void* sv, size_t num_shots, uint64_t seed, uint64_t* values_out,
                                 uint64_t* counts_out, size_t* num_unique) {
  Engine* e = as_engine(sv, 0);
  if (!e || !values_out || !counts_out || !num_unique) return -1;
  *num_unique = 0;
  if (!e->sync()) return -1;
  if (num_shots == 0) return 0;
  if (num_shots > ((size_t)1 << 30)) {
    set_error(E_ARG, "sample_counts: %zu shots exceed the supported count (2^30)", num_shots);
    return -1;
  }
  const size_t wbytes = (std::max(sample_work_bytes(e->nbits, num_shots), count_work_bytes(num_shots)) + 255) & ~(size_t)255;
  const size_t obytes = (num_shots * 8 + 255) & ~(size_t)255;
  char* dbuf = nullptr;
  if (!cuda_ok(cudaMallocAsync(reinterpret_cast<void**>(&dbuf), wbytes + 3 * obytes + 256, e->stream),
               "cudaMallocAsync sampling"))
    return -1;
  uint64_t* d_shots = reinterpret_cast<uint64_t*>(dbuf + wbytes);
  uint64_t* d_vals = reinterpret_cast<uint64_t*>(dbuf + wbytes + obytes);
  uint64_t* d_cnts = reinterpret_cast<uint64_t*>(dbuf + wbytes + 2 * obytes);
  uint64_t* d_n = reinterpret_cast<uint64_t*>(dbuf + wbytes + 3 * obytes);
  uint64_t nu = 0;
  bool ok = cuda_ok(sample_on_device(e->d_state, e->nbits, num_shots, seed, dbuf, d_shots, e->stream), "sampling") &&
            cuda_ok(count_outcomes(d_shots, num_shots, dbuf, d_vals, d_cnts, d_n, e->stream), "counts") &&
            cuda_ok(cudaMemcpyAsync(&nu, d_n, 8, cudaMemcpyDeviceToHost, e->stream), "D2H") &&
            cuda_ok(cudaStreamSynchronize(e->stream), "sync");
  if (ok)
    ok = cuda_ok(cudaMemcpyAsync(values_out, d_vals, nu * 8, cudaMemcpyDeviceToHost, e->stream), "D2H") &&
         cuda_ok(cudaMemcpyAsync(counts_out, d_cnts, nu * 8, cudaMemcpyDeviceToHost, e->stream), "D2H") &&
         cuda_ok(cudaStreamSynchronize(e->stream), "sync");
  cudaFreeAsync(dbuf, e->stream);
  cudaStreamSynchronize(e->stream);
  if (!ok) return -1;
  *num_unique = (size_t)nu;
  return 0;
}

int iq_mt64_uniform(uint64_t seed, size_t count, double* out) {
  if (!out) return -1;
  if (count == 0) return 0;
  double* d = nullptr;
  cudaStream_t st = nullptr;
  if (!cuda_ok(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "stream")) return -1;
  bool ok = cuda_ok(cudaMallocAsync(reinterpret_cast<void**>(&d), count * 8, st), "cudaMallocAsync") &&
            cuda_ok(launch_mt64_uniform(seed, count, d, st), "mt19937_64") &&
            cuda_ok(cudaMemcpyAsync(out, d, count * 8, cudaMemcpyDeviceToHost, st), "D2H") &&
            cuda_ok(cudaStreamSynchronize(st), "sync");
  if (d) cudaFreeAsync(d, st);
  cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  return ok ? 0 : -1;
}

double iq_statevector_entropy(void* sv, const size_t* qubits, size_t num_subsys_qubits) {
  Engine* e = as_engine(sv, 0);
  if (!e || !qubits) return 0.0;
  const int n = e->nbits;
  const size_t k = num_subsys_qubits;
  for (size_t i = 0; i < k; ++i)
    if (qubits[i] >= (size_t)n) {
      set_error(E_ARG, "entropy: qubit out of range");
      return kNaN;
    }
  if (k == 0 || k == (size_t)n) return 0.0;
  std::vector<int> keep;
  std::vector<bool> in(n, false);
  for (size_t i = 0; i < k; ++i) {
    if (in[qubits[i]]) {
      set_error(E_ARG, "entropy: repeated qubit");
      return kNaN;
    }
    in[qubits[i]] = true;
  }
  // the reduced state of the smaller side has the same nonzero spectrum
  if (k <= (size_t)n - k) {
    for (size_t i = 0; i < k; ++i) keep.push_back((int)qubits[i]);
  } else {
    for (int q = 0; q < n; ++q)
      if (!in[q]) keep.push_back(q);
  }
  const int kk = (int)keep.size();
  if (kk > reduced_spectrum_max_bits()) {
    set_error(E_UNSUPPORTED, "entropy: the smaller side has %d qubits; at most %d are supported", kk,
              reduced_spectrum_max_bits());
    return kNaN;
  }
  if (!e->sync()) return kNaN;
  if (kk >= 7) {
    // reduced state, tridiagonalisation and eigenvalues on the device (iq_entropy.cu)
    std::vector<double> w;
    if (!cuda_ok(reduced_spectrum(e->d_state, n, keep.data(), kk, w, e->stream), "reduced spectrum")) return kNaN;
    return entropy_from(w);
  }
  const size_t kd = (size_t)1 << kk;
  double2* d_rho = nullptr;
  if (!cuda_ok(cudaMallocAsync(&d_rho, kd * kd * sizeof(double2), e->stream), "cudaMallocAsync")) return kNaN;
  std::vector<cd> rho(kd * kd);
  ++g_launches;
  ++e->st_launches;
  bool ok = cuda_ok(launch_partial_trace(e->d_state, n, keep.data(), kk, d_rho, e->stream), "partial trace") &&
            cuda_ok(cudaMemcpyAsync(rho.data(), d_rho, kd * kd * sizeof(double2), cudaMemcpyDeviceToHost, e->stream),
                    "D2H") &&
            cuda_ok(cudaStreamSynchronize(e->stream), "sync");
  cudaFreeAsync(d_rho, e->stream);
  if (!ok) return kNaN;
  std::vector<double> w;
  if (!hermitian_eigenvalues(rho, (int)kd, w)) {
    set_error(E_STATE, "entropy: eigenvalue iteration did not converge");
    return kNaN;
  }
  return entropy_from(w);
}

void iq_statevector_expval_pauli(void* sv, const char* pauli_str, const size_t* qubits, size_t len, double* val_real,
                                 double* val_imag) {
  Engine* e = as_engine(sv, 0);
  if (!e || !pauli_str || !qubits || !val_real || !val_imag) return;
  uint64_t xm = 0, zm = 0;
  int ny = 0;
  for (size_t p = 0; p < len; ++p) {
    if (qubits[p] >= (size_t)e->nbits) {
      set_error(E_ARG, "expval_pauli: qubit out of range");
      *val_real = *val_imag = kNaN;
      return;
    }
    const uint64_t b = 1ULL << qubits[p];
    switch (pauli_str[p]) {
      case 'X': xm ^= b; break;
      case 'Y': xm ^= b; zm ^= b; ++ny; break;
      case 'Z': zm ^= b; break;
      default: break;
    }
  }
  if (!e->sync()) {
    *val_real = *val_imag = kNaN;
    return;
  }
  double2* part = reinterpret_cast<double2*>(e->partials());
  double2* res = reinterpret_cast<double2*>(e->result_slot());
  g_launches += 2;
  e->st_launches += 2;
  double out[2];
  // the reference skips amplitudes with |a_i|^2 < 1e-18 (statevector.cpp:267)
  if (!cuda_ok(launch_pauli_sum(e->d_state, e->dim, xm, zm, 1e-18, part, res, e->stream), "pauli reduction") ||
      !e->read_doubles(reinterpret_cast<double*>(res), 2, out)) {
    *val_real = *val_imag = kNaN;
    return;
  }
  // multiply by i^ny
  cd v(out[0], out[1]);
  static const cd ipow[4] = {cd(1, 0), cd(0, 1), cd(-1, 0), cd(0, -1)};
  v *= ipow[ny & 3];
  *val_real = v.real();
  *val_imag = v.imag();
}

// ------------------------------------------------------ SV additions

int iq_statevector_flush(void* sv) {
  Engine* e = as_engine(sv, 0);
  if (!e) return -1;
  return e->flush() ? 0 : -1;
}

int iq_statevector_sync(void* sv) {
  Engine* e = as_engine(sv, 0);
  if (!e) return -1;
  return e->sync() ? 0 : -1;
}

double iq_statevector_norm(void* sv) {
  Engine* e = as_engine(sv, 0);
  if (!e) return 0.0;
  double v = 0.0;
  if (!e->sumsq(0, 0, &v)) return kNaN;
  return v;
}

int iq_statevector_expval_z_all(void* sv, double* out) {
  Engine* e = as_engine(sv, 0);
  if (!e || !out) return -1;
  if (!e->sync()) return -1;
  double* res = e->result_slot();
  g_launches += 2;
  e->st_launches += 2;
  if (!cuda_ok(launch_zsums(e->d_state, e->nbits, e->partials(), res, e->stream), "z reduction")) return -1;
  std::vector<double> v(e->nbits + 1);
  if (!e->read_doubles(res, v.size(), v.data())) return -1;
  for (int q = 0; q < e->nbits; ++q) out[q] = v[0] - 2.0 * v[1 + q];
  return 0;
}

int iq_statevector_expval_pauli_sum(void* sv, size_t nterms, const double* coeffs, const char* paulis,
                                    double* val_real, double* val_imag) {
  Engine* e = as_engine(sv, 0);
  if (!e || !coeffs || !paulis || !val_real || !val_imag) return -1;
  const int n = e->nbits;
  if (!e->sync()) return -1;
  double2* part = reinterpret_cast<double2*>(e->partials());
  double2* res = reinterpret_cast<double2*>(e->result_slot());
  cd total(0.0, 0.0);
  static const cd ipow[4] = {cd(1, 0), cd(0, 1), cd(-1, 0), cd(0, -1)};
  for (size_t t = 0; t < nterms; ++t) {
    uint64_t xm = 0, zm = 0;
    int ny = 0;
    for (int q = 0; q < n; ++q) {
      const char c = paulis[t * n + q];
      const uint64_t b = 1ULL << q;
      if (c == 'X') xm ^= b;
      else if (c == 'Y') { xm ^= b; zm ^= b; ++ny; }
      else if (c == 'Z') zm ^= b;
      else if (c != 'I') {
        set_error(E_ARG, "expval_pauli_sum: invalid Pauli character");
        return -1;
      }
    }
    double out[2];
    g_launches += 2;
    e->st_launches += 2;
    if (!cuda_ok(launch_pauli_sum(e->d_state, e->dim, xm, zm, -1.0, part, res, e->stream), "pauli reduction") ||
        !e->read_doubles(reinterpret_cast<double*>(res), 2, out))
      return -1;
    total += coeffs[t] * cd(out[0], out[1]) * ipow[ny & 3];
  }
  *val_real = total.real();
  *val_imag = total.imag();
  return 0;
}

int iq_statevector_set_amplitudes(void* sv, const double* real_in, const double* imag_in) {
  Engine* e = as_engine(sv, 0);
  if (!e || !real_in || !imag_in) return -1;
  if (!e->select()) return -1;
  e->clear_queue();
  if (!e->ensure_stage()) return -1;
  const uint64_t per = kStageBytes / 16;
  for (uint64_t off = 0; off < e->dim; off += per) {
    const uint64_t n = std::min<uint64_t>(per, e->dim - off);
    double2* h = reinterpret_cast<double2*>(e->h_stage);
    if (!cuda_ok(cudaStreamSynchronize(e->stream), "sync")) return -1;
    for (uint64_t i = 0; i < n; ++i) h[i] = make_double2(real_in[off + i], imag_in[off + i]);
    if (!cuda_ok(cudaMemcpyAsync(e->d_state + off, h, n * 16, cudaMemcpyHostToDevice, e->stream), "H2D")) return -1;
  }
  return cuda_ok(cudaStreamSynchronize(e->stream), "sync") ? 0 : -1;
}

static int half_copy(void* sv, size_t bit, int value, void* d_buf, bool unpack) {
  Engine* e = as_engine(sv, 0);
  if (!e || !d_buf) return -1;
  if (bit >= (size_t)e->nbits || (value != 0 && value != 1)) {
    set_error(E_ARG, "%s_half: bit %zu / value %d out of range for %d qubits", unpack ? "unpack" : "pack", bit, value,
              e->nbits);
    return -1;
  }
  if (!e->flush()) return -1;
  ++g_launches;
  ++e->st_launches;
  if (!cuda_ok(launch_half_copy(e->d_state, e->nbits, (int)bit, value, static_cast<double2*>(d_buf), unpack, e->stream),
               "half copy"))
    return -1;
  return cuda_ok(cudaStreamSynchronize(e->stream), "sync") ? 0 : -1;
}

int iq_statevector_pack_half(void* sv, size_t bit, int value, void* d_dst) {
  return half_copy(sv, bit, value, d_dst, false);
}

int iq_statevector_unpack_half(void* sv, size_t bit, int value, const void* d_src) {
  return half_copy(sv, bit, value, const_cast<void*>(d_src), true);
}

void* iq_statevector_device_ptr(void* sv) {
  Engine* e = as_engine(sv, 0);
  if (!e) return nullptr;
  if (!e->flush()) return nullptr;
  return e->d_state;
}

void* iq_statevector_stream(void* sv) {
  Engine* e = as_engine(sv, 0);
  return e ? (void*)e->stream : nullptr;
}

size_t iq_statevector_num_qubits(void* sv) {
  Engine* e = as_engine(sv, 0);
  return e ? (size_t)e->nq : 0;
}

int iq_handle_set_option(void* h, const char* key, double v) {
  Engine* e = static_cast<Engine*>(h);
  if (!e || !key) return -1;
  if (!e->flush()) return -1;
  const int iv = (int)v;
  if (!strcmp(key, "tile_bits")) { if (iv < 7 || iv > kMaxTileBits) return -1; e->sp.M = iv; e->set_M = true; }
  else if (!strcmp(key, "chunk_bits")) { if (iv < 3 || iv > 7) return -1; e->sp.c = iv; e->set_c = true; }
  else if (!strcmp(key, "max_stages")) { if (iv < 1 || iv > kMaxStages) return -1; e->sp.max_stages = iv; }
  else if (!strcmp(key, "budget")) { if (v <= 0) return -1; e->sp.budget = v; e->set_budget = true; }
  else if (!strcmp(key, "nbuf")) { if (iv < 1 || iv > 4) return -1; e->tl.nbuf = iv; e->set_nbuf = true; }
  else if (!strcmp(key, "reg_slots")) { if (iv < 3 || iv > 5) return -1; e->sp.R = iv; }
  else if (!strcmp(key, "ctas_per_sm")) { if (iv < 1 || iv > 4) return -1; e->tl.ctas_per_sm = iv; e->set_ctas = true; }
  else if (!strcmp(key, "consumers")) { if (iv != 128) return -1; e->tl.consumers = iv; }
  else if (!strcmp(key, "eager")) e->eager = iv ? 1 : 0;
  else if (!strcmp(key, "fuse")) e->fuse = iv ? 1 : 0;
  else if (!strcmp(key, "flush_ops")) { if (iv < 1) return -1; e->flush_ops = iv; }
  else if (!strcmp(key, "profile")) e->profile = iv ? 1 : 0;
  else if (!strcmp(key, "jit")) { if (iv < 0 || iv > 2) return -1; e->jit = iv; }
  else if (!strcmp(key, "normalize")) e->normalize = iv ? 1 : 0;
  else if (!strcmp(key, "plan_style")) { if (iv < 0 || iv > 2) return -1; e->plan_style = iv; }
  else if (!strcmp(key, "jit_threads")) { if (iv != 0 && iv != 128 && iv != 256) return -1; e->jit_threads = iv; }
  else if (!strcmp(key, "inject_status")) {   // failure-path tests: as if a tile pass had timed out
    if (iv < 1 || iv > 2) return -1;
    if (!cuda_ok(cudaMemcpyAsync(e->d_status, &iv, sizeof(int), cudaMemcpyHostToDevice, e->stream), "inject status") ||
        !cuda_ok(cudaStreamSynchronize(e->stream), "stream sync"))
      return -1;
  }
  else { set_error(E_ARG, "unknown option '%s'", key); return -1; }
  return 0;
}

double iq_handle_get_option(void* h, const char* key) {
  Engine* e = static_cast<Engine*>(h);
  if (!e || !key) return kNaN;
  // the values the handle's next plan uses (its plan style's defaults where not set)
  const bool spec = e->spec_style();
  if (!strcmp(key, "tile_bits")) return e->plan_params(spec).M;
  if (!strcmp(key, "chunk_bits")) return e->plan_params(spec).c;
  if (!strcmp(key, "max_stages")) return e->sp.max_stages;
  if (!strcmp(key, "budget")) return e->plan_params(spec).budget;
  if (!strcmp(key, "nbuf")) return e->launch_params(spec).nbuf;
  if (!strcmp(key, "reg_slots")) return e->sp.R;
  if (!strcmp(key, "ctas_per_sm")) return e->launch_params(spec).ctas_per_sm;
  if (!strcmp(key, "consumers")) return e->tl.consumers;
  if (!strcmp(key, "eager")) return e->eager;
  if (!strcmp(key, "fuse")) return e->fuse;
  if (!strcmp(key, "flush_ops")) return e->flush_ops;
  if (!strcmp(key, "profile")) return e->profile;
  if (!strcmp(key, "jit")) return e->jit;
  if (!strcmp(key, "normalize")) return e->normalize;
  if (!strcmp(key, "plan_style")) return e->plan_style;
  if (!strcmp(key, "jit_threads")) return e->jit_threads;
  return kNaN;
}

int iq_handle_stats(void* h, double* out, size_t n) {
  Engine* e = static_cast<Engine*>(h);
  if (!e || !out) return 0;
  const double v[8] = {e->st_passes, e->st_ops, e->st_bytes,  e->st_launches,
                       e->st_flushes, e->st_tile, e->st_h2d, e->st_jit};
  const size_t m = std::min<size_t>(n, 8);
  for (size_t i = 0; i < m; ++i) out[i] = v[i];
  return (int)m;
}

int iq_handle_profile_read(void* h, double* ms_out, size_t max) {
  Engine* e = static_cast<Engine*>(h);
  if (!e || !ms_out) return 0;
  if (!e->select() || !cuda_ok(cudaStreamSynchronize(e->stream), "sync")) return 0;
  size_t n = 0;
  for (auto& pe : e->prof) {
    if (n < max) {
      float ms = 0.f;
      cudaEventElapsedTime(&ms, pe.first, pe.second);
      ms_out[n++] = ms;
    }
    cudaEventDestroy(pe.first);
    cudaEventDestroy(pe.second);
  }
  e->prof.clear();
  return (int)n;
}

// ============================================================ recorded programs

int iq_handle_record_begin(void* h) {
  Engine* e = static_cast<Engine*>(h);
  if (!e || !e->flush()) return -1;
  e->recording = true;
  return 0;
}

void* iq_handle_record_end(void* h) {
  Engine* e = static_cast<Engine*>(h);
  if (!e) return nullptr;
  if (!e->recording) {
    set_error(E_STATE, "record_end without record_begin");
    return nullptr;
  }
  e->recording = false;
  if (!e->select()) return nullptr;
  auto* pg = new Engine::Program();
  if (!e->build_program(*pg, true)) {
    if (pg->d_mats && pg->owns) cudaFree(pg->d_mats);
    delete pg;
    e->clear_queue();
    return nullptr;
  }
  e->clear_queue();
  return pg;
}

int iq_handle_program_run(void* h, void* prog) {
  Engine* e = static_cast<Engine*>(h);
  auto* pg = static_cast<Engine::Program*>(prog);
  if (!e || !pg) return -1;
  if (!e->flush() || !e->select()) return -1;
  return e->run_program(*pg) ? 0 : -1;
}

int iq_program_info(void* prog, double* out, size_t n) {
  auto* pg = static_cast<Engine::Program*>(prog);
  if (!pg || !out) return 0;
  double planned_cost = 0.0;
  for (auto& p : pg->plans) planned_cost += p.cost;
  const double v[4] = {(double)(pg->tiled ? pg->plans.size() : pg->sops.size()), (double)pg->nops,
                       (double)pg->pool_elems * sizeof(double2), planned_cost};
  const size_t m = std::min<size_t>(n, 4);
  for (size_t i = 0; i < m; ++i) out[i] = v[i];
  return (int)m;
}

int iq_program_pass_info(void* prog, size_t i, double* out, size_t n) {
  auto* pg = static_cast<Engine::Program*>(prog);
  if (!pg || !out || !pg->tiled || i >= pg->plans.size()) return 0;
  const PassPlan& p = pg->plans[i];
  const double v[6] = {(double)p.desc.nops, p.cost, (double)p.desc.nstages, (double)p.desc.M, (double)p.desc.c,
                       (double)p.desc.ntiles};
  const size_t m = std::min<size_t>(n, 6);
  for (size_t k = 0; k < m; ++k) out[k] = v[k];
  return (int)m;
}

void iq_program_free(void* prog) {
  auto* pg = static_cast<Engine::Program*>(prog);
  if (!pg) return;
  if (pg->owns && pg->d_mats) cudaFree(pg->d_mats);
  delete pg;
}

// ============================================================ specialised kernels

int iq_jit_info(double* out, size_t n, char* note, size_t note_len) {
  uint64_t compiled = 0, disk = 0;
  jit_counters(&compiled, &disk);
  const double v[2] = {(double)compiled, (double)disk};
  const size_t m = out ? std::min<size_t>(n, 2) : 0;
  for (size_t i = 0; i < m; ++i) out[i] = v[i];
  if (note && note_len) {
    std::lock_guard<std::mutex> lk(g_jit_mu);
    snprintf(note, note_len, "%s", g_jit_note.c_str());
  }
  return (int)m;
}

int iq_jit_wait(double timeout_s) { return jit_wait(timeout_s > 0 ? timeout_s : 0.0) ? 0 : -1; }

// ============================================================ density matrix

void* iq_density_matrix_create(size_t num_qubits) {
  Engine* e = new Engine();
  if (!e->init(1, num_qubits)) {
    e->release();
    delete e;
    return nullptr;
  }
  return e;
}

void iq_density_matrix_free(void* dm) {
  Engine* e = as_engine(dm, 1);
  if (!e) return;
  e->select();
  e->release();
  delete e;
}

void iq_density_matrix_reset(void* dm) {
  Engine* e = as_engine(dm, 1);
  if (!e || !e->select()) return;
  e->reset_state();
}

// rho <- U rho U^dagger: U on the row bits (n + q), conj(U) on the column bits (q)
static void dm_unitary(Engine* e, int k, const int* q_lsb, const std::vector<cd>& U) {
  int rows[kMaxK], cols[kMaxK];
  for (int i = 0; i < k; ++i) {
    rows[i] = e->nq + q_lsb[i];
    cols[i] = q_lsb[i];
  }
  std::vector<cd> Uc(U.size());
  for (size_t i = 0; i < U.size(); ++i) Uc[i] = std::conj(U[i]);
  if (!e->enqueue(k, rows, U.data())) return;
  e->enqueue(k, cols, Uc.data());
}

void iq_density_matrix_apply_1q_unitary(void* dm, size_t target, const double* u_real, const double* u_imag) {
  Engine* e = as_engine(dm, 1);
  if (!e || !u_real || !u_imag) return;
  if (target >= (size_t)e->nq) {
    set_error(E_ARG, "apply_1q_unitary: target qubit out of range");
    return;
  }
  std::vector<cd> U;
  load_matrix(1, u_real, u_imag, U);
  const int q[1] = {(int)target};
  dm_unitary(e, 1, q, U);
}

void iq_density_matrix_apply_2q_unitary(void* dm, size_t q0, size_t q1, const double* u_real, const double* u_imag) {
  Engine* e = as_engine(dm, 1);
  if (!e || !u_real || !u_imag) return;
  if (q0 >= (size_t)e->nq || q1 >= (size_t)e->nq || q0 == q1) {
    set_error(E_ARG, "apply_2q_unitary: invalid qubit indices");
    return;
  }
  std::vector<cd> U;
  load_matrix(2, u_real, u_imag, U);
  const int q[2] = {(int)q1, (int)q0};
  dm_unitary(e, 2, q, U);
}

// Kraus channel on k qubits (LSB-first list) as one 2k-bit superoperator
// S = sum_j K_j (x) conj(K_j) acting on (column bits, row bits).
static void dm_kraus(Engine* e, int k, const int* q_lsb, size_t nk, const double* kr, const double* ki) {
  const int d = 1 << k, D = d * d;
  std::vector<cd> S((size_t)D * D, cd(0.0, 0.0));
  for (size_t j = 0; j < nk; ++j) {
    const double* r = kr + j * d * d;
    const double* im = ki + j * d * d;
    for (int ro = 0; ro < d; ++ro)
      for (int co = 0; co < d; ++co)
        for (int ri = 0; ri < d; ++ri)
          for (int ci = 0; ci < d; ++ci) {
            const cd a(r[ro * d + ri], im[ro * d + ri]);
            const cd b(r[co * d + ci], im[co * d + ci]);
            // local index: column bits low, row bits high
            S[(size_t)(ro * d + co) * D + (ri * d + ci)] += a * std::conj(b);
          }
  }
  int bits[2 * kMaxK];
  for (int i = 0; i < k; ++i) {
    bits[i] = q_lsb[i];
    bits[k + i] = e->nq + q_lsb[i];
  }
  e->enqueue(2 * k, bits, S.data());
}

void iq_density_matrix_apply_kraus_1q(void* dm, size_t target, size_t num_kraus, const double* k_real,
                                      const double* k_imag) {
  Engine* e = as_engine(dm, 1);
  if (!e || !k_real || !k_imag) return;
  if (target >= (size_t)e->nq) {
    set_error(E_ARG, "apply_kraus_1q: target qubit out of range");
    return;
  }
  const int q[1] = {(int)target};
  dm_kraus(e, 1, q, num_kraus, k_real, k_imag);
}

void iq_density_matrix_apply_kraus_2q(void* dm, size_t q0, size_t q1, size_t num_kraus, const double* k_real,
                                      const double* k_imag) {
  Engine* e = as_engine(dm, 1);
  if (!e || !k_real || !k_imag) return;
  if (q0 >= (size_t)e->nq || q1 >= (size_t)e->nq || q0 == q1) {
    set_error(E_ARG, "apply_kraus_2q: invalid qubit indices");
    return;
  }
  const int q[2] = {(int)q1, (int)q0};
  dm_kraus(e, 2, q, num_kraus, k_real, k_imag);
}

void iq_density_matrix_get_elements(void* dm, double* real_out, double* imag_out) {
  Engine* e = as_engine(dm, 1);
  if (!e || !real_out || !imag_out) return;
  e->get_split(real_out, imag_out);
}

double iq_density_matrix_trace(void* dm) {
  Engine* e = as_engine(dm, 1);
  if (!e) return 0.0;
  double v = 0.0;
  if (!e->diag_sum(0, 0, &v)) return kNaN;
  return v;
}

double iq_density_matrix_purity(void* dm) {
  Engine* e = as_engine(dm, 1);
  if (!e) return 0.0;
  double v = 0.0;
  if (!e->sumsq(0, 0, &v)) return kNaN;
  return v;
}

double iq_density_matrix_measure_prob(void* dm, size_t target, int outcome) {
  Engine* e = as_engine(dm, 1);
  if (!e) return 0.0;
  if (target >= (size_t)e->nq) {
    set_error(E_ARG, "measure_prob: target qubit out of range");
    return kNaN;
  }
  if (outcome != 0 && outcome != 1) return 0.0;
  double p = 0.0;
  if (!e->diag_sum(1ULL << target, (uint64_t)outcome << target, &p)) return kNaN;
  return p > 0.0 ? p : 0.0;
}

double iq_density_matrix_entropy(void* dm) {
  Engine* e = as_engine(dm, 1);
  if (!e) return 0.0;
  if (!e->sync()) return kNaN;
  const uint64_t d = 1ULL << e->nq;
  if (d > 64) {   // the reference's diagonal approximation (density_matrix.cpp:312-320)
    g_launches += 2;
    e->st_launches += 2;
    double v = 0.0;
    if (!cuda_ok(launch_diag_entropy(e->d_state, d, e->partials(), e->result_slot(), e->stream), "entropy") ||
        !e->read_doubles(e->result_slot(), 1, &v))
      return kNaN;
    return v;
  }
  std::vector<cd> rho(d * d);
  if (!cuda_ok(cudaMemcpyAsync(rho.data(), e->d_state, d * d * 16, cudaMemcpyDeviceToHost, e->stream), "D2H") ||
      !cuda_ok(cudaStreamSynchronize(e->stream), "sync"))
    return kNaN;
  std::vector<double> w;
  if (!hermitian_eigenvalues(rho, (int)d, w)) {
    set_error(E_STATE, "entropy: eigenvalue iteration did not converge");
    return kNaN;
  }
  return entropy_from(w);
}

int iq_density_matrix_measure(void* dm, size_t target, double rand_val) {
  Engine* e = as_engine(dm, 1);
  if (!e) return 0;
  if (target >= (size_t)e->nq) {
    set_error(E_ARG, "measure: target qubit out of range");
    return -1;
  }
  double p0 = 0.0;
  if (!e->diag_sum(1ULL << target, 0, &p0)) return -1;
  if (p0 < 0.0) p0 = 0.0;
  const int outcome = (rand_val < p0) ? 0 : 1;
  double p = p0;
  if (outcome == 1) {
    if (!e->diag_sum(1ULL << target, 1ULL << target, &p)) return -1;
    if (p < 0.0) p = 0.0;
  }
  if (p < 1e-15) {
    set_error(E_STATE, "cannot collapse to a zero-probability outcome");
    return -1;
  }
  ++g_launches;
  ++e->st_launches;
  if (!cuda_ok(launch_dm_collapse(e->d_state, e->nq, 1ULL << target, (uint64_t)outcome << target, 1.0 / p, e->stream),
               "collapse"))
    return -1;
  return outcome;
}

void iq_density_matrix_reset_qubit(void* dm, size_t target) {
  Engine* e = as_engine(dm, 1);
  if (!e) return;
  if (target >= (size_t)e->nq) {
    set_error(E_ARG, "reset_qubit: target qubit out of range");
    return;
  }
  // Kraus {|0><0|, |0><1|} (density_matrix.cpp:258-269)
  const double kr[8] = {1, 0, 0, 0, 0, 1, 0, 0}, ki[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int q[1] = {(int)target};
  dm_kraus(e, 1, q, 2, kr, ki);
}

int iq_density_matrix_flush(void* dm) {
  Engine* e = as_engine(dm, 1);
  if (!e) return -1;
  return e->flush() ? 0 : -1;
}

void iq_density_matrix_get_diagonal(void* dm, double* out) {
  Engine* e = as_engine(dm, 1);
  if (!e || !out) return;
  if (!e->sync()) return;
  const uint64_t d = 1ULL << e->nq;
  // strided copy of the real parts of rho_ii (stride (d + 1) complex = (d + 1) * 16 bytes)
  cudaMemcpy2DAsync(out, sizeof(double), e->d_state, (d + 1) * 16, sizeof(double), d, cudaMemcpyDeviceToHost,
                    e->stream);
  cudaStreamSynchronize(e->stream);
}

void* iq_density_matrix_device_ptr(void* dm) {
  Engine* e = as_engine(dm, 1);
  if (!e) return nullptr;
  if (!e->flush()) return nullptr;
  return e->d_state;
}

// ============================================================ stabilizer / MPS (forwarded)

IQ_FORWARD(void*, iq_stabilizer_create, nullptr, (size_t n), (n))
IQ_FORWARD_VOID(iq_stabilizer_free, (void* s), (s))
IQ_FORWARD_VOID(iq_stabilizer_reset, (void* s), (s))
IQ_FORWARD_VOID(iq_stabilizer_reset_qubit, (void* s, size_t a, double r), (s, a, r))
IQ_FORWARD_VOID(iq_stabilizer_apply_h, (void* s, size_t a), (s, a))
IQ_FORWARD_VOID(iq_stabilizer_apply_s, (void* s, size_t a), (s, a))
IQ_FORWARD_VOID(iq_stabilizer_apply_sdg, (void* s, size_t a), (s, a))
IQ_FORWARD_VOID(iq_stabilizer_apply_cnot, (void* s, size_t a, size_t b), (s, a, b))
IQ_FORWARD_VOID(iq_stabilizer_apply_cz, (void* s, size_t a, size_t b), (s, a, b))
IQ_FORWARD_VOID(iq_stabilizer_apply_swap, (void* s, size_t a, size_t b), (s, a, b))
IQ_FORWARD_VOID(iq_stabilizer_apply_x, (void* s, size_t a), (s, a))
IQ_FORWARD_VOID(iq_stabilizer_apply_y, (void* s, size_t a), (s, a))
IQ_FORWARD_VOID(iq_stabilizer_apply_z, (void* s, size_t a), (s, a))
IQ_FORWARD(int, iq_stabilizer_measure, 0, (void* s, size_t a, double r), (s, a, r))
IQ_FORWARD_VOID(iq_stabilizer_to_string, (void* s, char* b, size_t m), (s, b, m))
IQ_FORWARD(void*, iq_mps_create, nullptr, (size_t n, size_t bd, double cut), (n, bd, cut))
IQ_FORWARD_VOID(iq_mps_free, (void* m), (m))
IQ_FORWARD_VOID(iq_mps_reset, (void* m), (m))
IQ_FORWARD_VOID(iq_mps_apply_1q, (void* m, size_t t, const double* r, const double* i), (m, t, r, i))
IQ_FORWARD_VOID(iq_mps_apply_2q, (void* m, size_t a, size_t b, const double* r, const double* i), (m, a, b, r, i))
IQ_FORWARD(double, iq_mps_entropy, 0.0, (void* m, size_t b), (m, b))
IQ_FORWARD_VOID(iq_mps_to_statevector, (void* m, double* r, double* i), (m, r, i))
IQ_FORWARD(int, iq_mps_measure, 0, (void* m, size_t t, double r), (m, t, r))

}  // extern "C"
