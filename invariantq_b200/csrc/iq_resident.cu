// iq_resident.cu -- persistent executor for the small circuits of a gradient
// batch.
//
// A circuit of n <= kResidentMaxQubits qubits keeps psi and lambda (2 x 16 B x
// 2^n, 128 KiB at 12 qubits) in one CTA's shared memory for its whole adjoint
// gradient: forward gate by gate, lambda = H psi, then the backward sweep
// (per rotation: the term Im<lambda|P|psi> and the inverse rotation on both
// vectors in one sweep over the pairs), with no global-memory traffic but the
// parameters in and the energy and gradient out.  All (circuit, parameter set)
// items of a batch are the entries of a device-side queue, largest first; one
// persistent launch of as many CTAs as fit the GPU pops them with an atomic
// counter until the queue is empty (no CTA ever waits for another).  The
// launch, with the parameter upload before it and the result download after
// it, is captured once per batch structure as a CUDA graph and replayed.
//
// Rotations are exp(-i t P / 2); U3 = e^{i(phi+lambda)/2} Rz(phi) Ry(theta)
// Rz(lambda) with the global phase dropped, P(l) as Rz(l) (the energy does not
// see a global phase) -- the conventions of the tile-pass executor
// (ansatz_forward / ansatz_backward in iq_sched.cpp).  The gradient term and
// the inverse rotation are the expressions the tile kernels use
// (grad_term / unrotate in iq_pipe.cuh).  Each item is computed by one CTA in
// a fixed order: results are reproducible bit for bit.
#include "iq_resident.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

#include "iq_pipe.cuh"

namespace iqb {
namespace {

constexpr int kResThreads = 256;

struct ResCirc {
  int n, nops, op0, nparams;
  int ngroups, g0, t0, pad;
  uint64_t param0;   // first parameter of set 0 in the parameter array
  uint64_t e0;       // first energy slot
  uint64_t grad0;    // first gradient slot (set-major, nparams per set)
};

__device__ __forceinline__ uint32_t insert0(uint32_t p, int q) {
  const uint32_t lo = p & ((1u << q) - 1u);
  return ((p >> q) << (q + 1)) | lo;
}

// forward (sign = -1) or inverse (sign = +1) rotation exp(-/+ i t P / 2) on one
// pair, as the structured matrix unrotate() takes
template <int GEN>
__device__ __forceinline__ void rot_pair(double c, double s, double2& x0, double2& x1) {
  double2 y0, y1;
  if (GEN == 2) unrotate<2>(x0, x1, y0, y1, make_double2(c, s), make_double2(0.0, 0.0), make_double2(c, -s));
  else if (GEN == 1) unrotate<1>(x0, x1, y0, y1, make_double2(c, 0.0), make_double2(s, 0.0), make_double2(c, 0.0));
  else unrotate<0>(x0, x1, y0, y1, make_double2(c, 0.0), make_double2(0.0, s), make_double2(c, 0.0));
  x0 = y0;
  x1 = y1;
}

// rotation generator (0 X, 1 Y, 2 Z) and parameter of the rotations of a gate, forward order
__device__ __forceinline__ int gate_rotations(const int4 op, int gen[3], int par[3]) {
  switch (op.x) {
    case GATE_RX: gen[0] = 0; par[0] = op.w; return 1;
    case GATE_RY: gen[0] = 1; par[0] = op.w; return 1;
    case GATE_RZ: case GATE_P: gen[0] = 2; par[0] = op.w; return 1;
    case GATE_U3: gen[0] = 2; par[0] = op.w + 2; gen[1] = 1; par[1] = op.w; gen[2] = 2; par[2] = op.w + 1; return 3;
    default: return 0;
  }
}

// a fixed one-qubit gate (or its inverse) on one pair
__device__ __forceinline__ void fixed1_pair(int kind, bool inverse, double2& x0, double2& x1) {
  if (kind == GATE_H) {
    const double r = 0.70710678118654752440;
    const double2 a = x0, b = x1;
    x0 = make_double2(r * (a.x + b.x), r * (a.y + b.y));
    x1 = make_double2(r * (a.x - b.x), r * (a.y - b.y));
  } else if (kind == GATE_X) {
    const double2 t = x0;
    x0 = x1;
    x1 = t;
  } else {   // SX = 1/2 [[1+i, 1-i], [1-i, 1+i]]; its inverse is the conjugate
    const double sg = inverse ? -1.0 : 1.0;
    const double2 a = x0, b = x1;
    // (1 + i sg) a / 2 + (1 - i sg) b / 2 and the mirror
    x0 = make_double2(0.5 * (a.x - sg * a.y + b.x + sg * b.y), 0.5 * (a.y + sg * a.x + b.y - sg * b.x));
    x1 = make_double2(0.5 * (a.x + sg * a.y + b.x - sg * b.y), 0.5 * (a.y - sg * a.x + b.y + sg * b.x));
  }
}

// block sum in a fixed order (warps by shuffles, then the warp sums in order); valid in thread 0
__device__ __forceinline__ double block_sum_fixed(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < kResThreads / 32; ++w) t += red[w];
  __syncthreads();
  return t;
}

template <int GEN>
__device__ __forceinline__ double backward_rotation(double2* psi, double2* lam, uint32_t pairs, int q, double c,
                                                    double s) {
  double acc = 0.0;
  for (uint32_t p = threadIdx.x; p < pairs; p += kResThreads) {
    const uint32_t i0 = insert0(p, q), i1 = i0 | (1u << q);
    double2 p0 = psi[i0], p1 = psi[i1], l0 = lam[i0], l1 = lam[i1];
    acc += grad_term<GEN>(p0, p1, l0, l1);
    rot_pair<GEN>(c, s, p0, p1);
    rot_pair<GEN>(c, s, l0, l1);
    psi[i0] = p0; psi[i1] = p1; lam[i0] = l0; lam[i1] = l1;
  }
  return acc;
}

template <int GEN>
__device__ __forceinline__ void forward_rotation(double2* psi, uint32_t pairs, int q, double c, double s) {
  for (uint32_t p = threadIdx.x; p < pairs; p += kResThreads) {
    const uint32_t i0 = insert0(p, q), i1 = i0 | (1u << q);
    double2 a = psi[i0], b = psi[i1];
    rot_pair<GEN>(c, -s, a, b);
    psi[i0] = a;
    psi[i1] = b;
  }
}

// fixed gate on one vector (inverse for the backward sweep; all but SX are self-inverse)
__device__ void fixed_gate(double2* v, uint32_t dim, const int4 op, bool inverse) {
  if (op.x == GATE_CZ) {
    const uint32_t m = (1u << op.y) | (1u << op.z);
    for (uint32_t x = threadIdx.x; x < dim; x += kResThreads)
      if ((x & m) == m) v[x] = make_double2(-v[x].x, -v[x].y);
    return;
  }
  if (op.x == GATE_CX) {   // control op.y, target op.z
    for (uint32_t p = threadIdx.x; p < dim / 2; p += kResThreads) {
      const uint32_t i0 = insert0(p, op.z);
      if ((i0 >> op.y) & 1u) {
        const uint32_t i1 = i0 | (1u << op.z);
        const double2 t = v[i0];
        v[i0] = v[i1];
        v[i1] = t;
      }
    }
    return;
  }
  for (uint32_t p = threadIdx.x; p < dim / 2; p += kResThreads) {
    const uint32_t i0 = insert0(p, op.y), i1 = i0 | (1u << op.y);
    double2 a = v[i0], b = v[i1];
    fixed1_pair(op.x, inverse, a, b);
    v[i0] = a;
    v[i1] = b;
  }
}

__global__ void __launch_bounds__(kResThreads) resident_adjoint_kernel(
    const ResCirc* __restrict__ circs, const int2* __restrict__ items, int nitems, int* __restrict__ head,
    const int4* __restrict__ ops, const uint64_t* __restrict__ gx, const int* __restrict__ gfirst,
    const uint64_t* __restrict__ tz, const double2* __restrict__ tc, const double* __restrict__ params,
    double* __restrict__ e_out, double* __restrict__ g_out, int dim_max) {
  extern __shared__ __align__(16) unsigned char res_smem[];
  double2* const psi = reinterpret_cast<double2*>(res_smem);
  double* const grads = reinterpret_cast<double*>(psi + 2 * (size_t)dim_max);
  __shared__ double red[kResThreads / 32];
  __shared__ int s_item;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_item = atomicAdd(head, 1);
    __syncthreads();
    const int it = s_item;
    __syncthreads();
    if (it >= nitems) return;
    const int2 w = items[it];
    const ResCirc C = circs[w.x];
    const uint32_t dim = 1u << C.n, pairs = dim >> 1;
    double2* const lam = psi + dim;
    const double* th = params + C.param0 + (uint64_t)w.y * C.nparams;
    for (uint32_t x = tid; x < dim; x += kResThreads) psi[x] = make_double2(x == 0 ? 1.0 : 0.0, 0.0);
    for (int p = tid; p < C.nparams; p += kResThreads) grads[p] = 0.0;
    __syncthreads();
    // forward
    for (int i = 0; i < C.nops; ++i) {
      const int4 op = ops[C.op0 + i];
      int gen[3], par[3];
      const int nr = gate_rotations(op, gen, par);
      for (int r = 0; r < nr; ++r) {
        double s, c;
        sincos(0.5 * th[par[r]], &s, &c);
        if (gen[r] == 0) forward_rotation<0>(psi, pairs, op.y, c, s);
        else if (gen[r] == 1) forward_rotation<1>(psi, pairs, op.y, c, s);
        else forward_rotation<2>(psi, pairs, op.y, c, s);
        __syncthreads();
      }
      if (!nr) {
        fixed_gate(psi, dim, op, false);
        __syncthreads();
      }
    }
    // lambda = H psi and the energy
    double e = 0.0;
    for (uint32_t x = tid; x < dim; x += kResThreads) {
      const double2 px = psi[x];
      double2 l = make_double2(0.0, 0.0);
      for (int g = 0; g < C.ngroups; ++g) {
        const uint64_t xm = gx[C.g0 + g];
        const uint32_t src = x ^ (uint32_t)xm;
        const double2 a = psi[src];
        double2 f = make_double2(0.0, 0.0);
        for (int t = gfirst[C.g0 + g]; t < gfirst[C.g0 + g + 1]; ++t) {
          const double2 cf = tc[C.t0 + t];
          if (__popcll((uint64_t)src & tz[C.t0 + t]) & 1) { f.x -= cf.x; f.y -= cf.y; }
          else { f.x += cf.x; f.y += cf.y; }
        }
        l = cfma(l, f, a);
      }
      lam[x] = l;
      e += px.x * l.x + px.y * l.y;
    }
    e = block_sum_fixed(e, red);   // ends with a barrier: lambda complete
    if (tid == 0) e_out[C.e0 + w.y] = e;
    // backward: per rotation (last first) the term, then the inverse on both vectors
    for (int i = C.nops - 1; i >= 0; --i) {
      const int4 op = ops[C.op0 + i];
      int gen[3], par[3];
      const int nr = gate_rotations(op, gen, par);
      for (int r = nr - 1; r >= 0; --r) {
        double s, c;
        sincos(0.5 * th[par[r]], &s, &c);
        double acc;
        if (gen[r] == 0) acc = backward_rotation<0>(psi, lam, pairs, op.y, c, s);
        else if (gen[r] == 1) acc = backward_rotation<1>(psi, lam, pairs, op.y, c, s);
        else acc = backward_rotation<2>(psi, lam, pairs, op.y, c, s);
        acc = block_sum_fixed(acc, red);
        if (tid == 0) grads[par[r]] += acc;
      }
      if (!nr) {
        fixed_gate(psi, dim, op, true);
        fixed_gate(lam, dim, op, true);
        __syncthreads();
      }
    }
    __syncthreads();
    for (int p = tid; p < C.nparams; p += kResThreads) g_out[C.grad0 + (uint64_t)w.y * C.nparams + p] = grads[p];
    __syncthreads();
  }
}

size_t smem_bytes(int nmax, int pmax) { return 2 * (sizeof(double2) << nmax) + (size_t)pmax * sizeof(double); }

// one batch structure: device arrays, pinned staging and the captured graph
struct Plan {
  int dev = -1;
  cudaStream_t stream = nullptr;
  cudaGraphExec_t exec = nullptr;
  size_t nparams_total = 0, nenergies = 0, ngrads = 0;
  std::vector<void*> dbufs;
  double* h_params = nullptr;
  double* h_e = nullptr;
  double* h_g = nullptr;
  ~Plan() {
    if (stream) cudaStreamSynchronize(stream);
    if (exec) cudaGraphExecDestroy(exec);
    for (void* p : dbufs) cudaFree(p);
    if (h_params) cudaFreeHost(h_params);
    if (h_e) cudaFreeHost(h_e);
    if (h_g) cudaFreeHost(h_g);
    if (stream) cudaStreamDestroy(stream);
  }
};

uint64_t fnv(uint64_t h, const void* p, size_t n) {
  const unsigned char* b = static_cast<const unsigned char*>(p);
  for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

uint64_t structure_key(int dev, const std::vector<ResidentJob>& jobs) {
  uint64_t h = 1469598103934665603ull;
  h = fnv(h, &dev, sizeof(dev));
  for (const ResidentJob& j : jobs) {
    const uint64_t hdr[3] = {(uint64_t)j.n, (uint64_t)j.nparams, (uint64_t)j.nsets};
    h = fnv(h, hdr, sizeof(hdr));
    h = fnv(h, j.ops->data(), j.ops->size() * sizeof(AnsatzOp));
    h = fnv(h, j.groups, sizeof(HamTerms));
    h = fnv(h, j.zmask->data(), j.zmask->size() * sizeof(uint64_t));
    h = fnv(h, j.coef->data(), j.coef->size() * sizeof(double2));
  }
  return h;
}

std::mutex g_mu;
std::map<uint64_t, std::unique_ptr<Plan>>* g_plans = new std::map<uint64_t, std::unique_ptr<Plan>>();
constexpr size_t kMaxPlans = 16;

bool cuda_ok(cudaError_t e, const char* what, std::string& err) {
  if (e == cudaSuccess) return true;
  cudaGetLastError();
  err = std::string("resident executor: ") + what + ": " + cudaGetErrorString(e);
  return false;
}

template <class T>
bool upload(Plan& p, const std::vector<T>& v, T** out, std::string& err) {
  void* d = nullptr;
  if (!cuda_ok(cudaMalloc(&d, std::max<size_t>(v.size(), 1) * sizeof(T)), "cudaMalloc", err)) return false;
  p.dbufs.push_back(d);
  if (!v.empty() && !cuda_ok(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "H2D", err))
    return false;
  *out = static_cast<T*>(d);
  return true;
}

std::unique_ptr<Plan> build(int dev, const std::vector<ResidentJob>& jobs, std::string& err) {
  std::unique_ptr<Plan> p(new Plan);
  p->dev = dev;
  std::vector<ResCirc> circs;
  std::vector<int2> items;
  std::vector<int4> ops;
  std::vector<uint64_t> gx, tz;
  std::vector<int> gfirst;
  std::vector<double2> tc;
  std::vector<std::pair<double, int2>> order;
  int nmax = 1, pmax = 1;
  for (size_t c = 0; c < jobs.size(); ++c) {
    const ResidentJob& j = jobs[c];
    ResCirc rc{};
    rc.n = j.n;
    rc.nops = (int)j.ops->size();
    rc.op0 = (int)ops.size();
    rc.nparams = j.nparams;
    rc.ngroups = j.groups->ngroups;
    rc.g0 = (int)gx.size();
    rc.t0 = (int)tz.size();
    rc.param0 = p->nparams_total;
    rc.e0 = p->nenergies;
    rc.grad0 = p->ngrads;
    for (const AnsatzOp& o : *j.ops) ops.push_back(make_int4(o.kind, o.q0, o.q1, o.param));
    for (int g = 0; g < rc.ngroups; ++g) {
      gx.push_back(j.groups->xmask[g]);
      gfirst.push_back(j.groups->first[g]);
    }
    gfirst.push_back(j.groups->first[rc.ngroups]);
    // gfirst is indexed by g0 + g with one closing entry per circuit: keep the
    // group arrays aligned by padding gx with the closing slot
    gx.push_back(0);
    tz.insert(tz.end(), j.zmask->begin(), j.zmask->end());
    tc.insert(tc.end(), j.coef->begin(), j.coef->end());
    p->nparams_total += j.nsets * (size_t)j.nparams;
    p->nenergies += j.nsets;
    p->ngrads += j.nsets * (size_t)j.nparams;
    nmax = std::max(nmax, j.n);
    pmax = std::max(pmax, j.nparams);
    for (size_t s = 0; s < j.nsets; ++s)
      order.push_back({std::ldexp((double)(j.ops->size() + 1), j.n), make_int2((int)c, (int)s)});
    circs.push_back(rc);
  }
  // largest items first, ties in input order
  std::stable_sort(order.begin(), order.end(),
                   [](const std::pair<double, int2>& a, const std::pair<double, int2>& b) { return a.first > b.first; });
  for (auto& o : order) items.push_back(o.second);

  if (!cuda_ok(cudaSetDevice(dev), "cudaSetDevice", err) ||
      !cuda_ok(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "stream", err))
    return nullptr;
  ResCirc* d_circs;
  int2* d_items;
  int4* d_ops;
  uint64_t *d_gx, *d_tz;
  int* d_gfirst;
  double2* d_tc;
  if (!upload(*p, circs, &d_circs, err) || !upload(*p, items, &d_items, err) || !upload(*p, ops, &d_ops, err) ||
      !upload(*p, gx, &d_gx, err) || !upload(*p, gfirst, &d_gfirst, err) || !upload(*p, tz, &d_tz, err) ||
      !upload(*p, tc, &d_tc, err))
    return nullptr;
  std::vector<double> zeros_p(p->nparams_total), zeros_e(p->nenergies), zeros_g(p->ngrads);
  std::vector<int> zero_head(1, 0);
  double *d_params, *d_e, *d_g;
  int* d_head;
  if (!upload(*p, zeros_p, &d_params, err) || !upload(*p, zeros_e, &d_e, err) || !upload(*p, zeros_g, &d_g, err) ||
      !upload(*p, zero_head, &d_head, err))
    return nullptr;
  if (!cuda_ok(cudaMallocHost(&p->h_params, std::max<size_t>(p->nparams_total, 1) * 8), "pinned", err) ||
      !cuda_ok(cudaMallocHost(&p->h_e, std::max<size_t>(p->nenergies, 1) * 8), "pinned", err) ||
      !cuda_ok(cudaMallocHost(&p->h_g, std::max<size_t>(p->ngrads, 1) * 8), "pinned", err))
    return nullptr;

  const size_t smem = smem_bytes(nmax, pmax);
  if (!cuda_ok(cudaFuncSetAttribute(resident_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
               "shared-memory limit", err))
    return nullptr;
  int per_sm = 0, sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (!cuda_ok(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, resident_adjoint_kernel, kResThreads, smem),
               "occupancy", err))
    return nullptr;
  if (per_sm < 1) { err = "resident executor: a CTA does not fit an SM"; return nullptr; }
  const int grid = (int)std::min<size_t>(items.size(), (size_t)per_sm * sms);

  // capture: parameters up, queue head reset, the persistent launch, results down
  cudaGraph_t graph = nullptr;
  if (!cuda_ok(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal), "begin capture", err))
    return nullptr;
  cudaMemcpyAsync(d_params, p->h_params, std::max<size_t>(p->nparams_total, 1) * 8, cudaMemcpyHostToDevice, p->stream);
  cudaMemsetAsync(d_head, 0, sizeof(int), p->stream);
  resident_adjoint_kernel<<<grid, kResThreads, smem, p->stream>>>(d_circs, d_items, (int)items.size(), d_head, d_ops,
                                                                  d_gx, d_gfirst, d_tz, d_tc, d_params, d_e, d_g,
                                                                  1 << nmax);
  cudaMemcpyAsync(p->h_e, d_e, std::max<size_t>(p->nenergies, 1) * 8, cudaMemcpyDeviceToHost, p->stream);
  cudaMemcpyAsync(p->h_g, d_g, std::max<size_t>(p->ngrads, 1) * 8, cudaMemcpyDeviceToHost, p->stream);
  const cudaError_t ce = cudaStreamEndCapture(p->stream, &graph);
  if (!cuda_ok(ce, "end capture", err)) {
    if (graph) cudaGraphDestroy(graph);
    return nullptr;
  }
  const cudaError_t ie = cudaGraphInstantiate(&p->exec, graph, 0);
  cudaGraphDestroy(graph);
  if (!cuda_ok(ie, "graph instantiate", err)) return nullptr;
  return p;
}

}  // namespace

bool resident_run(int dev, const std::vector<ResidentJob>& jobs, std::string& err, double* host_ms) {
  if (jobs.empty()) return true;
  for (const ResidentJob& j : jobs)
    if (j.n < 1 || j.n > kResidentMaxQubits || j.nparams > kResidentMaxParams || !j.ops || !j.groups) {
      err = "resident executor: a circuit outside its limits";
      return false;
    }
  const auto t0 = std::chrono::steady_clock::now();
  std::lock_guard<std::mutex> g(g_mu);
  const uint64_t key = structure_key(dev, jobs);
  auto it = g_plans->find(key);
  if (it == g_plans->end()) {
    if (g_plans->size() >= kMaxPlans) g_plans->erase(g_plans->begin());
    std::unique_ptr<Plan> p = build(dev, jobs, err);
    if (!p) return false;
    it = g_plans->emplace(key, std::move(p)).first;
  }
  Plan& p = *it->second;
  size_t off = 0;
  for (const ResidentJob& j : jobs) {
    const size_t cnt = j.nsets * (size_t)j.nparams;
    if (cnt) std::memcpy(p.h_params + off, j.params, cnt * sizeof(double));
    off += cnt;
  }
  if (!cuda_ok(cudaSetDevice(dev), "cudaSetDevice", err) ||
      !cuda_ok(cudaGraphLaunch(p.exec, p.stream), "graph launch", err) ||
      !cuda_ok(cudaStreamSynchronize(p.stream), "sync", err))
    return false;
  size_t eo = 0, go = 0;
  for (const ResidentJob& j : jobs) {
    for (size_t s = 0; s < j.nsets; ++s) {
      if (j.energy_out) j.energy_out[s] = p.h_e[eo + s];
      if (j.grad_out)
        std::memcpy(j.grad_out + s * (size_t)j.nparams, p.h_g + go + s * (size_t)j.nparams, j.nparams * sizeof(double));
    }
    eo += j.nsets;
    go += j.nsets * (size_t)j.nparams;
  }
  if (host_ms) *host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return true;
}

void resident_release() {
  std::lock_guard<std::mutex> g(g_mu);
  g_plans->clear();
}

}  // namespace iqb
