// iq_c64.cu -- kernels of the complex64 adjoint-gradient variant: amplitudes
// stored as float2 (8 B each, half the bytes of complex128), every operation
// computed in FP64 from the loaded values and rounded once on store, every
// reduction (gradient terms, energy) accumulated in FP64 with fixed-order
// block sums.  One launch per item of the ansatz: a run of one-qubit gates on
// one qubit (one pass over the pairs of that qubit's bit), or a CZ / CX.
#include <cuda_runtime.h>

#include "iq_c64.h"

namespace iqb {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double2 ld(const float2* p, uint64_t i) {
  const float2 v = p[i];
  return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ void st(float2* p, uint64_t i, double2 v) { p[i] = make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ double2 mul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ uint64_t pair0(uint64_t i, int q) {   // i with a zero inserted at bit q
  return ((i >> q) << (q + 1)) | (i & ((1ULL << q) - 1));
}

// out = m x for the 2x2 row-major matrix m (re/im interleaved)
__device__ __forceinline__ void apply2(const double* m, double2& x0, double2& x1) {
  const double2 a = make_double2(m[0], m[1]), b = make_double2(m[2], m[3]);
  const double2 c = make_double2(m[4], m[5]), d = make_double2(m[6], m[7]);
  const double2 y0 = add(mul(a, x0), mul(b, x1));
  const double2 y1 = add(mul(c, x0), mul(d, x1));
  x0 = y0;
  x1 = y1;
}

// inverse rotation exp(+i t P / 2), P = X (0), Y (1), Z (2), c = cos t/2, s = sin t/2
__device__ __forceinline__ void unrotate(int gen, double c, double s, double2& x0, double2& x1) {
  double2 y0, y1;
  if (gen == 0) {
    y0 = make_double2(c * x0.x - s * x1.y, c * x0.y + s * x1.x);
    y1 = make_double2(c * x1.x - s * x0.y, c * x1.y + s * x0.x);
  } else if (gen == 1) {
    y0 = make_double2(c * x0.x + s * x1.x, c * x0.y + s * x1.y);
    y1 = make_double2(c * x1.x - s * x0.x, c * x1.y - s * x0.y);
  } else {
    y0 = mul(make_double2(c, s), x0);
    y1 = mul(make_double2(c, -s), x1);
  }
  x0 = y0;
  x1 = y1;
}

// this pair's share of Im <lambda| P |psi> on the qubit
__device__ __forceinline__ double gterm(int gen, double2 p0, double2 p1, double2 l0, double2 l1) {
  if (gen == 0) return (l0.x * p1.y - l0.y * p1.x) + (l1.x * p0.y - l1.y * p0.x);
  if (gen == 1) return (l1.x * p0.x + l1.y * p0.y) - (l0.x * p1.x + l0.y * p1.y);
  return (l0.x * p0.y - l0.y * p0.x) - (l1.x * p1.y - l1.y * p1.x);
}

__device__ __forceinline__ double block_reduce(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) r += sh[i];   // fixed order
  return r;
}

__global__ void apply1q_kernel(float2* __restrict__ s, int n, int q, C64Mat m) {
  const uint64_t half = 1ULL << (n - 1);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = pair0(i, q), i1 = i0 | (1ULL << q);
    double2 x0 = ld(s, i0), x1 = ld(s, i1);
    apply2(m.m, x0, x1);
    st(s, i0, x0);
    st(s, i1, x1);
  }
}

// CZ: negate where both bits are set (touches a quarter of the amplitudes)
__global__ void cz_kernel(float2* __restrict__ s, int n, int a, int b) {
  const uint64_t quarter = 1ULL << (n - 2);
  const int lo = a < b ? a : b, hi = a < b ? b : a;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < quarter; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = pair0(pair0(i, lo), hi) | (1ULL << a) | (1ULL << b);
    const float2 v = s[j];
    s[j] = make_float2(-v.x, -v.y);
  }
}

// CX: swap the target's pair where the control bit is set
__global__ void cx_kernel(float2* __restrict__ s, int n, int c, int t) {
  const uint64_t quarter = 1ULL << (n - 2);
  const int lo = c < t ? c : t, hi = c < t ? t : c;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < quarter; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j0 = pair0(pair0(i, lo), hi) | (1ULL << c), j1 = j0 | (1ULL << t);
    const float2 v0 = s[j0], v1 = s[j1];
    s[j0] = v1;
    s[j1] = v0;
  }
}

// One run of one-qubit gates walked backwards on psi and lambda together:
// for each rotation (last first) record its gradient term, then un-apply it;
// fixed gates are un-applied with their inverse.  partials[term][block].
__global__ void grad_run_kernel(float2* __restrict__ psi, float2* __restrict__ lam, int n, C64Run run,
                                double* __restrict__ partials) {
  __shared__ double sh[32];
  double acc[kC64MaxRunOps];
#pragma unroll
  for (int j = 0; j < kC64MaxRunOps; ++j) acc[j] = 0.0;
  const int q = run.q;
  const uint64_t half = 1ULL << (n - 1);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t i0 = pair0(i, q), i1 = i0 | (1ULL << q);
    double2 p0 = ld(psi, i0), p1 = ld(psi, i1), l0 = ld(lam, i0), l1 = ld(lam, i1);
#pragma unroll
    for (int j = kC64MaxRunOps - 1; j >= 0; --j) {
      if (j >= run.nops) continue;
      const C64Op& o = run.ops[j];
      if (o.gen >= 0) {
        acc[j] += gterm(o.gen, p0, p1, l0, l1);
        unrotate(o.gen, o.c, o.s, p0, p1);
        unrotate(o.gen, o.c, o.s, l0, l1);
      } else {
        apply2(o.inv, p0, p1);
        apply2(o.inv, l0, l1);
      }
    }
    st(psi, i0, p0);
    st(psi, i1, p1);
    st(lam, i0, l0);
    st(lam, i1, l1);
  }
#pragma unroll
  for (int j = 0; j < kC64MaxRunOps; ++j) {
    if (j >= run.nops || run.ops[j].gen < 0) continue;
    const double v = block_reduce(acc[j], sh);
    if (threadIdx.x == 0) partials[(size_t)run.ops[j].term * gridDim.x + blockIdx.x] = v;
  }
}

// lambda = H psi (FP64 arithmetic, float2 storage) and block sums of Re <psi|lambda>
__global__ void hamiltonian_kernel(const float2* __restrict__ psi, uint64_t dim, HamTerms h,
                                   const uint64_t* __restrict__ zmask, const double2* __restrict__ coef,
                                   float2* __restrict__ lam, double* __restrict__ partials) {
  __shared__ double sh[32];
  double e = 0.0;
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
    const double2 px = ld(psi, x);
    double2 l = make_double2(0.0, 0.0);
    for (int g = 0; g < h.ngroups; ++g) {
      const uint64_t src = x ^ h.xmask[g];
      const double2 a = (h.xmask[g] == 0) ? px : ld(psi, src);
      double2 f = make_double2(0.0, 0.0);
      for (int t = h.first[g]; t < h.first[g + 1]; ++t) {
        const double2 c = coef[t];
        if (__popcll(src & zmask[t]) & 1) { f.x -= c.x; f.y -= c.y; }
        else { f.x += c.x; f.y += c.y; }
      }
      l = add(l, mul(f, a));
    }
    st(lam, x, l);
    e += px.x * l.x + px.y * l.y;
  }
  const double v = block_reduce(e, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = v;
}

__global__ void basis_kernel(float2* __restrict__ s, uint64_t dim) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x)
    s[i] = make_float2(i == 0 ? 1.0f : 0.0f, 0.0f);
}

}  // namespace

cudaError_t c64_set_basis(float2* s, int n, cudaStream_t st) {
  basis_kernel<<<kC64Blocks, kThreads, 0, st>>>(s, 1ULL << n);
  return cudaGetLastError();
}
cudaError_t c64_apply1q(float2* s, int n, int q, const C64Mat& m, cudaStream_t st) {
  apply1q_kernel<<<kC64Blocks, kThreads, 0, st>>>(s, n, q, m);
  return cudaGetLastError();
}
cudaError_t c64_cz(float2* s, int n, int a, int b, cudaStream_t st) {
  cz_kernel<<<kC64Blocks, kThreads, 0, st>>>(s, n, a, b);
  return cudaGetLastError();
}
cudaError_t c64_cx(float2* s, int n, int c, int t, cudaStream_t st) {
  cx_kernel<<<kC64Blocks, kThreads, 0, st>>>(s, n, c, t);
  return cudaGetLastError();
}
cudaError_t c64_grad_run(float2* psi, float2* lam, int n, const C64Run& run, double* partials, cudaStream_t st) {
  grad_run_kernel<<<kC64Blocks, kThreads, 0, st>>>(psi, lam, n, run, partials);
  return cudaGetLastError();
}
cudaError_t c64_hamiltonian(const float2* psi, int n, const HamTerms& h, const uint64_t* zmask, const double2* coef,
                            float2* lam, double* partials, cudaStream_t st) {
  hamiltonian_kernel<<<kC64Blocks, kThreads, 0, st>>>(psi, 1ULL << n, h, zmask, coef, lam, partials);
  return cudaGetLastError();
}

}  // namespace iqb
