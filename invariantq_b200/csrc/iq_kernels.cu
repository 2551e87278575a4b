// iq_kernels.cu -- host launchers and the non-tile sm_100a kernels: tensor-map
// encoding, the launcher of the tile pass (kernel in iq_tile.cuh, instantiated
// in iq_tile_r4.cu / iq_tile_r5.cu), the one-operation global-memory kernel,
// FP64 reductions, elementwise kernels, sampling and the partial trace.
#include <cudaTypedefs.h>

#include <cstdio>
#include <cstring>
#include <mutex>

#include "iq_kernels.h"

namespace iqb {

// ------------------------------------------------------------------ helpers

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cfma(double2 acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ double2 ld_mat(const double2* m, int i) { return m[i]; }

constexpr int kMaxBuf = 4;

// tile buffers + alignment slack + this pass's matrix block
size_t tile_pass_smem_bytes(int M, int R, int nbuf, uint32_t mat_elems, uint32_t ngrad) {
  return (size_t)nbuf * (16u << M) + 1024 + (size_t)mat_elems * 16 + (size_t)ngrad * (tile_pass_threads(R) / 8) * 8;
}


unsigned tile_pass_grid(const PassDesc& d, const TileLaunch& tl, int num_sms) {
  uint64_t grid = (uint64_t)num_sms * (uint64_t)(tl.ctas_per_sm < 1 ? 1 : tl.ctas_per_sm);
  if (grid > d.ntiles) grid = d.ntiles;
  return (unsigned)grid;
}

cudaError_t launch_tile_pass(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status,
                             const TileLaunch& tl, int num_sms, cudaStream_t st, double* grad_partials) {
  const int nbuf = tl.nbuf < 1 ? 1 : (tl.nbuf > kMaxBuf ? kMaxBuf : tl.nbuf);
  const size_t smem = tile_pass_smem_bytes(d.M, d.R, nbuf, d.mat_elems, d.ngrad);
  const unsigned grid = tile_pass_grid(d, tl, num_sms);
  if (d.ngrad && !grad_partials) return cudaErrorInvalidValue;
  if (d.R == 3) return launch_tile_r3(tm, d, mats, dev_status, nbuf, grid, smem, st, grad_partials);
  if (d.R == 4) return launch_tile_r4(tm, d, mats, dev_status, nbuf, grid, smem, st, grad_partials);
  return launch_tile_r5(tm, d, mats, dev_status, nbuf, grid, smem, st, grad_partials);
}

// ------------------------------------------------------------ tensor maps

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  });
  return fn;
}

int encode_pass_tmap(CUtensorMap* tm, void* state, int nbits, const PassDesc& d, char* err, size_t errlen) {
  auto fn = encode_fn();
  if (!fn) {
    snprintf(err, errlen, "cuTensorMapEncodeTiled unavailable from the driver");
    return -1;
  }
  uint64_t g[5], st[4];
  uint32_t b[5];
  pass_tmap_layout(d, nbits, g, st, b);
  cuuint64_t gd[5], gs[4];
  cuuint32_t box[5], es[5] = {1, 1, 1, 1, 1};
  for (int i = 0; i < 5; ++i) { gd[i] = g[i]; box[i] = b[i]; }
  for (int i = 0; i < 4; ++i) gs[i] = st[i];
  CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, state, gd, gs, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    snprintf(err, errlen, "cuTensorMapEncodeTiled failed (%d) for nbits=%d c=%d nbox=%d", (int)r, nbits, (int)d.c,
             (int)d.nbox);
    return -1;
  }
  return 0;
}

// ------------------------------------------------------- simple path

struct SimpleArgs {
  int k;
  int q[kMaxK];
  int qs[kMaxK];   // sorted ascending
  uint32_t mat;
};

template <int K>
__global__ void simple_op_kernel(double2* __restrict__ s, int nbits, SimpleArgs a, const double2* __restrict__ mats) {
  constexpr int D = 1 << K;
  // (matrix read through the read-only path: this kernel takes it from global memory)
  const uint64_t groups = 1ULL << (nbits - K);
  const double2* m = mats + a.mat;
  uint64_t qb[K];
#pragma unroll
  for (int i = 0; i < K; ++i) qb[i] = 1ULL << a.q[i];
  for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < groups;
       g += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t base = g;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      const int h = a.qs[i];
      base = ((base >> h) << (h + 1)) | (base & ((1ULL << h) - 1));
    }
    double2 x[D];
#pragma unroll
    for (int v = 0; v < D; ++v) {
      uint64_t id = base;
#pragma unroll
      for (int i = 0; i < K; ++i)
        if ((v >> i) & 1) id |= qb[i];
      x[v] = s[id];
    }
#pragma unroll 1
    for (int r = 0; r < D; ++r) {
      double2 acc = cmul(ld_mat(m, r * D), x[0]);
#pragma unroll
      for (int c = 1; c < D; ++c) acc = cfma(acc, ld_mat(m, r * D + c), x[c]);
      uint64_t id = base;
#pragma unroll
      for (int i = 0; i < K; ++i)
        if ((r >> i) & 1) id |= qb[i];
      s[id] = acc;
    }
  }
}

static unsigned grid_for(uint64_t work, int threads) {
  uint64_t g = (work + threads - 1) / threads;
  const uint64_t cap = 148ull * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (unsigned)g;
}

cudaError_t launch_simple_op(double2* s, int nbits, const SimpleOp& op, const double2* mats, cudaStream_t st) {
  SimpleArgs a;
  a.k = op.k;
  a.mat = op.mat;
  for (int i = 0; i < op.k; ++i) a.q[i] = a.qs[i] = op.q[i];
  for (int i = 0; i < op.k; ++i)
    for (int j = i + 1; j < op.k; ++j)
      if (a.qs[j] < a.qs[i]) { int t = a.qs[i]; a.qs[i] = a.qs[j]; a.qs[j] = t; }
  const uint64_t groups = 1ULL << (nbits - op.k);
  const int th = 128;
  const unsigned g = grid_for(groups, th);
  switch (op.k) {
    case 1: simple_op_kernel<1><<<g, th, 0, st>>>(s, nbits, a, mats); break;
    case 2: simple_op_kernel<2><<<g, th, 0, st>>>(s, nbits, a, mats); break;
    case 3: simple_op_kernel<3><<<g, th, 0, st>>>(s, nbits, a, mats); break;
    case 4: simple_op_kernel<4><<<g, th, 0, st>>>(s, nbits, a, mats); break;
    case 5: simple_op_kernel<5><<<g, th, 0, st>>>(s, nbits, a, mats); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// ------------------------------------------------------------ reductions

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// block-wide sum; result valid in thread 0
__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
    t = warp_sum(t);
  }
  return t;
}

__global__ void final_sum_kernel(const double* __restrict__ p, int n, double* __restrict__ out) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
  v = block_sum(v);
  if (threadIdx.x == 0) *out = v;
}

__global__ void sumsq_masked_kernel(const double2* __restrict__ s, uint64_t dim, uint64_t mask, uint64_t val,
                                    double* __restrict__ partials) {
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    if ((i & mask) == val) {
      const double2 a = s[i];
      acc += a.x * a.x + a.y * a.y;
    }
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

cudaError_t launch_sumsq_masked(const double2* s, uint64_t dim, uint64_t mask, uint64_t val, double* partials,
                                double* out, cudaStream_t st) {
  sumsq_masked_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(s, dim, mask, val, partials);
  final_sum_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, out);
  return cudaGetLastError();
}

__global__ void diag_sum_kernel(const double2* __restrict__ rho, uint64_t dim, uint64_t mask, uint64_t val,
                                double* __restrict__ partials) {
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x)
    if ((i & mask) == val) acc += rho[i * (dim + 1)].x;
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

cudaError_t launch_diag_sum(const double2* rho, uint64_t dim, uint64_t mask, uint64_t val, double* partials,
                            double* out, cudaStream_t st) {
  diag_sum_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(rho, dim, mask, val, partials);
  final_sum_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, out);
  return cudaGetLastError();
}

__global__ void diag_entropy_kernel(const double2* __restrict__ rho, uint64_t dim, double* __restrict__ partials) {
  double acc = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    double p = rho[i * (dim + 1)].x;
    if (p < 0.0) p = 0.0;
    if (p > 1e-14) acc -= p * log2(p);
  }
  acc = block_sum(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

cudaError_t launch_diag_entropy(const double2* rho, uint64_t dim, double* partials, double* out, cudaStream_t st) {
  diag_entropy_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(rho, dim, partials);
  final_sum_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, out);
  return cudaGetLastError();
}

__global__ void pauli_sum_kernel(const double2* __restrict__ s, uint64_t dim, uint64_t xmask, uint64_t zmask,
                                 double thresh, double2* __restrict__ partials) {
  double re = 0.0, im = 0.0;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 a = s[i];
    if (a.x * a.x + a.y * a.y < thresh) continue;
    const double2 b = s[i ^ xmask];
    // conj(b) * a
    double pr = b.x * a.x + b.y * a.y;
    double pi = b.x * a.y - b.y * a.x;
    if (__popcll(i & zmask) & 1) { pr = -pr; pi = -pi; }
    re += pr;
    im += pi;
  }
  re = block_sum(re);
  im = block_sum(im);
  if (threadIdx.x == 0) partials[blockIdx.x] = make_double2(re, im);
}

__global__ void final_csum_kernel(const double2* __restrict__ p, int n, double2* __restrict__ out) {
  double re = 0.0, im = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    re += p[i].x;
    im += p[i].y;
  }
  re = block_sum(re);
  im = block_sum(im);
  if (threadIdx.x == 0) *out = make_double2(re, im);
}

cudaError_t launch_pauli_sum(const double2* s, uint64_t dim, uint64_t xmask, uint64_t zmask, double thresh,
                             double2* partials, double2* out, cudaStream_t st) {
  pauli_sum_kernel<<<kRedBlocks, kRedThreads, 0, st>>>(s, dim, xmask, zmask, thresh, partials);
  final_csum_kernel<<<1, 1024, 0, st>>>(partials, kRedBlocks, out);
  return cudaGetLastError();
}

// Per-bit occupation sums.  Thread layout: blocks sweep super-chunks of
// 256 * 8 consecutive amplitudes; within one, element j*256 + tid has bits 0..7
// = tid, bits 8..10 = j, higher bits from the super-chunk index.
constexpr int kZThreads = 256;
constexpr int kZJ = 8;
constexpr int kZMaxBits = 40;

size_t zsums_partials_doubles(int nbits) { return (size_t)kRedBlocks * (nbits + 1); }

__global__ void zsums_kernel(const double2* __restrict__ s, int nbits, double* __restrict__ partials) {
  const uint64_t dim = 1ULL << nbits;
  const uint64_t chunk = (uint64_t)kZThreads * kZJ;
  double tot = 0.0, sj[3] = {0.0, 0.0, 0.0};
  double hi[kZMaxBits - 11];
#pragma unroll
  for (int b = 0; b < kZMaxBits - 11; ++b) hi[b] = 0.0;
  const int tid = threadIdx.x;
  for (uint64_t base = (uint64_t)blockIdx.x * chunk; base < dim; base += (uint64_t)gridDim.x * chunk) {
    double ct = 0.0;
#pragma unroll
    for (int j = 0; j < kZJ; ++j) {
      const uint64_t i = base + (uint64_t)j * kZThreads + tid;
      if (i < dim) {
        const double2 a = s[i];
        const double p = a.x * a.x + a.y * a.y;
        ct += p;
        if (j & 1) sj[0] += p;
        if (j & 2) sj[1] += p;
        if (j & 4) sj[2] += p;
      }
    }
    tot += ct;
#pragma unroll
    for (int b = 11; b < kZMaxBits; ++b)
      if (b < nbits && ((base >> b) & 1)) hi[b - 11] += ct;
  }
  // bit b < 8: whole thread total if tid bit set; 8..10: sj; >= 11: hi
#pragma unroll
  for (int b = 0; b <= kZMaxBits; ++b) {
    if (b > nbits) break;
    double v;
    if (b == 0) v = tot;
    else {
      const int bit = b - 1;
      if (bit < 8) v = ((tid >> bit) & 1) ? tot : 0.0;
      else if (bit < 11) v = sj[bit - 8];
      else v = hi[bit - 11];
    }
    v = block_sum(v);
    if (threadIdx.x == 0) partials[(size_t)b * gridDim.x + blockIdx.x] = v;
  }
}

__global__ void zsums_final_kernel(const double* __restrict__ partials, int nblocks, int nvals, double* __restrict__ out) {
  const int b = blockIdx.x;
  if (b >= nvals) return;
  double v = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) v += partials[(size_t)b * nblocks + i];
  v = block_sum(v);
  if (threadIdx.x == 0) out[b] = v;
}

cudaError_t launch_zsums(const double2* s, int nbits, double* partials, double* out, cudaStream_t st) {
  if (nbits > kZMaxBits) return cudaErrorInvalidValue;
  zsums_kernel<<<kRedBlocks, kZThreads, 0, st>>>(s, nbits, partials);
  zsums_final_kernel<<<nbits + 1, 256, 0, st>>>(partials, kRedBlocks, nbits + 1, out);
  return cudaGetLastError();
}

cudaError_t preload_zsums() {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, zsums_kernel);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, zsums_final_kernel);
  return e;
}

// ------------------------------------------------------------ elementwise

__global__ void collapse_kernel(double2* __restrict__ s, uint64_t dim, uint64_t mask, uint64_t val, double f) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x) {
    if ((i & mask) == val) {
      double2 a = s[i];
      a.x *= f;
      a.y *= f;
      s[i] = a;
    } else {
      s[i] = make_double2(0.0, 0.0);
    }
  }
}

cudaError_t launch_collapse(double2* s, uint64_t dim, uint64_t mask, uint64_t val, double factor, cudaStream_t st) {
  collapse_kernel<<<grid_for(dim, 256), 256, 0, st>>>(s, dim, mask, val, factor);
  return cudaGetLastError();
}

__global__ void dm_collapse_kernel(double2* __restrict__ rho, int n, uint64_t mask, uint64_t val, double f) {
  const uint64_t dim = 1ULL << n, tot = dim * dim;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < tot; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t r = i >> n, c = i & (dim - 1);
    if ((r & mask) == val && (c & mask) == val) {
      double2 a = rho[i];
      a.x *= f;
      a.y *= f;
      rho[i] = a;
    } else {
      rho[i] = make_double2(0.0, 0.0);
    }
  }
}

cudaError_t launch_dm_collapse(double2* rho, int n, uint64_t mask, uint64_t val, double factor, cudaStream_t st) {
  const uint64_t tot = 1ULL << (2 * n);
  dm_collapse_kernel<<<grid_for(tot, 256), 256, 0, st>>>(rho, n, mask, val, factor);
  return cudaGetLastError();
}

__global__ void set_basis_kernel(double2* __restrict__ s, uint64_t dim) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < dim; i += (uint64_t)gridDim.x * blockDim.x)
    s[i] = make_double2(i == 0 ? 1.0 : 0.0, 0.0);
}

cudaError_t launch_set_basis(double2* s, uint64_t dim, cudaStream_t st) {
  set_basis_kernel<<<grid_for(dim, 256), 256, 0, st>>>(s, dim);
  return cudaGetLastError();
}

// nsets arrays of dim (a power of two) amplitudes end to end, each set to e_0
__global__ void set_basis_sets_kernel(double2* __restrict__ s, uint64_t dim, uint64_t total) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x)
    s[i] = make_double2((i & (dim - 1)) == 0 ? 1.0 : 0.0, 0.0);
}

cudaError_t launch_set_basis_sets(double2* s, uint64_t dim, int nsets, cudaStream_t st) {
  const uint64_t total = dim * (uint64_t)(nsets < 1 ? 1 : nsets);
  set_basis_sets_kernel<<<grid_for(total, 256), 256, 0, st>>>(s, dim, total);
  return cudaGetLastError();
}

// The half of the 2^nbits amplitudes whose index bit `bit` equals `val`, in
// increasing index order: dst[i] = s[insert val at bit `bit` into i] (pack), or
// the reverse (unpack).  Runs of 2^bit consecutive amplitudes: coalesced for
// bit >= 5.
__global__ void half_copy_kernel(double2* __restrict__ s, int bit, int val, double2* __restrict__ buf, uint64_t half,
                                 int unpack) {
  const uint64_t lo = (1ULL << bit) - 1;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < half; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t j = ((i & ~lo) << 1) | ((uint64_t)val << bit) | (i & lo);
    if (unpack) s[j] = buf[i];
    else buf[i] = s[j];
  }
}

cudaError_t launch_half_copy(double2* s, int nbits, int bit, int val, double2* buf, bool unpack, cudaStream_t st) {
  if (bit < 0 || bit >= nbits) return cudaErrorInvalidValue;
  const uint64_t half = 1ULL << (nbits - 1);
  half_copy_kernel<<<grid_for(half, 256), 256, 0, st>>>(s, bit, val & 1, buf, half, unpack ? 1 : 0);
  return cudaGetLastError();
}

__global__ void split_kernel(const double2* __restrict__ s, uint64_t n, double* __restrict__ re, double* __restrict__ im) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 a = s[i];
    re[i] = a.x;
    im[i] = a.y;
  }
}

cudaError_t launch_split(const double2* s, uint64_t count, double* re, double* im, cudaStream_t st) {
  split_kernel<<<grid_for(count, 256), 256, 0, st>>>(s, count, re, im);
  return cudaGetLastError();
}

__global__ void probs_kernel(const double2* __restrict__ s, uint64_t n, double* __restrict__ p) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const double2 a = s[i];
    p[i] = a.x * a.x + a.y * a.y;
  }
}

cudaError_t launch_probs(const double2* s, uint64_t count, double* p, cudaStream_t st) {
  probs_kernel<<<grid_for(count, 256), 256, 0, st>>>(s, count, p);
  return cudaGetLastError();
}

// ------------------------------------------------------------ sampling

__global__ void block_sums_kernel(const double2* __restrict__ s, uint64_t nblk, int bbits, double* __restrict__ out) {
  // one warp per block of 2^bbits amplitudes, summed in index order per lane then across lanes
  const int lane = threadIdx.x & 31;
  const uint64_t w = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t len = 1ULL << bbits;
  for (uint64_t b = w; b < nblk; b += nw) {
    double acc = 0.0;
    for (uint64_t i = lane; i < len; i += 32) {
      const double2 a = s[b * len + i];
      acc += a.x * a.x + a.y * a.y;
    }
    acc = warp_sum(acc);
    if (lane == 0) out[b] = acc;
  }
}

cudaError_t launch_block_sums(const double2* s, uint64_t dim, int bbits, double* out, cudaStream_t st) {
  const uint64_t nblk = dim >> bbits;
  block_sums_kernel<<<grid_for(nblk * 32, 256), 256, 0, st>>>(s, nblk, bbits, out);
  return cudaGetLastError();
}

__global__ void block_search_kernel(const double2* __restrict__ s, int bbits, const uint64_t* __restrict__ blk,
                                    const double* __restrict__ base, const double* __restrict__ target,
                                    uint64_t* __restrict__ out, int shots) {
  // one warp per shot: sequential 32-wide windows, inclusive warp scan
  const int lane = threadIdx.x & 31;
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= shots) return;
  const uint64_t len = 1ULL << bbits;
  const uint64_t b0 = blk[w] * len;
  double run = base[w];
  const double r = target[w];
  uint64_t found = b0 + len - 1;
  for (uint64_t off = 0; off < len; off += 32) {
    const double2 a = s[b0 + off + lane];
    double v = a.x * a.x + a.y * a.y;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      const double t = __shfl_up_sync(0xffffffffu, v, d);
      if (lane >= d) v += t;
    }
    const double cum = run + v;
    const unsigned hit = __ballot_sync(0xffffffffu, cum >= r);
    if (hit) {
      found = b0 + off + (__ffs(hit) - 1);
      break;
    }
    run += __shfl_sync(0xffffffffu, v, 31);
  }
  if (lane == 0) out[w] = found;
}

cudaError_t launch_block_search(const double2* s, int bbits, const uint64_t* blk, const double* base,
                                const double* target, uint64_t* out, int shots, cudaStream_t st) {
  if (shots <= 0) return cudaSuccess;
  const int th = 256;
  const int blocks = (shots * 32 + th - 1) / th;
  block_search_kernel<<<blocks, th, 0, st>>>(s, bbits, blk, base, target, out, shots);
  return cudaGetLastError();
}

// ---------------------------------------------------- partial trace (entropy)

struct KeepArgs {
  int k;
  int keep[12];
  int nt;
  int traced[40];
};

__global__ void partial_trace_kernel(const double2* __restrict__ s, KeepArgs a, double2* __restrict__ out) {
  // one block per (r, c) with r <= c; threads sweep the environment
  const uint64_t kd = 1ULL << a.k;
  const uint64_t pair = blockIdx.x;
  // decode upper-triangle pair index
  uint64_t r = 0, rem = pair;
  while (rem >= kd - r) { rem -= kd - r; ++r; }
  const uint64_t c = r + rem;
  uint64_t ir = 0, ic = 0;
  for (int b = 0; b < a.k; ++b) {
    if ((r >> b) & 1) ir |= 1ULL << a.keep[b];
    if ((c >> b) & 1) ic |= 1ULL << a.keep[b];
  }
  const uint64_t td = 1ULL << a.nt;
  double re = 0.0, im = 0.0;
  for (uint64_t env = threadIdx.x; env < td; env += blockDim.x) {
    uint64_t e = 0;
    for (int b = 0; b < a.nt; ++b)
      if ((env >> b) & 1) e |= 1ULL << a.traced[b];
    const double2 x = s[ir | e], y = s[ic | e];
    // x * conj(y)
    re += x.x * y.x + x.y * y.y;
    im += x.y * y.x - x.x * y.y;
  }
  re = block_sum(re);
  im = block_sum(im);
  if (threadIdx.x == 0) {
    out[r * kd + c] = make_double2(re, im);
    out[c * kd + r] = make_double2(re, -im);
  }
}

cudaError_t launch_partial_trace(const double2* s, int nbits, const int* keep, int k, double2* out, cudaStream_t st) {
  if (k < 1 || k > 12) return cudaErrorInvalidValue;
  KeepArgs a;
  a.k = k;
  for (int i = 0; i < k; ++i) a.keep[i] = keep[i];
  a.nt = 0;
  for (int q = 0; q < nbits; ++q) {
    bool in = false;
    for (int i = 0; i < k; ++i) in |= keep[i] == q;
    if (!in) a.traced[a.nt++] = q;
  }
  const uint64_t kd = 1ULL << k;
  const uint64_t npairs = kd * (kd + 1) / 2;
  partial_trace_kernel<<<(unsigned)npairs, 256, 0, st>>>(s, a, out);
  return cudaGetLastError();
}

// ---------------------------------------------------- adjoint gradients

// lambda = H psi written next to psi in the joint array (joint[2x] = psi[x],
// joint[2x + 1] = lambda[x]; skipped when joint is null) and the block sums of
// Re conj(psi) lambda.
// H = sum over groups g of sum over terms t of c_t (-1)^popc((x ^ xmask_g) & zmask_t)
// psi[x ^ xmask_g]: Pauli strings sharing their X part share one gather.
__global__ void row_sum_kernel(const double* __restrict__ in, int cols, double* __restrict__ out);

// blockIdx.y = set: psi + set * pstride, lam + set * lstride, partials + set * gridDim.x
__global__ void hamiltonian_joint_kernel(const double2* __restrict__ psi, uint64_t pstride, uint64_t dim, HamTerms h,
                                         const uint64_t* __restrict__ zmask, const double2* __restrict__ coef,
                                         double2* __restrict__ lam_out, uint64_t lstride, double* __restrict__ partials) {
  psi += blockIdx.y * pstride;
  if (lam_out) lam_out += blockIdx.y * lstride;
  partials += (size_t)blockIdx.y * gridDim.x;
  double e = 0.0;
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
    const double2 px = psi[x];
    double2 lam = make_double2(0.0, 0.0);
    for (int g = 0; g < h.ngroups; ++g) {
      const uint64_t src = x ^ h.xmask[g];
      const double2 a = (h.xmask[g] == 0) ? px : psi[src];
      double2 f = make_double2(0.0, 0.0);
      for (int t = h.first[g]; t < h.first[g + 1]; ++t) {
        const double2 c = coef[t];
        if (__popcll(src & zmask[t]) & 1) { f.x -= c.x; f.y -= c.y; }
        else { f.x += c.x; f.y += c.y; }
      }
      lam = cfma(lam, f, a);
    }
    if (lam_out) lam_out[x] = lam;
    e += px.x * lam.x + px.y * lam.y;
  }
  e = block_sum(e);
  if (threadIdx.x == 0) partials[blockIdx.x] = e;
}

cudaError_t launch_hamiltonian_joint(const double2* psi, uint64_t pstride, int n, int nsets, const HamTerms& h,
                                     const uint64_t* zmask, const double2* coef, double2* lam, uint64_t lstride,
                                     double* partials, double* energy, cudaStream_t st) {
  if (nsets < 1) nsets = 1;
  hamiltonian_joint_kernel<<<dim3(kRedBlocks, nsets), kRedThreads, 0, st>>>(psi, pstride, 1ULL << n, h, zmask, coef,
                                                                            lam, lstride, partials);
  row_sum_kernel<<<nsets, 256, 0, st>>>(partials, kRedBlocks, energy);
  return cudaGetLastError();
}

// nsets joint arrays of jdim amplitudes end to end: psi half [0, dim) set to
// e_0, everything above 2 * dim (zero padding of small circuits) to zero; the
// lambda half [dim, 2 * dim) is left for the Hamiltonian kernel
__global__ void init_joint_kernel(double2* __restrict__ s, uint64_t dim, uint64_t jdim, uint64_t total) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t l = i & (jdim - 1);
    if (l < dim) s[i] = make_double2(l == 0 ? 1.0 : 0.0, 0.0);
    else if (l >= 2 * dim) s[i] = make_double2(0.0, 0.0);
  }
}

cudaError_t launch_init_joint(double2* s, int n, uint64_t jdim, int nsets, cudaStream_t st) {
  const uint64_t total = jdim * (uint64_t)(nsets < 1 ? 1 : nsets);
  init_joint_kernel<<<grid_for(total, 256), 256, 0, st>>>(s, 1ULL << n, jdim, total);
  return cudaGetLastError();
}

// complex64 storage of the same: psi_s at psi + s * pstride (float2), lambda_s
// written to lam + s * lstride (float2, rounded once), every product and sum in FP64
__global__ void hamiltonian_c64_kernel(const float2* __restrict__ psi, uint64_t pstride, uint64_t dim, HamTerms h,
                                       const uint64_t* __restrict__ zmask, const double2* __restrict__ coef,
                                       float2* __restrict__ lam_out, uint64_t lstride, double* __restrict__ partials) {
  psi += blockIdx.y * pstride;
  if (lam_out) lam_out += blockIdx.y * lstride;
  partials += (size_t)blockIdx.y * gridDim.x;
  double e = 0.0;
  for (uint64_t x = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; x < dim; x += (uint64_t)gridDim.x * blockDim.x) {
    const float2 pf = psi[x];
    const double2 px = make_double2(pf.x, pf.y);
    double2 lam = make_double2(0.0, 0.0);
    for (int g = 0; g < h.ngroups; ++g) {
      const uint64_t src = x ^ h.xmask[g];
      const float2 af = psi[src];
      const double2 a = (h.xmask[g] == 0) ? px : make_double2(af.x, af.y);
      double2 f = make_double2(0.0, 0.0);
      for (int t = h.first[g]; t < h.first[g + 1]; ++t) {
        const double2 c = coef[t];
        if (__popcll(src & zmask[t]) & 1) { f.x -= c.x; f.y -= c.y; }
        else { f.x += c.x; f.y += c.y; }
      }
      lam = cfma(lam, f, a);
    }
    if (lam_out) lam_out[x] = make_float2(__double2float_rn(lam.x), __double2float_rn(lam.y));
    e += px.x * lam.x + px.y * lam.y;
  }
  e = block_sum(e);
  if (threadIdx.x == 0) partials[blockIdx.x] = e;
}

cudaError_t launch_hamiltonian_c64(const float2* psi, uint64_t pstride, int n, int nsets, const HamTerms& h,
                                   const uint64_t* zmask, const double2* coef, float2* lam, uint64_t lstride,
                                   double* partials, double* energy, cudaStream_t st) {
  if (nsets < 1) nsets = 1;
  hamiltonian_c64_kernel<<<dim3(kRedBlocks, nsets), kRedThreads, 0, st>>>(psi, pstride, 1ULL << n, h, zmask, coef,
                                                                          lam, lstride, partials);
  row_sum_kernel<<<nsets, 256, 0, st>>>(partials, kRedBlocks, energy);
  return cudaGetLastError();
}

__global__ void init_joint_c64_kernel(float2* __restrict__ s, uint64_t dim, uint64_t jdim, uint64_t total) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t l = i & (jdim - 1);
    if (l < dim) s[i] = make_float2(l == 0 ? 1.0f : 0.0f, 0.0f);
    else if (l >= 2 * dim) s[i] = make_float2(0.0f, 0.0f);
  }
}

cudaError_t launch_init_joint_c64(float2* s, int n, uint64_t jdim, int nsets, cudaStream_t st) {
  const uint64_t total = jdim * (uint64_t)(nsets < 1 ? 1 : nsets);
  init_joint_c64_kernel<<<grid_for(total, 256), 256, 0, st>>>(s, 1ULL << n, jdim, total);
  return cudaGetLastError();
}

// out[r] = sum_c in[r * cols + c], in order (one block per row)
__global__ void row_sum_kernel(const double* __restrict__ in, int cols, double* __restrict__ out) {
  double v = 0.0;
  for (int c = threadIdx.x; c < cols; c += blockDim.x) v += in[(size_t)blockIdx.x * cols + c];
  v = block_sum(v);
  if (threadIdx.x == 0) out[blockIdx.x] = v;
}

cudaError_t launch_row_sums(const double* in, int rows, int cols, double* out, cudaStream_t st) {
  if (rows <= 0) return cudaSuccess;
  row_sum_kernel<<<rows, 256, 0, st>>>(in, cols, out);
  return cudaGetLastError();
}

}  // namespace iqb
