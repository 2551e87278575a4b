// iq_sampling.cu -- measurement shots entirely on the device.
//
// The reference samples on the host (StateVector::sample,
// core/src/statevector.cpp:235-256): a serial cumulative distribution over
// all 2^n probabilities, std::mt19937_64 seeded with the caller's seed,
// std::uniform_real_distribution<double>(0, 1) per shot, lower_bound, clamp to
// 2^n - 1; its driver then builds the counts dictionary in Python
// (invariantq/simulator/statevector.py:105-114).  Here every step runs on the
// GPU, drawing the same random numbers so the shots are the reference's:
//
//   1. block sums of |a|^2 over blocks of 2^bb amplitudes (launch_block_sums);
//   2. their inclusive prefix (one CTA: contiguous runs per thread, then the
//      run totals in order);
//   3. the mt19937_64 stream (Matsumoto & Nishimura's 64-bit Mersenne Twister,
//      the engine the C++ standard specifies: the state of 312 words is
//      regenerated by 156 threads in two dependent halves, then tempered in
//      parallel) mapped to [0, 1) as std::generate_canonical<double, 53> does
//      for a 64-bit engine: the draw converted to double, times 2^-64, values
//      that round up to 1 replaced by the largest double below 1;
//   4. per shot a binary search for its block, then the warp search inside
//      the block (launch_block_search);
//   5. for counts: the shot indices sorted (bitonic network in global memory,
//      padded to a power of two), run-length encoded into ascending outcomes
//      and their counts.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "iq_kernels.h"

namespace iqb {
namespace {

constexpr int kMtN = 312, kMtM = 156;
constexpr uint64_t kMtA = 0xB5026F5AA96619E9ULL;
constexpr uint64_t kMtUpper = 0xFFFFFFFF80000000ULL, kMtLower = 0x000000007FFFFFFFULL;

__device__ __forceinline__ uint64_t mt_mix(uint64_t cur, uint64_t nxt) {
  const uint64_t x = (cur & kMtUpper) | (nxt & kMtLower);
  return (x >> 1) ^ ((x & 1ULL) ? kMtA : 0ULL);
}

__device__ __forceinline__ uint64_t mt_temper(uint64_t z) {
  z ^= (z >> 29) & 0x5555555555555555ULL;
  z ^= (z << 17) & 0x71D67FFFEDA60000ULL;
  z ^= (z << 37) & 0xFFF7EEE000000000ULL;
  z ^= (z >> 43);
  return z;
}

// generate_canonical<double, 53> of one 64-bit draw
__device__ __forceinline__ double mt_unit(uint64_t z) {
  double r = __ull2double_rn(z) * 0x1p-64;
  if (r >= 1.0) r = 0x1.fffffffffffffp-1;
  return r;
}

// One CTA of kMtM threads: `count` uniform draws of the stream seeded with `seed`.
__global__ void __launch_bounds__(kMtM) mt64_uniform_kernel(uint64_t seed, uint64_t count, double* __restrict__ out) {
  __shared__ uint64_t mt[kMtN];
  const int t = threadIdx.x;
  if (t == 0) {   // seeding is a serial recurrence (312 steps)
    mt[0] = seed;
    for (int i = 1; i < kMtN; ++i) mt[i] = 6364136223846793005ULL * (mt[i - 1] ^ (mt[i - 1] >> 62)) + (uint64_t)i;
  }
  __syncthreads();
  for (uint64_t done = 0; done < count; done += kMtN) {
    // operands of the second half (words 156..311), read before the first half writes
    const int i2 = kMtM + t;
    const uint64_t cur2 = mt[i2];
    const uint64_t nxt2 = (i2 + 1 < kMtN) ? mt[i2 + 1] : 0ULL;
    const uint64_t new1 = mt[t + kMtM] ^ mt_mix(mt[t], mt[t + 1]);   // words 0..155: all old operands
    __syncthreads();
    mt[t] = new1;
    __syncthreads();
    // words 156..310 take word i + m - n of the new first half; word 311 also the new word 0
    const uint64_t nx = (i2 + 1 < kMtN) ? nxt2 : mt[0];
    const uint64_t new2 = mt[i2 + kMtM - kMtN] ^ mt_mix(cur2, nx);
    __syncthreads();
    mt[i2] = new2;
    __syncthreads();
    for (int j = t; j < kMtN; j += kMtM) {
      const uint64_t k = done + (uint64_t)j;
      if (k < count) out[k] = mt_unit(mt_temper(mt[j]));
    }
    __syncthreads();
  }
}

// One CTA: inclusive prefix of in[0..n) into out (contiguous runs per thread).
__global__ void __launch_bounds__(1024) prefix_kernel(const double* __restrict__ in, uint64_t n, double* __restrict__ out) {
  __shared__ double tot[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const uint64_t per = (n + T - 1) / T;
  const uint64_t b = (uint64_t)t * per, e = (b + per < n) ? b + per : n;
  double s = 0.0;
  for (uint64_t i = b; i < e; ++i) s += in[i];
  tot[t] = s;
  __syncthreads();
  if (t == 0) {
    double run = 0.0;
    for (int k = 0; k < T; ++k) {
      const double v = tot[k];
      tot[k] = run;
      run += v;
    }
  }
  __syncthreads();
  double run = tot[t];
  for (uint64_t i = b; i < e; ++i) {
    run += in[i];
    out[i] = run;
  }
}

// per shot: first block whose inclusive prefix is >= r (clamped to the last)
__global__ void find_block_kernel(const double* __restrict__ incl, uint64_t nblk, const double* __restrict__ r,
                                  int shots, uint64_t* __restrict__ blk, double* __restrict__ base) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= shots) return;
  const double x = r[k];
  uint64_t lo = 0, hi = nblk;
  while (lo < hi) {
    const uint64_t mid = lo + ((hi - lo) >> 1);
    if (incl[mid] < x) lo = mid + 1;
    else hi = mid;
  }
  if (lo >= nblk) lo = nblk - 1;
  blk[k] = lo;
  base[k] = lo ? incl[lo - 1] : 0.0;
}

__global__ void pad_kernel(const uint64_t* __restrict__ in, int n, uint64_t* __restrict__ out, int npow) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < npow) out[i] = i < n ? in[i] : ~0ULL;
}

// one compare-exchange step (k, j) of the bitonic network, ascending
__global__ void bitonic_step_kernel(uint64_t* __restrict__ a, int npow, int k, int j) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= npow) return;
  const int p = i ^ j;
  if (p <= i) return;
  const uint64_t x = a[i], y = a[p];
  const bool up = (i & k) == 0;
  if ((x > y) == up) {
    a[i] = y;
    a[p] = x;
  }
}

// One CTA: run-length encoding of the sorted a[0..n) into ascending outcomes and counts.
__global__ void __launch_bounds__(1024) rle_kernel(const uint64_t* __restrict__ a, int n, uint64_t* __restrict__ vals,
                                                   uint64_t* __restrict__ cnts, uint64_t* __restrict__ nuniq) {
  __shared__ int heads[1024];
  const int t = threadIdx.x, T = blockDim.x;
  const int per = (n + T - 1) / T;
  const int b = t * per, e = (b + per < n) ? b + per : n;
  int h = 0;
  for (int i = b; i < e; ++i) h += (i == 0 || a[i] != a[i - 1]);
  heads[t] = h;
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int k = 0; k < T; ++k) {
      const int v = heads[k];
      heads[k] = run;
      run += v;
    }
    *nuniq = (uint64_t)run;
  }
  __syncthreads();
  int u = heads[t];   // index of the first run this thread's range starts
  for (int i = b; i < e; ++i)
    if (i == 0 || a[i] != a[i - 1]) {
      int j = i + 1;
      while (j < n && a[j] == a[i]) ++j;
      vals[u] = a[i];
      cnts[u] = (uint64_t)(j - i);
      ++u;
    }
}

}  // namespace

cudaError_t launch_mt64_uniform(uint64_t seed, uint64_t count, double* out, cudaStream_t st) {
  mt64_uniform_kernel<<<1, kMtM, 0, st>>>(seed, count, out);
  return cudaGetLastError();
}

cudaError_t sample_on_device(const double2* s, int nbits, uint64_t shots, uint64_t seed, void* work, uint64_t* d_out,
                             cudaStream_t st) {
  const int bb = nbits < 12 ? nbits : 12;
  const uint64_t nblk = (1ULL << nbits) >> bb;
  double* bs = static_cast<double*>(work);
  double* incl = bs + nblk;
  double* r = incl + nblk;
  double* base = r + shots;
  uint64_t* blk = reinterpret_cast<uint64_t*>(base + shots);
  cudaError_t e = launch_block_sums(s, 1ULL << nbits, bb, bs, st);
  if (e != cudaSuccess) return e;
  prefix_kernel<<<1, 1024, 0, st>>>(bs, nblk, incl);
  mt64_uniform_kernel<<<1, kMtM, 0, st>>>(seed, shots, r);
  find_block_kernel<<<(unsigned)((shots + 255) / 256), 256, 0, st>>>(incl, nblk, r, (int)shots, blk, base);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  count_launches(5);
  return launch_block_search(s, bb, blk, base, r, d_out, (int)shots, st);
}

size_t sample_work_bytes(int nbits, uint64_t shots) {
  const int bb = std::min(12, nbits);
  const uint64_t nblk = (1ULL << nbits) >> bb;
  return (2 * nblk + 3 * shots) * 8 + 256;
}

cudaError_t count_outcomes(const uint64_t* d_shots, uint64_t shots, void* work, uint64_t* d_vals, uint64_t* d_cnts,
                           uint64_t* d_nuniq, cudaStream_t st) {
  int npow = 1;
  while ((uint64_t)npow < shots) npow <<= 1;
  uint64_t* a = static_cast<uint64_t*>(work);
  const unsigned g = (unsigned)((npow + 255) / 256);
  pad_kernel<<<g, 256, 0, st>>>(d_shots, (int)shots, a, npow);
  uint64_t launches = 2;
  for (int k = 2; k <= npow; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      bitonic_step_kernel<<<g, 256, 0, st>>>(a, npow, k, j);
      ++launches;
    }
  rle_kernel<<<1, 1024, 0, st>>>(a, (int)shots, d_vals, d_cnts, d_nuniq);
  count_launches(launches);
  return cudaGetLastError();
}

size_t count_work_bytes(uint64_t shots) {
  uint64_t npow = 1;
  while (npow < shots) npow <<= 1;
  return npow * 8 + 256;
}

}  // namespace iqb
