// iq_entropy.cu -- the spectrum of a reduced state, on the GPU, for the
// entanglement entropy of a state vector across a cut (the reference computes
// it in StateVector::entanglement_entropy, core/src/statevector.cpp:293-410,
// with a capped Jacobi iteration on the host; its drivers call it on every run
// for the half cut range(n // 2), invariantq/simulator/statevector.py:87-90).
//
// For a kept qubit set K (|K| = k, kd = 2^k) and the traced set E (ed = 2^(n-k)):
//
//   1. Gram kernel: rho[r][c] = sum_e psi[dep_K(r) | dep_E(e)] conj(psi[dep_K(c) | dep_E(e)]),
//      an FP64 complex rank-ed Hermitian product (rho = M M^H for the kd x ed
//      matrix M of the reshaped state), tiled 64 x 64 per CTA through shared
//      memory, upper-triangle tiles only, with the environment split across
//      CTAs in fixed chunks (deterministic: partial tiles summed in order).
//   2. Householder reduction of rho to real symmetric tridiagonal form, one
//      reflector per column (vector kernel, Hermitian matrix-vector product,
//      rank-2 update), all on the device.
//   3. Eigenvalues of the tridiagonal matrix by bisection on Sturm counts, one
//      thread per eigenvalue.
//
// Bit i of the kept index r is qubit keep[i]; the spectrum does not depend on
// the order.  Only the eigenvalues (kd doubles) come back to the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <vector>

#include "iq_kernels.h"

namespace iqb {
namespace {

constexpr int kGT = 64;        // Gram tile (rows and columns)
constexpr int kGK = 16;        // environment entries per shared-memory step
constexpr int kGThreads = 256;

// block-wide sum, result in every thread
__device__ double block_allsum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
  return t;
}

// index of environment entry e: dep_E(e) = lo[e & lomask] | hi[e >> lobits]
struct EnvDep {
  const uint64_t* lo;
  const uint64_t* hi;
  int lobits;
};

__device__ __forceinline__ uint64_t env_index(const EnvDep& d, uint64_t e) {
  return d.lo[e & ((1ULL << d.lobits) - 1)] | d.hi[e >> d.lobits];
}

// grid.x = upper-triangle tile pairs (tr <= tc), grid.y = environment split s.
// part[s][tile][64 x 64] for nsplit > 1, else written straight into rho.
__global__ void __launch_bounds__(kGThreads) gram_kernel(const double2* __restrict__ psi,
                                                         const uint64_t* __restrict__ depk, EnvDep dep, int tiles,
                                                         uint64_t kd, uint64_t env_per_split,
                                                         double2* __restrict__ part, double2* __restrict__ rho) {
  __shared__ double2 As[kGK][kGT];
  __shared__ double2 Bs[kGK][kGT];
  // decode the tile pair
  int tr = 0, rem = blockIdx.x;
  while (rem >= tiles - tr) {
    rem -= tiles - tr;
    ++tr;
  }
  const int tc = tr + rem;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const uint64_t e_begin = (uint64_t)blockIdx.y * env_per_split, e_end = e_begin + env_per_split;
  // loader coordinates: row rl of the tile, environment entries el, el + 4, el + 8, el + 12
  const int rl = tid & 63, el = tid >> 6;
  const uint64_t ra = (uint64_t)tr * kGT + rl, rb = (uint64_t)tc * kGT + rl;
  const uint64_t ia = (ra < kd) ? depk[ra] : 0, ib = (rb < kd) ? depk[rb] : 0;
  double acc_re[4][4], acc_im[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc_re[i][j] = acc_im[i][j] = 0.0;
  for (uint64_t e0 = e_begin; e0 < e_end; e0 += kGK) {
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int ek = el + 4 * m;
      const uint64_t e = e0 + ek;
      const bool in = e < e_end;
      const uint64_t ie = in ? env_index(dep, e) : 0;
      As[ek][rl] = (in && ra < kd) ? psi[ia | ie] : make_double2(0.0, 0.0);
      Bs[ek][rl] = (in && rb < kd) ? psi[ib | ie] : make_double2(0.0, 0.0);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGK; ++kk) {
      double2 a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          // a * conj(b)
          acc_re[i][j] = fma(a[i].x, b[j].x, fma(a[i].y, b[j].y, acc_re[i][j]));
          acc_im[i][j] = fma(a[i].y, b[j].x, fma(-a[i].x, b[j].y, acc_im[i][j]));
        }
    }
    __syncthreads();
  }
  if (part) {
    double2* out = part + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * (kGT * kGT);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) out[(ty + 16 * i) * kGT + tx + 16 * j] = make_double2(acc_re[i][j], acc_im[i][j]);
    return;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint64_t r = (uint64_t)tr * kGT + ty + 16 * i, c = (uint64_t)tc * kGT + tx + 16 * j;
      if (r < kd && c < kd && (tr != tc || r <= c)) {
        rho[r * kd + c] = make_double2(acc_re[i][j], r == c ? 0.0 : acc_im[i][j]);
        if (r != c) rho[c * kd + r] = make_double2(acc_re[i][j], -acc_im[i][j]);
      }
    }
}

// sums the nsplit partial tiles in split order and writes rho (both triangles)
__global__ void gram_reduce_kernel(const double2* __restrict__ part, int pairs, int tiles, int nsplit, uint64_t kd,
                                   double2* __restrict__ rho) {
  const uint64_t total = (uint64_t)pairs * kGT * kGT;
  for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < total;
       t += (uint64_t)gridDim.x * blockDim.x) {
    const int pair = (int)(t / (kGT * kGT));
    const int w = (int)(t % (kGT * kGT)), rl = w / kGT, cl = w % kGT;
    int tr = 0, rem = pair;
    while (rem >= tiles - tr) {
      rem -= tiles - tr;
      ++tr;
    }
    const int tc = tr + rem;
    const uint64_t r = (uint64_t)tr * kGT + rl, c = (uint64_t)tc * kGT + cl;
    if (r >= kd || c >= kd || (tr == tc && r > c)) continue;
    double re = 0.0, im = 0.0;
    for (int s = 0; s < nsplit; ++s) {
      const double2 v = part[((size_t)s * pairs + pair) * (kGT * kGT) + w];
      re += v.x;
      im += v.y;
    }
    rho[r * kd + c] = make_double2(re, r == c ? 0.0 : im);
    if (r != c) rho[c * kd + r] = make_double2(re, -im);
  }
}

// ---- Householder tridiagonalisation (A Hermitian, row-major, n x n)

// Reflector for column k: x_j = A[j][k] = conj(A[k][j]) for j > k.
// v = (x - alpha e_{k+1}) / |x - alpha e_{k+1}|, alpha = -phase(x_{k+1}) |x|.
// Writes v[j] (j > k), d[k] = Re A[k][k], e[k] = |alpha|, flag = 0 when x = 0.
__global__ void hh_vector_kernel(const double2* __restrict__ A, int n, int k, double2* __restrict__ v,
                                 double* __restrict__ d, double* __restrict__ e, int* __restrict__ flag) {
  __shared__ double red[32];
  const size_t row = (size_t)k * n;
  double s = 0.0;
  for (int j = k + 1 + threadIdx.x; j < n; j += blockDim.x) {
    const double2 a = A[row + j];
    s += a.x * a.x + a.y * a.y;
  }
  const double xn2 = block_allsum(s, red);
  const double xn = sqrt(xn2);
  const double2 a0 = A[row + k + 1];
  const double2 x0 = make_double2(a0.x, -a0.y);
  const double ax0 = hypot(x0.x, x0.y);
  const double2 ph = ax0 > 0.0 ? make_double2(x0.x / ax0, x0.y / ax0) : make_double2(1.0, 0.0);
  const double2 alpha = make_double2(-ph.x * xn, -ph.y * xn);
  const double2 v0 = make_double2(x0.x - alpha.x, x0.y - alpha.y);
  // |v|^2 = |x0 - alpha|^2 + (|x|^2 - |x0|^2)
  const double vn2 = v0.x * v0.x + v0.y * v0.y + (xn2 - (x0.x * x0.x + x0.y * x0.y));
  const bool ok = xn > 0.0 && vn2 > 0.0;
  const double inv = ok ? 1.0 / sqrt(vn2) : 0.0;
  for (int j = k + 1 + threadIdx.x; j < n; j += blockDim.x) {
    double2 x;
    if (j == k + 1) {
      x = v0;
    } else {
      const double2 a = A[row + j];
      x = make_double2(a.x, -a.y);
    }
    v[j] = make_double2(x.x * inv, x.y * inv);
  }
  if (threadIdx.x == 0) {
    d[k] = A[row + k].x;
    e[k] = xn;
    *flag = ok ? 1 : 0;
  }
}

// p_i = sum_{j > k} A[i][j] v_j for i > k; one warp per row
__global__ void hh_hemv_kernel(const double2* __restrict__ A, int n, int k, const double2* __restrict__ v,
                               const int* __restrict__ flag, double2* __restrict__ p) {
  if (!*flag) return;
  const int lane = threadIdx.x & 31;
  const int i = k + 1 + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= n) return;
  const double2* row = A + (size_t)i * n;
  double re = 0.0, im = 0.0;
  for (int j = k + 1 + lane; j < n; j += 32) {
    const double2 a = row[j], b = v[j];
    re = fma(a.x, b.x, fma(-a.y, b.y, re));
    im = fma(a.x, b.y, fma(a.y, b.x, im));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_xor_sync(0xffffffffu, re, o);
    im += __shfl_xor_sync(0xffffffffu, im, o);
  }
  if (lane == 0) p[i] = make_double2(re, im);
}

// K = v^H p, w = 2 (p - K v)
__global__ void hh_w_kernel(int n, int k, const double2* __restrict__ v, const double2* __restrict__ p,
                            const int* __restrict__ flag, double2* __restrict__ w) {
  if (!*flag) return;
  __shared__ double red[32];
  double kr = 0.0, ki = 0.0;
  for (int j = k + 1 + threadIdx.x; j < n; j += blockDim.x) {
    const double2 a = v[j], b = p[j];
    // conj(a) * b
    kr += a.x * b.x + a.y * b.y;
    ki += a.x * b.y - a.y * b.x;
  }
  kr = block_allsum(kr, red);
  __syncthreads();
  ki = block_allsum(ki, red);
  for (int j = k + 1 + threadIdx.x; j < n; j += blockDim.x) {
    const double2 a = v[j], b = p[j];
    w[j] = make_double2(2.0 * (b.x - (kr * a.x - ki * a.y)), 2.0 * (b.y - (kr * a.y + ki * a.x)));
  }
}

// A[i][j] -= v_i conj(w_j) + w_i conj(v_j) for i, j > k
__global__ void hh_her2_kernel(double2* __restrict__ A, int n, int k, const double2* __restrict__ v,
                               const double2* __restrict__ w, const int* __restrict__ flag) {
  if (!*flag) return;
  const int j = k + 1 + blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const double2 vj = v[j], wj = w[j];
  for (int i = k + 1 + blockIdx.y; i < n; i += gridDim.y) {
    const double2 vi = v[i], wi = w[i];
    double2 a = A[(size_t)i * n + j];
    // v_i conj(w_j) + w_i conj(v_j)
    const double re = vi.x * wj.x + vi.y * wj.y + wi.x * vj.x + wi.y * vj.y;
    const double im = vi.y * wj.x - vi.x * wj.y + wi.y * vj.x - wi.x * vj.y;
    a.x -= re;
    a.y -= im;
    A[(size_t)i * n + j] = a;
  }
}

// the last 2 x 2 block
__global__ void hh_tail_kernel(const double2* __restrict__ A, int n, double* __restrict__ d, double* __restrict__ e) {
  if (threadIdx.x != 0) return;
  if (n >= 2) {
    d[n - 2] = A[(size_t)(n - 2) * n + n - 2].x;
    const double2 b = A[(size_t)(n - 1) * n + n - 2];
    e[n - 2] = hypot(b.x, b.y);
  }
  d[n - 1] = A[(size_t)(n - 1) * n + n - 1].x;
}

// number of eigenvalues of the tridiagonal (d, e) below x (Sturm count)
__device__ int sturm_count(const double* __restrict__ d, const double* __restrict__ e, int n, double x,
                           double pivmin) {
  int cnt = 0;
  double q = d[0] - x;
  if (fabs(q) < pivmin) q = -pivmin;
  if (q < 0.0) ++cnt;
  for (int i = 1; i < n; ++i) {
    q = (d[i] - x) - (e[i - 1] * e[i - 1]) / q;
    if (fabs(q) < pivmin) q = -pivmin;
    if (q < 0.0) ++cnt;
  }
  return cnt;
}

// eig[i] = i-th smallest eigenvalue, by bisection inside the Gershgorin interval
__global__ void bisect_kernel(const double* __restrict__ d, const double* __restrict__ e, int n,
                              double* __restrict__ eig) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double lo = d[0], hi = d[0], emax2 = 0.0;
  for (int t = 0; t < n; ++t) {
    const double r = (t > 0 ? e[t - 1] : 0.0) + (t + 1 < n ? e[t] : 0.0);
    lo = fmin(lo, d[t] - r);
    hi = fmax(hi, d[t] + r);
    if (t + 1 < n) emax2 = fmax(emax2, e[t] * e[t]);
  }
  const double span = fmax(fabs(lo), fabs(hi));
  lo -= 2.0 * DBL_EPSILON * span * n + 1e-300;
  hi += 2.0 * DBL_EPSILON * span * n + 1e-300;
  const double pivmin = 1e-290 * fmax(1.0, emax2);
  for (int it = 0; it < 256; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (hi - lo <= 2.0 * DBL_EPSILON * fmax(fabs(lo), fabs(hi)) + 1e-300 || mid <= lo || mid >= hi) break;
    if (sturm_count(d, e, n, mid, pivmin) > i) hi = mid;
    else lo = mid;
  }
  eig[i] = 0.5 * (lo + hi);
}

uint64_t deposit(uint64_t x, const int* bits, int nb) {
  uint64_t r = 0;
  for (int b = 0; b < nb; ++b)
    if ((x >> b) & 1) r |= 1ULL << bits[b];
  return r;
}

}  // namespace

int reduced_spectrum_max_bits() { return 13; }

cudaError_t reduced_spectrum(const double2* psi, int nbits, const int* keep, int k, std::vector<double>& eig,
                             cudaStream_t st) {
  if (k < 1 || k > reduced_spectrum_max_bits() || k >= nbits) return cudaErrorInvalidValue;
  std::vector<int> traced;
  for (int q = 0; q < nbits; ++q) {
    bool in = false;
    for (int i = 0; i < k; ++i) in |= keep[i] == q;
    if (!in) traced.push_back(q);
  }
  const int nt = (int)traced.size();
  const uint64_t kd = 1ULL << k, ed = 1ULL << nt;
  const int lobits = (nt + 1) / 2, hibits = nt - lobits;
  std::vector<uint64_t> h_depk(kd), h_lo(1ULL << lobits), h_hi(1ULL << hibits);
  for (uint64_t r = 0; r < kd; ++r) h_depk[r] = deposit(r, keep, k);
  for (uint64_t x = 0; x < h_lo.size(); ++x) h_lo[x] = deposit(x, traced.data(), lobits);
  for (uint64_t x = 0; x < h_hi.size(); ++x) h_hi[x] = deposit(x, traced.data() + lobits, hibits);

  const int tiles = (int)((kd + kGT - 1) / kGT);
  const int pairs = tiles * (tiles + 1) / 2;
  // split the environment so that at least ~4 CTAs per SM run, in chunks of >= 256 entries
  int nsplit = 1;
  while ((uint64_t)pairs * nsplit < 4 * 148 && ed / (2ULL * nsplit) >= 256) nsplit *= 2;
  const uint64_t per = ed / nsplit;

  const size_t n = (size_t)kd;
  const size_t bytes_rho = n * n * sizeof(double2);
  const size_t bytes_part = nsplit > 1 ? (size_t)nsplit * pairs * kGT * kGT * sizeof(double2) : 0;
  const size_t bytes_vec = 3 * n * sizeof(double2) + 3 * n * sizeof(double) + sizeof(int);
  const size_t bytes_dep = (h_depk.size() + h_lo.size() + h_hi.size()) * sizeof(uint64_t);
  char* buf = nullptr;
  const size_t total = bytes_rho + bytes_part + bytes_vec + bytes_dep + 1024;
  cudaError_t err = cudaMallocAsync(&buf, total, st);
  if (err != cudaSuccess) return err;
  auto align = [](size_t x) { return (x + 255) & ~(size_t)255; };
  size_t off = 0;
  double2* rho = reinterpret_cast<double2*>(buf + off);
  off = align(off + bytes_rho);
  double2* part = bytes_part ? reinterpret_cast<double2*>(buf + off) : nullptr;
  off = align(off + bytes_part);
  double2* v = reinterpret_cast<double2*>(buf + off);
  double2* p = v + n;
  double2* w = p + n;
  double* d = reinterpret_cast<double*>(w + n);
  double* e = d + n;
  double* ev = e + n;
  int* flag = reinterpret_cast<int*>(ev + n);
  off = align(off + bytes_vec);
  uint64_t* depk = reinterpret_cast<uint64_t*>(buf + off);
  uint64_t* lo = depk + h_depk.size();
  uint64_t* hi = lo + h_lo.size();

  err = cudaMemcpyAsync(depk, h_depk.data(), h_depk.size() * 8, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(lo, h_lo.data(), h_lo.size() * 8, cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) err = cudaMemcpyAsync(hi, h_hi.data(), h_hi.size() * 8, cudaMemcpyHostToDevice, st);
  uint64_t launches = 0;
  if (err == cudaSuccess) {
    EnvDep dep{lo, hi, lobits};
    gram_kernel<<<dim3(pairs, nsplit), kGThreads, 0, st>>>(psi, depk, dep, tiles, kd, per, part, rho);
    ++launches;
    if (nsplit > 1) {
      gram_reduce_kernel<<<std::min<uint64_t>(((uint64_t)pairs * kGT * kGT + 255) / 256, 148 * 16), 256, 0, st>>>(
          part, pairs, tiles, nsplit, kd, rho);
      ++launches;
    }
    err = cudaGetLastError();
  }
  const int nn = (int)n;
  for (int kcol = 0; err == cudaSuccess && kcol + 2 < nn; ++kcol) {
    const int m = nn - kcol - 1;
    hh_vector_kernel<<<1, 1024, 0, st>>>(rho, nn, kcol, v, d, e, flag);
    hh_hemv_kernel<<<(m + 7) / 8, 256, 0, st>>>(rho, nn, kcol, v, flag, p);
    hh_w_kernel<<<1, 1024, 0, st>>>(nn, kcol, v, p, flag, w);
    const int gy = std::min(m, 256);
    hh_her2_kernel<<<dim3((m + 127) / 128, gy), 128, 0, st>>>(rho, nn, kcol, v, w, flag);
    launches += 4;
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) {
    hh_tail_kernel<<<1, 32, 0, st>>>(rho, nn, d, e);
    bisect_kernel<<<(nn + 127) / 128, 128, 0, st>>>(d, e, nn, ev);
    launches += 2;
    err = cudaGetLastError();
  }
  count_launches(launches);
  eig.assign(n, 0.0);
  if (err == cudaSuccess) err = cudaMemcpyAsync(eig.data(), ev, n * sizeof(double), cudaMemcpyDeviceToHost, st);
  const cudaError_t ferr = cudaFreeAsync(buf, st);
  const cudaError_t serr = cudaStreamSynchronize(st);
  if (err == cudaSuccess) err = ferr;
  if (err == cudaSuccess) err = serr;
  return err;
}

}  // namespace iqb
