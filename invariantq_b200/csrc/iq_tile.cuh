// iq_tile.cuh -- the tile-pass kernel template (device code), shared by the
// translation units that instantiate it (iq_tile_r4.cu, iq_tile_r5.cu).
//
// One launch = one pass over the complex128 array (16 B per amplitude read
// once, written once).  Tiles of 2^M amplitudes move between HBM and shared
// memory with TMA tensor copies (cp.async.bulk.tensor, 128-byte swizzle,
// mbarrier completion) through a ring of tile buffers; the CTA's threads apply
// the pass's register stages (see iq_plan.h) to the resident tile.  This
// replaces the reference's per-gate OpenMP sweeps (core/src/statevector.cpp:
// 26-152) and its two-pass density-matrix updates (core/src/density_matrix.cpp:
// 18-163): a density matrix is the same array with 2n index bits, U rho
// U^dagger is U on the row bits and conj(U) on the column bits, and a Kraus
// channel is the superoperator sum_k K_k (x) conj(K_k) on the (row, column) bits.
//
// Every wait on an mbarrier is bounded; a wait that runs out sets a status word
// the host reads, and the CTA finishes its loop without further copies.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <atomic>

#include "iq_kernels.h"
#include "iq_pipe.cuh"

namespace iqb {

// Raise a kernel's dynamic shared-memory limit to everything the device allows
// beside the kernel's static shared memory, once per device.  Setting it per
// launch to the launch's own size races between host threads: another thread's
// smaller setting can land between this thread's setting and its launch.
// Occupancy still follows each launch's actual dynamic size.
template <class K>
inline cudaError_t allow_full_dynamic_smem(K kern, std::atomic<uint64_t>& done) {
  int dev = 0;
  cudaError_t r = cudaGetDevice(&dev);
  if (r != cudaSuccess) return r;
  const uint64_t bit = 1ULL << (dev & 63);
  if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
  int optin = 0;
  r = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  if (r != cudaSuccess) return r;
  cudaFuncAttributes fa{};
  r = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(kern));
  if (r != cudaSuccess) return r;
  r = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes);
  if (r == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
  return r;
}

// ------------------------------------------------------- register-slot ops
//
// Every operation reads the register array `s` and writes all of its outputs
// to `d`.  With R = 4 the stage alternates between two arrays (ping-pong), so
// results go straight to their final registers.  With R = 5 (32 amplitudes per
// thread) there is room for one array only and the same code runs in place
// (s and d alias); the INPLACE flag selects orders that stay correct then.

template <int R, int S>
__device__ __forceinline__ void d1r(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m,
                                    bool real = false) {
  const double2 u0 = ld_mat(m, 0), u1 = ld_mat(m, 1), u2 = ld_mat(m, 2), u3 = ld_mat(m, 3);
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & (1 << S)) continue;
    const double2 x = s[v], y = s[v | (1 << S)];
    if (real) {   // OPF_REAL: the imaginary parts are zero and not read
      d[v] = rlin(u0.x, x, u1.x, y);
      d[v | (1 << S)] = rlin(u2.x, x, u3.x, y);
    } else {
      d[v] = cfma(cmul(u0, x), u1, y);
      d[v | (1 << S)] = cfma(cmul(u2, x), u3, y);
    }
  }
}

// normalised 2x2 (OP_N1R): row 0's entry in column COL is exactly 1
template <int R, int S, int COL>
__device__ __forceinline__ void n1r(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m) {
  const double2 u = ld_mat(m, 1 - COL), u2 = ld_mat(m, 2), u3 = ld_mat(m, 3);
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & (1 << S)) continue;
    const double2 x = s[v], y = s[v | (1 << S)];
    d[v] = COL == 0 ? cfma(x, u, y) : cfma(y, u, x);
    d[v | (1 << S)] = cfma(cmul(u2, x), u3, y);
  }
}

// normalised real rotation (OP_R1R): FORM 0 [[1, -t], [t, 1]] (t = Re m[2]),
// FORM 1 [[u, -1], [1, u]] (u = Re m[0]); 2 FMAs per amplitude
template <int R, int S, int FORM>
__device__ __forceinline__ void r1r(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m) {
  const double w = FORM == 0 ? ld_mat(m, 2).x : ld_mat(m, 0).x;
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & (1 << S)) continue;
    const double2 x = s[v], y = s[v | (1 << S)];
    d[v] = rot_row0<FORM>(w, x, y);
    d[v | (1 << S)] = rot_row1<FORM>(w, x, y);
  }
}

template <int R, int S, bool SW, bool UNIT>
__device__ __forceinline__ void m1r_t(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m) {
  double2 p0 = make_double2(1.0, 0.0), p1 = p0;
  if (!UNIT) { p0 = ld_mat(m, 0); p1 = ld_mat(m, 1); }
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & (1 << S)) continue;
    double2 x = s[v], y = s[v | (1 << S)];
    if (SW) { const double2 t = x; x = y; y = t; }
    if (!UNIT) { x = cmul(p0, x); y = cmul(p1, y); }
    d[v] = x;
    d[v | (1 << S)] = y;
  }
}

template <int R, int S>
__device__ __forceinline__ void m1r(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m, int perm,
                                    bool unit) {
  if (perm & 1) {
    if (unit) m1r_t<R, S, true, true>(s, d, m);
    else m1r_t<R, S, true, false>(s, d, m);
  } else if (unit) {
    m1r_t<R, S, false, true>(s, d, m);
  } else {
    m1r_t<R, S, false, false>(s, d, m);
  }
}

// dense 4x4 on slots A (matrix bit 0) and B (matrix bit 1).  Row-outer when
// writing a separate array (one matrix row live at a time), group-outer in place.
template <int R, int A, int B, bool INPLACE>
__device__ __forceinline__ void d2r(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m) {
  if constexpr (INPLACE) {
#pragma unroll
    for (int v = 0; v < (1 << R); ++v) {
      if (v & ((1 << A) | (1 << B))) continue;
      const int idx[4] = {v, v | (1 << A), v | (1 << B), v | (1 << A) | (1 << B)};
      const double2 x[4] = {s[idx[0]], s[idx[1]], s[idx[2]], s[idx[3]]};
      double2 o[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        double2 acc = cmul(ld_mat(m, 4 * r + 0), x[0]);
        acc = cfma(acc, ld_mat(m, 4 * r + 1), x[1]);
        acc = cfma(acc, ld_mat(m, 4 * r + 2), x[2]);
        acc = cfma(acc, ld_mat(m, 4 * r + 3), x[3]);
        o[r] = acc;
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) d[idx[r]] = o[r];
    }
  } else {
    // two rows per step: 16 independent accumulation chains per thread
#pragma unroll
    for (int r = 0; r < 4; r += 2) {
      const double2 u0 = ld_mat(m, 4 * r + 0), u1 = ld_mat(m, 4 * r + 1), u2 = ld_mat(m, 4 * r + 2),
                    u3 = ld_mat(m, 4 * r + 3);
      const double2 w0 = ld_mat(m, 4 * r + 4), w1 = ld_mat(m, 4 * r + 5), w2 = ld_mat(m, 4 * r + 6),
                    w3 = ld_mat(m, 4 * r + 7);
      const int ro = ((r & 1) << A) | (((r >> 1) & 1) << B);
      const int ro1 = (((r + 1) & 1) << A) | ((((r + 1) >> 1) & 1) << B);
#pragma unroll
      for (int v = 0; v < (1 << R); ++v) {
        if (v & ((1 << A) | (1 << B))) continue;
        const double2 x0 = s[v], x1 = s[v | (1 << A)], x2 = s[v | (1 << B)], x3 = s[v | (1 << A) | (1 << B)];
        double2 acc = cmul(u0, x0), acc1 = cmul(w0, x0);
        acc = cfma(acc, u1, x1);
        acc1 = cfma(acc1, w1, x1);
        acc = cfma(acc, u2, x2);
        acc1 = cfma(acc1, w2, x2);
        acc = cfma(acc, u3, x3);
        acc1 = cfma(acc1, w3, x3);
        d[v | ro] = acc;
        d[v | ro1] = acc1;
      }
    }
  }
}

// Monomial 4x4 on slots A (matrix bit 0) and B (matrix bit 1): output row r
// takes input column (PERM >> 2r) & 3 times phase r (inputs read before writes).
template <int R, int A, int B, int PERM, bool UNIT>
__device__ __forceinline__ void m2r_t(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m) {
  double2 p[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) p[r] = UNIT ? make_double2(1.0, 0.0) : ld_mat(m, r);
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & ((1 << A) | (1 << B))) continue;
    const int idx[4] = {v, v | (1 << A), v | (1 << B), v | (1 << A) | (1 << B)};
    const double2 x[4] = {s[idx[0]], s[idx[1]], s[idx[2]], s[idx[3]]};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double2 y = x[(PERM >> (2 * r)) & 3];
      d[idx[r]] = UNIT ? y : cmul(p[r], y);
    }
  }
}

__device__ __forceinline__ double2 sel4(int i, double2 x0, double2 x1, double2 x2, double2 x3) {
  const double2 lo = (i & 1) ? x1 : x0;
  const double2 hi = (i & 1) ? x3 : x2;
  return (i & 2) ? hi : lo;
}

template <int R, int A, int B>
__device__ __forceinline__ void m2r_generic(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m,
                                            int perm, bool unit) {
  const int c0 = perm & 3, c1 = (perm >> 2) & 3, c2 = (perm >> 4) & 3, c3 = (perm >> 6) & 3;
  double2 p0 = make_double2(1.0, 0.0), p1 = p0, p2 = p0, p3 = p0;
  if (!unit) { p0 = ld_mat(m, 0); p1 = ld_mat(m, 1); p2 = ld_mat(m, 2); p3 = ld_mat(m, 3); }
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & ((1 << A) | (1 << B))) continue;
    const int i0 = v, i1 = v | (1 << A), i2 = v | (1 << B), i3 = v | (1 << A) | (1 << B);
    const double2 x0 = s[i0], x1 = s[i1], x2 = s[i2], x3 = s[i3];
    double2 o0 = sel4(c0, x0, x1, x2, x3), o1 = sel4(c1, x0, x1, x2, x3);
    double2 o2 = sel4(c2, x0, x1, x2, x3), o3 = sel4(c3, x0, x1, x2, x3);
    if (!unit) { o0 = cmul(p0, o0); o1 = cmul(p1, o1); o2 = cmul(p2, o2); o3 = cmul(p3, o3); }
    d[i0] = o0;
    d[i1] = o1;
    d[i2] = o2;
    d[i3] = o3;
  }
}

constexpr int kPermId = 0xE4;     // [0, 1, 2, 3]: diagonal gates (CZ, CP, CRZ)
constexpr int kPermCx1 = 0xB4;    // [0, 1, 3, 2]: X on bit 0 controlled by bit 1
constexpr int kPermCx0 = 0x6C;    // [0, 3, 2, 1]: X on bit 1 controlled by bit 0
constexpr int kPermSwap = 0xD8;   // [0, 2, 1, 3]

template <int R, int A, int B>
__device__ __forceinline__ void m2r(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m, int perm,
                                    bool unit) {
  if (unit) {
    switch (perm) {
      case kPermId: m2r_t<R, A, B, kPermId, true>(s, d, m); return;
      case kPermCx1: m2r_t<R, A, B, kPermCx1, true>(s, d, m); return;
      case kPermCx0: m2r_t<R, A, B, kPermCx0, true>(s, d, m); return;
      case kPermSwap: m2r_t<R, A, B, kPermSwap, true>(s, d, m); return;
      default: break;
    }
  } else if (perm == kPermId) {
    m2r_t<R, A, B, kPermId, false>(s, d, m);
    return;
  }
  m2r_generic<R, A, B>(s, d, m, perm, unit);
}

// shared-memory slot offset of register v: XOR of the (swizzled) slot bits
// set in v; v is a compile-time constant after unrolling, so this folds to a
// few XORs of values computed once per stage
template <int R>
__device__ __forceinline__ uint32_t voff(int v, const uint32_t (&sb)[R]) {
  uint32_t o = 0;
#pragma unroll
  for (int i = 0; i < R; ++i)
    if ((v >> i) & 1) o ^= sb[i];
  return o;
}

// dense 2^K block on slots 0..K-1, written straight to the tile (ends the stage);
// rows are a runtime loop so only one row of the matrix is live at a time
template <int R, int K>
__device__ __forceinline__ void dkr_store(const double2 (&a)[1 << R], const double2* m, double2* tile,
                                          const uint32_t (&sb)[R], uint32_t base) {
  constexpr int D = 1 << K;
#pragma unroll
  for (int g = 0; g < (1 << R); g += D) {
    const uint32_t goff = base ^ voff<R>(g, sb);
#pragma unroll 1
    for (int r = 0; r < D; ++r) {
      double2 acc = cmul(ld_mat(m, r * D), a[g]);
#pragma unroll
      for (int c = 1; c < D; ++c) acc = cfma(acc, ld_mat(m, r * D + c), a[g + c]);
      uint32_t roff = 0;
#pragma unroll
      for (int i = 0; i < K; ++i)
        if ((r >> i) & 1) roff ^= sb[i];
      tile[goff ^ roff] = acc;
    }
  }
}

// lane-bit 1q ops: partner amplitude lives in lane ^ (1 << lb) of the octet

template <int R>
__device__ __forceinline__ void d1l(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m, int lb,
                                    int lane8, unsigned omask, bool real = false) {
  const int my = (lane8 >> lb) & 1;
  const double2 cs = my ? ld_mat(m, 3) : ld_mat(m, 0);
  const double2 co = my ? ld_mat(m, 2) : ld_mat(m, 1);
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    const double2 x = s[v];
    const double2 p = shfl_xor2(x, 1 << lb, omask);
    d[v] = real ? rlin(cs.x, x, co.x, p) : cfma(cmul(cs, x), co, p);
  }
}

template <int R, int FORM>
__device__ __forceinline__ void r1l(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m, int lb,
                                    int lane8, unsigned omask) {
  const bool hi = (lane8 >> lb) & 1;
  const double w = FORM == 0 ? ld_mat(m, 2).x : ld_mat(m, 0).x;
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    const double2 x = s[v];
    const double2 p = shfl_xor2(x, 1 << lb, omask);
    d[v] = rot_lane<FORM>(w, hi, x, p);
  }
}

template <int R>
__device__ __forceinline__ void m1l(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m, int lb,
                                    int lane8, unsigned omask, int perm, bool unit) {
  const int my = (lane8 >> lb) & 1;
  const double2 ph = unit ? make_double2(1.0, 0.0) : (my ? ld_mat(m, 1) : ld_mat(m, 0));
  const bool sw = perm & 1;
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    double2 x = s[v];
    if (sw) x = shfl_xor2(x, 1 << lb, omask);
    d[v] = unit ? x : cmul(ph, x);
  }
}

// OP_X2R on slots A (bit 0) and B (bit 1); flags bit 0 / 1: corners / middle real
template <int R, int A, int B>
__device__ __forceinline__ void x2r(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m, int flags) {
  const double2 m0 = ld_mat(m, 0), m3 = ld_mat(m, 3), m12 = ld_mat(m, 12), m15 = ld_mat(m, 15), m5 = ld_mat(m, 5),
                m10 = ld_mat(m, 10);
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & ((1 << A) | (1 << B))) continue;
    double2 x0 = s[v], x1 = s[v | (1 << A)], x2 = s[v | (1 << B)], x3 = s[v | (1 << A) | (1 << B)];
    switch (flags & 3) {
      case 3: xpat4<true, true>(x0, x1, x2, x3, m0, m3, m12, m15, m5, m10); break;
      case 1: xpat4<true, false>(x0, x1, x2, x3, m0, m3, m12, m15, m5, m10); break;
      case 2: xpat4<false, true>(x0, x1, x2, x3, m0, m3, m12, m15, m5, m10); break;
      default: xpat4<false, false>(x0, x1, x2, x3, m0, m3, m12, m15, m5, m10); break;
    }
    d[v] = x0;
    d[v | (1 << A)] = x1;
    d[v | (1 << B)] = x2;
    d[v | (1 << A) | (1 << B)] = x3;
  }
}

template <int R, int B, int GEN, int FORM>
__device__ __forceinline__ double grad2(const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m) {
  const double2 u0 = ld_mat(m, 0), u1 = ld_mat(m, 1), u3 = ld_mat(m, 3);
  double acc = 0.0;
#pragma unroll
  for (int v = 0; v < (1 << R); ++v) {
    if (v & (1 | (1 << B))) continue;
    const double2 p0 = s[v], p1 = s[v | (1 << B)], l0 = s[v | 1], l1 = s[v | 1 | (1 << B)];
    acc += grad_term<GEN>(p0, p1, l0, l1);
    unrotate<GEN, FORM>(p0, p1, d[v], d[v | (1 << B)], u0, u1, u3);
    unrotate<GEN, FORM>(l0, l1, d[v | 1], d[v | 1 | (1 << B)], u0, u1, u3);
  }
  return acc;
}

// ------------------------------------------------------- runtime dispatch

template <int R, int S = 0>
__device__ __forceinline__ void disp_d1r(int sl, const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m,
                                         bool real) {
  if constexpr (S < R) {
    if (sl == S) d1r<R, S>(s, d, m, real);
    else disp_d1r<R, S + 1>(sl, s, d, m, real);
  }
}
template <int R, int S = 0>
__device__ __forceinline__ void disp_n1r(int sl, int col, const double2 (&s)[1 << R], double2 (&d)[1 << R],
                                         const double2* m) {
  if constexpr (S < R) {
    if (sl == S) {
      if (col) n1r<R, S, 1>(s, d, m);
      else n1r<R, S, 0>(s, d, m);
    } else {
      disp_n1r<R, S + 1>(sl, col, s, d, m);
    }
  }
}
template <int R, int S = 0>
__device__ __forceinline__ void disp_r1r(int sl, int form, const double2 (&s)[1 << R], double2 (&d)[1 << R],
                                         const double2* m) {
  if constexpr (S < R) {
    if (sl == S) {
      if (form) r1r<R, S, 1>(s, d, m);
      else r1r<R, S, 0>(s, d, m);
    } else {
      disp_r1r<R, S + 1>(sl, form, s, d, m);
    }
  }
}
template <int R, int S = 0>
__device__ __forceinline__ void disp_m1r(int sl, const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m,
                                         int perm, bool unit) {
  if constexpr (S < R) {
    if (sl == S) m1r<R, S>(s, d, m, perm, unit);
    else disp_m1r<R, S + 1>(sl, s, d, m, perm, unit);
  }
}
template <int R, bool IP, int A, int B = 0>
__device__ __forceinline__ void disp_d2r_b(int sb, const double2 (&s)[1 << R], double2 (&d)[1 << R],
                                           const double2* m) {
  if constexpr (B < R) {
    if constexpr (A != B) {
      if (sb == B) { d2r<R, A, B, IP>(s, d, m); return; }
    }
    disp_d2r_b<R, IP, A, B + 1>(sb, s, d, m);
  }
}
template <int R, bool IP, int A = 0>
__device__ __forceinline__ void disp_d2r(int sa, int sb, const double2 (&s)[1 << R], double2 (&d)[1 << R],
                                         const double2* m) {
  if constexpr (A < R) {
    if (sa == A) disp_d2r_b<R, IP, A>(sb, s, d, m);
    else disp_d2r<R, IP, A + 1>(sa, sb, s, d, m);
  }
}
template <int R, int A, int B = 0>
__device__ __forceinline__ void disp_m2r_b(int sb, const double2 (&s)[1 << R], double2 (&d)[1 << R], const double2* m,
                                           int perm, bool unit) {
  if constexpr (B < R) {
    if constexpr (A != B) {
      if (sb == B) { m2r<R, A, B>(s, d, m, perm, unit); return; }
    }
    disp_m2r_b<R, A, B + 1>(sb, s, d, m, perm, unit);
  }
}
template <int R, int A = 0>
__device__ __forceinline__ void disp_m2r(int sa, int sb, const double2 (&s)[1 << R], double2 (&d)[1 << R],
                                         const double2* m, int perm, bool unit) {
  if constexpr (A < R) {
    if (sa == A) disp_m2r_b<R, A>(sb, s, d, m, perm, unit);
    else disp_m2r<R, A + 1>(sa, sb, s, d, m, perm, unit);
  }
}
template <int R, int K = 3>
__device__ __forceinline__ void disp_dkr(int k, const double2 (&a)[1 << R], const double2* m, double2* tile,
                                         const uint32_t (&sb)[R], uint32_t base) {
  if constexpr (K <= R) {
    if (k == K) dkr_store<R, K>(a, m, tile, sb, base);
    else disp_dkr<R, K + 1>(k, a, m, tile, sb, base);
  }
}

template <int R, int GEN, int FORM, int B = 1>
__device__ __forceinline__ double disp_grad2_b(int sb, const double2 (&s)[1 << R], double2 (&d)[1 << R],
                                               const double2* m) {
  if constexpr (B < R) {
    if (sb == B) return grad2<R, B, GEN, FORM>(s, d, m);
    return disp_grad2_b<R, GEN, FORM, B + 1>(sb, s, d, m);
  }
  return 0.0;
}

// Apply one operation from s to d; returns true when it wrote the tile itself.
template <int R, bool IP>
__device__ __forceinline__ bool apply_op(const OpDesc& od, const double2 (&s)[1 << R], double2 (&d)[1 << R],
                                         const double2* mats, int lane8, unsigned omask, double2* tile,
                                         const uint32_t (&sb)[R], uint32_t base, double* sgrad,
                                         uint32_t grad_base) {
  (void)grad_base;
  const double2* m = mats + od.mat;
  const bool unit = od.flags & OPF_UNIT_PHASE;
  switch (od.kind) {
    case OP_GRAD2: {
      // the planner puts the select bit in slot 0
      double acc;
      // generator (perm) and the inverse rotation's form (flags, a GradForm)
      switch (od.perm * 4 + od.flags) {
        case 0: acc = disp_grad2_b<R, 0, 0>(od.b, s, d, m); break;
        case 1: acc = disp_grad2_b<R, 0, 1>(od.b, s, d, m); break;
        case 2: acc = disp_grad2_b<R, 0, 2>(od.b, s, d, m); break;
        case 4: acc = disp_grad2_b<R, 1, 0>(od.b, s, d, m); break;
        case 5: acc = disp_grad2_b<R, 1, 1>(od.b, s, d, m); break;
        case 6: acc = disp_grad2_b<R, 1, 2>(od.b, s, d, m); break;
        case 9: acc = disp_grad2_b<R, 2, 1>(od.b, s, d, m); break;
        default: acc = disp_grad2_b<R, 2, 0>(od.b, s, d, m); break;
      }
      grad_accumulate(acc, sgrad + od.gidx, lane8, omask);
      break;
    }
    case OP_D1R: disp_d1r<R>(od.a, s, d, m, od.flags & OPF_REAL); break;
    case OP_N1R: disp_n1r<R>(od.a, od.perm, s, d, m); break;
    case OP_R1R: disp_r1r<R>(od.a, od.perm, s, d, m); break;
    case OP_R1L:
      if (od.perm) r1l<R, 1>(s, d, m, od.a, lane8, omask);
      else r1l<R, 0>(s, d, m, od.a, lane8, omask);
      break;
    case OP_D1L: d1l<R>(s, d, m, od.a, lane8, omask, od.flags & OPF_REAL); break;
    case OP_X2R:
      switch (od.a * 8 + od.b) {
#define IQ_X2R_CASE(A, B)                                               \
  case A * 8 + B:                                                       \
    if constexpr (A < R && B < R && A != B) x2r<R, A, B>(s, d, m, od.flags); \
    break;
        IQ_X2R_CASE(0, 1) IQ_X2R_CASE(0, 2) IQ_X2R_CASE(0, 3) IQ_X2R_CASE(0, 4)
        IQ_X2R_CASE(1, 0) IQ_X2R_CASE(1, 2) IQ_X2R_CASE(1, 3) IQ_X2R_CASE(1, 4)
        IQ_X2R_CASE(2, 0) IQ_X2R_CASE(2, 1) IQ_X2R_CASE(2, 3) IQ_X2R_CASE(2, 4)
        IQ_X2R_CASE(3, 0) IQ_X2R_CASE(3, 1) IQ_X2R_CASE(3, 2) IQ_X2R_CASE(3, 4)
        IQ_X2R_CASE(4, 0) IQ_X2R_CASE(4, 1) IQ_X2R_CASE(4, 2) IQ_X2R_CASE(4, 3)
#undef IQ_X2R_CASE
        default: break;
      }
      break;
    case OP_D2R:
      // one jump over the ordered slot pair (a, b) instead of nested compares
      switch (od.a * 8 + od.b) {
#define IQ_D2R_CASE(A, B)                                               \
  case A * 8 + B:                                                       \
    if constexpr (A < R && B < R && A != B) d2r<R, A, B, IP>(s, d, m); \
    break;
        IQ_D2R_CASE(0, 1) IQ_D2R_CASE(0, 2) IQ_D2R_CASE(0, 3) IQ_D2R_CASE(0, 4)
        IQ_D2R_CASE(1, 0) IQ_D2R_CASE(1, 2) IQ_D2R_CASE(1, 3) IQ_D2R_CASE(1, 4)
        IQ_D2R_CASE(2, 0) IQ_D2R_CASE(2, 1) IQ_D2R_CASE(2, 3) IQ_D2R_CASE(2, 4)
        IQ_D2R_CASE(3, 0) IQ_D2R_CASE(3, 1) IQ_D2R_CASE(3, 2) IQ_D2R_CASE(3, 4)
        IQ_D2R_CASE(4, 0) IQ_D2R_CASE(4, 1) IQ_D2R_CASE(4, 2) IQ_D2R_CASE(4, 3)
#undef IQ_D2R_CASE
        default: break;
      }
      break;
    case OP_M1R: disp_m1r<R>(od.a, s, d, m, od.perm, unit); break;
    case OP_M1L: m1l<R>(s, d, m, od.a, lane8, omask, od.perm, unit); break;
    case OP_M2R:
      switch (od.a * 8 + od.b) {
#define IQ_M2R_CASE(A, B)                                                          \
  case A * 8 + B:                                                                  \
    if constexpr (A < R && B < R && A != B) m2r<R, A, B>(s, d, m, od.perm, unit); \
    break;
        IQ_M2R_CASE(0, 1) IQ_M2R_CASE(0, 2) IQ_M2R_CASE(0, 3) IQ_M2R_CASE(0, 4)
        IQ_M2R_CASE(1, 0) IQ_M2R_CASE(1, 2) IQ_M2R_CASE(1, 3) IQ_M2R_CASE(1, 4)
        IQ_M2R_CASE(2, 0) IQ_M2R_CASE(2, 1) IQ_M2R_CASE(2, 3) IQ_M2R_CASE(2, 4)
        IQ_M2R_CASE(3, 0) IQ_M2R_CASE(3, 1) IQ_M2R_CASE(3, 2) IQ_M2R_CASE(3, 4)
        IQ_M2R_CASE(4, 0) IQ_M2R_CASE(4, 1) IQ_M2R_CASE(4, 2) IQ_M2R_CASE(4, 3)
#undef IQ_M2R_CASE
        default: break;
      }
      break;
    case OP_DKR: disp_dkr<R>(od.k, s, m, tile, sb, base); return true;
    default: break;
  }
  return false;
}

// One stage over the resident tile (consumer threads only).  Tile amplitude j
// lives in shared-memory slot swz(j); every offset below is kept swizzled.
template <int R>
__device__ __forceinline__ void run_stage(double2* tile, const PassDesc& P, int s, const double2* mats,
                                          int ctid, int ncons, double* gslots) {
  constexpr int NV = 1 << R;
  const StageDesc& sd = P.st[s];
  double* sgrad = gslots + (ctid >> 3) * P.ngrad;   // this octet's row of gradient accumulators
  const int lane8 = ctid & 7;
  const unsigned omask = 0xFFu << (ctid & 24);
  const uint32_t laneoff = ((uint32_t)(lane8 & 1) << sd.lane[0]) | ((uint32_t)((lane8 >> 1) & 1) << sd.lane[1]) |
                           ((uint32_t)((lane8 >> 2) & 1) << sd.lane[2]);
  uint32_t sb[R];
#pragma unroll
  for (int i = 0; i < R; ++i) sb[i] = swz(1u << sd.S[i]);
  const int nsub = 1 << sd.nt;
  const int op0 = sd.op0, op1 = sd.op1;
  for (int u = ctid >> 3; u < nsub; u += ncons >> 3) {
    uint32_t base = laneoff;
    for (int i = 0; i < sd.nt; ++i) base |= (uint32_t)((u >> i) & 1) << sd.tb[i];
    base = swz(base);
    double2 a[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) a[v] = tile[base ^ voff<R>(v, sb)];
    bool stored = false;
    if constexpr (R <= 4) {
      // ops alternate a -> b, b -> a (two inlined dispatch sites only); after an
      // odd count the result is in b and is stored from there
      double2 b[NV];
      bool inb = false;
      for (int o = op0; o < op1; o += 2) {
        stored |= apply_op<R, false>(P.ops[o], a, b, mats, lane8, omask, tile, sb, base, sgrad, P.grad_base);
        if (o + 1 < op1) stored |= apply_op<R, false>(P.ops[o + 1], b, a, mats, lane8, omask, tile, sb, base, sgrad, P.grad_base);
        else inb = true;
      }
      if (!stored) {
        if (inb) {
#pragma unroll
          for (int v = 0; v < NV; ++v) tile[base ^ voff<R>(v, sb)] = b[v];
        } else {
#pragma unroll
          for (int v = 0; v < NV; ++v) tile[base ^ voff<R>(v, sb)] = a[v];
        }
      }
      continue;
    } else {
      for (int o = op0; o < op1; ++o) stored |= apply_op<R, true>(P.ops[o], a, a, mats, lane8, omask, tile, sb, base, sgrad, P.grad_base);
    }
    if (!stored) {
#pragma unroll
      for (int v = 0; v < NV; ++v) tile[base ^ voff<R>(v, sb)] = a[v];
    }
  }
}

// The interpreting kernel's stages: run_stage over the pass descriptor.
template <int R, int NT>
struct InterpStages {
  const PassDesc& P;
  __device__ __forceinline__ void operator()(double2* buf, const double2* smat, double* gslots, bool work) {
    for (int s = 0; s < P.nstages; ++s) {
      if (work) run_stage<R>(buf, P, s, smat, threadIdx.x, NT, gslots);
      __syncthreads();
    }
  }
};

// The interpreting tile-pass kernel: NT threads per CTA run the pass's stages
// (run_stage) on each tile the pipeline makes resident.
template <int R, int NT, int MINB>
__global__ void __launch_bounds__(NT, MINB)
    tile_pass_kernel(const __grid_constant__ CUtensorMap tm, const __grid_constant__ PassDesc P,
                     const double2* __restrict__ mats, int* __restrict__ status, int nbuf,
                     double* __restrict__ grad_partials) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  InterpStages<R, NT> stages{P};
  set_tile_pass<NT>(tm, P, mats, status, nbuf, grad_partials, smem_raw, stages);
}

}  // namespace iqb
