// iq_pipe.cuh -- device code shared by the tile-pass kernels: complex
// arithmetic helpers, mbarrier / TMA wrappers, bounded waits, and the tile
// pipeline (a ring of shared-memory tile buffers fed and drained by TMA tensor
// copies).  The interpreting kernel (iq_tile.cuh) and the kernels generated
// per pass at run time (iq_jit.cpp, compiled with NVRTC) both run their
// stages inside tile_pipeline(), so both move tiles the same way.  The file
// compiles under nvcc and under NVRTC (__CUDACC_RTC__: no system headers).
#pragma once
#if defined(__CUDACC_RTC__)
struct __align__(64) CUtensorMap { unsigned long long opaque[16]; };   // layout of the driver's 128-byte map
#else
#include <cuda.h>
#include <cuda_runtime.h>
#endif

#include "iq_plan.h"

namespace iqb {

// ------------------------------------------------------------------ helpers

// explicit FMA forms: the interpreting and the generated kernels contract
// every complex product the same way, whatever the operands' origin
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -(a.y * b.y)), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cfma(double2 acc, double2 a, double2 b) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// operation matrices are read from the pass's block in shared memory
__device__ __forceinline__ double2 ld_mat(const double2* m, int i) { return m[i]; }

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ uint32_t mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done;
}

// try_wait that lets the hardware park the thread until the phase completes or
// `hint_ns` passes, so a waiting warp issues no instructions meanwhile (a plain
// try_wait returns almost at once and the polling loop would take issue slots
// from the warps that compute)
constexpr uint32_t kWaitSuspendNs = 20000;
__device__ __forceinline__ uint32_t mbar_try_wait_suspend(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity), "r"(hint_ns)
      : "memory");
  return done;
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                            int c4, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_u32(dst)),
      "l"(tm), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store_5d(const CUtensorMap* tm, int c0, int c1, int c2, int c3, int c4,
                                             const void* src) {
  asm volatile(
      "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group"
      " [%0, {%2, %3, %4, %5, %6}], [%1];" ::"l"(tm),
      "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
      : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// Wait limit of one mbarrier phase: 2 s of %globaltimer (a tile load or a
// consumer stage takes microseconds).
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded wait that ignores the abort flag: used to let copies already in
// flight land before the CTA exits after an abort.
__device__ __forceinline__ void drain_wait(uint64_t* bar, uint32_t parity) {
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait_suspend(bar, parity, kWaitSuspendNs))
    if (global_ns() - t0 > kWaitLimitNs) return;
}

// Bounded wait on an mbarrier phase.  Returns false (and raises the abort flag
// plus the status word) when the limit runs out, or as soon as another thread
// of the CTA has aborted.
__device__ __forceinline__ bool bounded_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag,
                                             int* status, int code, uint64_t limit_ns = kWaitLimitNs) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_wait_suspend(bar, parity, kWaitSuspendNs)) return true;
    if (*abort_flag) return false;
    if (global_ns() - t0 > limit_ns) break;
  }
  *abort_flag = 1;
  atomicCAS(status, 0, code);
  return false;
}


// rows of a normalised real rotation (OP_R1R) applied to the pair (x, y):
// FORM 0 [[1, -w], [w, 1]], FORM 1 [[w, -1], [1, w]]
template <int FORM>
__device__ __forceinline__ double2 rot_row0(double w, double2 x, double2 y) {
  return FORM == 0 ? make_double2(fma(-w, y.x, x.x), fma(-w, y.y, x.y))
                   : make_double2(fma(w, x.x, -y.x), fma(w, x.y, -y.y));
}
template <int FORM>
__device__ __forceinline__ double2 rot_row1(double w, double2 x, double2 y) {
  return FORM == 0 ? make_double2(fma(w, x.x, y.x), fma(w, x.y, y.y))
                   : make_double2(fma(w, y.x, x.x), fma(w, y.y, x.y));
}

// a normalised rotation on a lane bit: own amplitude x, partner's p, hi = this
// lane's value of the bit.  FORM 0: y = x + (hi ? w : -w) p; FORM 1:
// y = w x + (hi ? p : -p)
template <int FORM>
__device__ __forceinline__ double2 rot_lane(double w, bool hi, double2 x, double2 p) {
  if (FORM == 0) {
    const double c = hi ? w : -w;
    return make_double2(fma(c, p.x, x.x), fma(c, p.y, x.y));
  }
  return make_double2(fma(w, x.x, hi ? p.x : -p.x), fma(w, x.y, hi ? p.y : -p.y));
}

// a x + b y for real a, b (the rows of a real 2x2: OPF_REAL): 2 FP64 operations per component
__device__ __forceinline__ double2 rlin(double a, double2 x, double b, double2 y) {
  return make_double2(fma(b, y.x, a * x.x), fma(b, y.y, a * x.y));
}

// OP_X2R on one amplitude quadruple x0..x3 (local index bit 0 = slot a, bit 1
// = slot b) with the 4x4 m (row-major): corners (0,0), (0,3), (3,0), (3,3) mix
// x0 and x3, the middle (1,1), (2,2) scales x1 and x2.  CR / MR: the corner /
// middle entries are real (their imaginary parts are not read).
template <bool CR, bool MR>
__device__ __forceinline__ void xpat4(double2& x0, double2& x1, double2& x2, double2& x3, double2 m0, double2 m3,
                                      double2 m12, double2 m15, double2 m5, double2 m10) {
  double2 y0, y3;
  if (CR) {
    y0 = make_double2(fma(m3.x, x3.x, m0.x * x0.x), fma(m3.x, x3.y, m0.x * x0.y));
    y3 = make_double2(fma(m15.x, x3.x, m12.x * x0.x), fma(m15.x, x3.y, m12.x * x0.y));
  } else {
    y0 = cfma(cmul(m0, x0), m3, x3);
    y3 = cfma(cmul(m12, x0), m15, x3);
  }
  if (MR) {
    x1 = make_double2(m5.x * x1.x, m5.x * x1.y);
    x2 = make_double2(m10.x * x2.x, m10.x * x2.y);
  } else {
    x1 = cmul(m5, x1);
    x2 = cmul(m10, x2);
  }
  x0 = y0;
  x3 = y3;
}

__device__ __forceinline__ double2 shfl_xor2(double2 v, int dl, unsigned mask) {
  return make_double2(__shfl_xor_sync(mask, v.x, dl, 8), __shfl_xor_sync(mask, v.y, dl, 8));
}

// Adjoint step on slot 0 (psi / lambda select bit) and slot B (the qubit):
// returns this thread's share of Im<lambda| P |psi> for generator P (GEN 0 = X,
// 1 = Y, 2 = Z), then un-applies the rotation exp(-i t P / 2) on the qubit in
// both halves.  m is the inverse rotation or a multiple of it, used through
// its structure (FORM, a GradForm): GEN 0: [[c, i s], [i s, c]], [[1, i t],
// [i t, 1]] or [[u, i], [i, u]]; GEN 1: [[c, s], [-s, c]], [[1, t], [-t, 1]] or
// [[u, 1], [-1, u]]; GEN 2: diag(e^{i t/2}, e^{-i t/2}) or diag(1, u3).
// Inputs are read before outputs are written (in-place safe).
template <int GEN, int FORM = 0>
__device__ __forceinline__ void unrotate(double2 x0, double2 x1, double2& y0, double2& y1, double2 u0, double2 u1,
                                         double2 u3) {
  if (GEN == 0 && FORM == 1) {          // y0 = x0 + i t x1, y1 = x1 + i t x0
    const double t = u1.y;
    y0 = make_double2(fma(-t, x1.y, x0.x), fma(t, x1.x, x0.y));
    y1 = make_double2(fma(-t, x0.y, x1.x), fma(t, x0.x, x1.y));
  } else if (GEN == 0 && FORM == 2) {   // y0 = u x0 + i x1, y1 = u x1 + i x0
    const double u = u0.x;
    y0 = make_double2(fma(u, x0.x, -x1.y), fma(u, x0.y, x1.x));
    y1 = make_double2(fma(u, x1.x, -x0.y), fma(u, x1.y, x0.x));
  } else if (GEN == 0) {         // y0 = c x0 + i s x1, y1 = i s x0 + c x1
    const double c = u0.x, sn = u1.y;
    y0 = make_double2(fma(c, x0.x, -sn * x1.y), fma(c, x0.y, sn * x1.x));
    y1 = make_double2(fma(c, x1.x, -sn * x0.y), fma(c, x1.y, sn * x0.x));
  } else if (GEN == 1 && FORM == 1) {   // y0 = x0 + t x1, y1 = x1 - t x0
    const double t = u1.x;
    y0 = make_double2(fma(t, x1.x, x0.x), fma(t, x1.y, x0.y));
    y1 = make_double2(fma(-t, x0.x, x1.x), fma(-t, x0.y, x1.y));
  } else if (GEN == 1 && FORM == 2) {   // y0 = u x0 + x1, y1 = u x1 - x0
    const double u = u0.x;
    y0 = make_double2(fma(u, x0.x, x1.x), fma(u, x0.y, x1.y));
    y1 = make_double2(fma(u, x1.x, -x0.x), fma(u, x1.y, -x0.y));
  } else if (GEN == 1) {  // y0 = c x0 + s x1, y1 = c x1 - s x0
    const double c = u0.x, sn = u1.x;
    y0 = make_double2(fma(c, x0.x, sn * x1.x), fma(c, x0.y, sn * x1.y));
    y1 = make_double2(fma(c, x1.x, -sn * x0.x), fma(c, x1.y, -sn * x0.y));
  } else if (FORM == 1) { // diag(1, u3)
    y0 = x0;
    y1 = cmul(u3, x1);
  } else {                // diagonal phases
    y0 = cmul(u0, x0);
    y1 = cmul(u3, x1);
  }
}


// this amplitude pair's share of Im <lambda| P |psi> for the generator P of an
// adjoint step (GEN 0 = X, 1 = Y, 2 = Z); explicit FMA forms, so every kernel
// rounds it the same way
template <int GEN>
__device__ __forceinline__ double grad_term(double2 p0, double2 p1, double2 l0, double2 l1) {
  if (GEN == 0) {         // X: (P psi)_0 = psi_1, (P psi)_1 = psi_0
    return fma(l0.x, p1.y, -(l0.y * p1.x)) + fma(l1.x, p0.y, -(l1.y * p0.x));
  } else if (GEN == 1) {  // Y: (P psi)_0 = -i psi_1, (P psi)_1 = i psi_0
    return fma(l1.x, p0.x, l1.y * p0.y) - fma(l0.x, p1.x, l0.y * p1.y);
  } else {                // Z: (P psi)_0 = psi_0, (P psi)_1 = -psi_1
    return fma(l0.x, p0.y, -(l0.y * p0.x)) - fma(l1.x, p1.y, -(l1.y * p1.x));
  }
}

// the octet's eight lanes hold the same registers of eight tile rows: sum
// their shares, and the octet's lane 0 -- the only writer of its row of
// accumulators -- adds it there.  Tiles reach a CTA, and tile rows reach an
// octet, in a fixed order, so the sums are reproducible bit for bit.
__device__ __forceinline__ void grad_accumulate(double acc, double* slot, int lane8, unsigned omask) {
  acc += __shfl_xor_sync(omask, acc, 1, 8);
  acc += __shfl_xor_sync(omask, acc, 2, 8);
  acc += __shfl_xor_sync(omask, acc, 4, 8);
  if (lane8 == 0) *slot += acc;
}

constexpr int kMaxBuf = 4;

template <int N>
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// The tile pipeline of one pass (NT threads, all of them compute; the lanes
// of every warp also issue the TMA copies).  Tiles cycle through `nbuf`
// shared-memory buffers at `tiles` (1024-byte aligned for the 128-byte
// swizzle): while tile i is computed, tiles up to i + depth are loading and
// the stores of earlier tiles are draining.  depth = nbuf - 2 for nbuf >= 3,
// else nbuf - 1, so the buffer a load re-arms always held a tile every thread
// has finished with, and its mbarrier is armed once per phase.
//
// body(buf, t, work) runs the pass's stages on the resident tile buf (global
// tile index t) with a __syncthreads() after each stage; `work` is uniform in
// the CTA and false after an abort (the body must then only keep the CTA's
// barriers in step).  Every thread of the CTA calls tile_pipeline.
template <int NT, class Body>
__device__ __forceinline__ void tile_pipeline(const CUtensorMap& tm, const PassDesc& P, double2* tiles,
                                              int* __restrict__ status, int nbuf, Body&& body) {
  __shared__ __align__(8) uint64_t bar_loaded[kMaxBuf];
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const uint32_t tile_elems = 1u << P.M;
  const uint64_t ntiles = P.ntiles;
  const uint64_t first = blockIdx.x;
  if (tid == 0) {
    for (int b = 0; b < nbuf; ++b) mbar_init(&bar_loaded[b], NT / 32);   // one arrival per warp
    abort_flag = 0;
    fence_mbar_init();
  }
  __syncthreads();

  const uint64_t cnt = (first < ntiles) ? (ntiles - 1 - first) / gridDim.x + 1 : 0;
  const int depth = nbuf >= 3 ? nbuf - 2 : nbuf - 1;   // < nbuf

  // ---- copy issue setup: every warp issues its share of a tile's copies
  // (issues j = warp + NW * (lane + 32 r)); the tile mbarrier expects one
  // arrival per warp.  Coordinates are linear in the disjoint address bits, so
  // each lane keeps the offsets of its issues and adds the tile's base
  // coordinates per tile.
  constexpr int NW = NT / 32;
  const int warp = tid >> 5;
  const int nbox = P.nbox;
  const int nissue = 1 << (P.nH - nbox);
  const uint32_t box_elems = 1u << (P.c + nbox);
  const uint32_t box_bytes = box_elems * 16u;
  constexpr int kMaxPerLane = 1;   // nissue <= 32 * NW
  int jc1[kMaxPerLane], jc3[kMaxPerLane], jc4[kMaxPerLane], jj[kMaxPerLane];
  uint32_t my_bytes = 0;           // bytes of this warp's issues per tile
#pragma unroll
  for (int r = 0; r < kMaxPerLane; ++r) {
    const int j = warp + NW * (lane + 32 * r);
    jj[r] = j;
    int c2;
    if (j < nissue) chunk_coords(issue_offset(j, P), P, jc1[r], c2, jc3[r], jc4[r]);
    else jc1[r] = jc3[r] = jc4[r] = 0;
  }
  for (int j = warp; j < nissue; j += NW) my_bytes += box_bytes;
  TileCoordMap cmap;               // tile index -> tensor-map coordinates (32-bit, per thread)
  tile_coord_map(P, cmap);
  auto base_coords = [&](uint64_t t, int& c1, int& c3, int& c4) {
    int c2;
    tile_coords((uint32_t)t, cmap, c1, c2, c3, c4);
  };
  auto issue_load = [&](uint64_t i) {   // whole warp, converged
    const int b = (int)(i % nbuf);
    int c1, c3, c4;
    base_coords(first + i * gridDim.x, c1, c3, c4);
    double2* buf = tiles + (size_t)b * tile_elems;
    if (lane == 0) mbar_arrive_expect_tx(&bar_loaded[b], my_bytes);
    __syncwarp();
#pragma unroll
    for (int r = 0; r < kMaxPerLane; ++r)
      if (jj[r] < nissue)
        tma_load_5d(buf + (size_t)jj[r] * box_elems, &tm, 0, c1 + jc1[r], 0, c3 + jc3[r], c4 + jc4[r],
                    &bar_loaded[b]);
  };
  auto issue_store = [&](uint64_t i) {  // whole warp; one bulk group per lane per tile
    const int b = (int)(i % nbuf);
    int c1, c3, c4;
    base_coords(first + i * gridDim.x, c1, c3, c4);
    double2* buf = tiles + (size_t)b * tile_elems;
#pragma unroll
    for (int r = 0; r < kMaxPerLane; ++r)
      if (jj[r] < nissue)
        tma_store_5d(&tm, 0, c1 + jc1[r], 0, c3 + jc3[r], c4 + jc4[r], buf + (size_t)jj[r] * box_elems);
    bulk_commit();
  };

  uint64_t issued = 0;             // tiles whose loads have been issued
  uint64_t first_unwaited = cnt;   // first tile whose load wait did not succeed
  for (; issued < (uint64_t)depth && issued < cnt; ++issued) issue_load(issued);

  for (uint64_t i = 0; i < cnt; ++i) {
    const int b = (int)(i % nbuf);
    // abort_flag is read after the previous iteration's barrier: uniform in the CTA
    const bool ab = __shfl_sync(0xffffffffu, (int)abort_flag, 0) != 0;
    if (i + depth < cnt && !ab) {
      // buffer (i + depth) % nbuf last held tile i + depth - nbuf (finished by
      // every thread: it is at most tile i - 1), whose store is followed by
      // nbuf - depth - 1 later stores: wait only for that store's read
      if (i + depth >= (uint64_t)nbuf) {
        if (nbuf - depth - 1 >= 1) bulk_wait_read<1>();
        else bulk_wait_read<0>();
      }
      __syncwarp();
      issue_load(i + depth);
      issued = i + depth + 1;
    }
    const bool ok = bounded_wait(&bar_loaded[b], (uint32_t)((i / nbuf) & 1), &abort_flag, status, DEV_WAIT_LOADED);
    const bool work = __syncthreads_and(ok && !abort_flag);
    if (!work && first_unwaited == cnt) first_unwaited = i;
    double2* buf = tiles + (size_t)b * tile_elems;
    body(buf, first + i * gridDim.x, work);
    fence_proxy_async_smem();
    __syncthreads();
    if (work) issue_store(i);
  }
  // after an abort, let loads that were issued but never consumed land first
  for (uint64_t i = first_unwaited; i < issued; ++i) drain_wait(&bar_loaded[i % nbuf], (uint32_t)((i / nbuf) & 1));
  bulk_wait_all();
}

// A pass over nsets arrays laid end to end (one per parameter set), each with
// its own matrix block and gradient terms (PassDesc::nsets, set_shift,
// set_mat_stride, grad_stride).  Dynamic shared memory: [tile buffers]
// [the current set's matrix block][gradient accumulators: one row of ngrad per
// octet of threads].  At a set boundary the CTA flushes the finished set's
// gradient sums (octet rows summed in order, one column per CTA of
// grad_partials) and loads the next set's matrices.  stages(buf, smat, gslots,
// work) runs the pass's stages on a resident tile, each followed by a
// __syncthreads() (or none at all when work is false: it is uniform in the CTA).
template <int NT, class Stages>
struct SetTileBody {
  const PassDesc& P;
  const double2* mats;
  double* grad_partials;
  double2* smat;
  double* gslots;
  uint32_t sshift;
  uint32_t cur_set;
  Stages& stages;

  __device__ __forceinline__ void flush_grads() {
    for (uint32_t i = threadIdx.x; i < P.ngrad; i += NT) {
      double v = 0.0;
      for (int o = 0; o < NT / 8; ++o) v += gslots[o * P.ngrad + i];
      grad_partials[((size_t)cur_set * P.grad_stride + P.grad_term[i]) * gridDim.x + blockIdx.x] = v;
    }
  }
  __device__ __forceinline__ void operator()(double2* buf, unsigned long long t, bool work) {
    const int tid = threadIdx.x;
    const uint32_t tset = (uint32_t)(t >> sshift);   // uniform in the CTA
    if (tset != cur_set) {   // every thread is past the previous tile's stages
      if (P.ngrad) {
        flush_grads();
        __syncthreads();
        for (uint32_t j = tid; j < P.ngrad * (NT / 8); j += NT) gslots[j] = 0.0;
      }
      cur_set = tset;
      for (uint32_t j = tid; j < P.mat_elems; j += NT)
        smat[j] = mats[P.mat_base + (size_t)cur_set * P.set_mat_stride + j];
      __syncthreads();
    }
    stages(buf, smat, gslots, work);
  }
};

template <int NT, class Stages>
__device__ __forceinline__ void set_tile_pass(const CUtensorMap& tm, const PassDesc& P, const double2* mats,
                                              int* status, int nbuf, double* grad_partials, unsigned char* smem_raw,
                                              Stages& stages);

// 1024-byte aligned start of the dynamic shared memory (the tile buffers)
__device__ __forceinline__ double2* aligned_tiles(unsigned char* smem_raw) {
  return reinterpret_cast<double2*>((reinterpret_cast<unsigned long long>(smem_raw) + 1023ull) & ~1023ull);
}

template <int NT, class Stages>
__device__ __forceinline__ void set_tile_pass(const CUtensorMap& tm, const PassDesc& P, const double2* mats,
                                              int* status, int nbuf, double* grad_partials, unsigned char* smem_raw,
                                              Stages& stages) {
  double2* tiles = aligned_tiles(smem_raw);
  const int tid = threadIdx.x;
  double2* smat = tiles + (size_t)nbuf * (1u << P.M);
  const unsigned long long first = blockIdx.x;
  // set of the tiles being processed (the CTA's tiles ascend, so each set is
  // met in one run); its matrices sit in smat, its gradient sums in gslots
  const uint32_t sshift = (P.nsets > 1) ? P.set_shift : 63u;
  const uint32_t set0 = (first < P.ntiles) ? (uint32_t)(first >> sshift) : 0u;
  for (uint32_t i = tid; i < P.mat_elems; i += NT) smat[i] = mats[P.mat_base + (size_t)set0 * P.set_mat_stride + i];
  double* gslots = reinterpret_cast<double*>(smat + P.mat_elems);
  for (uint32_t i = tid; i < P.ngrad * (NT / 8); i += NT) gslots[i] = 0.0;
  SetTileBody<NT, Stages> body{P, mats, grad_partials, smat, gslots, sshift, set0, stages};
  tile_pipeline<NT>(tm, P, tiles, status, nbuf, body);
  if (P.ngrad) {   // the last set's gradient partials
    __syncthreads();
    body.flush_grads();
  }
}

// ---- passes over complex64 (float2) arrays: the first stage loads its
// registers straight from global memory (widened to FP64), the last stage
// stores them there (rounded to FP32), and the stages between exchange
// through a shared-memory tile of float2 (each stage boundary rounds to FP32
// as the array does; all arithmetic is FP64).  Every CTA walks its tiles
// (blockIdx.x, + gridDim.x, ...); no asynchronous copies.

// Physical index bits of tile-local index L: bits below c are themselves, bit
// c + i is H[i].
__device__ __forceinline__ unsigned long long local_to_phys(uint32_t L, const PassDesc& P) {
  unsigned long long x = L & ((1u << P.c) - 1u);
  for (int i = 0; i < P.nH; ++i)
    if ((L >> (P.c + i)) & 1u) x |= 1ULL << P.H[i];
  return x;
}
__device__ __forceinline__ double2 ldn(const float2* p) {
  const float2 v = *p;
  return make_double2((double)v.x, (double)v.y);
}
__device__ __forceinline__ void stn(float2* p, double2 v) {
  *p = make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
}

// Dynamic shared memory: [one float2 tile of 2^M elements][the current set's
// matrix block][gradient accumulators: one row of ngrad per octet].
// stages(tile, smat, gslots, t) runs the pass's stages on tile t (each stage
// ends with a __syncthreads()).  Set switches as in SetTileBody.
template <int NT, class Stages>
__device__ __forceinline__ void direct_set_pass(const PassDesc& P, const double2* mats, double* grad_partials,
                                                unsigned char* smem_raw, Stages& stages) {
  double2* const tiles = aligned_tiles(smem_raw);
  float2* tile = reinterpret_cast<float2*>(tiles);
  double2* smat = tiles + (1u << (P.M - 1));   // after the tile's 8 << M bytes
  double* gslots = reinterpret_cast<double*>(smat + P.mat_elems);
  const int tid = threadIdx.x;
  const uint32_t sshift = (P.nsets > 1) ? P.set_shift : 63u;
  uint32_t cur_set = (blockIdx.x < P.ntiles) ? (uint32_t)(blockIdx.x >> sshift) : 0u;
  for (uint32_t i = tid; i < P.mat_elems; i += NT) smat[i] = mats[P.mat_base + (size_t)cur_set * P.set_mat_stride + i];
  for (uint32_t i = tid; i < P.ngrad * (NT / 8); i += NT) gslots[i] = 0.0;
  __syncthreads();
  auto flush = [&]() {
    for (uint32_t i = tid; i < P.ngrad; i += NT) {
      double v = 0.0;
      for (int o = 0; o < NT / 8; ++o) v += gslots[o * P.ngrad + i];
      grad_partials[((size_t)cur_set * P.grad_stride + P.grad_term[i]) * gridDim.x + blockIdx.x] = v;
    }
  };
  for (unsigned long long t = blockIdx.x; t < P.ntiles; t += gridDim.x) {
    const uint32_t tset = (uint32_t)(t >> sshift);
    if (tset != cur_set) {
      if (P.ngrad) {
        flush();
        __syncthreads();
        for (uint32_t j = tid; j < P.ngrad * (NT / 8); j += NT) gslots[j] = 0.0;
      }
      cur_set = tset;
      for (uint32_t j = tid; j < P.mat_elems; j += NT)
        smat[j] = mats[P.mat_base + (size_t)cur_set * P.set_mat_stride + j];
      __syncthreads();
    }
    stages(tile, smat, gslots, t);
  }
  if (P.ngrad) {
    __syncthreads();
    flush();
  }
}

}  // namespace iqb
