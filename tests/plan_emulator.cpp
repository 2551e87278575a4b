// plan_emulator.cpp -- TEST ONLY.  Executes the passes planned by
// invariantq_b200/csrc/iq_sched.cpp on the CPU with the semantics of
// tile_pass_kernel (iq_kernels.cu): tensor-map box copies computed from the
// shared addressing helpers in iq_plan.h, register stages with octet lanes,
// and every operation kind.  It lets the CPU test suite check the scheduler,
// the descriptor encoding and the tile addressing against the oracle.  It also
// checks that the box copies of a pass cover every amplitude exactly once.
#include <algorithm>
#include <complex>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../invariantq_b200/csrc/iq_plan.h"

using namespace iqb;
using cd = std::complex<double>;

namespace {

struct Emu {
  int nbits;
  std::vector<cd> pool;
  cd* state;
  std::string err;

  uint32_t blk = 0;   // current pass's matrix block
  std::vector<double> grads;   // gradient terms accumulated by OP_GRAD2
  cd mat(uint32_t off, int i) const { return pool[blk + off + i]; }

  bool copy_tile(const PassDesc& P, uint64_t t, std::vector<cd>& tile, bool load, std::vector<uint8_t>& seen) {
    uint64_t gd[5], gs[4];
    uint32_t box[5];
    pass_tmap_layout(P, nbits, gd, gs, box);
    const uint64_t base = tile_base(t, P);
    {   // the kernel's 32-bit tile-coordinate map gives the same first copy
      TileCoordMap m;
      tile_coord_map(P, m);
      int a[4], b[4];
      tile_coords((uint32_t)t, m, a[0], a[1], a[2], a[3]);
      chunk_coords(base, P, b[0], b[1], b[2], b[3]);
      for (int d = 0; d < 4; ++d)
        if (a[d] != b[d]) { err = "tile coordinate map disagrees with the 64-bit tile address"; return false; }
    }
    const int nissue = 1 << (P.nH - P.nbox);
    const uint32_t box_elems = 1u << (P.c + P.nbox);
    double* sd = reinterpret_cast<double*>(state);
    double* td = reinterpret_cast<double*>(tile.data());
    for (int j = 0; j < nissue; ++j) {
      int c[5];
      c[0] = 0;
      chunk_coords(base | issue_offset(j, P), P, c[1], c[2], c[3], c[4]);
      for (int d = 1; d < 5; ++d)
        if (c[d] < 0 || (uint64_t)c[d] + box[d] > gd[d]) { err = "box out of tensor bounds"; return false; }
      uint64_t lin = 0;
      for (uint32_t i4 = 0; i4 < box[4]; ++i4)
        for (uint32_t i3 = 0; i3 < box[3]; ++i3)
          for (uint32_t i2 = 0; i2 < box[2]; ++i2)
            for (uint32_t i1 = 0; i1 < box[1]; ++i1)
              for (uint32_t i0 = 0; i0 < box[0]; ++i0, ++lin) {
                const uint64_t g = (uint64_t)(c[0] + i0) * 8 + (uint64_t)(c[1] + i1) * gs[0] +
                                   (uint64_t)(c[2] + i2) * gs[1] + (uint64_t)(c[3] + i3) * gs[2] +
                                   (uint64_t)(c[4] + i4) * gs[3];
                if (g % 8) { err = "misaligned element"; return false; }
                const uint64_t gi = g / 8;
                if (gi >= (2ull << nbits)) { err = "global address out of range"; return false; }
                // TMA 128-byte swizzle: 16-byte unit u of the tile lands in slot swz(u)
                const uint64_t lin_d = (uint64_t)j * box_elems * 2 + lin;
                const uint64_t si = 2 * (uint64_t)swz((uint32_t)(lin_d / 2)) + (lin_d & 1);
                if (si >= tile.size() * 2) { err = "shared address out of range"; return false; }
                if (load) {
                  td[si] = sd[gi];
                  if (gi % 2 == 0) {
                    if (seen[gi / 2]) { err = "amplitude loaded twice in one pass"; return false; }
                    seen[gi / 2] = 1;
                  }
                } else {
                  sd[gi] = td[si];
                }
              }
    }
    return true;
  }

  // one stage: 2^nt octet-subcubes, 8 lanes each, 2^R registers per lane
  bool run_stage(const PassDesc& P, int s, std::vector<cd>& tile) {
    const StageDesc& sd = P.st[s];
    const int R = P.R, NV = 1 << R;
    auto voff = [&](int v) {
      uint32_t o = 0;
      for (int i = 0; i < R; ++i)
        if ((v >> i) & 1) o |= 1u << sd.S[i];
      return o;
    };
    for (uint32_t u = 0; u < (1u << sd.nt); ++u) {
      uint32_t ub = 0;
      for (int i = 0; i < sd.nt; ++i) ub |= ((u >> i) & 1u) << sd.tb[i];
      std::vector<std::vector<cd>> a(8, std::vector<cd>(NV));
      uint32_t base[8];
      for (int L = 0; L < 8; ++L) {
        base[L] = ub | ((L & 1u) << sd.lane[0]) | (((L >> 1) & 1u) << sd.lane[1]) | (((L >> 2) & 1u) << sd.lane[2]);
        for (int v = 0; v < NV; ++v) a[L][v] = tile[swz(base[L] | voff(v))];
      }
      bool stored = false;
      for (int o = sd.op0; o < sd.op1; ++o) {
        const OpDesc& od = P.ops[o];
        const bool unit = od.flags & OPF_UNIT_PHASE;
        switch (od.kind) {
          case OP_D1R:
          case OP_N1R:   // stored whole (its unit entry included)
          case OP_R1R: {
            // OPF_REAL (dense kinds): only the real parts are read
            const bool re = (od.flags & OPF_REAL) && od.kind == OP_D1R;
            auto m1 = [&](int i) { const cd e = mat(od.mat, i); return re ? cd(e.real(), 0.0) : e; };
            for (int L = 0; L < 8; ++L)
              for (int v = 0; v < NV; ++v) {
                if (v & (1 << od.a)) continue;
                const cd x = a[L][v], y = a[L][v | (1 << od.a)];
                a[L][v] = m1(0) * x + m1(1) * y;
                a[L][v | (1 << od.a)] = m1(2) * x + m1(3) * y;
              }
            break;
          }
          case OP_D1L:
          case OP_R1L: {   // the rotation's matrix is stored whole
            const bool re = (od.flags & OPF_REAL) && od.kind == OP_D1L;
            auto m1 = [&](int i) { const cd e = mat(od.mat, i); return re ? cd(e.real(), 0.0) : e; };
            auto old = a;
            for (int L = 0; L < 8; ++L) {
              const int my = (L >> od.a) & 1, pl = L ^ (1 << od.a);
              for (int v = 0; v < NV; ++v)
                a[L][v] = (my ? m1(3) : m1(0)) * old[L][v] + (my ? m1(2) : m1(1)) * old[pl][v];
            }
            break;
          }
          case OP_M1R:
            for (int L = 0; L < 8; ++L)
              for (int v = 0; v < NV; ++v) {
                if (v & (1 << od.a)) continue;
                cd x = a[L][v], y = a[L][v | (1 << od.a)];
                if (od.perm & 1) std::swap(x, y);
                if (!unit) { x *= mat(od.mat, 0); y *= mat(od.mat, 1); }
                a[L][v] = x;
                a[L][v | (1 << od.a)] = y;
              }
            break;
          case OP_M1L: {
            auto old = a;
            for (int L = 0; L < 8; ++L) {
              const int my = (L >> od.a) & 1, pl = L ^ (1 << od.a);
              for (int v = 0; v < NV; ++v) {
                cd x = (od.perm & 1) ? old[pl][v] : old[L][v];
                a[L][v] = unit ? x : mat(od.mat, my) * x;
              }
            }
            break;
          }
          case OP_X2R: {   // only the corners and the middle are read (their real parts when flagged)
            auto ent = [&](int i, bool real) { const cd e = mat(od.mat, i); return real ? cd(e.real(), 0.0) : e; };
            const bool cr = od.flags & 1, mr = od.flags & 2;
            const cd m0 = ent(0, cr), m3 = ent(3, cr), m12 = ent(12, cr), m15 = ent(15, cr), m5 = ent(5, mr),
                     m10 = ent(10, mr);
            for (int L = 0; L < 8; ++L)
              for (int v = 0; v < NV; ++v) {
                if (v & ((1 << od.a) | (1 << od.b))) continue;
                const int i0 = v, i1 = v | (1 << od.a), i2 = v | (1 << od.b), i3 = i1 | i2;
                const cd x0 = a[L][i0], x3 = a[L][i3];
                a[L][i0] = m0 * x0 + m3 * x3;
                a[L][i3] = m12 * x0 + m15 * x3;
                a[L][i1] *= m5;
                a[L][i2] *= m10;
              }
            break;
          }
          case OP_D2R:
          case OP_M2R:
            for (int L = 0; L < 8; ++L)
              for (int v = 0; v < NV; ++v) {
                if (v & ((1 << od.a) | (1 << od.b))) continue;
                int idx[4];
                cd x[4];
                for (int m = 0; m < 4; ++m) {
                  idx[m] = v | ((m & 1) << od.a) | (((m >> 1) & 1) << od.b);
                  x[m] = a[L][idx[m]];
                }
                for (int r = 0; r < 4; ++r) {
                  cd acc;
                  if (od.kind == OP_D2R) {
                    acc = 0.0;
                    for (int m = 0; m < 4; ++m) acc += mat(od.mat, 4 * r + m) * x[m];
                  } else {
                    acc = x[(od.perm >> (2 * r)) & 3];
                    if (!unit) acc *= mat(od.mat, r);
                  }
                  a[L][idx[r]] = acc;
                }
              }
            break;
          case OP_GRAD2: {
            if (od.a != 0) { err = "adjoint step with the select bit outside slot 0"; return false; }
            const uint32_t term = P.grad_term[od.gidx];
            if (term >= grads.size()) grads.resize(term + 1, 0.0);
            const int B = od.b;
            for (int L = 0; L < 8; ++L)
              for (int v = 0; v < NV; ++v) {
                if (v & (1 | (1 << B))) continue;
                const cd p0 = a[L][v], p1 = a[L][v | (1 << B)], l0 = a[L][v | 1], l1 = a[L][v | 1 | (1 << B)];
                cd t;
                if (od.perm == 0) t = std::conj(l0) * p1 + std::conj(l1) * p0;
                else if (od.perm == 1) t = std::conj(l0) * (cd(0, -1) * p1) + std::conj(l1) * (cd(0, 1) * p0);
                else t = std::conj(l0) * p0 - std::conj(l1) * p1;
                grads[term] += t.imag();
                a[L][v] = mat(od.mat, 0) * p0 + mat(od.mat, 1) * p1;
                a[L][v | (1 << B)] = mat(od.mat, 2) * p0 + mat(od.mat, 3) * p1;
                a[L][v | 1] = mat(od.mat, 0) * l0 + mat(od.mat, 1) * l1;
                a[L][v | 1 | (1 << B)] = mat(od.mat, 2) * l0 + mat(od.mat, 3) * l1;
              }
            break;
          }
          case OP_DKR: {
            const int k = od.k, D = 1 << k;
            if (o != sd.op1 - 1) { err = "dense block is not the last operation of its stage"; return false; }
            for (int L = 0; L < 8; ++L)
              for (int g = 0; g < NV; g += D)
                for (int r = 0; r < D; ++r) {
                  cd acc = 0.0;
                  for (int cc = 0; cc < D; ++cc) acc += mat(od.mat, r * D + cc) * a[L][g + cc];
                  tile[swz(base[L] | voff(g + r))] = acc;
                }
            stored = true;
            break;
          }
          default:
            err = "unknown operation kind";
            return false;
        }
      }
      if (!stored)
        for (int L = 0; L < 8; ++L)
          for (int v = 0; v < NV; ++v) tile[swz(base[L] | voff(v))] = a[L][v];
    }
    return true;
  }
};

// plan `ops` (optionally fused) and run every pass on `state`
// gap != 0: the operations act on the lower half (address bit `gap` = 0) of a
// state of gap + 1 bits, through passes planned for `gap` bits (PassDesc::gap)
int run_plan(Emu& e, std::vector<SchedOp> ops, int M, int c, int R, int max_stages, double budget, int fuse,
             int* npasses, int* ops_per_pass, char* errbuf, int errlen, int gap = 0,
             std::vector<PassPlan>* plans_out = nullptr) {
  if (fuse) {
    std::vector<cplx64> cp(reinterpret_cast<const cplx64*>(e.pool.data()),
                           reinterpret_cast<const cplx64*>(e.pool.data()) + e.pool.size());
    ops = fuse_two_qubit_blocks(ops, cp);
    e.pool.assign(reinterpret_cast<const cd*>(cp.data()), reinterpret_cast<const cd*>(cp.data()) + cp.size());
  }
  SchedParams p{};
  p.nbits = gap ? gap : e.nbits;
  p.M = M;
  p.c = c;
  p.R = R;
  p.max_stages = max_stages;
  p.budget = budget;
  std::vector<PassPlan> plans;
  std::string err;
  if (plan_passes(p, ops, plans, err) < 0) {
    snprintf(errbuf, errlen, "plan: %s", err.c_str());
    return -1;
  }
  for (PassPlan& pl : plans) pl.desc.gap = (uint8_t)gap;
  if (npasses) *npasses = (int)plans.size();
  std::vector<cplx64> packed;
  pack_pass_matrices(plans, reinterpret_cast<const cplx64*>(e.pool.data()), packed);
  e.pool.assign(reinterpret_cast<const cd*>(packed.data()), reinterpret_cast<const cd*>(packed.data()) + packed.size());
  for (size_t pi = 0; pi < plans.size(); ++pi) {
    const PassDesc& P = plans[pi].desc;
    e.blk = P.mat_base;
    if (ops_per_pass) ops_per_pass[pi] = plans[pi].nsrc;
    if (P.mat_elems > (uint32_t)kSmemMatElems) {
      snprintf(errbuf, errlen, "pass %zu: matrix block exceeds shared memory", pi);
      return -1;
    }
    std::vector<cd> tile((size_t)1 << P.M);
    std::vector<uint8_t> seen((size_t)1 << e.nbits, 0);
    for (uint64_t t = 0; t < P.ntiles; ++t) {
      if (!e.copy_tile(P, t, tile, true, seen)) break;
      for (int st = 0; st < P.nstages && e.err.empty(); ++st) e.run_stage(P, st, tile);
      if (!e.err.empty()) break;
      if (!e.copy_tile(P, t, tile, false, seen)) break;
    }
    if (e.err.empty())
      for (size_t i = 0; i < seen.size(); ++i) {
        const bool in_pass = !gap || !((i >> gap) & 1);
        if (seen[i] != (in_pass ? 1 : 0)) {
          e.err = in_pass ? "amplitude not covered by a pass" : "amplitude outside the pass's half touched";
          break;
        }
      }
    if (!e.err.empty()) {
      snprintf(errbuf, errlen, "pass %zu: %s", pi, e.err.c_str());
      return -1;
    }
  }
  if (plans_out) *plans_out = std::move(plans);
  return 0;
}

}  // namespace

// Adjoint gradient of <psi|H|psi> for an ansatz, run through the planned
// passes exactly as the GPU path does (forward on psi, lambda = H psi, joint
// array, backward sweep with adjoint steps).  H = sum_t coeffs[t] paulis[t]
// (n characters per term, character q acting on qubit q).
// single_set: the operation lists of a circuit with one parameter set (the
// forward decomposed into rotations and phases, scaled adjoint steps whose
// scales are undone in the order the planned passes run them).
extern "C" int emu_adjoint_forms(int n, int nops, const int* kinds, const int* q0, const int* q1, const int* pidx,
                                 const double* params, int nterms, const double* coeffs, const char* paulis, int M,
                                 int c, int R, int max_stages, double budget, double* energy, double* grad,
                                 int nparams, int single_set, char* errbuf, int errlen) {
  std::vector<AnsatzOp> ops(nops);
  for (int i = 0; i < nops; ++i) ops[i] = {kinds[i], q0[i], q1[i], pidx[i]};
  std::string err;
  if (ansatz_check(n, ops, err) < 0) {
    snprintf(errbuf, errlen, "%s", err.c_str());
    return -1;
  }
  // the joint array [psi | lambda] (select bit n; zero-padded high bits for
  // small circuits); the forward runs on its psi half
  const int nj = std::max(n + 1, 7);
  std::vector<cd> joint((size_t)1 << nj, 0.0);
  std::vector<cd> psi((size_t)1 << n, 0.0);
  psi[0] = 1.0;
  Emu f;
  AdjointOps jo;   // the executor's operation lists (fused, or the single-set forms)
  adjoint_ops(n, ops, params, true, true, single_set != 0, jo);
  const std::vector<SchedOp>& fw = jo.fw;
  f.pool.assign(reinterpret_cast<const cd*>(jo.fpool.data()),
                reinterpret_cast<const cd*>(jo.fpool.data()) + jo.fpool.size());
  if (n >= 7) {   // passes planned for n bits with the select bit as their gap
    joint[0] = 1.0;
    f.nbits = n + 1;
    f.state = joint.data();
    if (run_plan(f, fw, M, c, R, max_stages, budget, 0, nullptr, nullptr, errbuf, errlen, n) < 0) return -1;
    for (uint64_t x = 0; x < (1ULL << n); ++x) psi[x] = joint[x];
  } else {   // the runtime's one-operation kernel: dense matrix, LSB-first qubit list
    for (const SchedOp& o : fw) {
      const int d = 1 << o.k;
      for (uint64_t base = 0; base < (1ULL << n); ++base) {
        bool lead = true;
        for (int j = 0; j < o.k; ++j) lead &= !((base >> o.q[j]) & 1);
        if (!lead) continue;
        std::vector<uint64_t> idx(d);
        std::vector<cd> x(d);
        for (int v = 0; v < d; ++v) {
          idx[v] = base;
          for (int j = 0; j < o.k; ++j)
            if ((v >> j) & 1) idx[v] |= 1ULL << o.q[j];
          x[v] = psi[idx[v]];
        }
        for (int r = 0; r < d; ++r) {
          cd acc = 0.0;
          for (int cc = 0; cc < d; ++cc) acc += f.pool[o.dense + r * d + cc] * x[cc];
          psi[idx[r]] = acc;
        }
      }
    }
  }
  // lambda = H psi and the energy
  const uint64_t dim = 1ULL << n;
  std::vector<cd> lam(dim, 0.0);
  for (int t = 0; t < nterms; ++t) {
    uint64_t xm = 0, zm = 0;
    int ny = 0;
    for (int q = 0; q < n; ++q) {
      const char ch = paulis[t * n + q];
      if (ch == 'X') xm |= 1ULL << q;
      else if (ch == 'Y') { xm |= 1ULL << q; zm |= 1ULL << q; ++ny; }
      else if (ch == 'Z') zm |= 1ULL << q;
    }
    const cd ip[4] = {cd(1, 0), cd(0, 1), cd(-1, 0), cd(0, -1)};
    for (uint64_t j = 0; j < dim; ++j) {
      const uint64_t i = j ^ xm;
      const double sg = (__builtin_popcountll(i & zm) & 1) ? -1.0 : 1.0;
      lam[j] += coeffs[t] * ip[ny & 3] * sg * psi[i];
    }
  }
  cd e = 0.0;
  for (uint64_t x = 0; x < dim; ++x) e += std::conj(psi[x]) * lam[x];
  *energy = e.real();
  // backward on the joint array: psi at [0, 2^n), lambda at [2^n, 2^(n+1))
  Emu b;
  b.nbits = nj;   // small circuits: zero-padded high bits the gates never touch
  for (uint64_t x = 0; x < dim; ++x) { joint[x] = psi[x]; joint[dim + x] = lam[x]; }
  b.state = joint.data();
  const std::vector<int>& gp = jo.grad_param;
  b.pool.assign(reinterpret_cast<const cd*>(jo.bpool.data()),
                reinterpret_cast<const cd*>(jo.bpool.data()) + jo.bpool.size());
  b.grads.assign(gp.size(), 0.0);
  std::vector<PassPlan> plans;
  if (run_plan(b, jo.bw, M, c, R, max_stages, budget, 0, nullptr, nullptr, errbuf, errlen, 0, &plans) < 0) return -1;
  std::vector<double> scale;
  exec_grad_scales(&plans, jo.bw, scale);
  if (scale.size() != gp.size()) {
    snprintf(errbuf, errlen, "gradient scales: %zu for %zu terms", scale.size(), gp.size());
    return -1;
  }
  for (int p = 0; p < nparams; ++p) grad[p] = 0.0;
  for (size_t t = 0; t < gp.size(); ++t) grad[gp[t]] += b.grads[t] * scale[t];
  return 0;
}

extern "C" int emu_adjoint(int n, int nops, const int* kinds, const int* q0, const int* q1, const int* pidx,
                           const double* params, int nterms, const double* coeffs, const char* paulis, int M, int c,
                           int R, int max_stages, double budget, double* energy, double* grad, int nparams,
                           char* errbuf, int errlen) {
  return emu_adjoint_forms(n, nops, kinds, q0, q1, pidx, params, nterms, coeffs, paulis, M, c, R, max_stages, budget,
                           energy, grad, nparams, 0, errbuf, errlen);
}

extern "C" int emu_apply(int nbits, int M, int c, int R, int max_stages, double budget, int fuse, int nops,
                         const int* ks, const int* qs, const double* mats, const long long* mat_off,
                         double* state_il, int* npasses, int* ops_per_pass, char* errbuf, int errlen) {
  Emu e;
  e.nbits = nbits;
  e.state = reinterpret_cast<cd*>(state_il);
  std::vector<SchedOp> ops;
  for (int i = 0; i < nops; ++i) {
    SchedOp o{};
    o.k = (uint8_t)ks[i];
    for (int j = 0; j < ks[i]; ++j) o.q[j] = (uint8_t)qs[i * 5 + j];
    const int d = 1 << ks[i];
    const double* m = mats + 2 * mat_off[i];
    o.mat = (uint32_t)e.pool.size();
    o.dense = o.mat;
    for (int j = 0; j < d * d; ++j) e.pool.emplace_back(m[2 * j], m[2 * j + 1]);
    double ph[8];
    uint8_t perm = 0, unit = 0;
    if (ks[i] <= 2 && classify_monomial(m, ks[i], &perm, ph, &unit)) {
      o.mono = 1;
      o.perm = perm;
      o.unit = unit;
      o.mat = (uint32_t)e.pool.size();
      for (int j = 0; j < d; ++j) e.pool.emplace_back(ph[2 * j], ph[2 * j + 1]);
    } else if (ks[i] == 2) {
      o.xpat = (uint8_t)classify_xpattern(m);   // as the runtime's queue classifies it
    }
    ops.push_back(o);
  }
  if (fuse) {   // 1: blocks for the interpreting kernel; 2: the specialised kernels' planning
    std::vector<cplx64> cp(reinterpret_cast<const cplx64*>(e.pool.data()),
                           reinterpret_cast<const cplx64*>(e.pool.data()) + e.pool.size());
    ops = fuse_two_qubit_blocks(ops, cp, fuse == 2);
    if (fuse == 2) {
      decompose_one_qubit_ops(ops, cp);
      normalize_one_qubit_ops(ops, cp);
    }
    e.pool.assign(reinterpret_cast<const cd*>(cp.data()), reinterpret_cast<const cd*>(cp.data()) + cp.size());
  }
  SchedParams p{};
  p.nbits = nbits;
  p.M = M;
  p.c = c;
  p.R = R;
  p.max_stages = max_stages;
  p.budget = budget;
  std::vector<PassPlan> plans;
  std::string err;
  if (plan_passes(p, ops, plans, err) < 0) {
    snprintf(errbuf, errlen, "plan: %s", err.c_str());
    return -1;
  }
  *npasses = (int)plans.size();
  std::vector<cplx64> packed;
  pack_pass_matrices(plans, reinterpret_cast<const cplx64*>(e.pool.data()), packed);
  e.pool.assign(reinterpret_cast<const cd*>(packed.data()), reinterpret_cast<const cd*>(packed.data()) + packed.size());
  for (size_t pi = 0; pi < plans.size(); ++pi) {
    const PassDesc& P = plans[pi].desc;
    e.blk = P.mat_base;
    if (P.mat_elems > (uint32_t)kSmemMatElems) {
      snprintf(errbuf, errlen, "pass %zu: matrix block exceeds shared memory", pi);
      return -1;
    }
    if (ops_per_pass) ops_per_pass[pi] = plans[pi].nsrc;
    std::vector<cd> tile((size_t)1 << P.M);
    std::vector<uint8_t> seen((size_t)1 << nbits, 0);
    for (uint64_t t = 0; t < P.ntiles; ++t) {
      if (!e.copy_tile(P, t, tile, true, seen)) break;
      for (int s = 0; s < P.nstages && e.err.empty(); ++s) e.run_stage(P, s, tile);
      if (!e.err.empty()) break;
      if (!e.copy_tile(P, t, tile, false, seen)) break;
    }
    if (e.err.empty())
      for (size_t i = 0; i < seen.size(); ++i)
        if (!seen[i]) { e.err = "amplitude not covered by a pass"; break; }
    if (!e.err.empty()) {
      snprintf(errbuf, errlen, "pass %zu: %s", pi, e.err.c_str());
      return -1;
    }
  }
  return 0;
}

// Plan `ops` as emu_apply does and write the source of every pass's
// specialised kernel (iq_jitgen.cpp) into `out`, separated by lines
// "//@@PASS@@".  Returns the number of sources, or -1 (message in `out`).
extern "C" int emu_jit_sources(int nbits, int M, int c, int R, int max_stages, double budget, int fuse, int nops,
                               const int* ks, const int* qs, const double* mats, const long long* mat_off,
                               char* out, long long outlen) {
  std::vector<cd> pool;
  std::vector<SchedOp> ops;
  for (int i = 0; i < nops; ++i) {
    SchedOp o{};
    o.k = (uint8_t)ks[i];
    for (int j = 0; j < ks[i]; ++j) o.q[j] = (uint8_t)qs[i * 5 + j];
    const int d = 1 << ks[i];
    const double* m = mats + 2 * mat_off[i];
    o.mat = (uint32_t)pool.size();
    o.dense = o.mat;
    for (int j = 0; j < d * d; ++j) pool.emplace_back(m[2 * j], m[2 * j + 1]);
    double ph[8];
    uint8_t perm = 0, unit = 0;
    if (ks[i] <= 2 && classify_monomial(m, ks[i], &perm, ph, &unit)) {
      o.mono = 1;
      o.perm = perm;
      o.unit = unit;
      o.mat = (uint32_t)pool.size();
      for (int j = 0; j < d; ++j) pool.emplace_back(ph[2 * j], ph[2 * j + 1]);
    } else if (ks[i] == 2) {
      o.xpat = (uint8_t)classify_xpattern(m);   // as the runtime's queue classifies it
    }
    ops.push_back(o);
  }
  std::vector<cplx64> cp(reinterpret_cast<const cplx64*>(pool.data()),
                         reinterpret_cast<const cplx64*>(pool.data()) + pool.size());
  if (fuse) ops = fuse_two_qubit_blocks(ops, cp, fuse == 2);
  if (fuse == 2) {
    decompose_one_qubit_ops(ops, cp);
    normalize_one_qubit_ops(ops, cp);
  }
  SchedParams p{};
  p.nbits = nbits;
  p.M = M;
  p.c = c;
  p.R = R;
  p.max_stages = max_stages;
  p.budget = budget;
  std::vector<PassPlan> plans;
  std::string err, all;
  if (plan_passes(p, ops, plans, err) < 0) {
    snprintf(out, (size_t)outlen, "plan: %s", err.c_str());
    return -1;
  }
  std::vector<cplx64> packed;
  pack_pass_matrices(plans, cp.data(), packed);
  for (size_t i = 0; i < plans.size(); ++i) {
    const std::string s = jit_pass_source(plans[i].desc, err);
    if (s.empty()) {
      snprintf(out, (size_t)outlen, "pass %zu: %s", i, err.c_str());
      return -1;
    }
    if (i) all += "\n//@@PASS@@\n";
    all += s;
  }
  if ((long long)all.size() + 1 > outlen) {
    snprintf(out, (size_t)outlen, "output buffer too small (%zu bytes needed)", all.size() + 1);
    return -1;
  }
  memcpy(out, all.c_str(), all.size() + 1);
  return (int)plans.size();
}

// Sources of the kernels specialised to an ansatz's forward and backward
// passes (shared-memory matrices, gradient accumulators: the adjoint
// executor's form), planned as the executor plans them; separated by lines
// "//@@PASS@@".  Returns the number of passes, or -1 (message in `out`).
extern "C" int emu_adjoint_sources(int n, int nops, const int* kinds, const int* q0, const int* q1, const int* pidx,
                                   const double* params, int M, int c, int R, int max_stages, double budget,
                                   int narrow, char* out, long long outlen) {
  std::vector<AnsatzOp> ops(nops);
  for (int i = 0; i < nops; ++i) ops[i] = {kinds[i], q0[i], q1[i], pidx[i]};
  std::string err, all;
  if (ansatz_check(n, ops, err) < 0) {
    snprintf(out, (size_t)outlen, "%s", err.c_str());
    return -1;
  }
  int count = 0;
  // passes 0, 1: forward and backward as a shared plan runs them (fused
  // blocks); 2, 3: the single-set forms (rotations and phases, scaled steps)
  for (int pass = 0; pass < 4; ++pass) {
    AdjointOps jo;
    adjoint_ops(n, ops, params, true, true, pass >= 2, jo);
    const std::vector<SchedOp>& fused = (pass & 1) ? jo.bw : jo.fw;
    std::vector<cplx64>& pool = (pass & 1) ? jo.bpool : jo.fpool;
    SchedParams p{};
    p.nbits = (pass & 1) ? n + 1 : n;
    if (p.nbits < 7) continue;
    p.M = M;
    p.c = c;
    p.R = R;
    p.max_stages = max_stages;
    p.budget = budget;
    std::vector<PassPlan> plans;
    if (plan_passes(p, fused, plans, err) < 0) {
      snprintf(out, (size_t)outlen, "plan: %s", err.c_str());
      return -1;
    }
    std::vector<cplx64> packed;
    pack_pass_matrices(plans, pool.data(), packed);
    for (const PassPlan& pl : plans) {
      const std::string s = jit_pass_source(pl.desc, err, 2, 0, true, narrow != 0);
      if (s.empty()) {
        snprintf(out, (size_t)outlen, "%s", err.c_str());
        return -1;
      }
      if (count++) all += "\n//@@PASS@@\n";
      all += s;
    }
  }
  if ((long long)all.size() + 1 > outlen) {
    snprintf(out, (size_t)outlen, "output buffer too small (%zu bytes needed)", all.size() + 1);
    return -1;
  }
  memcpy(out, all.c_str(), all.size() + 1);
  return count;
}

// Human-readable stage layout of every planned pass (development aid for the
// planner): per stage the physical bits of the register slots and lanes and
// the operations (kind, slot/lane a, slot b).
extern "C" int emu_plan_dump(int nbits, int M, int c, int R, int max_stages, double budget, int fuse, int nops,
                             const int* ks, const int* qs, const double* mats, const long long* mat_off, char* out,
                             long long outlen) {
  std::vector<cd> pool;
  std::vector<SchedOp> ops;
  for (int i = 0; i < nops; ++i) {
    SchedOp o{};
    o.k = (uint8_t)ks[i];
    for (int j = 0; j < ks[i]; ++j) o.q[j] = (uint8_t)qs[i * 5 + j];
    const int d = 1 << ks[i];
    const double* m = mats + 2 * mat_off[i];
    o.mat = (uint32_t)pool.size();
    o.dense = o.mat;
    for (int j = 0; j < d * d; ++j) pool.emplace_back(m[2 * j], m[2 * j + 1]);
    double ph[8];
    uint8_t perm = 0, unit = 0;
    if (ks[i] <= 2 && classify_monomial(m, ks[i], &perm, ph, &unit)) {
      o.mono = 1;
      o.perm = perm;
      o.unit = unit;
      o.mat = (uint32_t)pool.size();
      for (int j = 0; j < d; ++j) pool.emplace_back(ph[2 * j], ph[2 * j + 1]);
    } else if (ks[i] == 2) {
      o.xpat = (uint8_t)classify_xpattern(m);   // as the runtime's queue classifies it
    }
    ops.push_back(o);
  }
  std::vector<cplx64> cp(reinterpret_cast<const cplx64*>(pool.data()),
                         reinterpret_cast<const cplx64*>(pool.data()) + pool.size());
  if (fuse) ops = fuse_two_qubit_blocks(ops, cp, fuse == 2);
  if (fuse == 2) {
    decompose_one_qubit_ops(ops, cp);
    normalize_one_qubit_ops(ops, cp);
  }
  SchedParams p{};
  p.nbits = nbits;
  p.M = M;
  p.c = c;
  p.R = R;
  p.max_stages = max_stages;
  p.budget = budget;
  std::vector<PassPlan> plans;
  std::string err, all;
  if (plan_passes(p, ops, plans, err) < 0) {
    snprintf(out, (size_t)outlen, "plan: %s", err.c_str());
    return -1;
  }
  static const char* kind[] = {"-", "D1R", "D1L", "D2R", "DKR", "M1R", "M1L", "M2R", "G2", "N1R", "R1R", "R1L", "X2R"};
  char buf[256];
  for (size_t pi = 0; pi < plans.size(); ++pi) {
    const PassDesc& d = plans[pi].desc;
    auto phys = [&](int j) { return j < d.c ? j : (int)d.H[j - d.c]; };
    snprintf(buf, sizeof buf, "pass %zu cost %.0f stages %d ops %u\n", pi, plans[pi].cost, d.nstages, d.nops);
    all += buf;
    for (int s = 0; s < d.nstages; ++s) {
      const StageDesc& sd = d.st[s];
      all += "  S[";
      for (int i = 0; i < d.R; ++i) { snprintf(buf, sizeof buf, "%d%s", phys(sd.S[i]), i + 1 < d.R ? " " : ""); all += buf; }
      all += "] L[";
      for (int i = 0; i < kLaneBits; ++i) { snprintf(buf, sizeof buf, "%d%s", phys(sd.lane[i]), i + 1 < kLaneBits ? " " : ""); all += buf; }
      uint32_t v[3], r = 0;
      for (int i = 0; i < 3; ++i) v[i] = swz(1u << sd.lane[i]) & 7u;
      for (int bit = 0; bit < 3; ++bit) {   // rank over GF(2) of the lanes' swizzle images
        int piv = -1;
        for (int i = (int)r; i < 3; ++i)
          if ((v[i] >> bit) & 1) { piv = i; break; }
        if (piv < 0) continue;
        std::swap(v[r], v[piv]);
        for (int i = 0; i < 3; ++i)
          if (i != (int)r && ((v[i] >> bit) & 1)) v[i] ^= v[r];
        ++r;
      }
      snprintf(buf, sizeof buf, "] rank%u", r);
      all += buf;
      for (int o = sd.op0; o < sd.op1; ++o) {
        const OpDesc& od = d.ops[o];
        if (od.k == 2) snprintf(buf, sizeof buf, " %s(%d,%d)", kind[od.kind], phys(sd.S[od.a]), phys(sd.S[od.b]));
        else if (od.kind == OP_D1L || od.kind == OP_M1L || od.kind == OP_R1L) snprintf(buf, sizeof buf, " %s(L%d)", kind[od.kind], phys(sd.lane[od.a]));
        else if (od.kind == OP_DKR) snprintf(buf, sizeof buf, " DKR%d", od.k);
        else snprintf(buf, sizeof buf, " %s(%d)", kind[od.kind], phys(sd.S[od.a]));
        all += buf;
      }
      all += "\n";
    }
  }
  if ((long long)all.size() + 1 > outlen) return -1;
  memcpy(out, all.c_str(), all.size() + 1);
  return (int)plans.size();
}

// OP_X2R's shape classification (classify_xpattern) of a 4x4 row-major matrix
// given as interleaved re/im doubles.
extern "C" int emu_classify_xpattern(const double* m) { return classify_xpattern(m); }

// Scales of a backward sweep's gradient terms in the order its planned passes
// run the operations (exec_grad_scales), for an ansatz planned as the adjoint
// executor plans a single-set circuit; also the queue-order scales
// ansatz_backward reports.  Returns the number of terms (-1: error).
extern "C" int emu_grad_scales(int n, int nops, const int* kinds, const int* q0, const int* q1, const int* pidx,
                               const double* params, int M, int c, double* exec_scale, double* queue_scale, int cap) {
  std::vector<AnsatzOp> ops(nops);
  for (int i = 0; i < nops; ++i) ops[i] = {kinds[i], q0[i], q1[i], pidx[i]};
  std::string err;
  if (ansatz_check(n, ops, err) < 0) return -1;
  AdjointOps jo;
  adjoint_ops(n, ops, params, true, true, true, jo);
  SchedParams p{};
  p.nbits = std::max(n + 1, 7);
  p.M = M;
  p.c = c;
  p.R = 4;
  p.max_stages = 8;
  p.budget = 200.0;
  std::vector<PassPlan> plans;
  if (plan_passes(p, jo.bw, plans, err) < 0) return -1;
  std::vector<double> sc;
  exec_grad_scales(&plans, jo.bw, sc);
  if ((int)sc.size() > cap || sc.size() != jo.grad_scale.size()) return -1;
  for (size_t t = 0; t < sc.size(); ++t) {
    exec_scale[t] = sc[t];
    queue_scale[t] = jo.grad_scale[t];
  }
  return (int)sc.size();
}
