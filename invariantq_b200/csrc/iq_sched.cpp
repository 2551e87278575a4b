// iq_sched.cpp -- host-side gate scheduler: turns the queue of gates and
// channels recorded through the C ABI into tile passes (see iq_plan.h).
//
// The reference applies every gate as its own sweep over the state
// (core/src/statevector.cpp:26-152, one OpenMP loop per call).  Here the
// queued operations are grouped greedily, in dependency order, into passes
// whose operations all act on the M index bits a tile holds, so a group of
// gates costs one read and one write of the array.  Inside a pass the
// operations are split into register stages (R register slots + 3 lane bits).
// Operations are applied in queue order per qubit, so the result is the same
// product of matrices the reference applies one call at a time.
#include "iq_plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <set>

namespace iqb {

double op_cost(const SchedOp& op) {
  if (op.mono) return op.unit ? 0.25 : 4.0;
  return 4.0 * double(1u << op.k);
}

int classify_monomial(const double* m, int k, uint8_t* perm, double* phases, uint8_t* unit) {
  if (k < 1 || k > 2) return 0;
  const int d = 1 << k;
  int colcount[4] = {0, 0, 0, 0};
  uint8_t p = 0;
  uint8_t u = 1;
  for (int r = 0; r < d; ++r) {
    int nz = -1;
    for (int c = 0; c < d; ++c) {
      const double re = m[2 * (r * d + c)], im = m[2 * (r * d + c) + 1];
      if (re != 0.0 || im != 0.0) {
        if (nz >= 0) return 0;
        nz = c;
      }
    }
    if (nz < 0) return 0;
    colcount[nz]++;
    p |= uint8_t(nz << (2 * r));
    phases[2 * r] = m[2 * (r * d + nz)];
    phases[2 * r + 1] = m[2 * (r * d + nz) + 1];
    if (phases[2 * r] != 1.0 || phases[2 * r + 1] != 0.0) u = 0;
  }
  for (int c = 0; c < d; ++c)
    if (colcount[c] != 1) return 0;
  *perm = p;
  *unit = u;
  return 1;
}

namespace {

struct Stage {
  int S[kMaxK];
  int nS = 0;
  bool dk = false;                 // holds one dense k>=3 block; closed
  std::vector<int> ops;
};

struct PassBuilder {
  const SchedParams& p;
  int c;
  std::vector<Stage> stages;
  explicit PassBuilder(const SchedParams& pp, int cc) : p(pp), c(cc) {}

  static bool inS(const Stage& s, int b) {
    for (int i = 0; i < s.nS; ++i)
      if (s.S[i] == b) return true;
    return false;
  }
  int lowcount(const Stage& s) const {
    int n = 0;
    for (int i = 0; i < s.nS; ++i) n += s.S[i] < c;
    return n;
  }
  // lowest 3 bits of [0, c) not in S
  bool isLane(const Stage& s, int b) const {
    if (b >= c || inS(s, b)) return false;
    int seen = 0;
    for (int x = 0; x < c && seen < kLaneBits; ++x) {
      if (inS(s, x)) continue;
      if (x == b) return true;
      ++seen;
    }
    return false;
  }
  // try to add operation bits to stage s (k <= 2); returns false if it does not fit
  bool tryAdd(Stage& s, const SchedOp& op) const {
    if (s.dk) return false;
    if (op.k == 1) {
      const int b = op.q[0];
      if (inS(s, b) || isLane(s, b)) return true;
      if (s.nS >= p.R) return false;
      if (b < c && lowcount(s) + 1 > c - kLaneBits) return false;
      s.S[s.nS++] = b;
      return true;
    }
    int need[2], nn = 0, lowadd = 0;
    for (int i = 0; i < 2; ++i)
      if (!inS(s, op.q[i])) { need[nn++] = op.q[i]; lowadd += op.q[i] < c; }
    if (s.nS + nn > p.R) return false;
    if (lowcount(s) + lowadd > c - kLaneBits) return false;
    for (int i = 0; i < nn; ++i) s.S[s.nS++] = need[i];
    return true;
  }
  // place op i; returns false if the pass cannot take it
  bool place(int idx, const SchedOp& op) {
    if (op.k >= 3) {
      if (op.k > p.R) return false;
      if ((int)stages.size() >= p.max_stages) return false;
      Stage s;
      s.dk = true;
      for (int i = 0; i < op.k; ++i) s.S[s.nS++] = op.q[i];
      s.ops.push_back(idx);
      stages.push_back(s);
      return true;
    }
    if (!stages.empty()) {
      Stage trial = stages.back();
      if (tryAdd(trial, op)) {
        trial.ops.push_back(idx);
        stages.back() = trial;
        return true;
      }
    }
    if ((int)stages.size() >= p.max_stages) return false;
    Stage s;
    if (!tryAdd(s, op)) return false;
    s.ops.push_back(idx);
    stages.push_back(s);
    return true;
  }
};

inline uint64_t opmask(const SchedOp& op) {
  uint64_t m = 0;
  for (int i = 0; i < op.k; ++i) m |= 1ULL << op.q[i];
  return m;
}

}  // namespace

int plan_passes(const SchedParams& p, const std::vector<SchedOp>& ops, std::vector<PassPlan>& out,
                std::string& err) {
  const int nb = p.nbits;
  const int nops = (int)ops.size();
  if (p.R < 4 || p.R > kMaxK) { err = "register slots must be 4 or 5"; return -1; }
  if (nb < p.R + kLaneBits) { err = "array too small for the tile kernel"; return -1; }
  const int M = std::min(p.M, nb);
  const bool whole = nb <= p.M;         // the whole array is one tile
  const int c = whole ? std::min(p.c, M) : p.c;
  if (M < p.R + kLaneBits || M > kMaxTileBits) { err = "tile bits out of range"; return -1; }
  if (c < 5 || c > 7) { err = "chunk bits must be 5..7"; return -1; }
  if (!whole && M - c < kMaxK) { err = "tile must hold the chunk plus 5 free bits"; return -1; }

  for (int i = 0; i < nops; ++i) {
    const SchedOp& o = ops[i];
    if (o.k < 1 || o.k > kMaxK) { err = "operation width out of range"; return -1; }
    for (int j = 0; j < o.k; ++j) {
      if (o.q[j] >= nb) { err = "operation bit out of range"; return -1; }
      for (int l = 0; l < j; ++l)
        if (o.q[l] == o.q[j]) { err = "repeated operation bit"; return -1; }
    }
    if (o.k > p.R) { err = "dense block wider than the register slots"; return -1; }
  }

  // per-bit queues of op indices (dependency order)
  std::vector<std::vector<int>> q(nb);
  std::vector<size_t> head(nb, 0);
  for (int i = 0; i < nops; ++i)
    for (int j = 0; j < ops[i].k; ++j) q[ops[i].q[j]].push_back(i);
  std::vector<int> headcnt(nops, 0);
  std::set<int> ready;
  for (int b = 0; b < nb; ++b)
    if (!q[b].empty()) {
      int i = q[b][0];
      if (++headcnt[i] == ops[i].k) ready.insert(i);
    }
  auto retire = [&](int i) {
    for (int j = 0; j < ops[i].k; ++j) {
      int b = ops[i].q[j];
      ++head[b];
      if (head[b] < q[b].size()) {
        int nx = q[b][head[b]];
        if (++headcnt[nx] == ops[nx].k) ready.insert(nx);
      }
    }
  };

  const uint64_t lowmask = (c >= 64) ? ~0ULL : ((1ULL << c) - 1);
  const uint64_t allmask = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  int scheduled = 0;
  while (scheduled < nops) {
    if (ready.empty()) { err = "scheduler found no ready operation"; return -1; }
    uint64_t local = whole ? allmask : lowmask;
    int free_slots = whole ? 0 : (M - c);
    PassBuilder pb(p, c);
    std::vector<int> taken;
    double cost = 0.0;
    for (;;) {
      bool progress = true;
      while (progress) {
        progress = false;
        for (auto it = ready.begin(); it != ready.end();) {
          const int i = *it;
          const SchedOp& o = ops[i];
          const double oc = op_cost(o);
          if ((opmask(o) & ~local) == 0 && (int)taken.size() < kMaxPassOps &&
              (taken.empty() || cost + oc <= p.budget) && pb.place(i, o)) {
            taken.push_back(i);
            cost += oc;
            it = ready.erase(it);
            retire(i);
            progress = true;
          } else {
            ++it;
          }
        }
      }
      if (free_slots == 0 || (int)taken.size() >= kMaxPassOps) break;
      int best = -1, bestmiss = 0;
      for (int i : ready) {
        const int miss = __builtin_popcountll(opmask(ops[i]) & ~local);
        if (miss > 0 && miss <= free_slots && (taken.empty() || cost + op_cost(ops[i]) <= p.budget)) {
          best = i;
          bestmiss = miss;
          break;
        }
      }
      if (best < 0) break;
      local |= opmask(ops[best]);
      free_slots -= bestmiss;
    }
    if (taken.empty()) { err = "scheduler could not place an operation"; return -1; }
    scheduled += (int)taken.size();

    // ---- finalize: tile-local numbering, padded register slots, encoded ops
    PassPlan plan;
    std::memset(&plan.desc, 0, sizeof(plan.desc));
    PassDesc& d = plan.desc;
    std::vector<int> H;
    for (int b = c; b < nb; ++b)
      if (local & (1ULL << b)) H.push_back(b);
    for (int b = nb - 1; (int)H.size() < M - c && b >= c; --b)
      if (!(local & (1ULL << b))) H.push_back(b);
    std::sort(H.begin(), H.end());
    int pos[64];
    for (int b = 0; b < 64; ++b) pos[b] = -1;
    for (int b = 0; b < c; ++b) pos[b] = b;
    for (size_t i = 0; i < H.size(); ++i) pos[H[i]] = c + (int)i;
    d.M = (uint8_t)M;
    d.c = (uint8_t)c;
    d.R = (uint8_t)p.R;
    d.nH = (uint8_t)H.size();
    d.nbox = (uint8_t)std::min<int>(2, (int)H.size());
    for (size_t i = 0; i < H.size(); ++i) d.H[i] = (uint8_t)H[i];
    d.ntiles = 1ULL << (nb - M);
    d.nstages = (uint8_t)pb.stages.size();
    int nout = 0;
    for (size_t si = 0; si < pb.stages.size(); ++si) {
      const Stage& s = pb.stages[si];
      StageDesc& sd = d.st[si];
      bool used[kMaxTileBits] = {};
      int slot_of[kMaxTileBits];
      for (int j = 0; j < kMaxTileBits; ++j) slot_of[j] = -1;
      int nS = 0;
      for (int i = 0; i < s.nS; ++i) {
        const int j = pos[s.S[i]];
        sd.S[nS] = (uint8_t)j;
        slot_of[j] = nS++;
        used[j] = true;
      }
      for (int j = M - 1; nS < p.R && j >= 0; --j)
        if (!used[j]) { sd.S[nS] = (uint8_t)j; slot_of[j] = nS++; used[j] = true; }
      int nl = 0;
      int lane_of[kMaxTileBits];
      for (int j = 0; j < kMaxTileBits; ++j) lane_of[j] = -1;
      for (int j = 0; j < M && nl < kLaneBits; ++j)
        if (!used[j]) { sd.lane[nl] = (uint8_t)j; lane_of[j] = nl++; used[j] = true; }
      sd.nt = 0;
      for (int j = 0; j < M; ++j)
        if (!used[j]) sd.tb[sd.nt++] = (uint8_t)j;
      sd.op0 = (uint16_t)nout;
      for (int i : s.ops) {
        const SchedOp& o = ops[i];
        OpDesc& od = d.ops[nout++];
        od.k = o.k;
        od.mat = o.mat;
        od.perm = o.perm;
        od.flags = o.unit ? OPF_UNIT_PHASE : 0;
        if (o.k == 1) {
          const int j = pos[o.q[0]];
          if (slot_of[j] >= 0) { od.kind = o.mono ? OP_M1R : OP_D1R; od.a = (uint8_t)slot_of[j]; }
          else if (lane_of[j] >= 0) { od.kind = o.mono ? OP_M1L : OP_D1L; od.a = (uint8_t)lane_of[j]; }
          else { err = "internal: 1q operation bit is neither a slot nor a lane"; return -1; }
        } else if (o.k == 2) {
          const int j0 = pos[o.q[0]], j1 = pos[o.q[1]];
          if (slot_of[j0] < 0 || slot_of[j1] < 0) { err = "internal: 2q operation outside slots"; return -1; }
          od.kind = o.mono ? OP_M2R : OP_D2R;
          od.a = (uint8_t)slot_of[j0];
          od.b = (uint8_t)slot_of[j1];
        } else {
          for (int t = 0; t < o.k; ++t)
            if (slot_of[pos[o.q[t]]] != t) { err = "internal: dense block slots out of order"; return -1; }
          od.kind = OP_DKR;
        }
      }
      sd.op1 = (uint16_t)nout;
    }
    d.nops = (uint32_t)nout;
    plan.nsrc = (int)taken.size();
    plan.cost = cost;
    out.push_back(plan);
  }
  return (int)out.size();
}

}  // namespace iqb
