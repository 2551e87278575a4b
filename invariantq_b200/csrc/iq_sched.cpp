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
#include <array>
#include <complex>
#include <set>

namespace iqb {

// complex elements of an operation's matrix data (dense 4^k, monomial 2^k phases)
int op_mat_elems(const SchedOp& op) {
  if (op.grad) return 4;
  return op.mono ? (1 << op.k) : (1 << (2 * op.k));
}

double op_cost(const SchedOp& op, double grad_cost) {
  if (op.grad) return grad_cost;   // 2x2 on both halves plus the gradient products
  if (op.mono) {
    if (op.unit) return 0.25;
    const int rows = 1 << op.k;
    const int nonunit = rows - __builtin_popcount(op.urows & ((1u << rows) - 1));
    return 4.0 * nonunit / rows;
  }
  if (op.rot) return 2.0;
  if (op.norm) return 6.0;
  if (op.realm && op.k == 1) return 4.0;
  if (op.xpat) return ((op.xpat & XPAT_CORNERS_REAL) ? 2.0 : 4.0) + ((op.xpat & XPAT_MIDDLE_REAL) ? 1.0 : 2.0);
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

int classify_xpattern(const double* m) {
  bool corners_real = true, middle_real = true;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      const double re = m[2 * (r * 4 + c)], im = m[2 * (r * 4 + c) + 1];
      const bool corner = (r == 0 || r == 3) && (c == 0 || c == 3);
      const bool middle = r == c && (r == 1 || r == 2);
      if (!corner && !middle && (re != 0.0 || im != 0.0)) return 0;
      if (corner && im != 0.0) corners_real = false;
      if (middle && im != 0.0) middle_real = false;
    }
  return 1 | (corners_real ? XPAT_CORNERS_REAL : 0) | (middle_real ? XPAT_MIDDLE_REAL : 0);
}

namespace {

struct Stage {
  int S[kMaxK];
  int nS = 0;
  uint64_t lanereq = 0;            // bits that 1q lane operations of this stage act on
  bool dk = false;                 // holds one dense k>=3 block; closed
  std::vector<int> ops;
};

struct PassBuilder {
  const SchedParams& p;
  int c;
  std::vector<Stage> stages;
  bool allow_new = true;   // false: an operation joins the current stage or waits
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
  // Chunk bits a stage may hold in slots: c - 3 keeps three chunk bits free for
  // lane operations.  A stage without lane operations may take one more: its
  // lanes can then use the first tile bit above the chunk, whose swizzled
  // image also has a low bit set, so the octet's accesses can stay on eight
  // bank groups (the lane choice below takes the best rank it finds).
  int lowlimit(const Stage& s, bool no_lanes_after) const {
    return c - kLaneBits + ((no_lanes_after && s.lanereq == 0) ? 1 : 0);
  }
  // Whether a stage without lane operations whose slots also take the nn bits
  // `add` keeps three lane candidates with independent swizzle images: the
  // low three bits of swz(1 << j) are bit j mod 3 for tile-local j < 6 and 0
  // above, so each class {k, k + 3} (k = 0, 1, 2) needs a member outside the
  // slots.  Tile-local bits >= c are high tile bits chosen when the pass is
  // finalised; physical bit j stands in for them (it is the one they are when
  // it is local in the pass).
  bool lanes_feasible(const Stage& s, const int* add, int nn) const {
    for (int k = 0; k < 3; ++k) {
      bool free_member = false;
      for (int j = k; j < 6 && !free_member; j += 3) {
        // j >= c: the high tile bit H[j - c] is at least physical bit j, and is
        // that bit whenever it is local; count it taken when a slot holds it
        bool taken = inS(s, j);
        for (int i = 0; i < nn; ++i) taken |= add[i] == j;
        free_member = !taken;
      }
      if (!free_member) return false;
    }
    return true;
  }
  // Register slots take at most c - 3 of the chunk bits [0, c), so three lane
  // bits always remain inside the chunk; lane operations name up to 3 of them.
  bool tryAdd(Stage& s, const SchedOp& op) const {
    if (s.dk) return false;
    if (op.k == 1) {
      const int b = op.q[0];
      const uint64_t bm = 1ULL << b;
      if (inS(s, b) || (s.lanereq & bm)) return true;
      if (b < c && __builtin_popcountll(s.lanereq) < kLaneBits && lowcount(s) <= c - kLaneBits) {
        s.lanereq |= bm;
        return true;
      }
      if (s.nS >= p.R) return false;
      if (b < c && lowcount(s) + 1 > c - kLaneBits) return false;
      s.S[s.nS++] = b;
      return true;
    }
    int need[2], nn = 0, lowadd = 0;
    for (int i = 0; i < 2; ++i)
      if (!inS(s, op.q[i])) { need[nn++] = op.q[i]; lowadd += op.q[i] < c; }
    if (s.nS + nn > p.R) return false;
    if (lowcount(s) + lowadd > lowlimit(s, op.grad != 0)) {
      // a stage without lane operations may hold more chunk bits as long as
      // its lanes can still be drawn with independent swizzle images; an empty
      // stage takes the operation regardless (its lanes may then share bank
      // groups: slower, still correct)
      if (s.lanereq != 0 || (s.nS > 0 && !lanes_feasible(s, need, nn))) return false;
    }
    for (int i = 0; i < nn; ++i) {
      s.S[s.nS++] = need[i];
      s.lanereq &= ~(1ULL << need[i]);   // earlier lane ops on this bit become slot ops
    }
    return true;
  }
  bool place(int idx, const SchedOp& op) {
    if (op.grad) {
      // adjoint steps want the psi / lambda select bit in register slot 0; slot
      // positions bind to operations only when the pass is finalised, so the
      // current stage can take the select bit into slot 0 (swapped there, or
      // inserted when a slot is free and the chunk-bit limit allows)
      if (!stages.empty() && !stages.back().dk) {
        Stage trial = stages.back();
        const int sel = op.q[0];
        bool ready = trial.nS > 0 && trial.S[0] == sel;
        if (!ready && inS(trial, sel)) {
          for (int i = 1; i < trial.nS; ++i)
            if (trial.S[i] == sel) std::swap(trial.S[0], trial.S[i]);
          ready = true;
        } else if (!ready && trial.nS < p.R && !(trial.lanereq & (1ULL << sel)) &&
                   (sel >= c || lowcount(trial) + 1 <= lowlimit(trial, true))) {
          for (int i = trial.nS; i > 0; --i) trial.S[i] = trial.S[i - 1];
          trial.S[0] = sel;
          ++trial.nS;
          ready = true;
        }
        if (ready && tryAdd(trial, op)) {
          trial.ops.push_back(idx);
          stages.back() = trial;
          return true;
        }
      }
      if ((int)stages.size() >= p.max_stages || (!allow_new && !stages.empty())) return false;
      Stage s;
      s.S[s.nS++] = op.q[0];
      if (!tryAdd(s, op)) return false;
      s.ops.push_back(idx);
      stages.push_back(s);
      return true;
    }
    if (op.k >= 3) {
      if (op.k > p.R) return false;
      if ((int)stages.size() >= p.max_stages || (!allow_new && !stages.empty())) return false;
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
    if ((int)stages.size() >= p.max_stages || (!allow_new && !stages.empty())) return false;
    Stage s;
    if (!tryAdd(s, op)) return false;
    s.ops.push_back(idx);
    stages.push_back(s);
    return true;
  }
};

// Rank over GF(2) of the low three bits of swz(1 << j) for the lane bits: the
// eight lanes of an octet hit distinct shared-memory bank groups iff it is 3.
int lane_rank(const int* l) {
  uint32_t v[3];
  for (int i = 0; i < 3; ++i) v[i] = swz(1u << l[i]) & 7u;
  int r = 0;
  for (int bit = 0; bit < 3; ++bit) {
    int piv = -1;
    for (int i = r; i < 3; ++i)
      if (v[i] & (1u << bit)) { piv = i; break; }
    if (piv < 0) continue;
    std::swap(v[r], v[piv]);
    for (int i = 0; i < 3; ++i)
      if (i != r && (v[i] & (1u << bit))) v[i] ^= v[r];
    ++r;
  }
  return r;
}

// Choose the 3 lane bits (tile-local) among `cand`, containing `req`, with the
// best bank-group rank (ties: lowest bits).
bool choose_lanes(const std::vector<int>& cand, uint32_t req, int out[3]) {
  int best = -1;
  const int n = (int)cand.size();
  for (int a = 0; a < n; ++a)
    for (int b = a + 1; b < n; ++b)
      for (int d = b + 1; d < n; ++d) {
        const int l[3] = {cand[a], cand[b], cand[d]};
        const uint32_t m = (1u << l[0]) | (1u << l[1]) | (1u << l[2]);
        if ((m & req) != req) continue;
        const int r = lane_rank(l);
        if (r > best) {
          best = r;
          out[0] = l[0]; out[1] = l[1]; out[2] = l[2];
          if (r == 3) return true;
        }
      }
  return best >= 0;
}

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
  if (p.R < 3 || p.R > kMaxK) { err = "register slots must be 3, 4 or 5"; return -1; }
  if (nb < p.R + kLaneBits) { err = "array too small for the tile kernel"; return -1; }
  const int M = std::min(p.M, nb);
  const bool whole = nb <= p.M;         // the whole array is one tile
  const int c = whole ? std::min(p.c, M) : p.c;
  if (M < p.R + kLaneBits || M > kMaxTileBits) { err = "tile bits out of range"; return -1; }
  if (c < 3 || c > 7) { err = "chunk bits must be 3..7"; return -1; }
  // a tile moves in 2^(M - c - 2) box copies, one per lane of the CTA's first 128 threads
  if (!whole && M - c - 2 > 7) { err = "too many tile copies: raise the chunk bits or lower the tile bits"; return -1; }
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

  // per-bit queues of op indices (dependency order).  An adjoint step applies
  // the same 2x2 to the psi and lambda halves and never mixes them, so steps on
  // different qubits commute (their gradient terms too: Im<lambda|P_b|psi> does
  // not change when a unitary on another qubit acts on both halves); when no
  // other operation touches the select bit, adjoint steps are ordered by their
  // qubit bit only.
  std::vector<uint8_t> other_use(nb, 0);
  for (int i = 0; i < nops; ++i)
    if (!ops[i].grad)
      for (int j = 0; j < ops[i].k; ++j) other_use[ops[i].q[j]] = 1;
  auto dep_first = [&](int i) { return (ops[i].grad && !other_use[ops[i].q[0]]) ? 1 : 0; };
  auto ndeps = [&](int i) { return ops[i].k - dep_first(i); };
  std::vector<std::vector<int>> q(nb);
  std::vector<size_t> head(nb, 0);
  for (int i = 0; i < nops; ++i)
    for (int j = dep_first(i); j < ops[i].k; ++j) q[ops[i].q[j]].push_back(i);
  std::vector<int> headcnt(nops, 0);
  std::set<int> ready;
  for (int b = 0; b < nb; ++b)
    if (!q[b].empty()) {
      int i = q[b][0];
      if (++headcnt[i] == ndeps(i)) ready.insert(i);
    }
  auto retire = [&](int i) {
    for (int j = dep_first(i); j < ops[i].k; ++j) {
      int b = ops[i].q[j];
      ++head[b];
      if (head[b] < q[b].size()) {
        int nx = q[b][head[b]];
        if (++headcnt[nx] == ndeps(nx)) ready.insert(nx);
      }
    }
  };

  const uint64_t lowmask = (c >= 64) ? ~0ULL : ((1ULL << c) - 1);
  const uint64_t allmask = (nb >= 64) ? ~0ULL : ((1ULL << nb) - 1);
  // the psi / lambda select bit of adjoint steps is local in every pass (as
  // the chunk bits are): otherwise passes widened by the fixed gates first
  // would leave it out and the steps could not join them
  uint64_t select_mask = 0;
  for (int i = 0; i < nops; ++i)
    if (ops[i].grad) select_mask |= 1ULL << ops[i].q[0];
  select_mask &= ~lowmask;
  int scheduled = 0;
  while (scheduled < nops) {
    if (ready.empty()) { err = "scheduler found no ready operation"; return -1; }
    uint64_t local = whole ? allmask : (lowmask | select_mask);
    int free_slots = whole ? 0 : (M - c - __builtin_popcountll(select_mask));
    PassBuilder pb(p, c);
    std::vector<int> taken;
    double cost = 0.0;
    int mat_elems = 0;
    int ngrad = 0;
    for (;;) {
      // every ready operation that fits the current stage joins it before an
      // operation may open the next stage
      bool progress = true;
      while (progress) {
        progress = false;
        for (int phase = 0; phase < 2 && !progress; ++phase) {
          pb.allow_new = phase == 1;
          for (auto it = ready.begin(); it != ready.end();) {
            const int i = *it;
            const SchedOp& o = ops[i];
            const double oc = op_cost(o, p.grad_cost);
            if ((opmask(o) & ~local) == 0 && (int)taken.size() < kMaxPassOps &&
                mat_elems + op_mat_elems(o) <= kSmemMatElems && (taken.empty() || cost + oc <= p.budget) &&
                (!o.grad || ngrad < kMaxPassGrads) && pb.place(i, o)) {
              taken.push_back(i);
              cost += oc;
              mat_elems += op_mat_elems(o);
              ngrad += o.grad ? 1 : 0;
              it = ready.erase(it);
              retire(i);
              progress = true;
              if (phase == 1) break;   // one operation opens the stage; the others try to join it
            } else {
              ++it;
            }
          }
        }
      }
      pb.allow_new = true;
      if (free_slots == 0 || (int)taken.size() >= kMaxPassOps) break;
      int best = -1, bestmiss = 0;
      for (int i : ready) {
        const int miss = __builtin_popcountll(opmask(ops[i]) & ~local);
        if (miss > 0 && miss <= free_slots && (taken.empty() || cost + op_cost(ops[i], p.grad_cost) <= p.budget)) {
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
    d.ngrad = 0;
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
      // lanes: chunk bits for stages with lane operations, any tile bit for the
      // others; padding slots come from the highest bits left over
      uint32_t req = 0;
      for (int b = 0; b < c; ++b)
        if (s.lanereq & (1ULL << b)) req |= 1u << pos[b];
      std::vector<int> cand;
      const int lim = s.lanereq ? c : M;
      for (int j = 0; j < lim; ++j)
        if (!used[j]) cand.push_back(j);
      // keep R - nS bits for padding out of the candidates' reach when possible
      int lanes[3];
      if (!choose_lanes(cand, req, lanes)) { err = "internal: no lane bits for a stage"; return -1; }
      int lane_of[kMaxTileBits];
      for (int j = 0; j < kMaxTileBits; ++j) lane_of[j] = -1;
      for (int l = 0; l < kLaneBits; ++l) {
        sd.lane[l] = (uint8_t)lanes[l];
        lane_of[lanes[l]] = l;
        used[lanes[l]] = true;
      }
      for (int j = M - 1; nS < p.R && j >= 0; --j)
        if (!used[j]) { sd.S[nS] = (uint8_t)j; slot_of[j] = nS++; used[j] = true; }
      if (nS < p.R) { err = "internal: not enough tile bits for the register slots"; return -1; }
      sd.nt = 0;
      for (int j = 0; j < M; ++j)
        if (!used[j]) sd.tb[sd.nt++] = (uint8_t)j;
      sd.op0 = (uint16_t)nout;
      for (int i : s.ops) {
        const SchedOp& o = ops[i];
        plan.src.push_back((uint32_t)i);
        OpDesc& od = d.ops[nout++];
        od.k = o.k;
        od.mat = o.mat;
        od.perm = o.perm;
        od.flags = o.unit ? OPF_UNIT_PHASE : 0;
        od.urows = o.mono ? o.urows : 0;
        if (o.k == 1) {
          const int j = pos[o.q[0]];
          if (slot_of[j] >= 0) {
            od.kind = o.mono ? OP_M1R : (o.rot ? OP_R1R : (o.norm ? OP_N1R : OP_D1R));
            if (od.kind == OP_D1R && o.realm) od.flags |= OPF_REAL;
            od.a = (uint8_t)slot_of[j];
            if (o.norm) od.perm = (uint8_t)(o.norm - 1);
            if (o.rot) od.perm = (uint8_t)(o.rot - 1);
          }
          else if (lane_of[j] >= 0) {
            od.kind = o.mono ? OP_M1L : (o.rot ? OP_R1L : OP_D1L);
            if (od.kind == OP_D1L && o.realm && !o.norm) od.flags |= OPF_REAL;
            od.a = (uint8_t)lane_of[j];
            if (o.rot) od.perm = (uint8_t)(o.rot - 1);
          }
          else { err = "internal: 1q operation bit is neither a slot nor a lane"; return -1; }
        } else if (o.k == 2) {
          const int j0 = pos[o.q[0]], j1 = pos[o.q[1]];
          if (slot_of[j0] < 0 || slot_of[j1] < 0) { err = "internal: 2q operation outside slots"; return -1; }
          od.kind = o.grad ? OP_GRAD2 : (o.mono ? OP_M2R : (o.xpat ? OP_X2R : OP_D2R));
          if (od.kind == OP_X2R) od.flags = (uint8_t)(o.xpat >> 1);   // XPAT_* >> 1: bit 0 corners, bit 1 middle real
          od.a = (uint8_t)slot_of[j0];
          od.b = (uint8_t)slot_of[j1];
          if (o.grad) {
            od.perm = o.gen;
            od.flags = o.rot;                  // the inverse rotation's form (GradForm)
            od.gidx = d.ngrad;                 // local index; the global term goes to grad_term
            d.grad_term[d.ngrad++] = o.gidx;
          }
        } else {
          for (int t = 0; t < o.k; ++t)
            if (slot_of[pos[o.q[t]]] != t) { err = "internal: dense block slots out of order"; return -1; }
          od.kind = OP_DKR;
        }
      }
      sd.op1 = (uint16_t)nout;
    }
    d.nops = (uint32_t)nout;
    d.grad_base = 0;
    plan.nsrc = (int)taken.size();
    plan.cost = cost;
    out.push_back(plan);
  }
  return (int)out.size();
}

namespace {

using M4 = std::array<cplx64, 16>;

inline cplx64 cm(cplx64 a, cplx64 b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
inline cplx64 ca(cplx64 a, cplx64 b) { return {a.re + b.re, a.im + b.im}; }

M4 mul4(const M4& A, const M4& B) {
  M4 C;
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      cplx64 acc{0.0, 0.0};
      for (int k = 0; k < 4; ++k) acc = ca(acc, cm(A[r * 4 + k], B[k * 4 + c]));
      C[r * 4 + c] = acc;
    }
  return C;
}

// 2x2 U acting on local bit `bit` of a two-bit index (bit 0 = list[0])
M4 lift1(const cplx64* U, int bit) {
  M4 L;
  for (auto& x : L) x = {0.0, 0.0};
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) {
      const int ob = bit ^ 1;
      if (((r >> ob) & 1) != ((c >> ob) & 1)) continue;
      L[r * 4 + c] = U[((r >> bit) & 1) * 2 + ((c >> bit) & 1)];
    }
  return L;
}

// 4x4 U on list (u0, u1) re-expressed on list (l0, l1) = (u1, u0)
M4 swap_bits(const cplx64* U) {
  M4 L;
  auto sw = [](int i) { return ((i & 1) << 1) | ((i >> 1) & 1); };
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c) L[sw(r) * 4 + sw(c)] = U[r * 4 + c];
  return L;
}

struct Block {
  int k = 0;
  int q[2] = {-1, -1};
  M4 m;                 // dense (1q blocks use the top-left 2x2 in m[0], m[1], m[4], m[5])
  bool dead = false;
  int src = -1;         // index of the original op when the block is that op unchanged
  bool changed = false;
  bool xpat = false;    // a run of OP_X2R-shaped operations on one pair, kept apart from one-qubit blocks
};

}  // namespace

std::vector<SchedOp> fuse_two_qubit_blocks(const std::vector<SchedOp>& ops, std::vector<cplx64>& pool,
                                           bool monomial_barrier) {
  const int nb = 64;
  std::vector<Block> blocks;
  std::vector<int> open(nb, -1), last(nb, -1);
  std::vector<int> passthrough;   // ops of width >= 3 keep their place as blocks with k = 0
  auto mat2 = [&](const SchedOp& o) {
    M4 m;
    const cplx64* U = pool.data() + o.dense;
    m[0] = U[0]; m[1] = U[1]; m[4] = U[2]; m[5] = U[3];
    return m;
  };
  for (size_t i = 0; i < ops.size(); ++i) {
    const SchedOp& o = ops[i];
    // wide blocks and adjoint steps pass through unchanged, and so do two-qubit
    // monomials (CX, CZ, SWAP) when they are cheaper alone than inside a 4x4
    // adjoint steps and the scalars of a scaled backward sweep (smul) keep their place unchanged
    const bool diagonal2 = o.k == 2 && o.mono && o.perm == 0xE4;   // rows read their own column
    if (monomial_barrier && o.k == 2 && (o.xpat || diagonal2) && !o.grad && o.smul == 0.0) {
      // channel-shaped operations (OP_X2R's shape; diagonal ones included)
      // stay out of one-qubit blocks (a unitary inside would make the block
      // dense); consecutive ones on the same pair multiply into one block of
      // the same shape.  A run of one operation keeps it unchanged.
      const int a = o.q[0], bq = o.q[1];
      const int B = last[a];
      const cplx64* U = pool.data() + o.dense;
      M4 Um;
      for (int j = 0; j < 16; ++j) Um[j] = U[j];
      if (B >= 0 && B == last[bq] && blocks[B].xpat) {
        Block& bl = blocks[B];
        bl.m = mul4(bl.q[0] == a ? Um : swap_bits(Um.data()), bl.m);
        bl.changed = true;
        bl.src = -1;
        continue;
      }
      open[a] = open[bq] = -1;
      last[a] = last[bq] = (int)blocks.size();
      Block b;
      b.k = 2;
      b.q[0] = a;
      b.q[1] = bq;
      b.m = Um;
      b.src = (int)i;
      b.xpat = true;
      blocks.push_back(b);
      continue;
    }
    if (o.k >= 3 || o.grad || o.smul != 0.0 || (monomial_barrier && o.k == 2 && o.mono)) {
      for (int j = 0; j < o.k; ++j) { open[o.q[j]] = -1; last[o.q[j]] = (int)blocks.size(); }
      Block b;
      b.k = 0;
      b.src = (int)i;
      blocks.push_back(b);
      continue;
    }
    if (o.k == 1) {
      const int a = o.q[0];
      const int B = open[a];
      if (B >= 0 && last[a] == B) {
        Block& bl = blocks[B];
        const cplx64 U[4] = {pool[o.dense], pool[o.dense + 1], pool[o.dense + 2], pool[o.dense + 3]};
        if (bl.k == 1) {
          M4 u1 = mat2(o);
          M4 r;
          for (auto& x : r) x = {0.0, 0.0};
          for (int rr = 0; rr < 2; ++rr)
            for (int cc = 0; cc < 2; ++cc)
              for (int kk = 0; kk < 2; ++kk)
                r[rr * 4 + cc] = ca(r[rr * 4 + cc], cm(u1[rr * 4 + kk], bl.m[kk * 4 + cc]));
          bl.m = r;
        } else {
          bl.m = mul4(lift1(U, bl.q[0] == a ? 0 : 1), bl.m);
        }
        bl.changed = true;
        bl.src = -1;
        continue;
      }
      Block b;
      b.k = 1;
      b.q[0] = a;
      b.m = mat2(o);
      b.src = (int)i;
      open[a] = last[a] = (int)blocks.size();
      blocks.push_back(b);
      continue;
    }
    // two-qubit op on list (a, b) (bit 0 = a)
    const int a = o.q[0], bq = o.q[1];
    const int Ba = open[a], Bb = open[bq];
    const cplx64* U = pool.data() + o.dense;
    M4 Um;
    for (int j = 0; j < 16; ++j) Um[j] = U[j];
    if (Ba >= 0 && Ba == Bb && last[a] == Ba && last[bq] == Ba && blocks[Ba].k == 2) {
      Block& bl = blocks[Ba];
      bl.m = mul4(bl.q[0] == a ? Um : swap_bits(Um.data()), bl.m);
      bl.changed = true;
      bl.src = -1;
      continue;
    }
    const bool okA = Ba < 0 || (blocks[Ba].k == 1 && last[a] == Ba);
    const bool okB = Bb < 0 || (blocks[Bb].k == 1 && last[bq] == Bb);
    const int posc = std::max(Ba, Bb);
    // the fused block goes to position posc: nothing after it may touch a or b
    const bool okPos = posc >= 0 && last[a] <= posc && last[bq] <= posc;
    Block nbk;
    nbk.k = 2;
    nbk.q[0] = a;
    nbk.q[1] = bq;
    if (okA && okB && okPos) {
      // the fused block sits at the later of the two one-qubit blocks; moving the
      // earlier one there is valid because it is the last block on its qubit
      M4 pre;
      for (auto& x : pre) x = {0.0, 0.0};
      for (int j = 0; j < 4; ++j) pre[j * 5] = {1.0, 0.0};
      if (Ba >= 0) {
        const cplx64 ua[4] = {blocks[Ba].m[0], blocks[Ba].m[1], blocks[Ba].m[4], blocks[Ba].m[5]};
        pre = mul4(lift1(ua, 0), pre);
      }
      if (Bb >= 0) {
        const cplx64 ub[4] = {blocks[Bb].m[0], blocks[Bb].m[1], blocks[Bb].m[4], blocks[Bb].m[5]};
        pre = mul4(lift1(ub, 1), pre);
      }
      nbk.m = mul4(Um, pre);
      nbk.changed = true;
      const int pos = std::max(Ba, Bb);
      const int other = std::min(Ba, Bb);
      if (other >= 0 && other != pos) blocks[other].dead = true;
      blocks[pos] = nbk;
      open[a] = open[bq] = last[a] = last[bq] = pos;
      continue;
    }
    nbk.m = Um;
    nbk.src = (int)i;
    open[a] = open[bq] = last[a] = last[bq] = (int)blocks.size();
    blocks.push_back(nbk);
  }
  std::vector<SchedOp> out;
  out.reserve(blocks.size());
  for (const Block& b : blocks) {
    if (b.dead) continue;
    if (b.src >= 0 && !b.changed) {
      out.push_back(ops[b.src]);
      continue;
    }
    SchedOp o{};
    o.k = (uint8_t)b.k;
    const int d = 1 << b.k;
    o.dense = (uint32_t)pool.size();
    double flat[32];
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) {
        const cplx64 v = b.m[r * 4 + c];
        pool.push_back(v);
        flat[2 * (r * d + c)] = v.re;
        flat[2 * (r * d + c) + 1] = v.im;
      }
    for (int j = 0; j < b.k; ++j) o.q[j] = (uint8_t)b.q[j];
    o.mat = o.dense;
    double ph[8];
    uint8_t perm = 0, unit = 0;
    if (classify_monomial(flat, b.k, &perm, ph, &unit)) {
      o.mono = 1;
      o.perm = perm;
      o.unit = unit;
      o.mat = (uint32_t)pool.size();
      for (int j = 0; j < d; ++j) pool.push_back({ph[2 * j], ph[2 * j + 1]});
    } else if (b.k == 2) {
      o.xpat = (uint8_t)classify_xpattern(flat);
    }
    out.push_back(o);
  }
  return out;
}

void normalize_one_qubit_ops(std::vector<SchedOp>& ops, std::vector<cplx64>& pool) {
  std::vector<int> dense1;
  for (size_t i = 0; i < ops.size(); ++i)
    if (ops[i].k == 1 && !ops[i].mono && !ops[i].grad && !ops[i].rot) dense1.push_back((int)i);
  for (size_t s0 = 0; s0 < dense1.size(); s0 += kNormSegment) {
    const size_t s1 = std::min(dense1.size(), s0 + kNormSegment);
    if (s1 - s0 < 2) break;
    cplx64 scale{1.0, 0.0};
    for (size_t j = s0; j + 1 < s1; ++j) {
      SchedOp& o = ops[dense1[j]];
      const cplx64* U = pool.data() + o.dense;
      const int col = (std::hypot(U[1].re, U[1].im) > std::hypot(U[0].re, U[0].im)) ? 1 : 0;
      const cplx64 s = U[col];
      const double n2 = s.re * s.re + s.im * s.im;
      const cplx64 inv{s.re / n2, -s.im / n2};
      const uint32_t at = (uint32_t)pool.size();
      for (int e = 0; e < 4; ++e) pool.push_back(e == col ? cplx64{1.0, 0.0} : cm(pool[o.dense + e], inv));
      o.dense = o.mat = at;
      o.norm = (uint8_t)(col + 1);
      o.realm = 0;
      scale = cm(scale, s);
    }
    SchedOp& c = ops[dense1[s1 - 1]];   // the run's carrier takes the product of the divisors
    const uint32_t at = (uint32_t)pool.size();
    for (int e = 0; e < 4; ++e) pool.push_back(cm(pool[c.dense + e], scale));
    c.dense = c.mat = at;
    c.realm = 0;
  }
}

namespace {

inline cplx64 cdiv(cplx64 a, cplx64 b) {
  const double n = b.re * b.re + b.im * b.im;
  return {(a.re * b.re + a.im * b.im) / n, (a.im * b.re - a.re * b.im) / n};
}
inline double cabs2(cplx64 a) { return a.re * a.re + a.im * a.im; }
inline bool is_one(cplx64 a) { return a.re == 1.0 && a.im == 0.0; }

struct Decomposer {
  std::vector<SchedOp>& out;
  std::vector<cplx64>& pool;
  std::vector<cplx64> pa, pb;   // pending output diagonal diag(pa[q], pb[q]) of each qubit
  cplx64 G{1.0, 0.0};           // scalar factored out of the emitted operations

  Decomposer(std::vector<SchedOp>& o, std::vector<cplx64>& p) : out(o), pool(p), pa(64, {1.0, 0.0}), pb(64, {1.0, 0.0}) {}

  uint32_t put(std::initializer_list<cplx64> v) {
    const uint32_t at = (uint32_t)pool.size();
    for (const cplx64& x : v) pool.push_back(x);
    return at;
  }
  // one-qubit diagonal diag(a, b) = a diag(1, b / a): the scalar goes to G
  void emit_phase(int q, cplx64 a, cplx64 b) {
    const cplx64 r = cdiv(b, a);
    G = cm(G, a);
    if (is_one(r)) return;
    SchedOp o{};
    o.k = 1;
    o.q[0] = (uint8_t)q;
    o.mono = 1;
    o.perm = 0;
    o.urows = 1;
    o.mat = put({{1.0, 0.0}, r});
    o.dense = put({{1.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}, r});
    out.push_back(o);
  }
  void flush(int q) {
    if (is_one(pa[q]) && is_one(pb[q])) return;
    emit_phase(q, pa[q], pb[q]);
    pa[q] = pb[q] = {1.0, 0.0};
  }
  void emit_scalar(int q) {
    if (is_one(G)) return;
    SchedOp o{};
    o.k = 1;
    o.q[0] = (uint8_t)q;
    o.mono = 1;
    o.perm = 0;
    o.mat = put({G, G});
    o.dense = put({G, {0.0, 0.0}, {0.0, 0.0}, G});
    out.push_back(o);
    G = {1.0, 0.0};
  }
  void emit_x(int q) {
    SchedOp o{};
    o.k = 1;
    o.q[0] = (uint8_t)q;
    o.mono = 1;
    o.perm = 1;
    o.unit = 1;
    o.urows = 3;
    o.mat = put({{1.0, 0.0}, {1.0, 0.0}});
    o.dense = put({{0.0, 0.0}, {1.0, 0.0}, {1.0, 0.0}, {0.0, 0.0}});
    out.push_back(o);
  }
  // real rotation [[c, -s], [s, c]] (c^2 + s^2 = 1), normalised by max(c, s)
  void emit_rotation(int q, double c, double s) {
    SchedOp o{};
    o.k = 1;
    o.q[0] = (uint8_t)q;
    if (c >= s) {
      const double t = s / c;
      G = cm(G, {c, 0.0});
      o.rot = 1;
      o.dense = put({{1.0, 0.0}, {-t, 0.0}, {t, 0.0}, {1.0, 0.0}});
    } else {
      const double u = c / s;
      G = cm(G, {s, 0.0});
      o.rot = 2;
      o.dense = put({{u, 0.0}, {-1.0, 0.0}, {1.0, 0.0}, {u, 0.0}});
    }
    o.mat = o.dense;
    out.push_back(o);
    // keep the scale of the intermediate state within 2^+-100
    const double g2 = cabs2(G);
    if (g2 < 0x1p-200 || g2 > 0x1p200) emit_scalar(q);
  }
  // dense one-qubit U (row-major) on q, after the pending diagonal of q
  void dense1(const SchedOp& src) {
    const int q = src.q[0];
    const cplx64* U0 = pool.data() + src.dense;
    const cplx64 A = cm(U0[0], pa[q]), B = cm(U0[1], pb[q]), C = cm(U0[2], pa[q]), D = cm(U0[3], pb[q]);
    const double n0 = cabs2(A) + cabs2(C), n1 = cabs2(B) + cabs2(D);
    const cplx64 ip{A.re * B.re + A.im * B.im + C.re * D.re + C.im * D.im,
                    A.re * B.im - A.im * B.re + C.re * D.im - C.im * D.re};   // conj(A) B + conj(C) D
    const bool unitary = std::fabs(n0 - 1.0) < 1e-12 && std::fabs(n1 - 1.0) < 1e-12 && cabs2(ip) < 1e-24;
    const double c0 = std::sqrt(cabs2(A)), s0 = std::sqrt(cabs2(C));
    if (unitary && s0 == 0.0 && cabs2(B) == 0.0) {     // diagonal: joins the pending diagonal
      pa[q] = A;
      pb[q] = D;
      return;
    }
    if (unitary && c0 == 0.0 && cabs2(D) == 0.0) {     // anti-diagonal: X, then diag(B, C)
      emit_x(q);
      pa[q] = B;
      pb[q] = C;
      return;
    }
    if (unitary && c0 > 0.0 && s0 > 0.0) {
      const double r = std::hypot(c0, s0);
      const double c = c0 / r, s = s0 / r;
      const cplx64 d0 = cdiv(A, {c, 0.0}), d1 = cdiv(C, {s, 0.0});
      const cplx64 e1 = cdiv({-B.re, -B.im}, cm(d0, {s, 0.0}));
      const cplx64 Dr = cm(cm(d1, {c, 0.0}), e1);           // the rebuilt entry D
      if (cabs2({Dr.re - D.re, Dr.im - D.im}) < 1e-28) {
        emit_phase(q, {1.0, 0.0}, e1);
        emit_rotation(q, c, s);
        pa[q] = d0;
        pb[q] = d1;
        return;
      }
    }
    // not unitary (or not rebuilt exactly enough): dense, with the pending diagonal in its columns
    SchedOp o = src;
    o.dense = o.mat = put({A, B, C, D});
    o.norm = 0;
    o.rot = 0;
    o.realm = 0;
    pa[q] = pb[q] = {1.0, 0.0};
    out.push_back(o);
  }
  // two-qubit monomial: the pending diagonals pass through the permutation and
  // factor per qubit; the non-factoring part is a phase on the |11> row
  void mono2(const SchedOp& src) {
    const int q0 = src.q[0], q1 = src.q[1];
    cplx64 ph[4];
    for (int r = 0; r < 4; ++r) ph[r] = src.unit ? cplx64{1.0, 0.0} : pool[src.mat + r];
    cplx64 Dp[4];
    for (int r = 0; r < 4; ++r) {
      const int col = (src.perm >> (2 * r)) & 3;
      const cplx64 dl = cm((col & 1) ? pb[q0] : pa[q0], (col & 2) ? pb[q1] : pa[q1]);
      Dp[r] = cm(ph[r], dl);
    }
    bool unit_modulus = true;
    for (int r = 0; r < 4; ++r) unit_modulus = unit_modulus && std::fabs(cabs2(ph[r]) - 1.0) < 1e-12;
    if (!unit_modulus) {
      // a non-unitary diagonal part (a channel's damping factors): carried on it
      // would make the next gates on these qubits non-unitary, so it keeps its
      // place with the pending diagonals folded into its phases
      SchedOp o = src;
      o.unit = 0;
      o.urows = 0;
      o.mat = put({Dp[0], Dp[1], Dp[2], Dp[3]});
      o.dense = (uint32_t)pool.size();
      for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c)
          pool.push_back(((src.perm >> (2 * r)) & 3) == c ? Dp[r] : cplx64{0.0, 0.0});
      pa[q0] = pa[q1] = pb[q0] = pb[q1] = {1.0, 0.0};
      out.push_back(o);
      return;
    }
    const cplx64 s0 = Dp[0];
    const cplx64 x1 = cdiv(Dp[1], s0), y1 = cdiv(Dp[2], s0);
    const cplx64 gamma = cdiv(Dp[3], cm(s0, cm(x1, y1)));
    G = cm(G, s0);
    pa[q0] = pa[q1] = {1.0, 0.0};
    pb[q0] = x1;
    pb[q1] = y1;
    SchedOp o = src;
    const bool unit = is_one(gamma);
    o.unit = unit ? 1 : 0;
    o.urows = unit ? 15 : 7;
    o.mat = put({{1.0, 0.0}, {1.0, 0.0}, {1.0, 0.0}, gamma});
    o.dense = (uint32_t)pool.size();
    for (int r = 0; r < 4; ++r)
      for (int c = 0; c < 4; ++c) {
        const bool hit = ((src.perm >> (2 * r)) & 3) == c;
        pool.push_back(hit ? (r == 3 ? gamma : cplx64{1.0, 0.0}) : cplx64{0.0, 0.0});
      }
    out.push_back(o);
  }
  // dense k-qubit operation: the pending diagonals scale its columns
  void dense_k(const SchedOp& src) {
    const int d = 1 << src.k;
    SchedOp o = src;
    o.dense = o.mat = (uint32_t)pool.size();
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) {
        cplx64 f{1.0, 0.0};
        for (int j = 0; j < src.k; ++j) f = cm(f, ((c >> j) & 1) ? pb[src.q[j]] : pa[src.q[j]]);
        pool.push_back(cm(pool[src.dense + r * d + c], f));
      }
    for (int j = 0; j < src.k; ++j) pa[src.q[j]] = pb[src.q[j]] = {1.0, 0.0};
    if (src.xpat)   // the diagonal scales columns: same shape, entries maybe complex now
      o.xpat = (uint8_t)classify_xpattern(reinterpret_cast<const double*>(pool.data() + o.dense));
    out.push_back(o);
  }
};

}  // namespace

void decompose_one_qubit_ops(std::vector<SchedOp>& ops, std::vector<cplx64>& pool) {
  std::vector<SchedOp> out;
  out.reserve(ops.size() * 2);
  Decomposer dc(out, pool);
  int last_q = 0;
  for (const SchedOp& o : ops) {
    if (o.grad) {
      for (int j = 0; j < o.k; ++j) dc.flush(o.q[j]);
      out.push_back(o);
    } else if (o.k == 1 && !o.mono) {
      dc.dense1(o);
    } else if (o.k == 1) {             // one-qubit monomial: diagonal, or X with phases
      const int q = o.q[0];
      const cplx64 p0 = o.unit ? cplx64{1.0, 0.0} : pool[o.mat], p1 = o.unit ? cplx64{1.0, 0.0} : pool[o.mat + 1];
      if (o.perm & 1) {
        dc.emit_x(q);
        const cplx64 a = cm(p0, dc.pb[q]), b = cm(p1, dc.pa[q]);
        dc.pa[q] = a;
        dc.pb[q] = b;
      } else {
        dc.pa[q] = cm(dc.pa[q], p0);
        dc.pb[q] = cm(dc.pb[q], p1);
      }
    } else if (o.k == 2 && o.mono) {
      dc.mono2(o);
    } else {
      dc.dense_k(o);
    }
    last_q = o.q[0];
  }
  for (int q = 0; q < 64; ++q) dc.flush(q);
  dc.emit_scalar(last_q);
  ops.swap(out);
}

// ------------------------------------------------------------ adjoint builder
namespace {

using cdd = std::complex<double>;

void push_op(std::vector<SchedOp>& out, std::vector<cplx64>& pool, int k, const int* q, const cdd* m) {
  SchedOp o{};
  o.k = (uint8_t)k;
  for (int i = 0; i < k; ++i) o.q[i] = (uint8_t)q[i];
  const int d = 1 << k;
  o.dense = o.mat = (uint32_t)pool.size();
  double flat[32];
  for (int i = 0; i < d * d; ++i) {
    pool.push_back({m[i].real(), m[i].imag()});
    flat[2 * i] = m[i].real();
    flat[2 * i + 1] = m[i].imag();
  }
  double ph[8];
  uint8_t perm = 0, unit = 0;
  if (classify_monomial(flat, k, &perm, ph, &unit)) {
    o.mono = 1;
    o.perm = perm;
    o.unit = unit;
    o.mat = (uint32_t)pool.size();
    for (int i = 0; i < d; ++i) {
      pool.push_back({ph[2 * i], ph[2 * i + 1]});
      if (ph[2 * i] == 1.0 && ph[2 * i + 1] == 0.0) o.urows |= (uint8_t)(1u << i);   // its product is skipped
    }
  } else if (k == 1) {
    bool real = true;
    for (int i = 0; i < 4; ++i) real = real && flat[2 * i + 1] == 0.0;
    o.realm = real ? 1 : 0;
  }
  out.push_back(o);
}

// exp(-i theta P / 2) for P = X (g 0), Y (1), Z (2)
void rotation(int g, double th, cdd* m) {
  const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
  const cdd I(0.0, 1.0);
  if (g == 0) { m[0] = c; m[1] = -I * s; m[2] = -I * s; m[3] = c; }
  else if (g == 1) { m[0] = c; m[1] = -s; m[2] = s; m[3] = c; }
  else { m[0] = std::exp(-I * (th / 2.0)); m[1] = 0.0; m[2] = 0.0; m[3] = std::exp(I * (th / 2.0)); }
}

void dagger2(const cdd* m, cdd* o) {
  o[0] = std::conj(m[0]); o[1] = std::conj(m[2]); o[2] = std::conj(m[1]); o[3] = std::conj(m[3]);
}

// the rotations a parametrised gate is made of, in forward order: (generator, parameter)
int rotations_of(const AnsatzOp& op, int gen[3], int par[3]) {
  switch (op.kind) {
    case GATE_RX: gen[0] = 0; par[0] = op.param; return 1;
    case GATE_RY: gen[0] = 1; par[0] = op.param; return 1;
    case GATE_RZ: case GATE_P: gen[0] = 2; par[0] = op.param; return 1;
    // U3(theta, phi, lambda) = e^{i (phi + lambda) / 2} Rz(phi) Ry(theta) Rz(lambda)
    case GATE_U3: gen[0] = 2; par[0] = op.param + 2; gen[1] = 1; par[1] = op.param; gen[2] = 2; par[2] = op.param + 1;
      return 3;
    default: return 0;
  }
}

void fixed_matrix(const AnsatzOp& op, int& k, int q[2], cdd* m) {
  const double r = 1.0 / std::sqrt(2.0);
  const cdd I(0.0, 1.0);
  for (int i = 0; i < 16; ++i) m[i] = 0.0;
  switch (op.kind) {
    case GATE_H: k = 1; q[0] = op.q0; m[0] = r; m[1] = r; m[2] = r; m[3] = -r; return;
    case GATE_X: k = 1; q[0] = op.q0; m[1] = 1.0; m[2] = 1.0; return;
    case GATE_SX: k = 1; q[0] = op.q0; m[0] = 0.5 * (1.0 + I); m[1] = 0.5 * (1.0 - I); m[2] = 0.5 * (1.0 - I);
      m[3] = 0.5 * (1.0 + I); return;
    case GATE_CZ: k = 2; q[0] = op.q1; q[1] = op.q0; m[0] = 1.0; m[5] = 1.0; m[10] = 1.0; m[15] = -1.0; return;
    case GATE_CX:   // local bit 1 = control q0, bit 0 = target q1
      k = 2; q[0] = op.q1; q[1] = op.q0; m[0] = 1.0; m[5] = 1.0; m[11] = 1.0; m[14] = 1.0; return;
    default: k = 0; return;
  }
}

}  // namespace

int ansatz_check(int n, const std::vector<AnsatzOp>& ops, std::string& err) {
  int np = 0;
  for (const AnsatzOp& o : ops) {
    if (o.kind < GATE_RX || o.kind > GATE_SX) { err = "unknown gate kind"; return -1; }
    if (o.q0 < 0 || o.q0 >= n) { err = "qubit out of range"; return -1; }
    if (o.kind == GATE_CZ || o.kind == GATE_CX) {
      if (o.q1 < 0 || o.q1 >= n || o.q1 == o.q0) { err = "invalid second qubit"; return -1; }
    }
    if (o.kind <= GATE_P) {
      if (o.param < 0) { err = "parametrised gate without a parameter index"; return -1; }
      np = std::max(np, o.param + (o.kind == GATE_U3 ? 3 : 1));
    }
  }
  return np;
}

void ansatz_forward(int n, const std::vector<AnsatzOp>& ops, const double* params, std::vector<SchedOp>& out,
                    std::vector<cplx64>& pool, bool phase_free) {
  (void)n;
  for (const AnsatzOp& o : ops) {
    int gen[3], par[3];
    const int nr = rotations_of(o, gen, par);
    if (nr) {
      for (int r = 0; r < nr; ++r) {
        cdd m[4];
        rotation(gen[r], params[par[r]], m);
        if (phase_free && gen[r] == 2) {   // e^{-i th/2} diag(1, e^{i th}): the common phase dropped
          const double th = params[par[r]];
          m[0] = 1.0;
          m[3] = cdd(std::cos(th), std::sin(th));
        }
        const int q[1] = {o.q0};
        push_op(out, pool, 1, q, m);
      }
      continue;
    }
    int k, q[2];
    cdd m[16];
    fixed_matrix(o, k, q, m);
    push_op(out, pool, k, q, m);
  }
}

void ansatz_backward(int n, const std::vector<AnsatzOp>& ops, const double* params, std::vector<SchedOp>& out,
                     std::vector<cplx64>& pool, std::vector<int>& grad_param, int select_bit, bool scaled,
                     std::vector<double>* grad_scale) {
  if (select_bit < 0) select_bit = n;
  auto bit = [&](int q) { return q + (q >= select_bit ? 1 : 0); };   // index bit of qubit q in the joint array
  double sigma = 1.0;   // stored amplitudes = true amplitudes / sigma
  for (size_t i = ops.size(); i-- > 0;) {
    const AnsatzOp& o = ops[i];
    int gen[3], par[3];
    const int nr = rotations_of(o, gen, par);
    if (nr) {
      for (int r = nr - 1; r >= 0; --r) {   // last rotation of the gate first
        const double th = params[par[r]];
        cdd md[4];
        uint8_t form = GRAD_PLAIN;
        double kappa = 1.0;
        if (gen[r] == 2) {
          // exp(+i th Z / 2) divided by its row-0 phase: diag(1, e^{-i th})
          form = GRAD_PHASE;
          md[0] = 1.0; md[1] = 0.0; md[2] = 0.0; md[3] = cdd(std::cos(th), -std::sin(th));
        } else if (scaled) {
          const double c = std::cos(th / 2.0), s = std::sin(th / 2.0);
          const cdd j = gen[r] == 0 ? cdd(0.0, 1.0) : cdd(1.0, 0.0);   // X: i s off the diagonal; Y: +s, -s
          const cdd jl = gen[r] == 0 ? cdd(0.0, 1.0) : cdd(-1.0, 0.0);
          if (std::fabs(c) >= std::fabs(s)) {
            form = GRAD_TAN;
            kappa = c;
            const double t = s / c;
            md[0] = 1.0; md[1] = j * t; md[2] = jl * t; md[3] = 1.0;
          } else {
            form = GRAD_COT;
            kappa = s;
            const double u = c / s;
            md[0] = u; md[1] = j; md[2] = jl; md[3] = u;
          }
        } else {
          cdd m[4];
          rotation(gen[r], th, m);
          dagger2(m, md);
        }
        SchedOp g{};
        g.k = 2;
        g.q[0] = (uint8_t)select_bit;     // psi / lambda select bit
        g.q[1] = (uint8_t)bit(o.q0);
        g.grad = 1;
        g.gen = (uint8_t)gen[r];
        g.rot = form;
        g.gidx = (uint32_t)grad_param.size();
        g.dense = g.mat = (uint32_t)pool.size();
        for (int j = 0; j < 4; ++j) pool.push_back({md[j].real(), md[j].imag()});
        g.smul = kappa;
        out.push_back(g);
        grad_param.push_back(par[r]);
        if (grad_scale) grad_scale->push_back(sigma * sigma);
        sigma *= kappa;
        if (std::fabs(sigma) < 0x1p-64 || std::fabs(sigma) > 0x1p64) {
          // back to the true scale: every amplitude of both halves times sigma
          const cdd sc[4] = {sigma, 0.0, 0.0, sigma};
          const int q[1] = {bit(o.q0)};
          push_op(out, pool, 1, q, sc);
          out.back().smul = 1.0 / sigma;
          sigma = 1.0;
        }
      }
      continue;
    }
    int k, q[2];
    cdd m[16], md[16];
    fixed_matrix(o, k, q, m);
    const int d = 1 << k;
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) md[r * d + c] = std::conj(m[c * d + r]);
    int qj[2] = {bit(q[0]), k > 1 ? bit(q[1]) : 0};
    push_op(out, pool, k, qj, md);
  }
}

void adjoint_ops(int n, const std::vector<AnsatzOp>& ops, const double* params, bool backward, bool fuse,
                 bool single_set, AdjointOps& j) {
  j.fw.clear(); j.bw.clear(); j.fpool.clear(); j.bpool.clear(); j.grad_param.clear(); j.grad_scale.clear();
  std::vector<SchedOp> raw;
  // a global phase of psi changes neither the energy nor any Im<lambda|P|psi>
  ansatz_forward(n, ops, params, raw, j.fpool, /*phase_free=*/!single_set);
  if (single_set) {
    j.fw = fuse_two_qubit_blocks(raw, j.fpool, true);
    decompose_one_qubit_ops(j.fw, j.fpool);
    normalize_one_qubit_ops(j.fw, j.fpool);
  } else {
    // forms that do not depend on the angles, every gate alone: RY (and any
    // real gate) a real 2x2 (4 FMAs per amplitude), RZ diag(1, e^{i th}) (2),
    // CZ / CX renamings -- cheaper than fused 4x4 blocks (16); `fuse` = false
    // keeps the plain matrices
    j.fw = raw;
    if (!fuse) {
      raw.clear();
      j.fpool.clear();
      ansatz_forward(n, ops, params, raw, j.fpool, false);
      for (SchedOp& o : raw) o.realm = 0;
      j.fw = raw;
    }
  }
  if (!backward) return;
  raw.clear();
  ansatz_backward(n, ops, params, raw, j.bpool, j.grad_param, n, single_set, &j.grad_scale);   // [psi | lambda]
  j.bw = fuse ? fuse_two_qubit_blocks(raw, j.bpool, single_set) : raw;
}

void exec_grad_scales(const std::vector<PassPlan>* plans, const std::vector<SchedOp>& ops, std::vector<double>& scale) {
  uint32_t nterms = 0;
  for (const SchedOp& o : ops)
    if (o.grad) nterms = std::max(nterms, o.gidx + 1);
  scale.assign(nterms, 1.0);
  double sigma = 1.0;
  auto visit = [&](const SchedOp& o) {
    if (o.grad) scale[o.gidx] = sigma * sigma;
    if (o.smul != 0.0) sigma *= o.smul;
  };
  if (!plans) {
    for (const SchedOp& o : ops) visit(o);
    return;
  }
  for (const PassPlan& pl : *plans)
    for (uint32_t i : pl.src) visit(ops[i]);
}

void pack_pass_matrices(std::vector<PassPlan>& plans, const cplx64* pool, std::vector<cplx64>& packed) {
  packed.clear();
  for (auto& pl : plans) {
    PassDesc& d = pl.desc;
    const uint32_t base = (uint32_t)packed.size();
    for (uint32_t i = 0; i < d.nops; ++i) {
      OpDesc& od = d.ops[i];
      const bool mono = od.kind == OP_M1R || od.kind == OP_M1L || od.kind == OP_M2R;
      const uint32_t n = od.kind == OP_GRAD2 ? 4u : (mono ? (1u << od.k) : (1u << (2 * od.k)));
      const uint32_t rel = (uint32_t)packed.size() - base;
      packed.insert(packed.end(), pool + od.mat, pool + od.mat + n);
      od.mat = rel;
    }
    d.mat_base = base;
    d.mat_elems = (uint32_t)packed.size() - base;
  }
}

}  // namespace iqb
