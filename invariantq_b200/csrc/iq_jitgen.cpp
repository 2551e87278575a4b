// iq_jitgen.cpp -- source generator of the per-pass tile kernels (compiled
// at run time by iq_jit.cpp).  Pure C++: the CPU tests link it with the
// scheduler and compile its output with NVRTC.
#include <sstream>
#include <string>
#include <vector>

#include "iq_plan.h"

namespace iqb {

namespace {

struct Gen {
  std::ostringstream o;
  int tmp = 0;
  std::string fresh() { return "t" + std::to_string(tmp++); }
};

// matrix entry i of the pass's block: a kernel parameter, or (kernels for
// several parameter sets) the current set's block in shared memory
thread_local bool g_set_mode = false;
std::string mat(uint32_t i) { return (g_set_mode ? "smat[" : "Mt.m[") + std::to_string(i) + "]"; }

// Straight-line code of one stage.  cur[v] names the value register v of the
// thread holds (v's bit i = register slot i).  Every operation is written with
// the interpreting kernel's expression for it (iq_tile.cuh), so the results
// agree bit for bit.
// gmode bit 0: the stage loads its registers from the complex64 array in
// global memory (gst + tile base tb + physical offsets) instead of the tile;
// bit 1: it stores them there; bit 2: the shared-memory tile is complex64
// (float2 `ftile`: values widened to FP64 on load, rounded on store).
bool gen_stage(Gen& g, const PassDesc& d, int s, int NT, std::string& err, int gmode = 0) {
  const StageDesc& sd = d.st[s];
  const int R = d.R, NV = 1 << R;
  const bool gload = gmode & 1, gstore = gmode & 2, use_smem = !(gload && gstore), ftile = gmode & 4;
  std::ostringstream& o = g.o;
  uint32_t sb[kMaxK];
  for (int i = 0; i < R; ++i) sb[i] = swz(1u << sd.S[i]);
  auto voffc = [&](int v) {
    uint32_t x = 0;
    for (int i = 0; i < R; ++i)
      if ((v >> i) & 1) x ^= sb[i];
    return x;
  };
  o << "    {  // stage " << s << "\n";
  o << "      const unsigned lo = ((unsigned)(lane8 & 1) << " << (int)sd.lane[0] << ") | ((unsigned)((lane8 >> 1) & 1) << "
    << (int)sd.lane[1] << ") | ((unsigned)((lane8 >> 2) & 1) << " << (int)sd.lane[2] << ");\n";
  if (gload || gstore)   // physical offsets of the register slots' tile-local bits
    for (int i = 0; i < R; ++i)
      o << "      const unsigned long long q" << i << " = local_to_phys(" << (1u << sd.S[i]) << "u, P);\n";
  auto goff = [&](int v) {
    std::string x = "gb";
    for (int i = 0; i < R; ++i)
      if ((v >> i) & 1) x += " | q" + std::to_string(i);
    return "gst + (" + x + ")";
  };
  o << "      for (int u = octet; u < " << (1 << sd.nt) << "; u += " << NT / 8 << ") {\n";
  o << "        unsigned base = lo";
  for (int i = 0; i < sd.nt; ++i) o << " | ((((unsigned)u >> " << i << ") & 1u) << " << (int)sd.tb[i] << ")";
  o << ";\n";
  if (gload || gstore) o << "        const unsigned long long gb = tb + local_to_phys(base, P);\n";
  o << "        base = swz(base);\n";
  // The swizzle only mixes bits 0..2: swz(base) ^ off = (swz(base) ^ (off & 7))
  // + (off & ~7), because above bit 2 the thread's and the slots' bits are
  // disjoint.  One pointer per distinct (off & 7) then reaches every register's
  // slot with a constant displacement.
  std::string ptr[8];
  for (int v = 0; v < NV && use_smem; ++v) {
    const uint32_t k = voffc(v) & 7u;
    if (!ptr[k].empty()) continue;
    ptr[k] = "p" + std::to_string(k);
    o << "        " << (ftile ? "float2* const " : "double2* const ") << ptr[k] << " = " << (ftile ? "ftile" : "tile")
      << " + (base ^ " << k << "u);\n";
  }
  auto at = [&](int v) { return ptr[voffc(v) & 7u] + "[" + std::to_string(voffc(v) & ~7u) + "]"; };
  auto atp = [&](int v) { return ptr[voffc(v) & 7u] + " + " + std::to_string(voffc(v) & ~7u); };
  std::vector<std::string> cur(NV);
  for (int v = 0; v < NV; ++v) {
    cur[v] = g.fresh();
    o << "        const double2 " << cur[v] << " = "
      << (gload ? "ldn(" + goff(v) + ")" : (ftile ? "ldn(" + atp(v) + ")" : at(v))) << ";\n";
  }
  auto def = [&](const std::string& expr) {
    const std::string n = g.fresh();
    o << "        const double2 " << n << " = " << expr << ";\n";
    return n;
  };
  for (int oi = sd.op0; oi < sd.op1; ++oi) {
    const OpDesc& od = d.ops[oi];
    const uint32_t m = od.mat;
    const bool unit = od.flags & OPF_UNIT_PHASE;
    switch (od.kind) {
      case OP_D1R: {
        const int A = 1 << od.a;
        const bool real = od.flags & OPF_REAL;
        for (int v = 0; v < NV; ++v) {
          if (v & A) continue;
          const std::string x = cur[v], y = cur[v | A];
          if (real) {
            cur[v] = def("rlin(" + mat(m + 0) + ".x, " + x + ", " + mat(m + 1) + ".x, " + y + ")");
            cur[v | A] = def("rlin(" + mat(m + 2) + ".x, " + x + ", " + mat(m + 3) + ".x, " + y + ")");
          } else {
            cur[v] = def("cfma(cmul(" + mat(m + 0) + ", " + x + "), " + mat(m + 1) + ", " + y + ")");
            cur[v | A] = def("cfma(cmul(" + mat(m + 2) + ", " + x + "), " + mat(m + 3) + ", " + y + ")");
          }
        }
        break;
      }
      case OP_N1R: {   // row 0's entry in column perm is exactly 1
        const int A = 1 << od.a;
        for (int v = 0; v < NV; ++v) {
          if (v & A) continue;
          const std::string x = cur[v], y = cur[v | A];
          cur[v] = od.perm ? def("cfma(" + y + ", " + mat(m + 0) + ", " + x + ")")
                           : def("cfma(" + x + ", " + mat(m + 1) + ", " + y + ")");
          cur[v | A] = def("cfma(cmul(" + mat(m + 2) + ", " + x + "), " + mat(m + 3) + ", " + y + ")");
        }
        break;
      }
      case OP_R1R: {   // normalised real rotation
        const int A = 1 << od.a;
        const std::string w = od.perm ? mat(m + 0) + ".x" : mat(m + 2) + ".x";
        const std::string F = od.perm ? "1" : "0";
        for (int v = 0; v < NV; ++v) {
          if (v & A) continue;
          const std::string x = cur[v], y = cur[v | A];
          cur[v] = def("rot_row0<" + F + ">(" + w + ", " + x + ", " + y + ")");
          cur[v | A] = def("rot_row1<" + F + ">(" + w + ", " + x + ", " + y + ")");
        }
        break;
      }
      case OP_R1L: {   // normalised rotation on a lane bit
        const int l = od.a;
        const std::string hi = g.fresh();
        const std::string w = od.perm ? mat(m + 0) + ".x" : mat(m + 2) + ".x";
        o << "        const bool " << hi << " = (lane8 >> " << l << ") & 1;\n";
        for (int v = 0; v < NV; ++v) {
          const std::string p = def("shfl_xor2(" + cur[v] + ", " + std::to_string(1 << l) + ", omask)");
          cur[v] = def("rot_lane<" + std::string(od.perm ? "1" : "0") + ">(" + w + ", " + hi + ", " + cur[v] + ", " + p + ")");
        }
        break;
      }
      case OP_M1R: {
        const int A = 1 << od.a;
        const bool sw = od.perm & 1;
        for (int v = 0; v < NV; ++v) {
          if (v & A) continue;
          std::string x = cur[v], y = cur[v | A];
          if (sw) std::swap(x, y);
          // rows whose phase is exactly 1 skip the product (same value as multiplying by 1)
          if (!unit) {
            if (!(od.urows & 1)) x = def("cmul(" + mat(m + 0) + ", " + x + ")");
            if (!(od.urows & 2)) y = def("cmul(" + mat(m + 1) + ", " + y + ")");
          }
          cur[v] = x;
          cur[v | A] = y;
        }
        break;
      }
      case OP_D1L: {
        const int l = od.a;
        const std::string hi = g.fresh(), cs = g.fresh(), co = g.fresh();
        o << "        const bool " << hi << " = (lane8 >> " << l << ") & 1;\n";
        o << "        const double2 " << cs << " = " << hi << " ? " << mat(m + 3) << " : " << mat(m + 0) << ";\n";
        o << "        const double2 " << co << " = " << hi << " ? " << mat(m + 2) << " : " << mat(m + 1) << ";\n";
        for (int v = 0; v < NV; ++v) {
          const std::string p = def("shfl_xor2(" + cur[v] + ", " + std::to_string(1 << l) + ", omask)");
          cur[v] = (od.flags & OPF_REAL) ? def("rlin(" + cs + ".x, " + cur[v] + ", " + co + ".x, " + p + ")")
                                         : def("cfma(cmul(" + cs + ", " + cur[v] + "), " + co + ", " + p + ")");
        }
        break;
      }
      case OP_M1L: {
        const int l = od.a;
        const bool sw = od.perm & 1;
        std::string ph;
        if (!unit) {
          const std::string hi = g.fresh();
          ph = g.fresh();
          o << "        const bool " << hi << " = (lane8 >> " << l << ") & 1;\n";
          o << "        const double2 " << ph << " = " << hi << " ? " << mat(m + 1) << " : " << mat(m + 0) << ";\n";
        }
        for (int v = 0; v < NV; ++v) {
          std::string x = cur[v];
          if (sw) x = def("shfl_xor2(" + x + ", " + std::to_string(1 << l) + ", omask)");
          if (!unit) x = def("cmul(" + ph + ", " + x + ")");
          cur[v] = x;
        }
        break;
      }
      case OP_D2R: {
        const int A = 1 << od.a, B = 1 << od.b;
        for (int v = 0; v < NV; ++v) {
          if (v & (A | B)) continue;
          const int idx[4] = {v, v | A, v | B, v | A | B};
          const std::string x[4] = {cur[idx[0]], cur[idx[1]], cur[idx[2]], cur[idx[3]]};
          for (int r = 0; r < 4; ++r) {
            std::string e = "cmul(" + mat(m + 4 * r) + ", " + x[0] + ")";
            for (int c = 1; c < 4; ++c) e = "cfma(" + e + ", " + mat(m + 4 * r + c) + ", " + x[c] + ")";
            cur[idx[r]] = def(e);
          }
        }
        break;
      }
      case OP_M2R: {
        const int A = 1 << od.a, B = 1 << od.b;
        for (int v = 0; v < NV; ++v) {
          if (v & (A | B)) continue;
          const int idx[4] = {v, v | A, v | B, v | A | B};
          const std::string x[4] = {cur[idx[0]], cur[idx[1]], cur[idx[2]], cur[idx[3]]};
          for (int r = 0; r < 4; ++r) {
            const std::string y = x[(od.perm >> (2 * r)) & 3];
            cur[idx[r]] = (unit || ((od.urows >> r) & 1)) ? y : def("cmul(" + mat(m + r) + ", " + y + ")");
          }
        }
        break;
      }
      case OP_X2R: {   // channel-shaped 4x4: corners mix x0 / x3, the middle scales x1, x2
        const int A = 1 << od.a, B = 1 << od.b;
        const std::string tmpl = std::string("xpat4<") + ((od.flags & 1) ? "true" : "false") + ", " +
                                 ((od.flags & 2) ? "true" : "false") + ">";
        const std::string mv = g.fresh();
        o << "        const double2 " << mv << "[6] = {" << mat(m + 0) << ", " << mat(m + 3) << ", " << mat(m + 12)
          << ", " << mat(m + 15) << ", " << mat(m + 5) << ", " << mat(m + 10) << "};\n";
        for (int v = 0; v < NV; ++v) {
          if (v & (A | B)) continue;
          const std::string x[4] = {g.fresh(), g.fresh(), g.fresh(), g.fresh()};
          const int idx[4] = {v, v | A, v | B, v | A | B};
          o << "        double2 " << x[0] << " = " << cur[idx[0]] << ", " << x[1] << " = " << cur[idx[1]] << ", "
            << x[2] << " = " << cur[idx[2]] << ", " << x[3] << " = " << cur[idx[3]] << ";\n";
          o << "        " << tmpl << "(" << x[0] << ", " << x[1] << ", " << x[2] << ", " << x[3] << ", " << mv << "[0], "
            << mv << "[1], " << mv << "[2], " << mv << "[3], " << mv << "[4], " << mv << "[5]);\n";
          for (int r = 0; r < 4; ++r) cur[idx[r]] = x[r];
        }
        break;
      }
      case OP_DKR: {
        const int D = 1 << od.k;
        if (od.k > R) { err = "dense block wider than the register slots"; return false; }
        std::vector<std::string> out(NV);
        for (int gb = 0; gb < NV; gb += D)
          for (int r = 0; r < D; ++r) {
            std::string e = "cmul(" + mat(m + r * D) + ", " + cur[gb] + ")";
            for (int c = 1; c < D; ++c) e = "cfma(" + e + ", " + mat(m + r * D + c) + ", " + cur[gb + c] + ")";
            out[gb + r] = def(e);
          }
        cur = out;
        break;
      }
      case OP_GRAD2: {   // adjoint step: select bit in slot 0, qubit in slot b (shared-memory matrices only)
        if (!g_set_mode) { err = "adjoint steps need the shared-memory form"; return false; }
        const int B = 1 << od.b;
        const std::string G = std::to_string((int)od.perm) + ", " + std::to_string((int)od.flags);   // generator, form
        const std::string acc = g.fresh(), u0 = g.fresh(), u1 = g.fresh(), u3 = g.fresh();
        o << "        const double2 " << u0 << " = " << mat(m + 0) << ", " << u1 << " = " << mat(m + 1) << ", " << u3
          << " = " << mat(m + 3) << ";\n";
        o << "        double " << acc << " = 0.0;\n";
        for (int v = 0; v < NV; ++v) {
          if (v & (1 | B)) continue;
          const std::string p0 = cur[v], p1 = cur[v | B], l0 = cur[v | 1], l1 = cur[v | 1 | B];
          o << "        " << acc << " += grad_term<" << (int)od.perm << ">(" << p0 << ", " << p1 << ", " << l0 << ", " << l1 << ");\n";
          const std::string a = g.fresh(), b = g.fresh(), c = g.fresh(), d2 = g.fresh();
          o << "        double2 " << a << ", " << b << ", " << c << ", " << d2 << ";\n";
          o << "        unrotate<" << G << ">(" << p0 << ", " << p1 << ", " << a << ", " << b << ", " << u0 << ", " << u1 << ", "
            << u3 << ");\n";
          o << "        unrotate<" << G << ">(" << l0 << ", " << l1 << ", " << c << ", " << d2 << ", " << u0 << ", " << u1
            << ", " << u3 << ");\n";
          cur[v] = a;
          cur[v | B] = b;
          cur[v | 1] = c;
          cur[v | 1 | B] = d2;
        }
        o << "        grad_accumulate(" << acc << ", gs + " << od.gidx << ", lane8, omask);\n";
        break;
      }
      default:
        err = "operation kind " + std::to_string((int)od.kind) + " is not specialised";
        return false;
    }
  }
  for (int v = 0; v < NV; ++v) {
    if (gstore) o << "        stn(" << goff(v) << ", " << cur[v] << ");\n";
    else if (ftile) o << "        stn(" << atp(v) << ", " << cur[v] << ");\n";
    else o << "        " << at(v) << " = " << cur[v] << ";\n";
  }
  o << "      }\n    }\n    __syncthreads();\n";
  return true;
}

}  // namespace

// Everything of `d` (and of the kernel form) that its generated source depends
// on, as a compact byte string: equal keys give equal sources.
std::string jit_pass_key(const PassDesc& d, int min_blocks, int threads, bool set_mode, bool narrow) {
  std::string k;
  k.reserve(64 + d.nstages * 32 + d.nops * 16);
  auto put = [&](uint32_t v) { k.append(reinterpret_cast<const char*>(&v), sizeof(v)); };
  put(1);   // key format
  put((uint32_t)min_blocks);
  put((uint32_t)threads);
  put(set_mode ? (narrow ? 2u : 1u) : 0u);
  put(d.M);
  put(d.c);
  put(d.R);
  put(d.nstages);
  put(d.mat_elems);
  put(d.ngrad);
  for (int s = 0; s < d.nstages; ++s) {
    const StageDesc& sd = d.st[s];
    k.append(reinterpret_cast<const char*>(sd.S), kMaxK);
    k.append(reinterpret_cast<const char*>(sd.lane), kLaneBits);
    k.push_back((char)sd.nt);
    k.append(reinterpret_cast<const char*>(sd.tb), sd.nt);
    put(sd.op0);
    put(sd.op1);
  }
  for (uint32_t i = 0; i < d.nops; ++i) {
    const OpDesc& o = d.ops[i];
    const char b[7] = {(char)o.kind, (char)o.a, (char)o.b, (char)o.k, (char)o.perm, (char)o.flags, (char)o.urows};
    k.append(b, 7);
    put(o.mat);
    put(o.gidx);
  }
  return k;
}

// Source of the kernel specialised to pass `d` (see iq_plan.h).
std::string jit_pass_source(const PassDesc& d, std::string& err, int min_blocks, int threads, bool set_mode,
                            bool narrow) {
  if (narrow && !set_mode) {
    err = "complex64 passes use the shared-memory form";
    return "";
  }
  if (!set_mode && (d.ngrad || d.nsets > 1)) {
    err = "passes over several parameter sets need the shared-memory form";
    return "";
  }
  g_set_mode = set_mode;
  if (d.R < 3 || d.R > kMaxK) {
    err = "register slots out of range";
    return "";
  }
  const int NT = (threads == 128 || threads == 256) ? threads : tile_pass_threads(d.R);
  const int MINB = d.R == 5 ? 1 : (min_blocks >= 1 && min_blocks <= 4 ? min_blocks : 2);
  const uint32_t nmat = d.mat_elems ? d.mat_elems : 1;
  Gen g;
  std::ostringstream& o = g.o;
  o << "// generated by iq_jitgen (iq-jit-2): NT=" << NT << " sets=" << (set_mode ? 1 : 0)
    << " narrow=" << (narrow ? 1 : 0) << " M=" << (int)d.M
    << " c=" << (int)d.c << " R=" << (int)d.R
    << " stages=" << (int)d.nstages << " ops=" << d.nops << "\n";
  o << "#include \"iq_pipe.cuh\"\nusing namespace iqb;\n";
  if (narrow) {
    o << "struct JitStages {\n  const PassDesc& P;\n  float2* gst;\n  int lane8, octet;\n  unsigned omask;\n";
    o << "  __device__ __forceinline__ void operator()(float2* ftile, const double2* smat, double* gslots, "
         "unsigned long long t) {\n";
    o << "    const unsigned long long tb = tile_base(t, P);\n";
    o << "    double* const gs = gslots + octet * " << d.ngrad << ";\n    (void)gs; (void)ftile;\n";
    for (int s = 0; s < d.nstages; ++s) {
      const int gm = (s == 0 ? 1 : 0) | (s == d.nstages - 1 ? 2 : 0) | 4;
      if (!gen_stage(g, d, s, NT, err, gm)) return "";
    }
    o << "  }\n};\n";
    o << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", " << MINB << ")\n"
      << "iq_jit_pass(const __grid_constant__ PassDesc P, const double2* __restrict__ mats,\n"
      << "            float2* __restrict__ state, double* __restrict__ grad_partials) {\n"
      << "  extern __shared__ __align__(1024) unsigned char smem_raw[];\n"
      << "  const int ctid = threadIdx.x;\n"
      << "  JitStages st{P, state, ctid & 7, ctid >> 3, 0xFFu << (ctid & 24)};\n"
      << "  direct_set_pass<" << NT << ">(P, mats, grad_partials, smem_raw, st);\n}\n";
    return o.str();
  }
  if (set_mode) {
    o << "struct JitStages {\n  int lane8, octet;\n  unsigned omask;\n";
    o << "  __device__ __forceinline__ void operator()(double2* tile, const double2* smat, double* gslots, bool work) {\n";
    o << "    if (!work) return;\n";
    o << "    double* const gs = gslots + octet * " << d.ngrad << ";\n    (void)gs;\n";
    for (int s = 0; s < d.nstages; ++s)
      if (!gen_stage(g, d, s, NT, err)) return "";
    o << "  }\n};\n";
    o << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", " << MINB << ")\n"
      << "iq_jit_pass(const __grid_constant__ CUtensorMap tm, const __grid_constant__ PassDesc P,\n"
      << "            const double2* __restrict__ mats, int* __restrict__ status, int nbuf,\n"
      << "            double* __restrict__ grad_partials) {\n"
      << "  extern __shared__ __align__(1024) unsigned char smem_raw[];\n"
      << "  const int ctid = threadIdx.x;\n"
      << "  JitStages st{ctid & 7, ctid >> 3, 0xFFu << (ctid & 24)};\n"
      << "  set_tile_pass<" << NT << ">(tm, P, mats, status, nbuf, grad_partials, smem_raw, st);\n}\n";
    return o.str();
  }
  o << "struct JitMats { double2 m[" << nmat << "]; };\n";
  o << "struct JitBody {\n  const JitMats& Mt;\n  int lane8, octet;\n  unsigned omask;\n";
  o << "  __device__ __forceinline__ void operator()(double2* tile, unsigned long long, bool work) {\n";
  o << "    if (!work) return;\n";
  for (int s = 0; s < d.nstages; ++s)
    if (!gen_stage(g, d, s, NT, err)) return "";
  o << "  }\n};\n";
  o << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", " << MINB << ")\n"
    << "iq_jit_pass(const __grid_constant__ CUtensorMap tm, const __grid_constant__ PassDesc P,\n"
    << "            const __grid_constant__ JitMats Mt, int* __restrict__ status, int nbuf) {\n"
    << "  extern __shared__ __align__(1024) unsigned char smem_raw[];\n"
    << "  double2* tiles = aligned_tiles(smem_raw);\n"
    << "  const int ctid = threadIdx.x;\n"
    << "  JitBody body{Mt, ctid & 7, ctid >> 3, 0xFFu << (ctid & 24)};\n"
    << "  tile_pipeline<" << NT << ">(tm, P, tiles, status, nbuf, body);\n}\n";
  return o.str();
}

}  // namespace iqb
