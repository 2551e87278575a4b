// iq_jit.cpp -- generator, NVRTC compilation and launch of per-pass tile
// kernels (see iq_jit.h).
#include "iq_jit.h"

#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <thread>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <set>

namespace iqb {

namespace {

// the headers the generated source includes, embedded at build time
#include "iq_jit_headers.inc"

constexpr int kMaxBufJit = 4;
// Kernels kept per process.  Modules stay loaded for the process's life (a
// launch may still use one), so past this many distinct pass structures new
// passes run on the interpreting kernel.
constexpr size_t kMaxKernels = 8192;

// ------------------------------------------------------------- NVRTC / driver

typedef int nvrtcResult_t;
typedef struct _nvrtcProgram* nvrtcProgram_t;
struct Nvrtc {
  nvrtcResult_t (*create)(nvrtcProgram_t*, const char*, const char*, int, const char* const*, const char* const*);
  nvrtcResult_t (*compile)(nvrtcProgram_t, int, const char* const*);
  nvrtcResult_t (*log_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*log)(nvrtcProgram_t, char*);
  nvrtcResult_t (*cubin_size)(nvrtcProgram_t, size_t*);
  nvrtcResult_t (*cubin)(nvrtcProgram_t, char*);
  nvrtcResult_t (*destroy)(nvrtcProgram_t*);
  nvrtcResult_t (*version)(int*, int*);
  bool ok = false;
  std::string why;
};

const Nvrtc& nvrtc() {
  static Nvrtc n;
  static std::once_flag once;
  std::call_once(once, [] {
    // One NVRTC per process: reuse a copy already loaded (torch preloads its
    // own with global symbol binding); a second copy loaded beside it would
    // have its internal calls bound to the first one's exported functions.
    void* h = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_NOLOAD);
    for (const char* name : {"libnvrtc.so.12", "/usr/local/cuda/lib64/libnvrtc.so.12"}) {
      if (h) break;
      h = dlopen(name, RTLD_NOW | RTLD_LOCAL | RTLD_DEEPBIND);
    }
    if (!h) { n.why = "libnvrtc.so.12 not found"; return; }
    auto get = [&](const char* s) { return dlsym(h, s); };
    n.create = reinterpret_cast<decltype(n.create)>(get("nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(get("nvrtcCompileProgram"));
    n.log_size = reinterpret_cast<decltype(n.log_size)>(get("nvrtcGetProgramLogSize"));
    n.log = reinterpret_cast<decltype(n.log)>(get("nvrtcGetProgramLog"));
    n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(get("nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(get("nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(get("nvrtcDestroyProgram"));
    n.version = reinterpret_cast<decltype(n.version)>(get("nvrtcVersion"));
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy && n.version;
    if (!n.ok) n.why = "libnvrtc lacks an entry point";
  });
  return n;
}

struct Driver {
  CUresult (*load)(CUmodule*, const void*);
  CUresult (*getfn)(CUfunction*, CUmodule, const char*);
  CUresult (*launch)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, CUstream,
                     void**, void**);
  CUresult (*setattr)(CUfunction, CUfunction_attribute, int);
  bool ok = false;
};

const Driver& driver() {
  static Driver d;
  static std::once_flag once;
  std::call_once(once, [] {
    auto get = [](const char* s) -> void* {
      void* p = nullptr;
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPoint(s, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return nullptr;
      return p;
    };
    d.load = reinterpret_cast<decltype(d.load)>(get("cuModuleLoadData"));
    d.getfn = reinterpret_cast<decltype(d.getfn)>(get("cuModuleGetFunction"));
    d.launch = reinterpret_cast<decltype(d.launch)>(get("cuLaunchKernel"));
    d.setattr = reinterpret_cast<decltype(d.setattr)>(get("cuFuncSetAttribute"));
    d.ok = d.load && d.getfn && d.launch && d.setattr;
  });
  return d;
}

uint64_t fnv1a(const std::string& s) {
  uint64_t h = 1469598103934665603ull;
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

bool compile_cubin(const std::string& src, std::string& cubin, std::string& err) {
  const Nvrtc& nv = nvrtc();
  nvrtcProgram_t prog = nullptr;
  const int nh = (int)(sizeof(kJitHeaderNames) / sizeof(kJitHeaderNames[0]));
  if (nv.create(&prog, src.c_str(), "iq_jit_pass.cu", nh, kJitHeaderSources, kJitHeaderNames) != 0) {
    err = "nvrtcCreateProgram failed";
    return false;
  }
  const char* opts[] = {"-arch=sm_100a", "-std=c++17", "-lineinfo", "-default-device"};
  const int r = nv.compile(prog, 4, opts);
  if (r != 0) {
    size_t n = 0;
    nv.log_size(prog, &n);
    std::string log(n, '\0');
    if (n) nv.log(prog, &log[0]);
    err = "NVRTC compile failed: " + log.substr(0, 1500);
    nv.destroy(&prog);
    return false;
  }
  size_t n = 0;
  nv.cubin_size(prog, &n);
  cubin.assign(n, '\0');
  nv.cubin(prog, &cubin[0]);
  nv.destroy(&prog);
  return true;
}

std::string cache_dir() {
  const char* e = getenv("IQ_JIT_CACHE");
  if (e && !strcmp(e, "off")) return "";
  if (e && *e) return e;
  const char* home = getenv("HOME");
  if (!home || !*home) return "";
  return std::string(home) + "/.cache/invariantq_b200/jit";
}

void mkdirs(const std::string& path) {
  std::string cur;
  std::stringstream ss(path);
  std::string part;
  if (!path.empty() && path[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    mkdir(cur.c_str(), 0755);
  }
}

bool read_file(const std::string& p, std::string& out) {
  std::ifstream f(p, std::ios::binary);
  if (!f) return false;
  std::ostringstream ss;
  ss << f.rdbuf();
  out = ss.str();
  return !out.empty();
}

void write_file_atomic(const std::string& p, const std::string& data) {
  const std::string tmp = p + "." + std::to_string(getpid()) + ".tmp";
  {
    std::ofstream f(tmp, std::ios::binary);
    if (!f) return;
    f.write(data.data(), (std::streamsize)data.size());
    if (!f) return;
  }
  rename(tmp.c_str(), p.c_str());
}

std::atomic<uint64_t> g_compiled{0}, g_disk{0};

}  // namespace

struct JitKernel {
  CUmodule mod = nullptr;
  CUfunction fn = nullptr;
  int nt = 128;
  bool sets = false;     // shared-memory matrices per parameter set (interpreting kernel's arguments)
  bool narrow = false;   // complex64 array, direct global loads and stores (jit_launch_narrow)
  std::atomic<int> smem_limit_set{0};
};

namespace {

// Compiled kernels by (device, source), the sources queued for background
// compilation, and the worker threads that compile them.  Never destroyed: at
// exit an atexit handler empties the queue and waits (bounded) for the
// compilations in progress; idle workers stay parked on the condition
// variable, which outlives them.
struct JitState {
  std::mutex mu;
  std::condition_variable cv, idle;
  // keyed by (device, jit_pass_key); queued tasks carry the source to compile
  std::map<std::pair<int, std::string>, std::unique_ptr<JitKernel>> cache;
  std::set<std::pair<int, std::string>> pending;
  struct Task { int dev; std::string key, src; };
  std::deque<Task> queue;
  std::vector<std::thread> workers;
  int busy = 0;
  bool stop = false;
  std::string last_error;
};

JitState& state() {
  static JitState* s = new JitState;
  return *s;
}

void drain_at_exit() {
  JitState& S = state();
  std::unique_lock<std::mutex> lk(S.mu);
  S.stop = true;
  for (auto& t : S.queue) S.pending.erase({t.dev, t.key});
  S.queue.clear();
  S.idle.wait_for(lk, std::chrono::seconds(60), [&] { return S.busy == 0; });
}

// cache file of a source: keyed by the NVRTC version, the headers the source
// includes (a change to the tile pipeline or the pass descriptor must not pick
// up a cubin built from the old text) and the source itself
std::string cubin_path(const std::string& dir, const std::string& src) {
  int maj = 0, min = 0;
  nvrtc().version(&maj, &min);
  char name[96];
  std::string tag = "nvrtc" + std::to_string(maj) + "." + std::to_string(min);
  for (const char* h : kJitHeaderSources) tag += h;
  snprintf(name, sizeof(name), "/%016llx.cubin", (unsigned long long)fnv1a(tag + src));
  return dir + name;
}

// cubin of `src`: from the cache directory, else compiled (and stored there)
bool get_cubin(const std::string& src, std::string& cubin, std::string& err) {
  const std::string dir = cache_dir();
  const std::string path = dir.empty() ? "" : cubin_path(dir, src);
  if (!path.empty() && read_file(path, cubin)) {
    g_disk.fetch_add(1);
    return true;
  }
  if (!compile_cubin(src, cubin, err)) return false;
  g_compiled.fetch_add(1);
  if (!path.empty()) {
    mkdirs(dir);
    write_file_atomic(path, cubin);
  }
  return true;
}

// CTA size written in the generated source's first line
int source_NT(const std::string& src) {
  const size_t p = src.find("NT=");
  return p == std::string::npos ? 128 : atoi(src.c_str() + p + 3);
}

// load a cubin into the current context's cache entry (caller holds no lock)
bool install(int dev, const std::string& key, const std::string& src, const std::string& cubin, std::string& err) {
  const Driver& dr = driver();
  auto k = std::make_unique<JitKernel>();
  if (dr.load(&k->mod, cubin.data()) != CUDA_SUCCESS) { err = "cuModuleLoadData failed"; return false; }
  if (dr.getfn(&k->fn, k->mod, "iq_jit_pass") != CUDA_SUCCESS) { err = "cuModuleGetFunction failed"; return false; }
  k->nt = source_NT(src);
  k->sets = src.find(" sets=1 ") != std::string::npos;
  k->narrow = src.find(" narrow=1 ") != std::string::npos;
  JitState& S = state();
  std::lock_guard<std::mutex> lk(S.mu);
  S.cache.emplace(std::make_pair(dev, key), std::move(k));   // keeps the first if two raced
  return true;
}

void worker_loop() {
  JitState& S = state();
  for (;;) {
    JitState::Task task;
    {
      std::unique_lock<std::mutex> lk(S.mu);
      // after stop (process exit) the worker stays parked here: returning would
      // run its thread-local teardown while the process is tearing down
      S.cv.wait(lk, [&] { return !S.stop && !S.queue.empty(); });
      task = std::move(S.queue.front());
      S.queue.pop_front();
      ++S.busy;
    }
    std::string cubin, err;
    bool ok = get_cubin(task.src, cubin, err);
    if (ok) {
      bool stopping;
      {
        std::lock_guard<std::mutex> lk(S.mu);
        stopping = S.stop;
      }
      ok = !stopping && cudaSetDevice(task.dev) == cudaSuccess && cudaFree(nullptr) == cudaSuccess &&
           install(task.dev, task.key, task.src, cubin, err);
    }
    {
      std::lock_guard<std::mutex> lk(S.mu);
      if (!ok && !err.empty()) S.last_error = err;
      S.pending.erase({task.dev, task.key});
      --S.busy;
    }
    S.idle.notify_all();
  }
}

bool jit_ready(std::string& err, int& dev) {
  const Nvrtc& nv = nvrtc();
  if (!nv.ok) { err = "NVRTC unavailable: " + nv.why; return false; }
  if (!driver().ok) { err = "driver module entry points unavailable"; return false; }
  if (cudaGetDevice(&dev) != cudaSuccess) { err = "cudaGetDevice failed"; return false; }
  // make the device's primary context current for the driver calls
  if (cudaFree(nullptr) != cudaSuccess) { err = "CUDA context unavailable"; return false; }
  return true;
}

}  // namespace

bool jit_prepare(const std::vector<const PassDesc*>& passes, std::vector<const JitKernel*>& out, std::string& err,
                 int min_blocks, int threads, bool set_mode, bool narrow) {
  out.assign(passes.size(), nullptr);
  int dev = 0;
  if (!jit_ready(err, dev)) return false;
  JitState& S = state();
  std::vector<std::string> keys(passes.size()), srcs(passes.size());
  std::vector<int> todo;                      // first pass of each structure not yet cached
  {
    std::set<std::string> seen;
    std::lock_guard<std::mutex> lk(S.mu);
    for (size_t i = 0; i < passes.size(); ++i) {
      keys[i] = jit_pass_key(*passes[i], min_blocks, threads, set_mode, narrow);
      auto it = S.cache.find({dev, keys[i]});
      if (it != S.cache.end()) { out[i] = it->second.get(); continue; }
      if (S.cache.size() + todo.size() >= kMaxKernels) continue;
      if (!seen.insert(keys[i]).second) continue;
      std::string e;
      srcs[i] = jit_pass_source(*passes[i], e, min_blocks, threads, set_mode, narrow);
      if (!srcs[i].empty()) todo.push_back((int)i);
    }
  }
  if (!todo.empty()) {
    std::vector<std::string> cubins(todo.size()), errs(todo.size());
    const unsigned hw = std::thread::hardware_concurrency();
    const int nthr = (int)std::min<size_t>(todo.size(), std::max(1u, std::min(hw ? hw : 1u, 32u)));
    std::atomic<int> next{0};
    std::vector<std::thread> th;
    for (int t = 0; t < nthr; ++t)
      th.emplace_back([&] {
        for (int w; (w = next.fetch_add(1)) < (int)todo.size();) get_cubin(srcs[todo[w]], cubins[w], errs[w]);
      });
    for (auto& t : th) t.join();
    for (size_t j = 0; j < todo.size(); ++j) {
      if (cubins[j].empty()) { err = errs[j]; return false; }
      if (!install(dev, keys[todo[j]], srcs[todo[j]], cubins[j], err)) return false;
    }
  }
  std::lock_guard<std::mutex> lk(S.mu);
  for (size_t i = 0; i < passes.size(); ++i)
    if (!out[i]) {
      auto it = S.cache.find({dev, keys[i]});
      if (it != S.cache.end()) out[i] = it->second.get();
    }
  return true;
}

void jit_lookup(const std::vector<const PassDesc*>& passes, std::vector<const JitKernel*>& out, bool queue_missing,
                int min_blocks, int threads, bool set_mode) {
  out.assign(passes.size(), nullptr);
  int dev = 0;
  std::string err;
  if (!jit_ready(err, dev)) return;
  JitState& S = state();
  bool queued = false;
  {
    std::lock_guard<std::mutex> lk(S.mu);
    for (size_t i = 0; i < passes.size(); ++i) {
      std::pair<int, std::string> key(dev, jit_pass_key(*passes[i], min_blocks, threads, set_mode));
      auto it = S.cache.find(key);
      if (it != S.cache.end()) { out[i] = it->second.get(); continue; }
      if (!queue_missing || S.pending.count(key) || S.cache.size() + S.pending.size() >= kMaxKernels) continue;
      std::string e;
      std::string src = jit_pass_source(*passes[i], e, min_blocks, threads, set_mode);
      if (src.empty()) continue;
      S.pending.insert(key);
      S.queue.push_back({dev, key.second, std::move(src)});
      queued = true;
    }
    if (queued && S.workers.empty()) {
      // NVRTC sets up (and registers the teardown of) its compiler state on
      // its first compilation.  Compile once here, on this thread, before the
      // exit handler that drains the workers is registered: exit handlers run
      // in reverse order, so the drain then runs before NVRTC's teardown and
      // no compilation is in flight when NVRTC's state goes away.
      std::string cubin, werr;
      compile_cubin("extern \"C\" __global__ void iq_jit_warmup() {}\n", cubin, werr);
      atexit(drain_at_exit);
      const unsigned hw = std::thread::hardware_concurrency();
      const int n = (int)std::max(1u, std::min(hw ? hw / 2 : 1u, 16u));
      for (int t = 0; t < n; ++t) {
        S.workers.emplace_back(worker_loop);
        S.workers.back().detach();
      }
    }
  }
  if (queued) S.cv.notify_all();
}

bool jit_wait(double timeout_s) {
  JitState& S = state();
  std::unique_lock<std::mutex> lk(S.mu);
  return S.idle.wait_for(lk, std::chrono::duration<double>(timeout_s),
                         [&] { return S.queue.empty() && S.busy == 0; });
}

cudaError_t jit_launch(const JitKernel* kc, const CUtensorMap& tm, const PassDesc& d, const double2* host_mats,
                       int* dev_status, const TileLaunch& tl, int num_sms, cudaStream_t st) {
  JitKernel* k = const_cast<JitKernel*>(kc);
  const Driver& dr = driver();
  int nbuf = tl.nbuf < 1 ? 1 : (tl.nbuf > kMaxBufJit ? kMaxBufJit : tl.nbuf);
  const size_t smem = 1024 + (size_t)nbuf * ((size_t)16 << d.M);
  if (!k->smem_limit_set.load(std::memory_order_acquire)) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // the kernel's static shared memory (pipeline barriers) is well under 1 KiB
    if (dr.setattr(k->fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, optin - 1024) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
    k->smem_limit_set.store(1, std::memory_order_release);
  }
  static const double2 zero_mat[1] = {{0.0, 0.0}};
  const double2* mats = d.mat_elems ? host_mats : zero_mat;
  void* args[] = {const_cast<CUtensorMap*>(&tm), const_cast<PassDesc*>(&d), const_cast<double2*>(mats), &dev_status,
                  &nbuf};
  const unsigned grid = tile_pass_grid(d, tl, num_sms);
  const CUresult r = dr.launch(k->fn, grid, 1, 1, (unsigned)k->nt, 1, 1, (unsigned)smem, (CUstream)st, args, nullptr);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

cudaError_t jit_launch_sets(const JitKernel* kc, const CUtensorMap& tm, const PassDesc& d, const double2* dev_mats,
                            int* dev_status, const TileLaunch& tl, int num_sms, cudaStream_t st, double* grad_partials) {
  JitKernel* k = const_cast<JitKernel*>(kc);
  if (!k->sets) return cudaErrorInvalidValue;
  if (d.ngrad && !grad_partials) return cudaErrorInvalidValue;
  const Driver& dr = driver();
  int nbuf = tl.nbuf < 1 ? 1 : (tl.nbuf > kMaxBufJit ? kMaxBufJit : tl.nbuf);
  const size_t smem = 1024 + (size_t)nbuf * ((size_t)16 << d.M) + (size_t)d.mat_elems * 16 +
                      (size_t)d.ngrad * (k->nt / 8) * 8;
  if (!k->smem_limit_set.load(std::memory_order_acquire)) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (dr.setattr(k->fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, optin - 1024) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
    k->smem_limit_set.store(1, std::memory_order_release);
  }
  void* args[] = {const_cast<CUtensorMap*>(&tm), const_cast<PassDesc*>(&d), &dev_mats, &dev_status, &nbuf,
                  &grad_partials};
  const unsigned grid = tile_pass_grid(d, tl, num_sms);
  const CUresult r = dr.launch(k->fn, grid, 1, 1, (unsigned)k->nt, 1, 1, (unsigned)smem, (CUstream)st, args, nullptr);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

cudaError_t jit_launch_narrow(const JitKernel* kc, const PassDesc& d, const double2* dev_mats, void* state,
                              const TileLaunch& tl, int num_sms, cudaStream_t st, double* grad_partials) {
  JitKernel* k = const_cast<JitKernel*>(kc);
  if (!k->narrow) return cudaErrorInvalidValue;
  if (d.ngrad && !grad_partials) return cudaErrorInvalidValue;
  const Driver& dr = driver();
  // [float2 tile][matrix block][gradient accumulators] (direct_set_pass)
  const size_t smem = 1024 + ((size_t)8 << d.M) + (size_t)d.mat_elems * 16 + (size_t)d.ngrad * (k->nt / 8) * 8;
  if (!k->smem_limit_set.load(std::memory_order_acquire)) {
    int dev = 0, optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (dr.setattr(k->fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, optin - 1024) != CUDA_SUCCESS)
      return cudaErrorInvalidValue;
    k->smem_limit_set.store(1, std::memory_order_release);
  }
  void* args[] = {const_cast<PassDesc*>(&d), &dev_mats, &state, &grad_partials};
  const unsigned grid = tile_pass_grid(d, tl, num_sms);
  const CUresult r = dr.launch(k->fn, grid, 1, 1, (unsigned)k->nt, 1, 1, (unsigned)smem, (CUstream)st, args, nullptr);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorLaunchFailure;
}

void jit_counters(uint64_t* compiled, uint64_t* loaded_from_disk) {
  if (compiled) *compiled = g_compiled.load();
  if (loaded_from_disk) *loaded_from_disk = g_disk.load();
}

}  // namespace iqb
