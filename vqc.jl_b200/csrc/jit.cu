// Run-time specialised FP32 tile kernels.
//
// The interpreted tile kernel (tile_f32.cuh, interp_ops) decodes every op of
// a pass at run time; on sm_100 that costs about as many integer and move
// instructions as the op's packed FMAs, because each of the many op variants
// leaves the amplitudes in different registers.  A pass's *structure* (its
// stages, and per op the type, target and control bits, matrix form and
// accumulated entries) is known when the circuit is planned, and the same
// structures recur from layer to layer and from call to call.  So the pass
// is written out as straight-line CUDA (every op a compile-time variant of
// the same device functions), compiled with NVRTC for sm_100a once per
// structure, and cached for the life of the process.  Everything that varies
// between calls with the same structure (angles, masks, addresses, slots)
// stays run-time data in the pass's descriptors, exactly as the interpreter
// reads them.
//
// VQC_JIT=0 / off: never (the generic tile kernel runs every pass); 1 / on:
// every FP32 tile pass; auto (default): passes of states with at least 2^18
// amplitudes; interp: the packed plan on its interpreter (testing).  If
// NVRTC cannot be loaded the generic kernel runs; if one compilation fails,
// that pass runs on the packed interpreter (both are GPU kernels).
#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <set>
#include <sstream>
#include <thread>

#include "tile_plan.cuh"

namespace vqc {

namespace {

#include "jit_src.inc"  // kJitTileDev, kJitTileF32: the device headers as text (generated at build time)

struct Nvrtc {
  bool ok = false;
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
};

const Nvrtc& nvrtc() {
  static Nvrtc n = [] {
    Nvrtc r;
    std::vector<std::string> cands = {"libnvrtc.so.12", "libnvrtc.so"};
    for (const char* env : {"CUDA_HOME", "CUDA_PATH"})
      if (const char* h = std::getenv(env)) cands.push_back(std::string(h) + "/lib64/libnvrtc.so.12");
    cands.push_back("/usr/local/cuda/lib64/libnvrtc.so.12");
    void* h = nullptr;
    for (const std::string& c : cands)
      if ((h = dlopen(c.c_str(), RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) return r;
    r.create = (decltype(r.create))dlsym(h, "nvrtcCreateProgram");
    r.compile = (decltype(r.compile))dlsym(h, "nvrtcCompileProgram");
    r.cubin_size = (decltype(r.cubin_size))dlsym(h, "nvrtcGetCUBINSize");
    r.cubin = (decltype(r.cubin))dlsym(h, "nvrtcGetCUBIN");
    r.log_size = (decltype(r.log_size))dlsym(h, "nvrtcGetProgramLogSize");
    r.log = (decltype(r.log))dlsym(h, "nvrtcGetProgramLog");
    r.destroy = (decltype(r.destroy))dlsym(h, "nvrtcDestroyProgram");
    r.ok = r.create && r.compile && r.cubin_size && r.cubin && r.log_size && r.log && r.destroy;
    return r;
  }();
  return n;
}

struct Entry {
  cudaLibrary_t lib = nullptr;
  cudaKernel_t kernel = nullptr;
  bool failed = false;
  std::string log;
};

std::mutex g_mu;
std::map<std::string, Entry>& cache() {
  static std::map<std::string, Entry> c;
  return c;
}

int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  return v && *v ? std::atoi(v) : dflt;
}

// NVRTC -> cubin for one source (thread-safe; no CUDA calls).
bool compile_one(const std::string& src, std::vector<char>& cubin, std::string& log) {
  const Nvrtc& nv = nvrtc();
  nvrtcProgram prog;
  const char* hdrs[2] = {kJitTileDev, kJitTileF32};
  const char* names[2] = {"tile_dev.cuh", "tile_f32.cuh"};
  if (nv.create(&prog, src.c_str(), "vqc_pass.cu", 2, hdrs, names) != NVRTC_SUCCESS) {
    log = "nvrtcCreateProgram failed";
    return false;
  }
  std::vector<const char*> opts = {"-arch=sm_100a", "-std=c++17", "-lineinfo", "--extra-device-vectorization"};
  if (env_int("VQC_JIT_VERBOSE", 0)) opts.push_back("--ptxas-options=-v");
  const nvrtcResult rc = nv.compile(prog, (int)opts.size(), opts.data());
  size_t ls = 0;
  nv.log_size(prog, &ls);
  log.assign(ls, '\0');
  if (ls) nv.log(prog, &log[0]);
  bool ok = rc == NVRTC_SUCCESS;
  if (ok) {
    size_t cs = 0;
    ok = nv.cubin_size(prog, &cs) == NVRTC_SUCCESS && cs > 0;
    if (ok) {
      cubin.resize(cs);
      ok = nv.cubin(prog, cubin.data()) == NVRTC_SUCCESS;
    }
  }
  nv.destroy(&prog);
  return ok;
}

// The code of one op of a stage (o = its index in the pass's op array; cx =
// the expression of the pass's coefficient array).
void emit_op(std::ostringstream& os, const DevOp& op, int o, const char* cx) {
  const int code = op.code, type = code & 15;
  const bool ctl = code & kCodeCtl, gctl = code & kCodeGCtl, acc = code & kCodeAcc;
  os << "    { const DevOp* op = x.ops + " << o << ";\n";
  if (gctl) os << "      if ((x.base & op->gmask) == op->gval) {\n";
  if (type == kOpU1) {
    const int tb = op_r0(code), rctl = (code >> 16) & 7, form = (code >> 11) & 7, kind = acc_kind_of(code);
    const int cb = rctl == 0 ? -1 : rctl - 1;
    os << "      const u64* c = " << cx << " + " << op.mat << ";\n";
    if (ctl) os << "      const bool run = (tthr & op->cmask) == op->cval;\n";
    if (acc) os << "      float s8[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};\n";
    os << "      " << (ctl ? "if (run) " : "") << "{\n";
    if (rctl == 7)
      os << "        u1_masked<" << tb << ", " << form << ", ADJ>(v, w, c, (uint32_t)op->rmask);\n";
    else
      os << "        u1_static<" << tb << ", " << cb << ", " << form << ", ADJ>(v, w, c);\n";
    if (acc) {
      if (rctl == 7)
        os << "        acc_masked<" << tb << ", " << kind << ">(v, w, (uint32_t)op->rmask, s8);\n";
      else
        os << "        acc_static<" << tb << ", " << cb << ", " << kind << ">(v, w, s8);\n";
    }
    os << "      }\n";
    if (acc) os << "      " << ((kind & kAccAH) ? "flush4" : "flush8") << "(s8, x.sacc, op->slot, NW);\n";
  } else if (type == kOpU2) {
    const int ja = op_r0(code), jb = op_r1(code);
    if (ctl) os << "      if ((tthr & op->cmask) == op->cval)\n";
    os << "      u2_op<" << ja << ", " << jb << ", ADJ>(v, w, reinterpret_cast<const float2*>(" << cx << " + " << op.mat
       << "), (uint32_t)op->rmask);\n";
  } else if (type == kOpDiag) {
    os << "      diag_op<ADJ>(v, w, op, reinterpret_cast<const float2*>(" << cx << " + " << op.mat
       << "), tthr, S->dep, x.base);\n";
  } else {
    os << "      float s8[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};\n"
       << "      accd_op(v, w, op, tthr, S->dep, x.base, s8);\n"
       << "      flush8(s8, x.sacc, op->slot, NW);\n";
  }
  if (gctl) os << "      }\n";
  os << "    }\n";
}

}  // namespace

int jit_mode() {
  const char* v = std::getenv("VQC_JIT");
  if (!v || !*v || !std::strcmp(v, "auto")) return 2;
  if (!std::strcmp(v, "0") || !std::strcmp(v, "off")) return 0;
  if (!std::strcmp(v, "interp")) return 3;
  return 1;
}

// The debug build (device-side index checks) runs every pass on the kernels
// compiled into the library, whose checks it can read.
#ifdef VQC_DEBUG_CHECKS
bool jit_available() { return false; }
#else
bool jit_available() { return nvrtc().ok; }
#endif

// Forward passes with the asynchronous tile copy (VQC_JIT_ASYNC=1; off by
// default): a second tile buffer in shared memory receives the next tile by
// cp.async while the current tile is computed.  Measured at n = 26: 0.43 ms
// per forward pass against 0.355 ms for the default (three resident CTAs
// instead of four, and one more barrier per tile, cost more than the copy
// saves; the default already prefetches the next tile into L2).
bool jit_async_fwd() { return env_int("VQC_JIT_ASYNC", 0) != 0; }
size_t jit_extra_smem(bool adj, int M, int rb) {
  return (!adj && rb == kRegBits && jit_async_fwd() && env_int("VQC_JIT_BAKE", 1)) ? (size_t(1) << (M - 1)) * 16 : 0;
}

// Resident CTAs per SM the compiled kernels' registers are budgeted for:
// 1024 threads for forward passes (64 registers), 768 when they hold a second
// tile buffer (85 registers: their shared memory admits three 256-thread CTAs
// anyway), 512 for the reverse sweep (128 registers); the wide forward passes
// (32 amplitudes per thread) 640 (five 128-thread CTAs, 96 registers).
int jit_min_blocks(bool adj, int M, int rb) {
  const int nt = 1 << (M - rb);
  if (adj) return env_int("VQC_JIT_MINB_ADJ", 512 / nt);
  if (rb != kRegBits) return std::max(1, env_int("VQC_JIT_MINB_WIDE", 640 / nt));
  return env_int("VQC_JIT_MINB_FWD", (jit_async_fwd() && env_int("VQC_JIT_BAKE", 1) ? 768 : 1024) / nt);
}

// The next tile's first-stage pairs prefetched into L2 during the current
// tile: measured at 2^26 amplitudes, the reverse sweep gains (1.059 against
// 1.094 ms per pass), the forward pass loses a little (0.354 against 0.350
// ms), so by default only reverse passes prefetch (VQC_JIT_L2PF=0/1 sets both).
static bool jit_l2_prefetch(bool adj) { return env_int("VQC_JIT_L2PF", adj ? 1 : 0) != 0; }

// Tile bits of the warp index in a stage's thread layout (thread bit j is the
// stage's j-th tile bit outside the register set; the warp index is thread
// bits 5 and up).
static uint32_t warp_tile_bits(const DevStageF& st, int thread_bits) {
  uint32_t m = 0;
  for (int j = 5; j < thread_bits; ++j) m |= st.thr[j >> 2][1 << (j & 3)];
  return m;
}

std::string jit_pass_source(int M, bool adj, const DevStageF* st, int nst, const DevOp* ops, int npool, bool batch,
                            int rb) {
  if (!batch && npool > kJitMaxCoef) return std::string();  // beyond the kernel-parameter space: interpreter
  std::ostringstream os;
  const int NT = 1 << (M - rb), NP = 1 << (rb - 1);
  // the wide passes exist only as compiled kernels with their offsets baked in
  const bool bake = rb != kRegBits || env_int("VQC_JIT_BAKE", 1) != 0;
  const bool async = !batch && jit_extra_smem(adj, M, rb) > 0;
  const bool warp_local = env_int("VQC_JIT_WARPSYNC", 1) != 0;
  os << "#include \"tile_f32.cuh\"\n"
     << "using namespace vqc;\nusing namespace vqc::f32t;\n";
  if (!batch) {
    // the pass's matrix pool travels as a kernel parameter (constant bank,
    // read uniformly by the whole grid) instead of through shared memory
    os << "struct Coef { unsigned long long c[" << std::max(npool, 2) << "]; };\n"
       << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", " << jit_min_blocks(adj, M, rb) << ")\n"
       << "vqc_pass(float2* psi, float2* lam, const DevPass* pass, const DevStageF* stages, const DevOp* ops,\n"
       << "         const float2* pool, double* partials, const __grid_constant__ Coef coef) {\n"
       << "  const int ncta = gridDim.x;\n";
  } else {
    // the serving loop: one request per blockIdx.y, each with its own state,
    // descriptors and coefficient pool (staged in shared memory)
    os << "extern \"C\" __global__ void __launch_bounds__(" << NT << ", " << jit_min_blocks(adj, M, rb) << ")\n"
       << "vqc_pass_batch(const TileItem* __restrict__ items) {\n"
       << "  const TileItem item = items[blockIdx.y];\n"
       << "  if ((int)blockIdx.x >= item.ncta) return;\n"
       << "  const int ncta = item.ncta;\n"
       << "  float2* psi = (float2*)item.psi;\n  float2* lam = (float2*)item.lam;\n"
       << "  const DevPass* pass = item.pass;\n  const DevStageF* stages = (const DevStageF*)item.stages;\n"
       << "  const DevOp* ops = item.ops;\n  const float2* pool = (const float2*)item.pool;\n"
       << "  double* partials = item.partials;\n";
  }
  os << "  constexpr int M = " << M << ";\n  constexpr bool ADJ = " << (adj ? "true" : "false") << ";\n"
     << "  constexpr int RB = " << rb << ";\n"
     << "  constexpr int NW = TileCtx<M, ADJ, RB>::NW;\n"
     << "  __shared__ DevPass P;\n  __shared__ uint64_t s_inc, s_base0;\n"
     << "  TileCtx<M, ADJ, RB> x;\n"
     << "  tile_setup<M, ADJ, " << (async ? 2 : 1)
     << ">(x, psi, lam, pass, stages, ops, pool, ncta, P, s_inc, s_base0, " << (batch ? "true" : "false") << ");\n"
     << "  Pk v[" << NP << "], w[" << NP << "];\n";
  if (batch) os << "  const u64* C = reinterpret_cast<const u64*>(x.pool);\n";
  const char* cx = batch ? "C" : "coef.c";
  if (async) {
    // the first stage's pair offsets, for the copies of the next tile
    os << "  constexpr uint32_t swm0[8] = {";
    for (int m = 0; m < 8; ++m) os << (m ? ", " : "") << st[0].swm[m] << "u";
    os << "};\n  constexpr int64_t gdep0[8] = {";
    for (int m = 0; m < 8; ++m) os << (m ? ", " : "") << st[0].gdep[m] << "ll";
    os << "};\n  ulonglong2* tbuf[2] = {x.sp, x.spb};\n"
       << "  if (x.ntiles_here > 0) tile_copy_async<M>(x, x.stages, x.base, tbuf[0], swm0, gdep0);\n";
  }
  os << "  for (int it = 0; it < x.ntiles_here; ++it) {\n";
  if (async)
    os << "    if (it + 1 < x.ntiles_here) {\n"
       << "      tile_copy_async<M>(x, x.stages, tile_base_after(x, s_inc), tbuf[(it + 1) & 1], swm0, gdep0);\n"
       << "      cp_async_wait<1>();\n    } else {\n      cp_async_wait<0>();\n    }\n"
       << "    __syncthreads();\n    x.sp = tbuf[it & 1];\n";
  for (int s = 0; s < nst; ++s) {
    os << "  {\n    const DevStageF* S = x.stages + " << s << ";\n";
    if (async && s == 0) {
      os << "    constexpr uint32_t swm[8] = {";
      for (int m = 0; m < 8; ++m) os << (m ? ", " : "") << st[s].swm[m] << "u";
      os << "};\n    constexpr int64_t gdep[8] = {";
      for (int m = 0; m < 8; ++m) os << (m ? ", " : "") << st[s].gdep[m] << "ll";
      os << "};\n    stage_load_raw<M>(x, S, x.sp, v, swm);\n";
    } else if (bake) {
      // the stage's pair offsets as constants (they depend on the pass's qubits)
      os << "    constexpr uint32_t swm[" << NP << "] = {";
      for (int m = 0; m < NP; ++m) os << (m ? ", " : "") << st[s].swm[m] << "u";
      os << "};\n    constexpr int64_t gdep[" << NP << "] = {";
      for (int m = 0; m < NP; ++m) os << (m ? ", " : "") << st[s].gdep[m] << "ll";
      os << "};\n    stage_load_k<M, ADJ>(x, S, " << (s == 0 ? "true" : "false") << ", v, w, swm, gdep);\n";
    } else {
      os << "    stage_load<M, ADJ>(x, S, " << (s == 0 ? "true" : "false") << ", v, w);\n";
    }
    if (s == 0 && bake && !async && jit_l2_prefetch(adj))
      os << "    if (it + 1 < x.ntiles_here) prefetch_next_l2<M, ADJ>(x, S, s_inc, gdep);\n";
    os << "    const uint32_t tthr = S->thr[0][x.tlo] | S->thr[1][x.thi];\n    (void)tthr;\n";
    for (int o = st[s].op_begin; o < st[s].op_end; ++o) emit_op(os, ops[o], o, cx);
    // the first stage of an asynchronous pass read its input from the buffer it
    // now writes (in the next stage's layout): every read must be done first
    if (async && s == 0 && nst > 1) os << "    __syncthreads();\n";
    // a CTA barrier only where the warp index moves to other tile bits (the
    // last stage: against the next tile's first stage)
    const bool cta = async || !warp_local ||
                     warp_tile_bits(st[s], M - rb) != warp_tile_bits(st[(s + 1) % nst], M - rb);
    if (bake)
      os << "    stage_store_k<M, ADJ>(x, S, " << (s == nst - 1 ? "true" : "false") << ", v, w, swm, gdep, "
         << (cta ? "true" : "false") << ");\n  }\n";
    else
      os << "    stage_store<M, ADJ>(x, S, " << (s == nst - 1 ? "true" : "false") << ", v, w);\n  }\n";
  }
  os << "    tile_next<M, ADJ>(x, s_inc);\n  }\n  tile_finish<M, ADJ>(x, partials);\n  (void)NW;\n}\n";
  return os.str();
}

// Kernels for `srcs` (nullptr where unavailable): cached ones at once, the
// rest compiled in parallel, then loaded.
namespace {
thread_local int t_thread_cap = 0;
}
void jit_set_thread_cap(int n) { t_thread_cap = n < 0 ? 0 : n; }

int jit_kernels(const std::vector<std::string>& srcs, std::vector<const void*>& out, const char* name) {
  out.assign(srcs.size(), nullptr);
  if (!jit_available()) return VQC_OK;
  std::vector<size_t> todo;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    std::map<std::string, size_t> seen;
    for (size_t i = 0; i < srcs.size(); ++i) {
      if (srcs[i].empty()) continue;
      auto it = cache().find(srcs[i]);
      if (it != cache().end()) {
        if (!it->second.failed) out[i] = (const void*)it->second.kernel;
      } else if (!seen.count(srcs[i])) {
        seen[srcs[i]] = i;
        todo.push_back(i);
      }
    }
  }
  if (!todo.empty()) {
    std::vector<std::vector<char>> bins(todo.size());
    std::vector<std::string> logs(todo.size());
    std::vector<char> ok(todo.size(), 0);
    const int hw = std::max(1, (int)std::thread::hardware_concurrency());
    const int nthr = std::max(1, std::min<int>((int)todo.size(), t_thread_cap > 0 ? std::min(t_thread_cap, hw) : hw));
    std::vector<std::thread> pool;
    std::mutex qm;
    size_t next = 0;
    for (int t = 0; t < nthr; ++t)
      pool.emplace_back([&] {
        while (true) {
          size_t k;
          {
            std::lock_guard<std::mutex> lk(qm);
            if (next >= todo.size()) return;
            k = next++;
          }
          ok[k] = compile_one(srcs[todo[k]], bins[k], logs[k]);
        }
      });
    for (auto& th : pool) th.join();
    std::lock_guard<std::mutex> lk(g_mu);
    for (size_t k = 0; k < todo.size(); ++k) {
      Entry e;
      e.log = logs[k];
      if (ok[k] && cudaLibraryLoadData(&e.lib, bins[k].data(), nullptr, nullptr, 0, nullptr, nullptr, 0) ==
                       cudaSuccess &&
          cudaLibraryGetKernel(&e.kernel, e.lib, name) == cudaSuccess) {
        e.failed = false;
      } else {
        e.failed = true;
        cudaGetLastError();
        if (env_int("VQC_JIT_VERBOSE", 0)) fprintf(stderr, "vqc jit: compile failed:\n%s\n", e.log.c_str());
      }
      if (env_int("VQC_JIT_VERBOSE", 0) && !e.failed) fprintf(stderr, "vqc jit: %s\n", e.log.c_str());
      cache()[srcs[todo[k]]] = e;
    }
    for (size_t i = 0; i < srcs.size(); ++i) {
      if (srcs[i].empty()) continue;
      auto it = cache().find(srcs[i]);
      if (it != cache().end() && !it->second.failed) out[i] = (const void*)it->second.kernel;
    }
    prof_note("jit_compiled_passes", (long long)todo.size());
  }
  return VQC_OK;
}

// Kernels of many passes by structure: a 128-bit hash of everything the
// generated source depends on keys a second cache, so a pass seen before
// costs a hash, not a source text.
namespace {
struct Hash128 {
  uint64_t a = 1469598103934665603ull, b = 0x9e3779b97f4a7c15ull;
  void add(const void* p, size_t n) {
    const unsigned char* c = (const unsigned char*)p;
    for (size_t i = 0; i < n; ++i) {
      a = (a ^ c[i]) * 1099511628211ull;
      b = (b + c[i]) * 0xff51afd7ed558ccdull;
      b ^= b >> 29;
    }
  }
  template <class T>
  void val(const T& v) {
    add(&v, sizeof(v));
  }
};
std::map<std::pair<uint64_t, uint64_t>, const void*>& hcache() {
  static std::map<std::pair<uint64_t, uint64_t>, const void*> c;
  return c;
}
}  // namespace

// Structures some thread is compiling now: another thread that misses them
// does not compile them again (it gets nullptr, the interpreter's case).
std::set<std::pair<uint64_t, uint64_t>>& inflight() {
  static std::set<std::pair<uint64_t, uint64_t>> s;
  return s;
}

int jit_pass_kernels(int M, bool adj, const std::vector<JitPassRef>& refs, std::vector<const void*>& out, bool batch,
                     bool compile, int rb) {
  out.assign(refs.size(), nullptr);
  if (!jit_available()) return VQC_OK;
  const int flags[8] = {env_int("VQC_JIT_BAKE", 1), jit_l2_prefetch(adj) ? 1 : 0, jit_min_blocks(adj, M, rb), M,
                        batch ? 0 : (int)jit_extra_smem(adj, M, rb), batch ? 1 : 0, rb, env_int("VQC_JIT_WARPSYNC", 1)};
  std::vector<std::pair<uint64_t, uint64_t>> keys(refs.size());
  std::vector<size_t> miss;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    for (size_t i = 0; i < refs.size(); ++i) {
      const JitPassRef& r = refs[i];
      if (!r.stages || (!batch && r.npool > kJitMaxCoef)) continue;
      Hash128 h;
      h.add(flags, sizeof(flags));
      h.val(adj);
      h.val(r.nstages);
      h.val(r.npool);
      for (int s = 0; s < r.nstages; ++s) {
        const DevStageF& st = r.stages[s];
        h.add(st.swm, sizeof(st.swm));
        h.add(st.gdep, sizeof(st.gdep));
        h.val(st.op_begin);
        h.val(st.op_end);
        for (int o = st.op_begin; o < st.op_end; ++o) {
          h.val(r.ops[o].code);
          h.val(r.ops[o].mat);
        }
      }
      keys[i] = {h.a, h.b};
      auto it = hcache().find(keys[i]);
      if (it != hcache().end())
        out[i] = it->second;
      else if (compile && !inflight().count(keys[i]) &&
               std::find_if(miss.begin(), miss.end(), [&](size_t m) { return keys[m] == keys[i]; }) == miss.end())
        miss.push_back(i);
    }
    for (size_t m : miss) inflight().insert(keys[m]);
  }
  if (miss.empty()) return VQC_OK;
  std::vector<std::string> srcs(miss.size());
  for (size_t k = 0; k < miss.size(); ++k) {
    const JitPassRef& r = refs[miss[k]];
    srcs[k] = jit_pass_source(M, adj, r.stages, r.nstages, r.ops, r.npool, batch, rb);
  }
  std::vector<const void*> ks;
  int rc = jit_kernels(srcs, ks, batch ? "vqc_pass_batch" : "vqc_pass");
  std::lock_guard<std::mutex> lk(g_mu);
  for (size_t m : miss) inflight().erase(keys[m]);
  if (rc) return rc;
  for (size_t k = 0; k < miss.size(); ++k) hcache()[keys[miss[k]]] = ks[k];  // (nullptr: failed; the interpreter runs it)
  for (size_t i = 0; i < refs.size(); ++i) {  // every pass of a structure compiled here (duplicates too)
    auto it = hcache().find(keys[i]);
    if (!out[i] && it != hcache().end()) out[i] = it->second;
  }
  return VQC_OK;
}

}  // namespace vqc
