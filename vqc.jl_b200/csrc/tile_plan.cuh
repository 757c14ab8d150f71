// Data structures of the tile engine shared by the single-state path
// (fused.cu) and the serving loop (serve.cu): the device descriptors of a
// pass, the planner's op form, and a serialised plan.
#pragma once

#include <vector>

#include "engine.h"
#include "tile_dev.cuh"

namespace vqc {

// Shared-memory bytes of one pass: tiles, accumulation slots, and the pass's
// own stage / op / matrix descriptors (read by every thread for every op, so
// they are staged once per CTA instead of being fetched through L1/L2).
template <class R, int M, bool ADJ>
__host__ __device__ constexpr size_t tile_bytes() {
  return (size_t)(ADJ ? 2 : 1) * (size_t(1) << M) * sizeof(cplx<R>);
}


struct PGrad {
  int param;             // caller's parameter index
  std::vector<cd> D;     // U1: 2x2 over the target (control subspace); AccD: 2^nd diagonal bins
};

struct FOp {
  int kind = 0;          // kOpU1, kOpU2, kOpDiag, kOpAccD
  int tq[2] = {-1, -1};  // target qubits (ascending)
  uint64_t cmask = 0, cval = 0;  // control qubits and their firing values (global bits)
  uint64_t qubits = 0;   // every qubit the op reads or writes
  std::vector<cd> mat;   // U1 2x2, U2 4x4 (bit 0 <-> tq[0]), diagonal 2^nd table
  int nd = 0;
  int dq[5] = {0, 0, 0, 0, 0};
  bool acc = false;
  std::vector<PGrad> grads;
};

struct PassShape {
  int nslots = 0, nstages = 0, nops = 0, npool = 0;
  bool general = true;  // false: every op of the pass is a one-qubit op
  bool packed = false;  // FP32 packed layout (DevStageF), for the compiled pass kernels
};

// An accumulating op of the reverse sweep and the row of 8 doubles (the
// reduced matrix A) its partial sums land in.
struct AccRef {
  int row;
  FOp op;
  bool ah = false;  // the row holds the anti-Hermitian projection (kAccAH)
};

struct PassLoc {
  bool standalone = false;
  int gate = -1;
  size_t pass = 0, stages = 0, ops = 0;
  size_t pool_begin = 0;  // in pool entries, a multiple of 16 bytes
  PassShape shape;
  int nslots = 0;
  int row0 = 0;
  int64_t ntiles = 0;
  double fma_ops = 0;  // FMA-pipe lane operations of the pass over the whole state
};

// A plan serialised for the device: one byte image holding every pass's
// DevPass, stages and ops, then the matrix pool; offsets in `locs`.
struct SerialPlan {
  std::vector<unsigned char> buf;
  std::vector<PassLoc> locs;
  size_t pool_off = 0;
  int rows = 0;  // accumulation rows (ADJ)
};


// Pauli-sum tables (expect.cu): terms grouped by flip mask x.
struct DevTerm {
  uint64_t z;
  double2 c;  // coefficient for the expectation, times i^{popcount(x & z)}
  double2 d;  // coefficient for the applied operator, same phase
};
struct DevGroup {
  uint64_t x;
  int start, count;
};

// One state's Pauli pass in a batched launch (serving path).
struct PauliItem {
  const void* ket;  // the state (also the bra: <psi|H|psi>)
  void* out;        // (H + H^dagger) psi for gradient requests, else unused
  int64_t N;
  const DevGroup* groups;
  int ng;
  const DevTerm* terms;
  int nt;
  double* partials;  // [gridDim.x][2]
};
struct PauliRed {
  const double* partials;
  int nblocks;
  double* out;  // energy (re, im)
};
int serve_pauli_image(int nq, const vqc_pauli* terms, int nterms, bool hermitian_part, std::vector<unsigned char>& img,
                      int& ng, int& nt);
int serve_launch_pauli(int dtype, bool write, const PauliItem* d_items, int nitems, int gridx, size_t smem,
                       cudaStream_t stream);
int serve_launch_pauli_reduce(const PauliRed* d_items, int nitems, cudaStream_t stream);

// Reduction of one request's per-CTA accumulation partials (serving path).
struct RedItem {
  const double* partials;  // [nblocks][nslots][8]
  int nblocks;
  int nslots;
  double* out;  // [nslots][8]
};

// A request's plan for the serving loop: forward passes, and for gradient
// requests the reverse passes and their accumulation rows.
struct ReqPlan {
  int M = 0;
  SerialPlan fwd, adj;
  std::vector<AccRef> accs;
  PassShape fwd_max, adj_max;
  int64_t ntiles = 0;
  // compiled batch kernels per pass (FP32 packed plans), empty for the generic kernel
  std::vector<const void*> fwd_k, adj_k;
};

// Run-time specialised FP32 tile kernels (jit.cu).
int jit_mode();        // 0 off, 1 on, 2 auto, 3 packed interpreter (VQC_JIT)
bool jit_available();  // NVRTC could be loaded
int jit_min_blocks(bool adj, int M, int rb = kRegBits);
// Shared-memory bytes a compiled pass needs beyond pass_smem (the second tile
// buffer of the asynchronous forward passes).
size_t jit_extra_smem(bool adj, int M, int rb = kRegBits);
// Source of a pass's kernel ("" when the pass is not compiled: its matrix
// pool, passed as a kernel parameter, would exceed kJitMaxCoef entries).
constexpr int kJitMaxCoef = 3800;
std::string jit_pass_source(int M, bool adj, const DevStageF* stages, int nstages, const DevOp* ops, int npool,
                            bool batch = false, int rb = kRegBits);
// Compiler threads jit_kernels may start from the calling thread (0: one per
// host core).  A background compiler sets a few so the threads that plan and
// launch keep their cores.
void jit_set_thread_cap(int n);
// Kernels for the given pass sources (nullptr for an empty source or a failed compile).
int jit_kernels(const std::vector<std::string>& srcs, std::vector<const void*>& out, const char* name = "vqc_pass");
// A serialised pass for jit_pass_kernels (stages == nullptr: not a tile pass).
struct JitPassRef {
  const DevStageF* stages = nullptr;
  int nstages = 0;
  const DevOp* ops = nullptr;
  int npool = 0;
};
// Kernels for many passes, looked up by a hash of their structure first.
// batch: the serving loop's kernels (vqc_pass_batch over an array of TileItems,
// coefficients from each item's pool) instead of the single-state ones.
// compile = false: look up only (a structure not compiled yet gives nullptr).
// rb: register bits per thread of the passes' stage layout (kRegBits, or
// kWideRegBits for wide forward passes).
int jit_pass_kernels(int M, bool adj, const std::vector<JitPassRef>& refs, std::vector<const void*>& out,
                     bool batch = false, bool compile = true, int rb = kRegBits);

// compiled: an FP32 packed plan with compiled batch kernels (fwd_k / adj_k)
// when every pass has one already, else the classic plan for the generic
// kernel; then *to_compile (if given) receives the packed plan whose missing
// kernels the caller compiles afterwards (serve_compile_plan) for later
// requests of the same structure.
int serve_build_plan(int n, int dtype, const std::vector<GateSpec>& fspecs, const std::vector<GateSpec>& rspecs,
                     const std::vector<std::vector<ParamInfo>>& params, bool want_grad, bool compiled, ReqPlan& rp,
                     ReqPlan* to_compile = nullptr);
void serve_compile_plan(const ReqPlan& packed, bool want_grad);
// CTAs per request of the compiled batch kernels ks of a plan's passes.
int serve_jit_gridx(int M, bool adj, const std::vector<const void*>& ks, const SerialPlan& sp, int64_t ntiles,
                    int device);
int serve_launch_jit(int M, bool adj, const void* kernel, const TileItem* d_items, int nitems, int gridx,
                     const PassShape& maxs, cudaStream_t stream);
int serve_tile_gridx(int dtype, int M, bool adj, const PassShape& maxs, int64_t max_ntiles, int device);
int serve_launch_tiles(int dtype, int M, bool adj, const TileItem* d_items, int nitems, int gridx,
                       const PassShape& maxs, cudaStream_t stream);
int serve_launch_reduce(const RedItem* d_items, int nitems, int maxslots, cudaStream_t stream);
void contract_grads(const std::vector<AccRef>& accs, const double* A, double* grads);

}  // namespace vqc
