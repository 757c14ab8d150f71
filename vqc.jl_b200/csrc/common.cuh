// Shared device/host definitions of libvqcb200: complex arithmetic on the
// interleaved float2 / double2 amplitude layout, the state handle, error
// plumbing, and the deterministic grid reduction used by every kernel that
// returns a number (norms, expectations, gradient partials).
#pragma once

#include <cuda_runtime.h>

#include <complex>
#include <cstdint>
#include <mutex>
#include <string>
#include <vector>

#include "vqc_b200.h"

namespace vqc {

// ----------------------------------------------------------------------------- debug checks
// Built with -DVQC_DEBUG_CHECKS (vqcb200._build.build(debug=True), the
// library libvqcb200_debug.so), every index wrapped in VQC_DCHECK(i, limit) is
// tested on the device before its access: a violation increments this
// translation unit's device record (keeping the first source line, index and
// limit) and the access is skipped, so nothing traps and the context stays
// usable.  vqc_debug_status() sums the records of every translation unit.
// In the release build VQC_DCHECK is the constant true and compiles away.
struct DebugRecord {
  unsigned hits;
  int line;
  long long index, limit;
};
typedef int (*DebugReader)(DebugRecord* out, int reset);
int register_debug_reader(DebugReader r);
#ifdef VQC_DEBUG_CHECKS
static __device__ DebugRecord g_vqc_dbg;
__device__ __forceinline__ bool dcheck(long long i, long long lim, int line) {
  if (i >= 0 && i < lim) return true;
  if (atomicAdd(&g_vqc_dbg.hits, 1u) == 0u) {
    g_vqc_dbg.line = line;
    g_vqc_dbg.index = i;
    g_vqc_dbg.limit = lim;
  }
  return false;
}
#define VQC_DCHECK(i, lim) (::vqc::dcheck((long long)(i), (long long)(lim), __LINE__))
static int vqc_dbg_read(DebugRecord* out, int reset) {
  if (cudaMemcpyFromSymbol(out, g_vqc_dbg, sizeof(DebugRecord)) != cudaSuccess) return -1;
  if (reset) {
    const DebugRecord z{};
    if (cudaMemcpyToSymbol(g_vqc_dbg, &z, sizeof(z)) != cudaSuccess) return -1;
  }
  return 0;
}
[[maybe_unused]] static const int vqc_dbg_registered = register_debug_reader(&vqc_dbg_read);
#else
#define VQC_DCHECK(i, lim) true
#endif

// ----------------------------------------------------------------------------- complex
template <class R>
struct CT;
template <>
struct CT<float> {
  using T = float2;
};
template <>
struct CT<double> {
  using T = double2;
};
template <class R>
using cplx = typename CT<R>::T;

template <class R>
__host__ __device__ __forceinline__ cplx<R> mkc(R a, R b) {
  cplx<R> r;
  r.x = a;
  r.y = b;
  return r;
}
// a * b
template <class V>
__host__ __device__ __forceinline__ V cmul(V a, V b) {
  V r;
  r.x = a.x * b.x - a.y * b.y;
  r.y = a.x * b.y + a.y * b.x;
  return r;
}
// acc + a * b
template <class V>
__host__ __device__ __forceinline__ V cfma(V a, V b, V acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(-a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(a.y, b.x, acc.y);
  return acc;
}
// acc + conj(a) * b
template <class V>
__host__ __device__ __forceinline__ V cfma_conj(V a, V b, V acc) {
  acc.x = fma(a.x, b.x, acc.x);
  acc.x = fma(a.y, b.y, acc.x);
  acc.y = fma(a.x, b.y, acc.y);
  acc.y = fma(-a.y, b.x, acc.y);
  return acc;
}
__device__ __forceinline__ double2 to_d2(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_d2(double2 a) { return a; }

// ----------------------------------------------------------------------------- errors
void set_error(const std::string& msg);
int fail(int code, const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define VQC_CK(call)                                   \
  do {                                                 \
    cudaError_t _e = (call);                           \
    if (_e != cudaSuccess) return ::vqc::cuda_fail(_e, #call); \
  } while (0)

// ----------------------------------------------------------------------------- device info
struct DeviceInfo {
  int sms = 148;
  int max_smem_optin = 0;
};
const DeviceInfo& device_info(int device);

// Every reduction launches a fixed grid for a given size, so its sum order
// (and result) does not change from call to call.
constexpr int kRedThreads = 256;
constexpr int kMaxAcc = 64;  // doubles reduced per launch
// The last two doubles of a handle's pinned result buffer receive a result
// copied without waiting (the gradient's energy, read after the reverse
// sweep); fetch_result never reaches them.
constexpr int kDeferredSlot = kMaxAcc - 2;
int reduction_grid(int device, int64_t work_items);

// ----------------------------------------------------------------------------- scratch
// Per-handle device scratch for reductions: `partials` holds one row of
// kMaxAcc doubles per block, `counter` elects the last block (zero between
// launches), `result` receives the reduced values.
struct Scratch {
  double* partials = nullptr;
  unsigned* counter = nullptr;
  double* result = nullptr;
  int max_blocks = 0;
};

}  // namespace vqc

// The state handle (opaque in the C ABI).
struct vqc_state_s {
  int nq = 0;      // stored qubits (2n for a density matrix)
  int n_dm = 0;    // density-matrix qubits, 0 for a state vector
  int dtype = VQC_C128;
  int device = 0;
  void* d = nullptr;  // 2^nq amplitudes
  cudaStream_t stream = nullptr;
  vqc::Scratch scr;
  double* h_result = nullptr;  // pinned host copy of scr.result
  void* opbuf = nullptr;       // device buffer for op lists (terms, passes)
  size_t opbuf_bytes = 0;
  void* work[3] = {nullptr, nullptr, nullptr};  // state-sized workspaces (gradients)
  double* accbuf = nullptr;    // gradient partial sums, one row per parameterised gate
  size_t accbuf_rows = 0;
  void* fused_scratch = nullptr;  // per-CTA partial sums of the tile engine
  size_t fused_scratch_bytes = 0;
  std::mutex mu;
  size_t amp_bytes() const { return dtype == VQC_C64 ? 8 : 16; }
  int64_t size() const { return int64_t(1) << nq; }
};

namespace vqc {
int launch_grid(int device, int64_t items, int threads = 256, int per_sm = 16);
int set_basis(vqc_state h, int64_t index);
int dot_device(vqc_state h, const void* x, const void* y, int64_t N, int dtype);
int convert_copy(vqc_state dst, vqc_state src);
// Orders dst's stream after the work queued so far on src's stream.
int stream_after(vqc_state dst, vqc_state src);
// Device workspace of the handle: `count` buffers of the state's size.
int workspace(vqc_state h, int count, void** bufs);
// Makes h's device current; returns a status.
int enter(vqc_state h);
// Grows h->opbuf to at least `bytes` and copies `src` into it (stream-ordered).
int upload_ops(vqc_state h, const void* src, size_t bytes);
int reserve_ops(vqc_state h, size_t bytes);
int upload_ops_at(vqc_state h, size_t off, const void* src, size_t bytes);
// Copies `n` reduced doubles from h->scr.result to h->h_result and waits.
int fetch_result(vqc_state h, int n);
}  // namespace vqc

namespace vqc {
// ----------------------------------------------------------------------------- profiling
// Per-kernel-class launch timing with CUDA events on the launching stream,
// switched on by vqc_profile_enable(1).  Each record carries the launch's
// algorithmic bytes (the data the operation must move at minimum), so
// achieved bandwidth = bytes / time per class, and, where the kernel is bound
// by arithmetic, its FMA-pipe operations (lane operations of the FMA pipe:
// fused multiply-adds, multiplies and adds, counted once each) as flops =
// 2 x operations, against the measured FMA peak (vqc_fma_peak).
struct ProfScope {
  int token = -1;
  ProfScope(cudaStream_t s, const char* cls, double bytes, double flops = 0);
  ~ProfScope();
  cudaStream_t stream;
};
// Adds `count` to a counter class of the profile (no timing), e.g. the
// number of passes and stages the planner produced.
void prof_note(const char* cls, long long count);
}  // namespace vqc

// ----------------------------------------------------------------------------- grid reduction
namespace vqc {

// Block sum of NACC per-thread doubles, then a last-block sum over the grid's
// block partials in block order.  Deterministic for a fixed grid size.
// out[i] (device memory) receives the grid total of acc[i].  All NT threads
// of the block (NT = its block size) must call it.
template <int NACC, int NT = kRedThreads>
__device__ __forceinline__ void grid_reduce(double (&acc)[NACC], const Scratch& s, double* out) {
  __shared__ double sm[NT / 32][NACC];
  __shared__ bool last;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < NACC; ++i) {
    double v = acc[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sm[warp][i] = v;
  }
  __syncthreads();
  if (threadIdx.x < NACC) {
    double v = 0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) v += sm[w][threadIdx.x];
    s.partials[(size_t)blockIdx.x * kMaxAcc + threadIdx.x] = v;
  }
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(s.counter, 1u) == gridDim.x - 1);
  __syncthreads();
  if (!last) return;
  __threadfence();
  for (int i = 0; i < NACC; ++i) {
    double v = 0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += NT)
      v += __ldcg(&s.partials[(size_t)b * kMaxAcc + i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) sm[warp][0] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0;
      for (int w = 0; w < NT / 32; ++w) t += sm[w][0];
      out[i] = t;
    }
  }
  if (threadIdx.x == 0) *s.counter = 0;
}

}  // namespace vqc
