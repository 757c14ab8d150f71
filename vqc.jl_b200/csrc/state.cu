// State handles: StateVector{T} / DensityMatrix{T} storage on the device
// (statevector.jl:1-65, densitymatrix.jl:1-61), plus the shared plumbing
// (errors, device info, per-handle scratch, result fetch).
#include <cstdio>
#include <cstring>
#include <map>

#include "common.cuh"

namespace vqc {

static thread_local std::string g_err;

void set_error(const std::string& msg) { g_err = msg; }
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  g_err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? VQC_ERR_OOM : VQC_ERR_CUDA;
}

const DeviceInfo& device_info(int device) {
  static std::mutex mu;
  static std::map<int, DeviceInfo> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(device);
  if (it != cache.end()) return it->second;
  DeviceInfo di;
  cudaDeviceGetAttribute(&di.sms, cudaDevAttrMultiProcessorCount, device);
  cudaDeviceGetAttribute(&di.max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (di.sms <= 0) di.sms = 148;
  return cache[device] = di;
}

int reduction_grid(int device, int64_t work_items) {
  const int64_t cap = int64_t(device_info(device).sms) * 8;
  int64_t want = (work_items + kRedThreads - 1) / kRedThreads;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

int enter(vqc_state h) {
  if (!h) return fail(VQC_ERR_ARG, "null state handle");
  VQC_CK(cudaSetDevice(h->device));
  return VQC_OK;
}

int upload_ops(vqc_state h, const void* src, size_t bytes) {
  if (bytes == 0) return VQC_OK;
  if (bytes > h->opbuf_bytes) {
    if (h->opbuf) {
      VQC_CK(cudaStreamSynchronize(h->stream));
      VQC_CK(cudaFree(h->opbuf));
      h->opbuf = nullptr;
      h->opbuf_bytes = 0;
    }
    size_t cap = 1 << 16;
    while (cap < bytes) cap <<= 1;
    VQC_CK(cudaMalloc(&h->opbuf, cap));
    h->opbuf_bytes = cap;
  }
  // Pageable source: the copy is staged before the call returns, so the caller
  // may reuse `src` at once.
  VQC_CK(cudaMemcpyAsync(h->opbuf, src, bytes, cudaMemcpyHostToDevice, h->stream));
  return VQC_OK;
}

// The op buffer holds at least `bytes` (a larger buffer replaces it after the
// stream has drained: call before uploading anything the coming launches read).
int reserve_ops(vqc_state h, size_t bytes) {
  if (bytes <= h->opbuf_bytes) return VQC_OK;
  if (h->opbuf) {
    VQC_CK(cudaStreamSynchronize(h->stream));
    VQC_CK(cudaFree(h->opbuf));
    h->opbuf = nullptr;
    h->opbuf_bytes = 0;
  }
  size_t cap = 1 << 16;
  while (cap < bytes) cap <<= 1;
  VQC_CK(cudaMalloc(&h->opbuf, cap));
  h->opbuf_bytes = cap;
  return VQC_OK;
}

// Upload into the op buffer at byte offset `off` (reserved with reserve_ops);
// stream-ordered like upload_ops, so launches queued before it keep reading
// the bytes they were given elsewhere in the buffer.
int upload_ops_at(vqc_state h, size_t off, const void* src, size_t bytes) {
  if (bytes == 0) return VQC_OK;
  if (off + bytes > h->opbuf_bytes) return fail(VQC_ERR_ARG, "internal: op upload beyond the reserved buffer");
  VQC_CK(cudaMemcpyAsync((unsigned char*)h->opbuf + off, src, bytes, cudaMemcpyHostToDevice, h->stream));
  return VQC_OK;
}

int stream_after(vqc_state dst, vqc_state src) {
  if (src == dst || src->stream == dst->stream) return VQC_OK;
  cudaEvent_t ev;
  VQC_CK(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  VQC_CK(cudaEventRecord(ev, src->stream));
  VQC_CK(cudaStreamWaitEvent(dst->stream, ev, 0));
  VQC_CK(cudaEventDestroy(ev));
  return VQC_OK;
}

int workspace(vqc_state h, int count, void** bufs) {
  for (int i = 0; i < count; ++i) {
    if (!h->work[i]) VQC_CK(cudaMalloc(&h->work[i], h->size() * h->amp_bytes()));
    bufs[i] = h->work[i];
  }
  return VQC_OK;
}

// ----------------------------------------------------------------------------- profiling
namespace {
struct ProfRec {
  std::string cls;
  cudaEvent_t a, b;
  double bytes, flops;
};
std::mutex g_prof_mu;
bool g_prof_on = false;
std::vector<ProfRec> g_prof;
struct ProfSum {
  std::string cls;
  long long launches = 0;
  double ms = 0, bytes = 0, flops = 0;
};
std::vector<ProfSum> g_prof_sum;
}  // namespace

ProfScope::ProfScope(cudaStream_t s, const char* cls, double bytes, double flops) : stream(s) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on) return;
  ProfRec r{cls, nullptr, nullptr, bytes, flops};
  if (cudaEventCreate(&r.a) != cudaSuccess || cudaEventCreate(&r.b) != cudaSuccess) return;
  cudaEventRecord(r.a, s);
  token = (int)g_prof.size();
  g_prof.push_back(r);
}

ProfScope::~ProfScope() {
  if (token < 0) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (token < (int)g_prof.size()) cudaEventRecord(g_prof[token].b, stream);
}

void prof_note(const char* cls, long long count) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_on) return;
  for (auto& x : g_prof_sum)
    if (x.cls == cls) {
      x.launches += count;
      return;
    }
  ProfSum t;
  t.cls = cls;
  t.launches = count;
  g_prof_sum.push_back(t);
}

std::vector<DebugReader>& debug_readers() {
  static std::vector<DebugReader> r;
  return r;
}
int register_debug_reader(DebugReader r) {
  debug_readers().push_back(r);
  return 0;
}

static void prof_collect() {
  for (auto& r : g_prof) {
    float ms = 0;
    cudaEventSynchronize(r.b);
    cudaEventElapsedTime(&ms, r.a, r.b);
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
    ProfSum* t = nullptr;
    for (auto& x : g_prof_sum)
      if (x.cls == r.cls) t = &x;
    if (!t) {
      g_prof_sum.push_back(ProfSum{r.cls});
      t = &g_prof_sum.back();
    }
    t->launches += 1;
    t->ms += ms;
    t->bytes += r.bytes;
    t->flops += r.flops;
  }
  g_prof.clear();
}

int fetch_result(vqc_state h, int n) {
  if (n > kDeferredSlot) return fail(VQC_ERR_ARG, "internal: result fetch beyond the reserved slot");
  VQC_CK(cudaMemcpyAsync(h->h_result, h->scr.result, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  VQC_CK(cudaStreamSynchronize(h->stream));
  return VQC_OK;
}

// ----------------------------------------------------------------------------- kernels
template <class R>
__global__ void k_set_basis(cplx<R>* v, int64_t N, int64_t one) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = mkc<R>(i == one ? R(1) : R(0), R(0));
}

// The slice of qubit q at `value`, scaled: dst[j] = scale * src[j with bit
// `value` inserted at q] (measure / post_select dropping the qubit,
// measure.jl:38-46, postselect.jl:37-44).
template <class R>
__global__ void k_take_qubit(cplx<R>* __restrict__ dst, const cplx<R>* __restrict__ src, int64_t M, int q, int value,
                             double scale) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < M; j += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = ((j >> q) << (q + 1)) | ((int64_t)value << q) | (j & ((int64_t(1) << q) - 1));
    const cplx<R> a = src[i];
    dst[j] = mkc<R>((R)(scale * a.x), (R)(scale * a.y));
  }
}

// y <- a x + b y (complex a, b), the vector update of the Krylov methods.
template <class R>
__global__ void k_axpby(cplx<R>* __restrict__ y, const cplx<R>* __restrict__ x, int64_t N, double2 a, double2 b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 xv = to_d2(x[i]), yv = to_d2(y[i]);
    const double re = a.x * xv.x - a.y * xv.y + b.x * yv.x - b.y * yv.y;
    const double im = a.x * xv.y + a.y * xv.x + b.x * yv.y + b.y * yv.x;
    y[i] = mkc<R>((R)re, (R)im);
  }
}

template <class RD, class RS>
__global__ void k_convert(cplx<RD>* dst, const cplx<RS>* src, int64_t N) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    cplx<RS> a = src[i];
    dst[i] = mkc<RD>((RD)a.x, (RD)a.y);
  }
}

// sum conj(x_i) y_i in FP64 (y == x gives the squared norm).
template <class R>
__global__ void __launch_bounds__(kRedThreads) k_dot(const cplx<R>* x, const cplx<R>* y, int64_t N, Scratch s) {
  double acc[2] = {0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    double2 a = to_d2(x[i]), b = to_d2(y[i]);
    acc[0] = fma(a.x, b.x, fma(a.y, b.y, acc[0]));
    acc[1] = fma(a.x, b.y, fma(-a.y, b.x, acc[1]));
  }
  grid_reduce<2>(acc, s, s.result);
}

int launch_grid(int device, int64_t items, int threads, int per_sm) {
  int64_t cap = int64_t(device_info(device).sms) * per_sm;
  int64_t want = (items + threads - 1) / threads;
  if (want < 1) want = 1;
  return (int)(want < cap ? want : cap);
}

int set_basis(vqc_state h, int64_t index) {
  const int g = launch_grid(h->device, h->size());
  if (h->dtype == VQC_C64)
    k_set_basis<float><<<g, 256, 0, h->stream>>>((float2*)h->d, h->size(), index);
  else
    k_set_basis<double><<<g, 256, 0, h->stream>>>((double2*)h->d, h->size(), index);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

int dot_device(vqc_state h, const void* x, const void* y, int64_t N, int dtype) {
  const int g = reduction_grid(h->device, N);
  if (dtype == VQC_C64)
    k_dot<float><<<g, kRedThreads, 0, h->stream>>>((const float2*)x, (const float2*)y, N, h->scr);
  else
    k_dot<double><<<g, kRedThreads, 0, h->stream>>>((const double2*)x, (const double2*)y, N, h->scr);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

int convert_copy(vqc_state dst, vqc_state src) {
  const int g = launch_grid(dst->device, dst->size());
  if (dst->dtype == src->dtype) {
    VQC_CK(cudaMemcpyAsync(dst->d, src->d, dst->size() * dst->amp_bytes(), cudaMemcpyDeviceToDevice, dst->stream));
  } else if (dst->dtype == VQC_C64) {
    k_convert<float, double><<<g, 256, 0, dst->stream>>>((float2*)dst->d, (const double2*)src->d, dst->size());
  } else {
    k_convert<double, float><<<g, 256, 0, dst->stream>>>((double2*)dst->d, (const float2*)src->d, dst->size());
  }
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

int create_storage(int nq, int n_dm, int dtype, int device, vqc_state* out) {
  if (!out) return fail(VQC_ERR_ARG, "null output handle");
  *out = nullptr;
  if (dtype != VQC_C64 && dtype != VQC_C128) return fail(VQC_ERR_ARG, "dtype must be VQC_C64 or VQC_C128");
  if (nq < 1 || nq > 36) return fail(VQC_ERR_ARG, "number of qubits must be in 1..36");
  int ndev = 0;
  VQC_CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(VQC_ERR_ARG, "device index out of range");
  VQC_CK(cudaSetDevice(device));
  auto* h = new vqc_state_s();
  h->nq = nq;
  h->n_dm = n_dm;
  h->dtype = dtype;
  h->device = device;
  auto cleanup = [&](int code) {
    if (h->d) cudaFree(h->d);
    if (h->scr.partials) cudaFree(h->scr.partials);
    if (h->scr.counter) cudaFree(h->scr.counter);
    if (h->scr.result) cudaFree(h->scr.result);
    if (h->h_result) cudaFreeHost(h->h_result);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return code;
  };
  cudaError_t e = cudaMalloc(&h->d, h->size() * h->amp_bytes());
  if (e != cudaSuccess) return cleanup(cuda_fail(e, "cudaMalloc(state)"));
  const int maxb = device_info(device).sms * 8;
  h->scr.max_blocks = maxb;
  if ((e = cudaMalloc(&h->scr.partials, sizeof(double) * kMaxAcc * maxb)) != cudaSuccess ||
      (e = cudaMalloc(&h->scr.counter, sizeof(unsigned) * 4)) != cudaSuccess ||
      (e = cudaMalloc(&h->scr.result, sizeof(double) * kMaxAcc)) != cudaSuccess ||
      (e = cudaMallocHost(&h->h_result, sizeof(double) * kMaxAcc)) != cudaSuccess ||
      (e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaMemsetAsync(h->scr.counter, 0, sizeof(unsigned) * 4, h->stream)) != cudaSuccess)
    return cleanup(cuda_fail(e, "state scratch"));
  int rc = set_basis(h, 0);
  if (rc) return cleanup(rc);
  *out = h;
  return VQC_OK;
}

}  // namespace vqc

using namespace vqc;

extern "C" {

const char* vqc_last_error(void) { return g_err.c_str(); }
const char* vqc_version(void) { return "vqcb200 0.1 (sm_100a)"; }

int vqc_device_count(void) {
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceCount");
  return n;
}

int vqc_state_create(int n, int dtype, int device, vqc_state* out) { return create_storage(n, 0, dtype, device, out); }

int vqc_dm_create(int n, int dtype, int device, vqc_state* out) {
  if (n < 1 || n > 18) return fail(VQC_ERR_ARG, "density matrix qubits must be in 1..18");
  return create_storage(2 * n, n, dtype, device, out);
}

int vqc_state_destroy(vqc_state h) {
  if (!h) return VQC_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->d) cudaFree(h->d);
  if (h->opbuf) cudaFree(h->opbuf);
  for (void* w : h->work)
    if (w) cudaFree(w);
  if (h->accbuf) cudaFree(h->accbuf);
  if (h->fused_scratch) cudaFree(h->fused_scratch);
  cudaFree(h->scr.partials);
  cudaFree(h->scr.counter);
  cudaFree(h->scr.result);
  cudaFreeHost(h->h_result);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return VQC_OK;
}

int vqc_state_nqubits(vqc_state h) { return h ? h->nq : VQC_ERR_ARG; }
int vqc_dm_nqubits(vqc_state h) { return h && h->n_dm ? h->n_dm : fail(VQC_ERR_ARG, "not a density matrix"); }
int vqc_state_dtype(vqc_state h) { return h ? h->dtype : VQC_ERR_ARG; }
void* vqc_state_device_ptr(vqc_state h) { return h ? h->d : nullptr; }

int vqc_state_upload(vqc_state h, const void* host, size_t bytes) {
  int rc = enter(h);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!host || bytes != h->size() * h->amp_bytes()) return fail(VQC_ERR_ARG, "upload: byte count mismatch");
  VQC_CK(cudaMemcpyAsync(h->d, host, bytes, cudaMemcpyHostToDevice, h->stream));
  return VQC_OK;
}

int vqc_state_download(vqc_state h, void* host, size_t bytes) {
  int rc = enter(h);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(h->mu);
  if (!host || bytes != h->size() * h->amp_bytes()) return fail(VQC_ERR_ARG, "download: byte count mismatch");
  VQC_CK(cudaMemcpyAsync(host, h->d, bytes, cudaMemcpyDeviceToHost, h->stream));
  VQC_CK(cudaStreamSynchronize(h->stream));
  return VQC_OK;
}

int vqc_state_reset(vqc_state h) {
  int rc = enter(h);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(h->mu);
  return set_basis(h, 0);
}

int vqc_state_axpby(vqc_state y, const double* a, vqc_state x, const double* b) {
  int rc = enter(y);
  if (rc) return rc;
  if (!x || !a || !b || x->nq != y->nq || x->dtype != y->dtype || x->device != y->device)
    return fail(VQC_ERR_ARG, "axpby: same size, dtype and device");
  std::lock_guard<std::mutex> lk(y->mu);
  std::unique_lock<std::mutex> lx(x->mu, std::defer_lock);
  if (x != y) lx.lock();
  if (x != y && (rc = stream_after(y, x))) return rc;
  const int g = launch_grid(y->device, y->size());
  const double2 da = make_double2(a[0], a[1]), db = make_double2(b[0], b[1]);
  if (y->dtype == VQC_C64)
    k_axpby<float><<<g, 256, 0, y->stream>>>((float2*)y->d, (const float2*)x->d, y->size(), da, db);
  else
    k_axpby<double><<<g, 256, 0, y->stream>>>((double2*)y->d, (const double2*)x->d, y->size(), da, db);
  VQC_CK(cudaGetLastError());
  return x != y ? stream_after(x, y) : VQC_OK;
}

int vqc_state_take_qubit(vqc_state src, int q, int value, double scale, vqc_state dst) {
  int rc = enter(src);
  if (rc) return rc;
  if (!dst || src->n_dm || dst->n_dm || src->nq < 1 || dst->nq != src->nq - 1 || dst->dtype != src->dtype ||
      dst->device != src->device)
    return fail(VQC_ERR_ARG, "take_qubit: dst must be a state of one qubit fewer, same dtype and device");
  if (q < 0 || q >= src->nq || (value != 0 && value != 1)) return fail(VQC_ERR_ARG, "take_qubit: bad qubit or value");
  std::lock_guard<std::mutex> lk(src->mu);
  if ((rc = stream_after(src, dst))) return rc;
  const int64_t M = dst->size();
  const int g = launch_grid(src->device, M);
  if (src->dtype == VQC_C64)
    k_take_qubit<float><<<g, 256, 0, src->stream>>>((float2*)dst->d, (const float2*)src->d, M, q, value, scale);
  else
    k_take_qubit<double><<<g, 256, 0, src->stream>>>((double2*)dst->d, (const double2*)src->d, M, q, value, scale);
  VQC_CK(cudaGetLastError());
  return stream_after(dst, src);
}

int vqc_state_copy(vqc_state dst, vqc_state src) {
  int rc = enter(dst);
  if (rc) return rc;
  if (!src || src->nq != dst->nq || src->n_dm != dst->n_dm) return fail(VQC_ERR_ARG, "copy: shape mismatch");
  if (src->device != dst->device) return fail(VQC_ERR_ARG, "copy: handles on different devices");
  if (src == dst) return VQC_OK;
  std::lock_guard<std::mutex> lk(dst->mu);
  if ((rc = stream_after(dst, src))) return rc;
  return convert_copy(dst, src);
}

int vqc_state_norm(vqc_state h, double* out) {
  int rc = enter(h);
  if (rc) return rc;
  if (!out) return fail(VQC_ERR_ARG, "null output");
  std::lock_guard<std::mutex> lk(h->mu);
  if ((rc = dot_device(h, h->d, h->d, h->size(), h->dtype))) return rc;
  if ((rc = fetch_result(h, 1))) return rc;
  *out = std::sqrt(h->h_result[0]);
  return VQC_OK;
}

int vqc_state_dot(vqc_state x, vqc_state y, double* out) {
  int rc = enter(x);
  if (rc) return rc;
  if (!y || !out || x->nq != y->nq || x->dtype != y->dtype || x->device != y->device)
    return fail(VQC_ERR_ARG, "dot: handles differ in size, dtype or device");
  std::lock_guard<std::mutex> lk(x->mu);
  if ((rc = stream_after(x, y))) return rc;
  if ((rc = dot_device(x, x->d, y->d, x->size(), x->dtype))) return rc;
  if ((rc = fetch_result(x, 2))) return rc;
  out[0] = x->h_result[0];
  out[1] = x->h_result[1];
  return VQC_OK;
}

void* vqc_state_stream(vqc_state h) { return h ? (void*)h->stream : nullptr; }

int vqc_profile_enable(int on) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (on) {
    prof_collect();
    g_prof_sum.clear();
  } else {
    prof_collect();
  }
  g_prof_on = on != 0;
  return VQC_OK;
}

int vqc_profile_count(void) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  prof_collect();
  return (int)g_prof_sum.size();
}

int vqc_profile_get(int i, char* name, int name_len, long long* launches, double* total_ms, double* total_bytes) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  prof_collect();
  if (i < 0 || i >= (int)g_prof_sum.size()) return fail(VQC_ERR_ARG, "profile index out of range");
  const ProfSum& t = g_prof_sum[i];
  if (name && name_len > 0) {
    std::strncpy(name, t.cls.c_str(), name_len - 1);
    name[name_len - 1] = 0;
  }
  if (launches) *launches = t.launches;
  if (total_ms) *total_ms = t.ms;
  if (total_bytes) *total_bytes = t.bytes;
  return VQC_OK;
}

int vqc_debug_status(int reset, long long* out) {
  DebugRecord first{};
  long long hits = 0;
  for (DebugReader r : debug_readers()) {
    DebugRecord d{};
    if (r(&d, reset)) return fail(VQC_ERR_CUDA, "reading a debug record failed");
    if (d.hits && !hits) first = d;
    hits += d.hits;
  }
  if (out) {
    out[0] = hits;
    out[1] = first.line;
    out[2] = first.index;
    out[3] = first.limit;
  }
  return (int)std::min<long long>(hits, 1 << 30);
}

int vqc_debug_build(void) {
#ifdef VQC_DEBUG_CHECKS
  return 1;
#else
  return 0;
#endif
}

int vqc_profile_flops(int i, double* total_flops) {
  std::lock_guard<std::mutex> lk(g_prof_mu);
  prof_collect();
  if (i < 0 || i >= (int)g_prof_sum.size()) return fail(VQC_ERR_ARG, "profile index out of range");
  if (total_flops) *total_flops = g_prof_sum[i].flops;
  return VQC_OK;
}

int vqc_state_sync(vqc_state h) {
  int rc = enter(h);
  if (rc) return rc;
  VQC_CK(cudaStreamSynchronize(h->stream));
  return VQC_OK;
}

}  // extern "C"
