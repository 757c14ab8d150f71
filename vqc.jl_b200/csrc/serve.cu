// The serving loop: continuous batching of many circuits on one GPU.
//
// Requests (a circuit, a Pauli observable, energy or energy + gradient) are
// submitted from any thread.  Planner threads turn each into device
// descriptors (the tile engine's passes, the Pauli tables).  One GPU worker
// thread runs the loop:
//   1. admit planned requests, first come first served, while their device
//      memory (states + descriptors + scratch) fits the budget and the slot
//      count allows; a request that never fits is rejected;
//   2. take the next step of EVERY admitted request -- a forward pass, the
//      Pauli pass (energy, and the cotangent (H + H^dagger) psi), a reverse
//      pass -- and launch the steps of a kind together (a 2-D grid: request x
//      tiles): FP32 tile passes grouped by pass structure, one launch of that
//      structure's compiled kernel per group (a background compiler thread,
//      with a few host cores, compiles each structure once after its first
//      request has been planned; requests of one qubit count share most
//      structures; until then they run on the generic kernel),
//      the others on the generic tile kernel in one launch per tile size;
//   3. wait for the launches, retire finished requests (results to the host,
//      memory back to the budget) and loop.
// Requests that arrive while others run are admitted at the next iteration,
// so their work overlaps the others' on the device.  The reference has no
// serving layer; the per-request arithmetic is the same as the single-state
// path (circuitdiff.jl / expecdiff.jl semantics), and a request's result does
// not depend on what it is batched with (each CTA touches one request; sums
// are reduced in a fixed order).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <thread>
#include <tuple>

#include "engine.h"
#include "tile_plan.cuh"

namespace vqc {

int launch_grid(int device, int64_t items, int threads, int per_sm);
constexpr size_t kCompileQueue = 64;  // packed plans waiting for the compiler thread

template <class R>
__global__ void k_zero_state(cplx<R>* v, int64_t N) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = mkc<R>(i == 0 ? R(1) : R(0), R(0));
}

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  int64_t ticket = 0;
  int n = 0;
  bool grad = false;
  std::vector<vqc_gate> gates;
  std::vector<double> mats;
  std::vector<vqc_param> params;
  std::vector<vqc_pauli> terms;
  double* grads_out = nullptr;
  // plan
  ReqPlan plan;
  ReqPlan to_compile;  // a packed plan whose kernels the planner compiles after handing the request on
  std::vector<unsigned char> image;  // fwd plan | adj plan | pauli tables
  size_t off_adj = 0, off_pauli = 0;
  int ng = 0, nt = 0;
  size_t pauli_smem = 0;
  int fwd_cap = 0;    // CTAs of its forward passes
  int adj_cap = 0;    // CTAs of its reverse passes
  int pauli_cap = 0;  // CTAs of its Pauli pass
  // device
  size_t dbytes = 0;
  unsigned char* dmem = nullptr;
  void* psi = nullptr;
  void* lam = nullptr;
  unsigned char* dimg = nullptr;
  double* partials = nullptr;
  double* rows = nullptr;
  double* energy_dev = nullptr;
  double* host_res = nullptr;  // pinned: energy (2) + rows (8 per row)
  size_t host_cap = 0;
  // progress
  int step = 0;
  int status = 0;  // 0 queued, 1 planned, 2 running, 3 done, < 0 error
  bool cancel = false;  // set by vqc_serve_cancel; a running request is retired at the next iteration
  std::string error;
  double energy[2] = {0, 0};
  double t_submit = 0, t_planned = 0, t_admit = 0, t_done = 0;
  int nfwd() const { return (int)plan.fwd.locs.size(); }
  int nadj() const { return grad ? (int)plan.adj.locs.size() : 0; }
  int nsteps() const { return nfwd() + 1 + nadj(); }
};

}  // namespace vqc

struct vqc_server_s {
  int device = 0;
  int dtype = VQC_C64;
  size_t budget = 0, in_use = 0;
  int max_active = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  std::mutex mu;
  std::condition_variable cv_plan, cv_ready, cv_done;
  std::deque<std::shared_ptr<vqc::Request>> to_plan, ready;
  std::vector<std::shared_ptr<vqc::Request>> active;
  std::map<int64_t, std::shared_ptr<vqc::Request>> all;
  std::vector<std::thread> planners;
  std::thread worker;
  // packed plans whose kernels the compiler thread builds (bounded: a plan
  // that finds the queue full is dropped; a later request of its structure
  // queues it again)
  std::deque<vqc::ReqPlan> to_build;
  std::condition_variable cv_build;
  std::thread compiler;
  bool stop = false;
  int64_t next_ticket = 0;
  std::multimap<size_t, double*> pinned_free;  // pinned result buffers by size
  // launch item staging (pinned host + device), grown as needed
  unsigned char* h_items = nullptr;
  unsigned char* d_items = nullptr;
  size_t items_cap = 0;
  // statistics
  long long completed = 0, iterations = 0, launches = 0, items_launched = 0;
  double plan_s_max = 0, wait_s_max = 0, run_s_max = 0, plan_s_sum = 0, wait_s_sum = 0, run_s_sum = 0;
  // loop iterations with work: host time building and enqueueing, time waiting for the
  // device, host time retiring (seconds, summed)
  double loop_build_s = 0, loop_wait_s = 0, loop_retire_s = 0;
  long long loop_busy = 0;
  std::string fatal;
};

namespace vqc {

static int plan_request(vqc_server_s* s, Request& r) {
  std::vector<GateSpec> fspecs(r.gates.size());
  for (size_t i = 0; i < r.gates.size(); ++i) {
    const vqc_gate& g = r.gates[i];
    int rc = analyze_gate(r.n, g.nq, g.pos, r.mats.data() + g.mat, false, fspecs[i]);
    if (rc) return rc;
  }
  std::vector<GateSpec> rspecs;
  std::vector<std::vector<ParamInfo>> per_gate;
  if (r.grad) {
    int rc = prepare_reverse(r.n, r.gates.data(), (int)r.gates.size(), r.mats.data(), r.params.data(),
                             (int)r.params.size(), rspecs, per_gate);
    if (rc) return rc;
  }
  // FP32 requests run on compiled batch kernels (one per pass structure,
  // compiled here in the planner thread the first time a structure is seen)
  // unless run-time compilation is off (VQC_JIT=off) or fails
  int rc = serve_build_plan(r.n, s->dtype, fspecs, rspecs, per_gate, r.grad, jit_mode() != 0, r.plan, &r.to_compile);
  if (rc) return rc;
  std::vector<unsigned char> pimg;
  if ((rc = serve_pauli_image(r.n, r.terms.data(), (int)r.terms.size(), true, pimg, r.ng, r.nt))) return rc;
  auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
  r.off_adj = align(r.plan.fwd.buf.size());
  r.off_pauli = align(r.off_adj + r.plan.adj.buf.size());
  r.image.assign(r.off_pauli + pimg.size() + 16, 0);
  std::memcpy(r.image.data(), r.plan.fwd.buf.data(), r.plan.fwd.buf.size());
  if (r.grad) std::memcpy(r.image.data() + r.off_adj, r.plan.adj.buf.data(), r.plan.adj.buf.size());
  if (!pimg.empty()) std::memcpy(r.image.data() + r.off_pauli, pimg.data(), pimg.size());
  r.pauli_smem = pimg.size();
  const int64_t N = int64_t(1) << r.n;
  r.pauli_cap = (int)std::min<int64_t>((N + kRedThreads - 1) / kRedThreads, device_info(s->device).sms * 2);
  r.fwd_cap = r.plan.fwd_k.empty()
                  ? serve_tile_gridx(s->dtype, r.plan.M, false, r.plan.fwd_max, r.plan.ntiles, s->device)
                  : serve_jit_gridx(r.plan.M, false, r.plan.fwd_k, r.plan.fwd, r.plan.ntiles, s->device);
  r.adj_cap = !r.grad ? 0
              : r.plan.adj_k.empty()
                  ? serve_tile_gridx(s->dtype, r.plan.M, true, r.plan.adj_max, r.plan.ntiles, s->device)
                  : serve_jit_gridx(r.plan.M, true, r.plan.adj_k, r.plan.adj, r.plan.ntiles, s->device);
  const size_t amp = s->dtype == VQC_C64 ? 8 : 16;
  size_t off = 0;
  auto take = [&](size_t b) {
    const size_t o = off;
    off = align(off + b);
    return o;
  };
  const size_t o_psi = take(N * amp);
  const size_t o_lam = r.grad ? take(N * amp) : 0;
  const size_t o_img = take(r.image.size());
  const size_t o_part = take(std::max<size_t>((size_t)r.adj_cap * r.plan.adj_max.nslots * 8, (size_t)r.pauli_cap * 2) *
                             sizeof(double));
  const size_t o_rows = take((size_t)std::max(r.plan.adj.rows, 1) * 8 * sizeof(double));
  const size_t o_en = take(2 * sizeof(double));
  r.dbytes = off;
  (void)o_psi;
  // offsets are re-applied to the allocation at admission
  r.psi = (void*)o_psi;
  r.lam = (void*)o_lam;
  r.dimg = (unsigned char*)o_img;
  r.partials = (double*)o_part;
  r.rows = (double*)o_rows;
  r.energy_dev = (double*)o_en;
  return VQC_OK;
}

static void planner_main(vqc_server_s* s) {
  cudaSetDevice(s->device);  // occupancy queries of the planner run on the server's device
  while (true) {
    std::shared_ptr<Request> r;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_plan.wait(lk, [&] { return s->stop || !s->to_plan.empty(); });
      if (s->stop) return;
      r = s->to_plan.front();
      s->to_plan.pop_front();
    }
    const int rc = plan_request(s, *r);
    ReqPlan compile_later;
    std::swap(compile_later, r->to_compile);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (r->status < 0) {
        // cancelled while it was being planned
      } else if (rc) {
        r->status = rc;
        r->error = vqc_last_error();
        r->t_done = now_s();
        s->cv_done.notify_all();
      } else if (r->dbytes > s->budget) {
        r->status = VQC_ERR_BUSY;
        r->error = "request needs more device memory than the serving budget";
        r->t_done = now_s();
        s->cv_done.notify_all();
      } else {
        r->status = 1;
        r->t_planned = now_s();
        s->ready.push_back(r);
        s->cv_ready.notify_all();
      }
    }
    // the request is on its way; its structure is compiled for the next ones
    // by the compiler thread, so planning never waits for a compile
    if (!compile_later.fwd.locs.empty()) {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->to_build.size() < kCompileQueue) {
        s->to_build.push_back(std::move(compile_later));
        s->cv_build.notify_one();
      }
    }
  }
}

// Compiles queued structures with at most a quarter of the host cores (at
// least one), so the planners and the GPU worker are not starved meanwhile.
static void compiler_main(vqc_server_s* s) {
  cudaSetDevice(s->device);  // kernels are loaded into the server's device context
  jit_set_thread_cap(std::max(1u, std::thread::hardware_concurrency() / 4));
  while (true) {
    ReqPlan p;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_build.wait(lk, [&] { return s->stop || !s->to_build.empty(); });
      if (s->stop) return;
      p = std::move(s->to_build.front());
      s->to_build.pop_front();
    }
    serve_compile_plan(p, !p.adj.locs.empty());
  }
}

static void fail_all(vqc_server_s* s, const std::string& why) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->fatal = why;
  for (auto& kv : s->all)
    if (kv.second->status >= 0 && kv.second->status != 3) {
      kv.second->status = VQC_ERR_CUDA;
      kv.second->error = why;
    }
  s->cv_done.notify_all();
}

#define SRV_CK(call)                                                   \
  do {                                                                 \
    cudaError_t _e = (call);                                           \
    if (_e != cudaSuccess) {                                           \
      fail_all(s, std::string(#call) + ": " + cudaGetErrorString(_e)); \
      return;                                                          \
    }                                                                  \
  } while (0)

static void worker_main(vqc_server_s* s) {
  if (cudaSetDevice(s->device) != cudaSuccess) {
    fail_all(s, "cudaSetDevice failed in the serving worker");
    return;
  }
  const size_t amp = s->dtype == VQC_C64 ? 8 : 16;
  while (true) {
    // 1. admission
    std::vector<std::shared_ptr<Request>> admitted;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      if (s->active.empty())
        s->cv_ready.wait(lk, [&] { return s->stop || !s->ready.empty(); });
      if (s->stop) return;
      while (!s->ready.empty() && (int)s->active.size() + (int)admitted.size() < s->max_active &&
             s->in_use + s->ready.front()->dbytes <= s->budget) {
        auto r = s->ready.front();
        s->ready.pop_front();
        s->in_use += r->dbytes;
        r->status = 2;
        r->t_admit = now_s();
        admitted.push_back(r);
      }
    }
    for (auto& r : admitted) {
      SRV_CK(cudaMallocAsync((void**)&r->dmem, r->dbytes, s->stream));
      {
        size_t want = 64;
        while (want < 2 + 8 * (size_t)std::max(r->plan.adj.rows, 1)) want <<= 1;
        auto it = s->pinned_free.find(want);
        if (it != s->pinned_free.end()) {
          r->host_res = it->second;
          s->pinned_free.erase(it);
        } else {
          SRV_CK(cudaMallocHost((void**)&r->host_res, sizeof(double) * want));
        }
        r->host_cap = want;
      }
      unsigned char* b = r->dmem;
      r->psi = b + (size_t)r->psi;
      r->lam = r->grad ? b + (size_t)r->lam : nullptr;
      r->dimg = b + (size_t)r->dimg;
      r->partials = (double*)(b + (size_t)r->partials);
      r->rows = (double*)(b + (size_t)r->rows);
      r->energy_dev = (double*)(b + (size_t)r->energy_dev);
      SRV_CK(cudaMemcpyAsync(r->dimg, r->image.data(), r->image.size(), cudaMemcpyHostToDevice, s->stream));
      const int64_t N = int64_t(1) << r->n;
      const int g = launch_grid(s->device, N, 256, 16);
      if (s->dtype == VQC_C64)
        k_zero_state<float><<<g, 256, 0, s->stream>>>((float2*)r->psi, N);
      else
        k_zero_state<double><<<g, 256, 0, s->stream>>>((double2*)r->psi, N);
      SRV_CK(cudaGetLastError());
      std::lock_guard<std::mutex> lk(s->mu);
      s->active.push_back(r);
    }
    // cancelled requests leave before the launches are built (the previous
    // iteration's launches have completed: the loop waited for them)
    {
      std::vector<std::shared_ptr<Request>> keep;
      std::vector<std::shared_ptr<Request>> gone;
      {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto& r : s->active) (r->cancel ? gone : keep).push_back(r);
      }
      for (auto& r : gone) {
        SRV_CK(cudaFreeAsync(r->dmem, s->stream));
        r->dmem = nullptr;
        s->pinned_free.emplace(r->host_cap, r->host_res);
        r->host_res = nullptr;
      }
      if (!gone.empty()) {
        std::lock_guard<std::mutex> lk(s->mu);
        for (auto& r : gone) {
          s->in_use -= r->dbytes;
          r->status = VQC_ERR_CANCELED;
          r->error = "request cancelled";
          r->t_done = now_s();
        }
        s->active.swap(keep);
        s->cv_done.notify_all();
      }
    }
    if (s->active.empty()) continue;
    // 2. one launch per step kind (and tile size) over every active request
    const double t_build = now_s();
    // tile items grouped by (tile size, direction, compiled kernel or the generic one)
    struct Group {
      std::vector<TileItem> items;
      std::vector<std::shared_ptr<Request>> reqs;
      std::vector<const PassLoc*> locs;
      unsigned char* d = nullptr;
    };
    std::map<std::tuple<int, int, const void*>, Group> groups;
    std::vector<RedItem> red_items;
    std::vector<PauliItem> p_items[2];  // [0] energy only, [1] energy + cotangent
    std::vector<PauliRed> p_red[2];
    for (auto& r : s->active) {
      const int F = r->nfwd();
      const unsigned char* img = r->dimg;
      if (r->step < F) {
        const PassLoc& l = r->plan.fwd.locs[r->step];
        const void* k = r->plan.fwd_k.empty() ? nullptr : r->plan.fwd_k[r->step];
        Group& g = groups[std::make_tuple(r->plan.M, 0, k)];
        g.items.push_back(TileItem{r->psi, nullptr, (const DevPass*)(img + l.pass), (const void*)(img + l.stages),
                                   (const DevOp*)(img + l.ops), img + r->plan.fwd.pool_off + l.pool_begin * amp,
                                   nullptr, l.ntiles, r->fwd_cap, 0});
        g.reqs.push_back(r);
        g.locs.push_back(&l);
      } else if (r->step == F) {
        const unsigned char* pt = img + r->off_pauli;
        p_items[r->grad].push_back(PauliItem{r->psi, r->lam, int64_t(1) << r->n, (const DevGroup*)pt, r->ng,
                                             (const DevTerm*)(pt + sizeof(DevGroup) * r->ng), r->nt, r->partials});
        p_red[r->grad].push_back(PauliRed{r->partials, 0, r->energy_dev});
      } else {
        const int st = r->step - F - 1;
        const PassLoc& l = r->plan.adj.locs[st];
        const unsigned char* ai = img + r->off_adj;
        const void* k = r->plan.adj_k.empty() ? nullptr : r->plan.adj_k[st];
        Group& g = groups[std::make_tuple(r->plan.M, 1, k)];
        g.items.push_back(TileItem{r->psi, r->lam, (const DevPass*)(ai + l.pass), (const void*)(ai + l.stages),
                                   (const DevOp*)(ai + l.ops), ai + r->plan.adj.pool_off + l.pool_begin * amp,
                                   r->partials, l.ntiles, r->adj_cap, 0});
        g.reqs.push_back(r);
        g.locs.push_back(&l);
        if (l.nslots > 0)
          red_items.push_back(RedItem{r->partials, r->adj_cap, l.nslots, r->rows + (size_t)l.row0 * 8});
      }
    }
    // stage every item array in one pinned buffer, one copy
    size_t need = 0;
    auto add = [&](size_t b) { need = ((need + 15) & ~size_t(15)) + b; };
    for (auto& kv : groups) add(sizeof(TileItem) * kv.second.items.size());
    add(sizeof(PauliItem) * p_items[0].size());
    add(sizeof(PauliItem) * p_items[1].size());
    int p_gridx = 0;
    size_t p_smem = 0;
    for (int v = 0; v < 2; ++v)
      for (size_t i = 0; i < p_items[v].size(); ++i) {
        const int64_t N = p_items[v][i].N;
        p_gridx = std::max(p_gridx, (int)std::min<int64_t>((N + kRedThreads - 1) / kRedThreads,
                                                           device_info(s->device).sms * 2));
        p_smem = std::max(p_smem, sizeof(DevGroup) * p_items[v][i].ng + sizeof(DevTerm) * p_items[v][i].nt);
      }
    for (int v = 0; v < 2; ++v)
      for (size_t i = 0; i < p_items[v].size(); ++i) {
        const int64_t N = p_items[v][i].N;
        p_red[v][i].nblocks = (int)std::min<int64_t>(p_gridx, (N + kRedThreads - 1) / kRedThreads);
      }
    add(sizeof(RedItem) * red_items.size());
    add(sizeof(PauliRed) * p_red[0].size());
    add(sizeof(PauliRed) * p_red[1].size());
    if (need > s->items_cap) {
      SRV_CK(cudaStreamSynchronize(s->stream));
      if (s->h_items) cudaFreeHost(s->h_items);
      if (s->d_items) cudaFree(s->d_items);
      s->items_cap = std::max<size_t>(need * 2, 1 << 16);
      SRV_CK(cudaMallocHost((void**)&s->h_items, s->items_cap));
      SRV_CK(cudaMalloc((void**)&s->d_items, s->items_cap));
    }
    size_t pos = 0;
    auto put = [&](const void* src, size_t b) {
      pos = (pos + 15) & ~size_t(15);
      const size_t o = pos;
      if (b) std::memcpy(s->h_items + o, src, b);
      pos += b;
      return s->d_items + o;
    };
    for (auto& kv : groups) kv.second.d = put(kv.second.items.data(), sizeof(TileItem) * kv.second.items.size());
    unsigned char* d_p[2];
    unsigned char* d_pred[2];
    for (int v = 0; v < 2; ++v) {
      d_p[v] = put(p_items[v].data(), sizeof(PauliItem) * p_items[v].size());
      d_pred[v] = put(p_red[v].data(), sizeof(PauliRed) * p_red[v].size());
    }
    unsigned char* d_red = put(red_items.data(), sizeof(RedItem) * red_items.size());
    SRV_CK(cudaMemcpyAsync(s->d_items, s->h_items, pos, cudaMemcpyHostToDevice, s->stream));
    long long nl = 0, ni = 0;
    // forward groups, the Pauli passes, then the reverse groups (a request takes one step per iteration)
    auto launch_groups = [&](int adj) -> bool {
      for (auto& kv : groups) {
        if (std::get<1>(kv.first) != adj) continue;
        const int M = std::get<0>(kv.first);
        const void* k = std::get<2>(kv.first);
        Group& g = kv.second;
        PassShape mx;
        mx.packed = k != nullptr;
        int gridx = 0;
        for (size_t i = 0; i < g.items.size(); ++i) {
          const PassShape& sh = g.locs[i]->shape;
          mx.nslots = std::max(mx.nslots, sh.nslots);
          mx.nstages = std::max(mx.nstages, sh.nstages);
          mx.nops = std::max(mx.nops, sh.nops);
          mx.npool = std::max(mx.npool, sh.npool);
          gridx = std::max(gridx, g.items[i].ncta);
        }
        const int rc = k ? serve_launch_jit(M, adj != 0, k, (const TileItem*)g.d, (int)g.items.size(), gridx, mx,
                                            s->stream)
                         : serve_launch_tiles(s->dtype, M, adj != 0, (const TileItem*)g.d, (int)g.items.size(),
                                              gridx, mx, s->stream);
        if (rc) {
          fail_all(s, vqc_last_error());
          return false;
        }
        ++nl;
        ni += (long long)g.items.size();
      }
      return true;
    };
    if (!launch_groups(0)) return;
    for (int v = 0; v < 2; ++v) {
      if (p_items[v].empty()) continue;
      if (serve_launch_pauli(s->dtype, v == 1, (const PauliItem*)d_p[v], (int)p_items[v].size(), p_gridx, p_smem,
                             s->stream) ||
          serve_launch_pauli_reduce((const PauliRed*)d_pred[v], (int)p_red[v].size(), s->stream)) {
        fail_all(s, vqc_last_error());
        return;
      }
      ++nl;
      ni += (long long)p_items[v].size();
    }
    if (!launch_groups(1)) return;
    if (!red_items.empty()) {
      int ms = 0;
      for (auto& it : red_items) ms = std::max(ms, it.nslots);
      if (serve_launch_reduce((const RedItem*)d_red, (int)red_items.size(), ms, s->stream)) {
        fail_all(s, vqc_last_error());
        return;
      }
    }
    // results of requests that finish with this step
    std::vector<std::shared_ptr<Request>> finishing;
    for (auto& r : s->active)
      if (r->step + 1 == r->nsteps()) {
        finishing.push_back(r);
        SRV_CK(cudaMemcpyAsync(r->host_res, r->energy_dev, 2 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
        if (r->grad && r->plan.adj.rows > 0)
          SRV_CK(cudaMemcpyAsync(r->host_res + 2, r->rows, sizeof(double) * 8 * r->plan.adj.rows,
                                 cudaMemcpyDeviceToHost, s->stream));
      }
    SRV_CK(cudaEventRecord(s->ev, s->stream));
    const double t_enqueued = now_s();
    SRV_CK(cudaEventSynchronize(s->ev));
    const double t_synced = now_s();
    // 3. retire
    std::vector<std::shared_ptr<Request>> still;
    for (auto& r : s->active) {
      if (r->step + 1 == r->nsteps()) {
        r->energy[0] = r->host_res[0];
        r->energy[1] = r->host_res[1];
        if (r->grad && r->grads_out) contract_grads(r->plan.accs, r->host_res + 2, r->grads_out);
        SRV_CK(cudaFreeAsync(r->dmem, s->stream));
        s->pinned_free.emplace(r->host_cap, r->host_res);
        r->host_res = nullptr;
        r->dmem = nullptr;
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use -= r->dbytes;
        r->t_done = now_s();
        if (r->cancel) {  // cancelled during its last step: the outcome is the cancellation
          r->status = VQC_ERR_CANCELED;
          r->error = "request cancelled";
          s->cv_done.notify_all();
          continue;
        }
        r->status = 3;
        ++s->completed;
        const double pl = r->t_planned - r->t_submit, wt = r->t_admit - r->t_planned, rn = r->t_done - r->t_admit;
        s->plan_s_sum += pl;
        s->wait_s_sum += wt;
        s->run_s_sum += rn;
        s->plan_s_max = std::max(s->plan_s_max, pl);
        s->wait_s_max = std::max(s->wait_s_max, wt);
        s->run_s_max = std::max(s->run_s_max, rn);
        s->cv_done.notify_all();
      } else {
        ++r->step;
        still.push_back(r);
      }
    }
    std::lock_guard<std::mutex> lk(s->mu);
    s->active.swap(still);
    if (nl > 0) {
      s->loop_build_s += t_enqueued - t_build;
      s->loop_wait_s += t_synced - t_enqueued;
      s->loop_retire_s += now_s() - t_synced;
      ++s->loop_busy;
    }
    ++s->iterations;
    s->launches += nl;
    s->items_launched += ni;
  }
}

}  // namespace vqc

using namespace vqc;

extern "C" {

int vqc_serve_open(int device, int dtype, size_t memory_bytes, int max_active, int planner_threads,
                   vqc_server* out) {
  if (!out) return fail(VQC_ERR_ARG, "null output");
  *out = nullptr;
  if (dtype != VQC_C64 && dtype != VQC_C128) return fail(VQC_ERR_ARG, "dtype must be VQC_C64 or VQC_C128");
  if (max_active < 1 || memory_bytes == 0) return fail(VQC_ERR_ARG, "budget and slot count must be positive");
  int ndev = 0;
  VQC_CK(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(VQC_ERR_ARG, "device index out of range");
  VQC_CK(cudaSetDevice(device));
  auto* s = new vqc_server_s();
  s->device = device;
  s->dtype = dtype;
  s->budget = memory_bytes;
  s->max_active = max_active;
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&s->ev, cudaEventDisableTiming)) != cudaSuccess) {
    delete s;
    return cuda_fail(e, "serving stream");
  }
  {
    // keep freed request memory in the stream-ordered pool instead of
    // returning it to the driver at every synchronisation
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t thr = UINT64_MAX;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
  }
  const int np = std::max(1, std::min(planner_threads, 16));
  for (int i = 0; i < np; ++i) s->planners.emplace_back(planner_main, s);
  s->worker = std::thread(worker_main, s);
  s->compiler = std::thread(compiler_main, s);
  *out = s;
  return VQC_OK;
}

int vqc_serve_submit(vqc_server s, int nqubits, const vqc_gate* gates, int ngates, const double* mats,
                     const vqc_param* params, int nparams, const vqc_pauli* terms, int nterms, int want_grad,
                     double* grads_out, int64_t* ticket) {
  if (!s || !ticket) return fail(VQC_ERR_ARG, "null server or ticket");
  if (ngates < 0 || (ngates > 0 && (!gates || !mats)) || nparams < 0 || (nparams > 0 && !params) || nterms < 0 ||
      (nterms > 0 && !terms))
    return fail(VQC_ERR_ARG, "bad request arrays");
  if (want_grad && nparams > 0 && !grads_out) return fail(VQC_ERR_ARG, "gradient requests need an output array");
  auto r = std::make_shared<Request>();
  r->n = nqubits;
  r->grad = want_grad != 0;
  r->gates.assign(gates, gates + ngates);
  size_t mlen = 0;
  for (int i = 0; i < ngates; ++i) {
    if (gates[i].nq < 1 || gates[i].nq > 5 || gates[i].mat < 0) return fail(VQC_ERR_ARG, "bad gate");
    mlen = std::max(mlen, (size_t)gates[i].mat + ((size_t)2 << (2 * gates[i].nq)));
  }
  for (int j = 0; j < nparams; ++j) {
    if (params[j].gate < 0 || params[j].gate >= ngates || params[j].dmat < 0) return fail(VQC_ERR_ARG, "bad parameter");
    mlen = std::max(mlen, (size_t)params[j].dmat + ((size_t)2 << (2 * gates[params[j].gate].nq)));
  }
  // a poisoned request (a NaN or infinite matrix entry or coefficient) is
  // turned away here: it never reaches the device or the batch
  for (size_t i = 0; i < mlen; ++i)
    if (!std::isfinite(mats[i])) return fail(VQC_ERR_ARG, "request has a non-finite gate or derivative matrix entry");
  for (int t = 0; t < nterms; ++t)
    if (!std::isfinite(terms[t].coeff_re) || !std::isfinite(terms[t].coeff_im))
      return fail(VQC_ERR_ARG, "request has a non-finite Pauli coefficient");
  r->mats.assign(mats, mats + mlen);
  if (r->grad) r->params.assign(params, params + nparams);
  r->terms.assign(terms, terms + nterms);
  r->grads_out = grads_out;
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->fatal.empty()) return fail(VQC_ERR_CUDA, s->fatal);
  r->ticket = s->next_ticket++;
  r->t_submit = now_s();
  s->all[r->ticket] = r;
  s->to_plan.push_back(r);
  s->cv_plan.notify_one();
  *ticket = r->ticket;
  return VQC_OK;
}

static int finish_ticket(vqc_server s, std::map<int64_t, std::shared_ptr<Request>>::iterator it, double* energy,
                         double* latency_s) {
  auto r = it->second;
  if (r->status < 0) {
    const int rc = r->status;
    set_error(r->error);
    s->all.erase(it);
    return rc;
  }
  if (energy) {
    energy[0] = r->energy[0];
    energy[1] = r->energy[1];
  }
  if (latency_s) *latency_s = r->t_done - r->t_submit;
  s->all.erase(it);
  return 1;
}

int vqc_serve_poll(vqc_server s, int64_t ticket, double* energy, double* latency_s) {
  if (!s) return fail(VQC_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return fail(VQC_ERR_ARG, "unknown ticket");
  if (it->second->status >= 0 && it->second->status != 3) return 0;
  return finish_ticket(s, it, energy, latency_s);
}

int vqc_serve_wait(vqc_server s, int64_t ticket, int timeout_ms, double* energy, double* latency_s) {
  if (!s) return fail(VQC_ERR_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return fail(VQC_ERR_ARG, "unknown ticket");
  auto r = it->second;
  const bool done = s->cv_done.wait_for(lk, std::chrono::milliseconds(std::max(timeout_ms, 0)),
                                        [&] { return r->status < 0 || r->status == 3; });
  if (!done) return fail(VQC_ERR_TIMEOUT, "request not finished within the timeout");
  return finish_ticket(s, s->all.find(ticket), energy, latency_s);
}

int vqc_serve_cancel(vqc_server s, int64_t ticket) {
  if (!s) return fail(VQC_ERR_ARG, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) return fail(VQC_ERR_ARG, "unknown ticket");
  auto r = it->second;
  if (r->status == 3 || r->status < 0) return 0;
  r->cancel = true;
  if (r->status == 0 || r->status == 1) {
    // not admitted: drop it from the queues now
    for (auto* q : {&s->to_plan, &s->ready}) {
      auto p = std::find(q->begin(), q->end(), r);
      if (p != q->end()) q->erase(p);
    }
    r->status = VQC_ERR_CANCELED;
    r->error = "request cancelled";
    r->t_done = now_s();
    s->cv_done.notify_all();
  }
  return 1;
}

int vqc_serve_stats(vqc_server s, long long* out) {
  if (!s || !out) return fail(VQC_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out[0] = s->completed;
  out[1] = s->iterations;
  out[2] = s->launches;
  out[3] = s->items_launched;
  out[4] = (long long)s->in_use;
  out[5] = (long long)s->active.size();
  out[6] = (long long)s->ready.size() + (long long)s->to_plan.size();
  return VQC_OK;
}

int vqc_serve_timing(vqc_server s, double* out) {
  if (!s || !out) return fail(VQC_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  const double n = (double)std::max<long long>(s->completed, 1);
  out[0] = s->plan_s_sum / n;
  out[1] = s->plan_s_max;
  out[2] = s->wait_s_sum / n;
  out[3] = s->wait_s_max;
  out[4] = s->run_s_sum / n;
  out[5] = s->run_s_max;
  return VQC_OK;
}

int vqc_serve_loop_timing(vqc_server s, double* out) {
  if (!s || !out) return fail(VQC_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  out[0] = s->loop_build_s;
  out[1] = s->loop_wait_s;
  out[2] = s->loop_retire_s;
  out[3] = (double)s->loop_busy;
  return VQC_OK;
}

int vqc_serve_close(vqc_server s) {
  if (!s) return VQC_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv_plan.notify_all();
    s->cv_ready.notify_all();
    s->cv_build.notify_all();
  }
  for (auto& t : s->planners) t.join();
  if (s->worker.joinable()) s->worker.join();
  if (s->compiler.joinable()) s->compiler.join();  // (finishes the compile in progress)
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->stream);
  for (auto& r : s->active) {
    if (r->dmem) cudaFreeAsync(r->dmem, s->stream);
    if (r->host_res) cudaFreeHost(r->host_res);
  }
  cudaStreamSynchronize(s->stream);
  if (s->h_items) cudaFreeHost(s->h_items);
  if (s->d_items) cudaFree(s->d_items);
  for (auto& kv : s->pinned_free) cudaFreeHost(kv.second);
  cudaEventDestroy(s->ev);
  cudaStreamDestroy(s->stream);
  delete s;
  return VQC_OK;
}

}  // extern "C"
