// apply!(::Gate, ::StateVector) and apply!(::QCircuit, state) on the device.
//
// Reference: applygates/generic/generic.jl:6-14 (front end, range check,
// <=5 qubits), :26-31 (circuit loop), the dense k-qubit loops of
// threaded_short_range.jl / threaded_long_range.jl and the specialised
// kernels of applygates/specific/*.jl.  One kernel family covers all of them:
// the gate's active subspace (engine.h) is applied per group of amplitudes,
// so diagonal gates touch only their non-unit entries and controlled gates
// only their controlled block, as the reference's specialised kernels do.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "subspace.cuh"

namespace vqc {

int order_matrix(int n, int k, const int* pos, const double* mat, int* sp, std::vector<cd>& M) {
  if (k < 1) return fail(VQC_ERR_ARG, "gate needs at least one position");
  if (k > 5) return fail(VQC_ERR_UNSUPPORTED, "only implement 5-qubit gates and less currently.");
  if (!pos || !mat) return fail(VQC_ERR_ARG, "null positions or matrix");
  int perm[5];
  for (int i = 0; i < k; ++i) {
    if (pos[i] < 0 || pos[i] >= n) return fail(VQC_ERR_ARG, "gate position out of range");
    int j = i;
    for (; j > 0 && pos[perm[j - 1]] > pos[i]; --j) perm[j] = perm[j - 1];
    perm[j] = i;
  }
  for (int i = 0; i < k; ++i) {
    sp[i] = pos[perm[i]];
    if (i && sp[i] == sp[i - 1]) return fail(VQC_ERR_ARG, "duplicate gate positions");
  }
  const int d = 1 << k;
  auto remap = [&](int rs) {
    int r = 0;
    for (int i = 0; i < k; ++i)
      if (rs >> i & 1) r |= 1 << perm[i];
    return r;
  };
  M.assign((size_t)d * d, cd(0));
  for (int rs = 0; rs < d; ++rs) {
    const int r = remap(rs);
    for (int cs = 0; cs < d; ++cs) {
      const int c = remap(cs);
      M[(size_t)rs * d + cs] = cd(mat[2 * ((size_t)r * d + c)], mat[2 * ((size_t)r * d + c) + 1]);
    }
  }
  return VQC_OK;
}

int analyze_gate(int n, int k, const int* pos, const double* mat, bool dagger, GateSpec& g) {
  int rc = order_matrix(n, k, pos, mat, g.sp, g.U);
  if (rc) return rc;
  g.k = k;
  const int d = 1 << k;
  for (int i = 0; i < d * d; ++i)
    if (!std::isfinite(g.U[i].real()) || !std::isfinite(g.U[i].imag()))
      return fail(VQC_ERR_ARG, "gate matrix has a non-finite entry");
  if (dagger) {
    std::vector<cd> T((size_t)d * d);
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c) T[(size_t)r * d + c] = std::conj(g.U[(size_t)c * d + r]);
    g.U.swap(T);
  }
  g.ns = 0;
  for (int j = 0; j < d; ++j) {
    bool inactive = g.U[(size_t)j * d + j] == cd(1, 0);
    for (int c = 0; c < d && inactive; ++c)
      if (c != j && (g.U[(size_t)j * d + c] != cd(0) || g.U[(size_t)c * d + j] != cd(0))) inactive = false;
    if (!inactive) g.S[g.ns++] = j;
  }
  g.US.assign((size_t)g.ns * g.ns, cd(0));
  bool diag = true, mono = true;
  for (int a = 0; a < g.ns; ++a) {
    int nz = 0;
    for (int b = 0; b < g.ns; ++b) {
      cd u = g.U[(size_t)g.S[a] * d + g.S[b]];
      g.US[(size_t)a * g.ns + b] = u;
      if (u != cd(0)) {
        ++nz;
        g.mono_src[a] = b;
        if (a != b) diag = false;
      }
    }
    if (nz != 1) mono = false;
  }
  g.mode = diag && mono ? kDiag : (mono ? kMono : kDense);
  return VQC_OK;
}

template <class R, int MS, int MODE>
__global__ void __launch_bounds__(256) k_gate_sub(cplx<R>* __restrict__ v, const __grid_constant__ SubArgs<R, MS> a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.ngroups; g += stride) {
    const int64_t base = group_base(g, a.k, a.mask);
    cplx<R> x[MS];
    if (MODE == kDense) {
#pragma unroll
      for (int s = 0; s < MS; ++s)
        if (s < a.ns && VQC_DCHECK(base + a.off[s], a.namp)) x[s] = v[base + a.off[s]];
#pragma unroll
      for (int r = 0; r < MS; ++r) {
        if (r < a.ns) {
          cplx<R> acc = mkc<R>(R(0), R(0));
#pragma unroll
          for (int c = 0; c < MS; ++c)
            if (c < a.ns) acc = cfma(a.U[r * MS + c], x[c], acc);
          if (VQC_DCHECK(base + a.off[r], a.namp)) v[base + a.off[r]] = acc;
        }
      }
    } else if (MODE == kDiag) {
#pragma unroll
      for (int s = 0; s < MS; ++s)
        if (s < a.ns && VQC_DCHECK(base + a.off[s], a.namp)) v[base + a.off[s]] = cmul(a.U[s], v[base + a.off[s]]);
    } else {
#pragma unroll
      for (int s = 0; s < MS; ++s)
        if (s < a.ns && VQC_DCHECK(base + a.src_off[s], a.namp)) x[s] = v[base + a.src_off[s]];
#pragma unroll
      for (int s = 0; s < MS; ++s)
        if (s < a.ns && VQC_DCHECK(base + a.off[s], a.namp)) v[base + a.off[s]] = cmul(a.U[s], x[s]);
    }
  }
}

template <class R, int MS>
static int launch_ms(const GateSpec& g, void* v, int nq, int device, cudaStream_t stream) {
  SubArgs<R, MS> a;
  fill_sub_args<R, MS>(g, nq, a);
  const int grid = launch_grid(device, a.ngroups);
  ProfScope prof(stream, g.mode == kDense ? "gate_dense" : (g.mode == kDiag ? "gate_diag" : "gate_perm"),
                 2.0 * a.ngroups * g.ns * sizeof(cplx<R>));
  if (g.mode == kDense)
    k_gate_sub<R, MS, kDense><<<grid, 256, 0, stream>>>((cplx<R>*)v, a);
  else if (g.mode == kDiag)
    k_gate_sub<R, MS, kDiag><<<grid, 256, 0, stream>>>((cplx<R>*)v, a);
  else
    k_gate_sub<R, MS, kMono><<<grid, 256, 0, stream>>>((cplx<R>*)v, a);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

template <class R>
static int launch_r(const GateSpec& g, void* v, int nq, int device, cudaStream_t stream) {
  switch (ms_of(g.ns)) {
    case 1: return launch_ms<R, 1>(g, v, nq, device, stream);
    case 2: return launch_ms<R, 2>(g, v, nq, device, stream);
    case 4: return launch_ms<R, 4>(g, v, nq, device, stream);
    case 8: return launch_ms<R, 8>(g, v, nq, device, stream);
    case 16: return launch_ms<R, 16>(g, v, nq, device, stream);
    default: return launch_ms<R, 32>(g, v, nq, device, stream);
  }
}

int launch_gate(const GateSpec& g, void* v, int nq, int dtype, int device, cudaStream_t stream) {
  if (g.ns == 0) return VQC_OK;  // identity
  return dtype == VQC_C64 ? launch_r<float>(g, v, nq, device, stream) : launch_r<double>(g, v, nq, device, stream);
}

int apply_gate_raw(vqc_state h, int k, const int* pos, const double* mat) {
  GateSpec g;
  int rc = analyze_gate(h->nq, k, pos, mat, false, g);
  if (rc) return rc;
  return launch_gate(g, h->d, h->nq, h->dtype, h->device, h->stream);
}

int apply_circuit_raw(vqc_state h, const vqc_gate* gates, int ngates, const double* mats, bool dm, int fuse) {
  if (ngates < 0 || (ngates > 0 && (!gates || !mats))) return fail(VQC_ERR_ARG, "bad circuit arrays");
  if (fuse && !dm) return apply_circuit_fused(h, gates, ngates, mats);
  if (fuse && dm) {
    // rho <- U rho U^dagger is U on the row qubits and conj(U) on the column
    // qubits (generic.jl:54-64); as gates of the 2n-qubit vector both go to the
    // tile engine, which applies them (and the neighbouring gates) in one pass.
    const int n = h->n_dm;
    std::vector<vqc_gate> g2;
    std::vector<double> m2;
    g2.reserve(2 * (size_t)ngates);
    for (int i = 0; i < ngates; ++i) {
      const vqc_gate& gt = gates[i];
      if (gt.nq < 1) return fail(VQC_ERR_ARG, "gate needs at least one position");
      if (gt.nq > 5) return fail(VQC_ERR_UNSUPPORTED, "only implement 5-qubit gates and less currently.");
      const size_t len = (size_t)2 << (2 * gt.nq);
      vqc_gate a = gt, b = gt;
      for (int j = 0; j < gt.nq; ++j) {
        if (gt.pos[j] < 0 || gt.pos[j] >= n) return fail(VQC_ERR_ARG, "gate position out of range");
        b.pos[j] = gt.pos[j] + n;
      }
      a.mat = (int64_t)m2.size();
      m2.insert(m2.end(), mats + gt.mat, mats + gt.mat + len);
      b.mat = (int64_t)m2.size();
      for (size_t e = 0; e < len; ++e) m2.push_back(e & 1 ? -mats[gt.mat + e] : mats[gt.mat + e]);
      g2.push_back(a);
      g2.push_back(b);
    }
    return apply_circuit_fused(h, g2.data(), (int)g2.size(), m2.data());
  }
  for (int i = 0; i < ngates; ++i) {
    const vqc_gate& gt = gates[i];
    int rc = dm ? dm_apply_gate_raw(h, gt.nq, gt.pos, mats + gt.mat) : apply_gate_raw(h, gt.nq, gt.pos, mats + gt.mat);
    if (rc) return rc;
  }
  return VQC_OK;
}

}  // namespace vqc

using namespace vqc;

extern "C" {

int vqc_apply_gate(vqc_state h, int k, const int* pos, const double* mat) {
  int rc = enter(h);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(h->mu);
  return apply_gate_raw(h, k, pos, mat);
}

int vqc_apply_circuit(vqc_state h, const vqc_gate* gates, int ngates, const double* mats, int fuse) {
  int rc = enter(h);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(h->mu);
  return apply_circuit_raw(h, gates, ngates, mats, false, fuse);
}

int vqc_dm_apply_circuit(vqc_state h, const vqc_gate* gates, int ngates, const double* mats, int fuse) {
  int rc = enter(h);
  if (rc) return rc;
  if (!h->n_dm) return fail(VQC_ERR_ARG, "not a density matrix");
  std::lock_guard<std::mutex> lk(h->mu);
  return apply_circuit_raw(h, gates, ngates, mats, true, fuse);
}

}  // extern "C"
