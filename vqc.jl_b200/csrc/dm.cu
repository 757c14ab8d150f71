// Density matrices: DensityMatrix{T} (densitymatrix.jl:1-30), the unitary
// gate rho <- U rho U^dagger (applygates/generic/generic.jl:16-24, 54-64),
// partial_tr (ptrace.jl:4-53), basis probabilities (measure.jl:69-81;
// real(diag(storage(rho)))) and tr (densitymatrix.jl:58).
//
// rho of n qubits is the 2n-qubit vector of its column-major storage: bit q
// (q < n) of the flat index is row qubit q, bit n + q is column qubit q.
// The reference applies U on the row qubits and conj(U) on the column qubits
// in two passes; for k <= 2 this file applies W = conj(U) (x) U on the 2k
// positions (pos, pos + n) in ONE pass (half the HBM traffic), and in two
// passes for k >= 3 (W would exceed the 5-qubit kernel limit).
#include <algorithm>
#include <mutex>

#include "engine.h"
#include "subspace.cuh"

namespace vqc {

int dm_apply_gate_raw(vqc_state h, int k, const int* pos, const double* mat) {
  const int n = h->n_dm;
  if (k < 1) return fail(VQC_ERR_ARG, "gate needs at least one position");
  if (k > 5) return fail(VQC_ERR_UNSUPPORTED, "only implement 5-qubit gates and less currently.");
  if (!pos || !mat) return fail(VQC_ERR_ARG, "null positions or matrix");
  for (int i = 0; i < k; ++i)
    if (pos[i] < 0 || pos[i] >= n) return fail(VQC_ERR_ARG, "gate position out of range");
  const int d = 1 << k;
  if (2 * k <= 5) {
    const int D = d * d;
    std::vector<double> W((size_t)2 * D * D);
    for (int r2 = 0; r2 < d; ++r2)
      for (int r1 = 0; r1 < d; ++r1)
        for (int c2 = 0; c2 < d; ++c2)
          for (int c1 = 0; c1 < d; ++c1) {
            const cd u(mat[2 * (r1 * d + c1)], mat[2 * (r1 * d + c1) + 1]);
            const cd v(mat[2 * (r2 * d + c2)], mat[2 * (r2 * d + c2) + 1]);
            const cd w = u * std::conj(v);
            const size_t idx = (size_t)(r1 + d * r2) * D + (c1 + d * c2);
            W[2 * idx] = w.real();
            W[2 * idx + 1] = w.imag();
          }
    int p2[10];
    for (int i = 0; i < k; ++i) {
      p2[i] = pos[i];
      p2[k + i] = pos[i] + n;
    }
    return apply_gate_raw(h, 2 * k, p2, W.data());
  }
  int rc = apply_gate_raw(h, k, pos, mat);
  if (rc) return rc;
  std::vector<double> Uc((size_t)2 * d * d);
  for (size_t i = 0; i < (size_t)d * d; ++i) {
    Uc[2 * i] = mat[2 * i];
    Uc[2 * i + 1] = -mat[2 * i + 1];
  }
  int p2[5];
  for (int i = 0; i < k; ++i) p2[i] = pos[i] + n;
  return apply_gate_raw(h, k, p2, Uc.data());
}

// rho[r + L c] = psi[r] conj(psi[c])
template <class R>
__global__ void k_dm_from_state(cplx<R>* rho, const cplx<R>* psi, int n) {
  const int64_t L = int64_t(1) << n, N = L * L;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    const cplx<R> a = psi[i & (L - 1)], b = psi[i >> n];
    rho[i] = mkc<R>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
  }
}

// deposit the low bits of v into the set bits of mask
__device__ __forceinline__ int64_t deposit(int64_t v, uint64_t mask) {
  int64_t r = 0;
  while (mask) {
    const uint64_t low = mask & (~mask + 1);
    if (v & 1) r |= (int64_t)low;
    v >>= 1;
    mask ^= low;
  }
  return r;
}

// out[a + s1 b] = sum_c rho[(K(a)|T(c)) + L (K(b)|T(c))], FP64 accumulation.
template <class R>
__global__ void k_dm_ptrace(const cplx<R>* __restrict__ rho, int n, uint64_t kept, uint64_t traced, int nk, int nt,
                            double2* __restrict__ out) {
  const int64_t L = int64_t(1) << n, s1 = int64_t(1) << nk, s2 = int64_t(1) << nt;
  for (int64_t o = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; o < s1 * s1; o += (int64_t)gridDim.x * blockDim.x) {
    const int64_t a = o & (s1 - 1), b = o >> nk;
    const int64_t ra = deposit(a, kept), cb = deposit(b, kept);
    double2 acc = make_double2(0, 0);
    for (int64_t c = 0; c < s2; ++c) {
      const int64_t t = deposit(c, traced);
      if (!VQC_DCHECK((ra | t) + L * (cb | t), L * L)) continue;
      const double2 v = to_d2(rho[(ra | t) + L * (cb | t)]);
      acc.x += v.x;
      acc.y += v.y;
    }
    out[o] = acc;
  }
}

template <class R>
__global__ void k_dm_diag(const cplx<R>* __restrict__ rho, int n, double* __restrict__ out) {
  const int64_t L = int64_t(1) << n;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)rho[i + L * i].x;
}

template <class R>
__global__ void __launch_bounds__(kRedThreads) k_dm_trace(const cplx<R>* __restrict__ rho, int n, Scratch s) {
  const int64_t L = int64_t(1) << n;
  double acc[2] = {0, 0};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x) {
    const double2 v = to_d2(rho[i + L * i]);
    acc[0] += v.x;
    acc[1] += v.y;
  }
  grid_reduce<2>(acc, s, s.result);
}

// tr(op(A) M op(B)) for two density matrices (circuitdiff.jl:35-40, the
// expectation(x::DensityMatrix, m::Gate, y::DensityMatrix) of the DM
// pullback): M is a K-qubit operator on the row index (left
// multiplication), op = identity or the conjugate transpose.  Work item =
// (column j, row group r0 with the K target bits clear):
//   (M B)[r_s][j] = sum_t M[s][t] B[r_t][j],  sum_s A[j][r_s] (M B)[r_s][j].
// FP64 accumulation and grid reduction.
template <int K>
struct TraceProdArgs {
  double2 M[(1 << K) * (1 << K)];  // sorted-position order, row-major
  int64_t off[1 << K];             // row offset of target pattern t
  int sp[K];                       // sorted target bits
};

template <class R, int K>
__global__ void __launch_bounds__(kRedThreads)
    k_dm_trace_prod(const cplx<R>* __restrict__ a, const cplx<R>* __restrict__ b, int n, int dag_a, int dag_b,
                    const __grid_constant__ TraceProdArgs<K> g, Scratch s, double* res) {
  constexpr int D = 1 << K;
  const int64_t N = int64_t(1) << n, rows = N >> K, items = rows << n;
  double acc[2] = {0, 0};
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < items; it += (int64_t)gridDim.x * blockDim.x) {
    const int64_t j = it >> (n - K);
    int64_t r0 = it & (rows - 1);
#pragma unroll
    for (int q = 0; q < K; ++q) r0 = ((r0 >> g.sp[q]) << (g.sp[q] + 1)) | (r0 & ((int64_t(1) << g.sp[q]) - 1));
    double2 bv[D];
#pragma unroll
    for (int t = 0; t < D; ++t) {
      const int64_t r = r0 + g.off[t];
      if (!VQC_DCHECK(r + N * j, N * N) || !VQC_DCHECK(j + N * r, N * N)) {
        bv[t] = make_double2(0, 0);
        continue;
      }
      bv[t] = dag_b ? to_d2(b[j + N * r]) : to_d2(b[r + N * j]);
      if (dag_b) bv[t].y = -bv[t].y;
    }
#pragma unroll
    for (int q = 0; q < D; ++q) {
      double2 mb = make_double2(0, 0);
#pragma unroll
      for (int t = 0; t < D; ++t) mb = cfma(g.M[q * D + t], bv[t], mb);
      const int64_t r = r0 + g.off[q];
      double2 av = dag_a ? to_d2(a[r + N * j]) : to_d2(a[j + N * r]);
      if (dag_a) av.y = -av.y;
      acc[0] = fma(av.x, mb.x, fma(-av.y, mb.y, acc[0]));
      acc[1] = fma(av.x, mb.y, fma(av.y, mb.x, acc[1]));
    }
  }
  grid_reduce<2>(acc, s, res);
}

template <int K>
static int trace_prod_k(vqc_state a, vqc_state b, int dag_a, int dag_b, const int* sp, const std::vector<cd>& M,
                        double* out) {
  TraceProdArgs<K> g;
  for (int i = 0; i < (1 << K) * (1 << K); ++i) g.M[i] = make_double2(M[i].real(), M[i].imag());
  for (int q = 0; q < K; ++q) g.sp[q] = sp[q];
  for (int t = 0; t < (1 << K); ++t) g.off[t] = offset_of(t, K, sp);
  const int n = b->n_dm;
  const int grid = reduction_grid(b->device, (int64_t(1) << (2 * n - K)));
  ProfScope prof(b->stream, "dm_trace_prod", 2.0 * (double)b->size() * b->amp_bytes());
  if (b->dtype == VQC_C64)
    k_dm_trace_prod<float, K><<<grid, kRedThreads, 0, b->stream>>>((const float2*)a->d, (const float2*)b->d, n, dag_a,
                                                                    dag_b, g, b->scr, b->scr.result);
  else
    k_dm_trace_prod<double, K><<<grid, kRedThreads, 0, b->stream>>>((const double2*)a->d, (const double2*)b->d, n,
                                                                     dag_a, dag_b, g, b->scr, b->scr.result);
  VQC_CK(cudaGetLastError());
  int rc = fetch_result(b, 2);
  if (rc) return rc;
  out[0] = b->h_result[0];
  out[1] = b->h_result[1];
  return VQC_OK;
}

// The superoperator of a channel rho -> sum_i K_i rho K_i^dagger on k qubits
// (apply_qmaps.jl:67-77): the 2k-qubit gate on the vectorised rho over the
// positions (pos..., pos + n), index J = r + 2^k c (r: row bits, c: column
// bits), S[(r, c), (r', c')] = sum_i K_i[r][r'] conj(K_i[c][c']).  mode 1:
// S^dagger (apply_dagger!), mode 2: S^-1 (apply_inverse!).
static int channel_supermatrix(int k, int nkraus, const double* kraus, int mode, std::vector<cd>& S) {
  const int d = 1 << k, D = d * d;
  S.assign((size_t)D * D, cd(0));
  for (int i = 0; i < nkraus; ++i) {
    const double* K = kraus + (size_t)i * d * d * 2;
    auto at = [&](int r, int c) { return cd(K[(r * d + c) * 2], K[(r * d + c) * 2 + 1]); };
    for (int r = 0; r < d; ++r)
      for (int c = 0; c < d; ++c)
        for (int r2 = 0; r2 < d; ++r2)
          for (int c2 = 0; c2 < d; ++c2) S[(size_t)(r + d * c) * D + (r2 + d * c2)] += at(r, r2) * std::conj(at(c, c2));
  }
  if (mode == 1) {
    std::vector<cd> T(S.size());
    for (int a = 0; a < D; ++a)
      for (int b = 0; b < D; ++b) T[(size_t)a * D + b] = std::conj(S[(size_t)b * D + a]);
    S.swap(T);
  } else if (mode == 2) {  // Gauss-Jordan with partial pivoting, FP64
    std::vector<cd> A = S, I((size_t)D * D, cd(0));
    for (int a = 0; a < D; ++a) I[(size_t)a * D + a] = 1;
    double scale = 0;
    for (const cd& x : A) scale = std::max(scale, std::abs(x));
    for (int col = 0; col < D; ++col) {
      int piv = col;
      for (int r = col + 1; r < D; ++r)
        if (std::abs(A[(size_t)r * D + col]) > std::abs(A[(size_t)piv * D + col])) piv = r;
      if (std::abs(A[(size_t)piv * D + col]) <= 1e-13 * std::max(scale, 1e-300))
        return fail(VQC_ERR_ARG, "apply_inverse!: the channel's supermatrix is singular");
      if (piv != col)
        for (int c = 0; c < D; ++c) {
          std::swap(A[(size_t)piv * D + c], A[(size_t)col * D + c]);
          std::swap(I[(size_t)piv * D + c], I[(size_t)col * D + c]);
        }
      const cd inv = cd(1) / A[(size_t)col * D + col];
      for (int c = 0; c < D; ++c) {
        A[(size_t)col * D + c] *= inv;
        I[(size_t)col * D + c] *= inv;
      }
      for (int r = 0; r < D; ++r) {
        if (r == col) continue;
        const cd f = A[(size_t)r * D + col];
        if (f == cd(0)) continue;
        for (int c = 0; c < D; ++c) {
          A[(size_t)r * D + c] -= f * A[(size_t)col * D + c];
          I[(size_t)r * D + c] -= f * I[(size_t)col * D + c];
        }
      }
    }
    S.swap(I);
  }
  return VQC_OK;
}

}  // namespace vqc

using namespace vqc;

extern "C" {

int vqc_dm_trace_prod(vqc_state a, int dag_a, vqc_state b, int dag_b, int k, const int* pos, const double* mat,
                      double* out) {
  int rc = enter(b);
  if (rc) return rc;
  if (!a || !a->n_dm || !b->n_dm || a->n_dm != b->n_dm || a->dtype != b->dtype || a->device != b->device)
    return fail(VQC_ERR_ARG, "tr(A M B): two density matrices of the same size, dtype and device");
  if (!out || !pos || !mat) return fail(VQC_ERR_ARG, "null argument");
  if (k < 1 || k > 5) return fail(VQC_ERR_UNSUPPORTED, "only implement 5-qubit gates and less currently.");
  if (k > b->n_dm) return fail(VQC_ERR_ARG, "operator wider than the register");
  int sp[5];
  std::vector<cd> M;
  if ((rc = order_matrix(b->n_dm, k, pos, mat, sp, M))) return rc;
  std::lock_guard<std::mutex> lk(b->mu);
  std::unique_lock<std::mutex> la(a->mu, std::defer_lock);
  if (a != b) la.lock();
  if (a != b && (rc = stream_after(b, a))) return rc;
  switch (k) {
    case 1: rc = trace_prod_k<1>(a, b, dag_a, dag_b, sp, M, out); break;
    case 2: rc = trace_prod_k<2>(a, b, dag_a, dag_b, sp, M, out); break;
    case 3: rc = trace_prod_k<3>(a, b, dag_a, dag_b, sp, M, out); break;
    case 4: rc = trace_prod_k<4>(a, b, dag_a, dag_b, sp, M, out); break;
    default: rc = trace_prod_k<5>(a, b, dag_a, dag_b, sp, M, out); break;
  }
  if (rc) return rc;
  return a != b ? stream_after(a, b) : VQC_OK;
}

int vqc_dm_apply_channel(vqc_state rho, int k, const int* pos, int nkraus, const double* kraus, int mode) {
  int rc = enter(rho);
  if (rc) return rc;
  if (!rho->n_dm) return fail(VQC_ERR_ARG, "not a density matrix");
  if (k < 1 || k > 2)
    return fail(VQC_ERR_UNSUPPORTED, "channels on 1 or 2 qubits (the supermatrix is a gate on 2k <= 5 qubits)");
  if (!pos || !kraus || nkraus < 1) return fail(VQC_ERR_ARG, "channel: null positions or no Kraus operators");
  if (mode < 0 || mode > 2) return fail(VQC_ERR_ARG, "channel: mode must be 0 (apply), 1 (dagger) or 2 (inverse)");
  for (int i = 0; i < k; ++i) {
    if (pos[i] < 0 || pos[i] >= rho->n_dm) return fail(VQC_ERR_ARG, "channel position out of range");
    for (int j = 0; j < i; ++j)
      if (pos[i] == pos[j]) return fail(VQC_ERR_ARG, "duplicate channel positions");
  }
  std::vector<cd> S;
  if ((rc = channel_supermatrix(k, nkraus, kraus, mode, S))) return rc;
  std::vector<double> m(S.size() * 2);
  for (size_t i = 0; i < S.size(); ++i) {
    m[2 * i] = S[i].real();
    m[2 * i + 1] = S[i].imag();
  }
  int all[4];
  for (int i = 0; i < k; ++i) {
    all[i] = pos[i];
    all[k + i] = pos[i] + rho->n_dm;
  }
  std::lock_guard<std::mutex> lk(rho->mu);
  return apply_gate_raw(rho, 2 * k, all, m.data());
}


int vqc_dm_from_state(vqc_state rho, vqc_state psi) {
  int rc = enter(rho);
  if (rc) return rc;
  if (!rho->n_dm || !psi || psi->n_dm || psi->nq != rho->n_dm || psi->dtype != rho->dtype || psi->device != rho->device)
    return fail(VQC_ERR_ARG, "DensityMatrix(psi): shapes, dtypes or devices differ");
  std::lock_guard<std::mutex> lk(rho->mu);
  if ((rc = stream_after(rho, psi))) return rc;
  const int g = launch_grid(rho->device, rho->size());
  if (rho->dtype == VQC_C64)
    k_dm_from_state<float><<<g, 256, 0, rho->stream>>>((float2*)rho->d, (const float2*)psi->d, rho->n_dm);
  else
    k_dm_from_state<double><<<g, 256, 0, rho->stream>>>((double2*)rho->d, (const double2*)psi->d, rho->n_dm);
  VQC_CK(cudaGetLastError());
  return stream_after(psi, rho);
}

int vqc_dm_apply_gate(vqc_state rho, int k, const int* pos, const double* mat) {
  int rc = enter(rho);
  if (rc) return rc;
  if (!rho->n_dm) return fail(VQC_ERR_ARG, "not a density matrix");
  std::lock_guard<std::mutex> lk(rho->mu);
  return dm_apply_gate_raw(rho, k, pos, mat);
}

int vqc_dm_ptrace(vqc_state rho, int nsites, const int* sites, double* out) {
  int rc = enter(rho);
  if (rc) return rc;
  const int n = rho->n_dm;
  if (!n) return fail(VQC_ERR_ARG, "not a density matrix");
  if (!out || nsites < 0 || nsites > n || (nsites > 0 && !sites)) return fail(VQC_ERR_ARG, "bad sites");
  uint64_t traced = 0;
  for (int i = 0; i < nsites; ++i) {
    if (sites[i] < 0 || sites[i] >= n) return fail(VQC_ERR_ARG, "site out of range.");
    if (traced >> sites[i] & 1) return fail(VQC_ERR_ARG, "duplicate sites not allowed.");
    traced |= 1ull << sites[i];
  }
  const uint64_t kept = ((n >= 64) ? ~0ull : ((1ull << n) - 1)) & ~traced;
  const int nk = n - nsites;
  const int64_t s1 = int64_t(1) << nk;
  std::lock_guard<std::mutex> lk(rho->mu);
  double2* dout = nullptr;
  VQC_CK(cudaMallocAsync((void**)&dout, sizeof(double2) * s1 * s1, rho->stream));
  const int g = launch_grid(rho->device, s1 * s1);
  if (rho->dtype == VQC_C64)
    k_dm_ptrace<float><<<g, 256, 0, rho->stream>>>((const float2*)rho->d, n, kept, traced, nk, nsites, dout);
  else
    k_dm_ptrace<double><<<g, 256, 0, rho->stream>>>((const double2*)rho->d, n, kept, traced, nk, nsites, dout);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(out, dout, sizeof(double2) * s1 * s1, cudaMemcpyDeviceToHost, rho->stream);
  cudaFreeAsync(dout, rho->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(rho->stream);
  if (e != cudaSuccess) return cuda_fail(e, "partial trace");
  return VQC_OK;
}

int vqc_dm_probs(vqc_state rho, double* out) {
  int rc = enter(rho);
  if (rc) return rc;
  const int n = rho->n_dm;
  if (!n) return fail(VQC_ERR_ARG, "not a density matrix");
  if (!out) return fail(VQC_ERR_ARG, "null output");
  std::lock_guard<std::mutex> lk(rho->mu);
  const int64_t L = int64_t(1) << n;
  double* dout = nullptr;
  VQC_CK(cudaMallocAsync((void**)&dout, sizeof(double) * L, rho->stream));
  const int g = launch_grid(rho->device, L);
  if (rho->dtype == VQC_C64)
    k_dm_diag<float><<<g, 256, 0, rho->stream>>>((const float2*)rho->d, n, dout);
  else
    k_dm_diag<double><<<g, 256, 0, rho->stream>>>((const double2*)rho->d, n, dout);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, sizeof(double) * L, cudaMemcpyDeviceToHost, rho->stream);
  cudaFreeAsync(dout, rho->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(rho->stream);
  if (e != cudaSuccess) return cuda_fail(e, "probabilities");
  return VQC_OK;
}

int vqc_dm_trace(vqc_state rho, double* out) {
  int rc = enter(rho);
  if (rc) return rc;
  if (!rho->n_dm) return fail(VQC_ERR_ARG, "not a density matrix");
  if (!out) return fail(VQC_ERR_ARG, "null output");
  std::lock_guard<std::mutex> lk(rho->mu);
  const int g = reduction_grid(rho->device, int64_t(1) << rho->n_dm);
  if (rho->dtype == VQC_C64)
    k_dm_trace<float><<<g, kRedThreads, 0, rho->stream>>>((const float2*)rho->d, rho->n_dm, rho->scr);
  else
    k_dm_trace<double><<<g, kRedThreads, 0, rho->stream>>>((const double2*)rho->d, rho->n_dm, rho->scr);
  VQC_CK(cudaGetLastError());
  if ((rc = fetch_result(rho, 2))) return rc;
  out[0] = rho->h_result[0];
  out[1] = rho->h_result[1];
  return VQC_OK;
}

}  // extern "C"
