// CPU oracle for the VQC.jl state-vector hot path.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product library links, loads or
// calls this file; only tests/, __graft_entry__.smoke() and the cpu_baseline /
// reference arm of bench.py use it, as the checker and as the timed CPU
// restatement of the reference's multithreaded path.
//
// Parity status: UNPINNED against the reference's own outputs.  The reference
// (guochu/VQC.jl) is Julia, Julia is not installed here or on the GPU box, and
// its test-suite holds no golden vectors (all of its tests use unseeded random
// data).  This oracle is pinned instead by restating the reference's loops
// line for line and by the reference's relational / known-answer tests,
// restated under tests/ (serial vs threaded, specialised vs dense, LSB-first
// encodings, partial trace of a state vs of its density matrix, phase
// estimation, AD vs central finite differences).
//
// Conventions (identical to the reference):
//   * qubit q (0-based here, 1-based in the reference) <-> bit q of the
//     amplitude index (LSB first, statevector.jl:167-176);
//   * a k-qubit matrix U is row-major, 2^k x 2^k, complex interleaved
//     (re, im); bit b of a row/column index <-> positions[b]
//     (hamiltonian/util.jl:6-15 builds kron(reverse(ops)), i.e. the first
//     listed position is the least significant bit);
//   * a density matrix of n qubits is a 2n-qubit vector: bits 0..n-1 are the
//     row index, bits n..2n-1 the column index (densitymatrix.jl:27-30,
//     column-major L x L storage).
//
// Threading restates auxiliary/parallel_for.jl:3-61: a static split of the
// iteration range [0, total) over nthreads when total >= MIN_SIZE (1024),
// serial otherwise; reductions add one partial per thread.

#include <algorithm>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#include <thread>

namespace {

constexpr int64_t kMinSize = 1024;  // parallel_for.jl:3

// parallel_for.jl:6-7 get_size_1 / get_size_2
inline int64_t split_lo(int64_t total, int nt, int tid) { return total * tid / nt; }
inline int64_t split_hi(int64_t total, int nt, int tid) { return total * (tid + 1) / nt; }

// parallel_for.jl:12-23 parallel_run (Julia tasks -> one std::thread per
// slice of the static split).
template <class F>
void parallel_run(int64_t total, int nthreads, F f) {
  if (total >= kMinSize && nthreads > 1) {
    std::vector<std::thread> th;
    for (int tid = 0; tid < nthreads; ++tid) {
      int64_t ist = split_lo(total, nthreads, tid), ifn = split_hi(total, nthreads, tid);
      if (ifn > ist) th.emplace_back([=, &f] { f(ist, ifn); });
    }
    for (auto& t : th) t.join();
  } else {
    f(0, total);
  }
}

// parallel_for.jl:28-61 parallel_sum: one partial per thread, added in thread
// order (the reference adds them with atomics, so its order is arbitrary).
template <class A, class F>
A parallel_sum(int64_t total, int nthreads, F f) {
  if (total >= kMinSize && nthreads > 1) {
    std::vector<A> part(nthreads, A(0));
    std::vector<std::thread> th;
    for (int tid = 0; tid < nthreads; ++tid) {
      int64_t ist = split_lo(total, nthreads, tid), ifn = split_hi(total, nthreads, tid);
      if (ifn > ist) th.emplace_back([=, &f, &part] { part[tid] = f(ist, ifn); });
    }
    for (auto& t : th) t.join();
    A r(0);
    for (int t = 0; t < nthreads; ++t) r += part[t];
    return r;
  }
  return f(0, total);
}

// ordered_positions / ordered_mat of QuantumCircuits.jl (called at
// applygates/generic/generic.jl:43,50): sort the positions ascending and
// permute the matrix so that bit b of its index follows sorted position b.
template <class C>
void order_gate(int k, const int* pos, const C* U, int* sp, std::vector<C>& Us) {
  int perm[8];
  for (int i = 0; i < k; ++i) {  // insertion sort of at most 5 entries
    int j = i;
    for (; j > 0 && pos[perm[j - 1]] > pos[i]; --j) perm[j] = perm[j - 1];
    perm[j] = i;
  }
  for (int i = 0; i < k; ++i) sp[i] = pos[perm[i]];
  const int d = 1 << k;
  Us.assign((size_t)d * d, C(0));
  auto remap = [&](int rs) {  // index over sorted bits -> index over given bits
    int r = 0;
    for (int i = 0; i < k; ++i)
      if (rs >> i & 1) r |= 1 << perm[i];
    return r;
  };
  for (int rs = 0; rs < d; ++rs)
    for (int cs = 0; cs < d; ++cs) Us[(size_t)rs * d + cs] = U[(size_t)remap(rs) * d + remap(cs)];
}

// The group-base formula of applygates/generic/threaded_long_range.jl:3-55
// (and the specialised kernels, e.g. specific/czgate.jl:10-18): with sorted
// positions p_1 < ... < p_k and masks
//   mask_0 = 2^p_1 - 1,  mask_i = (2^p_{i+1} - 1) xor (2^{p_i + 1} - 1),
//   mask_k = (L - 1) xor (2^{p_k + 1} - 1),
// group i starts at sum_j ((i << j) & mask_j).  The serial nested-stride loops
// of serial_short_range.jl:2-71 enumerate the same groups in the same order.
struct GroupIndex {
  int k;
  int64_t mask[6];
  int64_t off[32];
  GroupIndex(int n, int k_, const int* sp) : k(k_) {
    const int64_t L = int64_t(1) << n;
    mask[0] = (int64_t(1) << sp[0]) - 1;
    for (int i = 1; i < k; ++i)
      mask[i] = ((int64_t(1) << sp[i]) - 1) ^ ((int64_t(2) << sp[i - 1]) - 1);
    mask[k] = (L - 1) ^ ((int64_t(2) << sp[k - 1]) - 1);
    for (int j = 0; j < (1 << k); ++j) {
      int64_t o = 0;
      for (int b = 0; b < k; ++b)
        if (j >> b & 1) o += int64_t(1) << sp[b];
      off[j] = o;
    }
  }
  inline int64_t base(int64_t i) const {
    int64_t l = 0;
    for (int j = 0; j <= k; ++j) l |= (i << j) & mask[j];
    return l;
  }
};

template <class T>
int apply_gate(std::complex<T>* v, int n, int k, const int* pos, const std::complex<T>* U, int nthreads) {
  using C = std::complex<T>;
  if (k < 1 || k > 5 || n < k) return -1;
  int sp[8];
  std::vector<C> Us;
  order_gate<C>(k, pos, U, sp, Us);
  for (int i = 0; i < k; ++i)
    if (sp[i] < 0 || sp[i] >= n || (i && sp[i] == sp[i - 1])) return -1;
  GroupIndex g(n, k, sp);
  const int d = 1 << k;
  const C* M = Us.data();
  parallel_run(int64_t(1) << (n - k), nthreads, [&](int64_t ist, int64_t ifn) {
    C vi[32], vo[32];
    for (int64_t i = ist; i < ifn; ++i) {
      const int64_t l = g.base(i);
      for (int j = 0; j < d; ++j) vi[j] = v[l + g.off[j]];
      for (int r = 0; r < d; ++r) {
        C acc(0);
        for (int c = 0; c < d; ++c) acc += M[r * d + c] * vi[c];
        vo[r] = acc;
      }
      for (int j = 0; j < d; ++j) v[l + g.off[j]] = vo[j];
    }
  });
  return 0;
}

// vout += U v on the given positions: hamiltonian/apply_qterms/short_range_serial.jl:3-96
template <class T>
int apply_gate_add(const std::complex<T>* v, std::complex<T>* vout, int n, int k, const int* pos,
                   const std::complex<T>* U, int nthreads) {
  using C = std::complex<T>;
  if (k < 1 || k > 5 || n < k) return -1;
  int sp[8];
  std::vector<C> Us;
  order_gate<C>(k, pos, U, sp, Us);
  for (int i = 0; i < k; ++i)
    if (sp[i] < 0 || sp[i] >= n || (i && sp[i] == sp[i - 1])) return -1;
  GroupIndex g(n, k, sp);
  const int d = 1 << k;
  const C* M = Us.data();
  parallel_run(int64_t(1) << (n - k), nthreads, [&](int64_t ist, int64_t ifn) {
    C vi[32];
    for (int64_t i = ist; i < ifn; ++i) {
      const int64_t l = g.base(i);
      for (int j = 0; j < d; ++j) vi[j] = v[l + g.off[j]];
      for (int r = 0; r < d; ++r) {
        C acc(0);
        for (int c = 0; c < d; ++c) acc += M[r * d + c] * vi[c];
        vout[l + g.off[r]] += acc;
      }
    }
  });
  return 0;
}

// sum over groups of vc^dagger M v: hamiltonian/expecs/expec_serial.jl:2-128
// (one state: vc == v) and expec_threaded_2.jl (two states).  Accumulates in
// the template type A (the reference accumulates in eltype(v)).
template <class T, class A>
int expect(const std::complex<T>* v, const std::complex<T>* vc, int n, int k, const int* pos,
           const std::complex<T>* Mm, std::complex<A>* out, int nthreads) {
  using C = std::complex<T>;
  using CA = std::complex<A>;
  if (k < 1 || k > 5 || n < k) return -1;
  int sp[8];
  std::vector<C> Us;
  order_gate<C>(k, pos, Mm, sp, Us);
  for (int i = 0; i < k; ++i)
    if (sp[i] < 0 || sp[i] >= n || (i && sp[i] == sp[i - 1])) return -1;
  if (!vc) vc = v;
  GroupIndex g(n, k, sp);
  const int d = 1 << k;
  std::vector<CA> MA(Us.begin(), Us.end());
  const CA* M = MA.data();
  *out = parallel_sum<CA>(int64_t(1) << (n - k), nthreads, [&](int64_t ist, int64_t ifn) {
    CA r(0);
    CA vi[32], vci[32];
    for (int64_t i = ist; i < ifn; ++i) {
      const int64_t l = g.base(i);
      for (int j = 0; j < d; ++j) {
        vi[j] = CA(v[l + g.off[j]]);
        vci[j] = CA(vc[l + g.off[j]]);
      }
      for (int a = 0; a < d; ++a) {
        CA acc(0);
        for (int c = 0; c < d; ++c) acc += M[a * d + c] * vi[c];
        r += std::conj(vci[a]) * acc;
      }
    }
    return r;
  });
  return 0;
}

// applygates/generic/generic.jl:54-64: U on the row qubits, then conj(U) on
// the column qubits (positions + n) of the 2n-qubit flattened density matrix.
template <class T>
int dm_apply_gate(std::complex<T>* rho, int n, int k, const int* pos, const std::complex<T>* U, int nthreads) {
  using C = std::complex<T>;
  if (k < 1 || k > 5 || n < k) return -1;
  const int d = 1 << k;
  int err = apply_gate<T>(rho, 2 * n, k, pos, U, nthreads);
  if (err) return err;
  for (int i = 0; i < k; ++i)
    if (pos[i] < 0 || pos[i] >= n) return -1;
  int pos2[8];
  for (int i = 0; i < k; ++i) pos2[i] = pos[i] + n;
  std::vector<C> Uc((size_t)d * d);
  for (size_t i = 0; i < Uc.size(); ++i) Uc[i] = std::conj(U[i]);
  return apply_gate<T>(rho, 2 * n, k, pos2, Uc.data(), nthreads);
}

// ptrace.jl:38-53 with auxiliary/indexop.jl:46-74: the kept qubits keep their
// ascending order and become qubits 0..n-m-1 of the result;
//   out[a + s1*b] = sum_c rho[row = a (+) c, col = b (+) c].
template <class T>
int validate_sites(int n, int m, const int* sites) {
  if (m < 0 || m > n) return -1;
  for (int i = 0; i < m; ++i) {
    if (sites[i] < 0 || sites[i] >= n) return -1;
    for (int j = 0; j < i; ++j)
      if (sites[j] == sites[i]) return -1;
  }
  return 0;
}

inline void site_maps(int n, int m, const int* sites, std::vector<int64_t>& kept_dep, std::vector<int64_t>& tr_dep) {
  uint64_t trmask = 0;
  for (int i = 0; i < m; ++i) trmask |= uint64_t(1) << sites[i];
  std::vector<int> kept, tr;
  for (int q = 0; q < n; ++q) (trmask >> q & 1 ? tr : kept).push_back(q);
  const int nk = (int)kept.size(), nt = (int)tr.size();
  kept_dep.assign(size_t(1) << nk, 0);
  tr_dep.assign(size_t(1) << nt, 0);
  for (int64_t a = 0; a < (int64_t(1) << nk); ++a)
    for (int b = 0; b < nk; ++b)
      if (a >> b & 1) kept_dep[a] |= int64_t(1) << kept[b];
  for (int64_t c = 0; c < (int64_t(1) << nt); ++c)
    for (int b = 0; b < nt; ++b)
      if (c >> b & 1) tr_dep[c] |= int64_t(1) << tr[b];
}

template <class T>
int dm_ptrace(const std::complex<T>* rho, int n, int m, const int* sites, std::complex<T>* out) {
  using C = std::complex<T>;
  if (validate_sites<T>(n, m, sites)) return -1;
  std::vector<int64_t> kd, td;
  site_maps(n, m, sites, kd, td);
  const int64_t s1 = (int64_t)kd.size(), s2 = (int64_t)td.size(), L = int64_t(1) << n;
  for (int64_t b = 0; b < s1; ++b)
    for (int64_t a = 0; a < s1; ++a) {
      C acc(0);
      for (int64_t c = 0; c < s2; ++c) acc += rho[(kd[a] | td[c]) + L * (kd[b] | td[c])];
      out[a + s1 * b] = acc;
    }
  return 0;
}

// ptrace.jl:13-27: the state-vector form, vt * vt' after the same permutation.
template <class T>
int sv_ptrace(const std::complex<T>* psi, int n, int m, const int* sites, std::complex<T>* out) {
  using C = std::complex<T>;
  if (validate_sites<T>(n, m, sites)) return -1;
  std::vector<int64_t> kd, td;
  site_maps(n, m, sites, kd, td);
  const int64_t s1 = (int64_t)kd.size(), s2 = (int64_t)td.size();
  for (int64_t b = 0; b < s1; ++b)
    for (int64_t a = 0; a < s1; ++a) {
      C acc(0);
      for (int64_t c = 0; c < s2; ++c) acc += psi[kd[a] | td[c]] * std::conj(psi[kd[b] | td[c]]);
      out[a + s1 * b] = acc;
    }
  return 0;
}

// real(diag(storage(rho))): the full basis distribution of a density matrix
// (densitymatrix.jl:30; measure.jl:69-81 sums the zero branch of it).
template <class T>
int dm_probs(const std::complex<T>* rho, int n, T* out) {
  const int64_t L = int64_t(1) << n;
  for (int64_t i = 0; i < L; ++i) out[i] = rho[i + L * i].real();
  return 0;
}

// measure.jl:69-81 compute_probability_zero for a density matrix.
template <class T>
double dm_prob_zero(const std::complex<T>* rho, int n, int q) {
  const int64_t L = int64_t(1) << n;
  double r = 0;
  for (int64_t i = 0; i < L; ++i)
    if (!(i >> q & 1)) r += (double)rho[i + L * i].real();
  return r;
}

}  // namespace

#define CD(p) reinterpret_cast<std::complex<double>*>(p)
#define CCD(p) reinterpret_cast<const std::complex<double>*>(p)
#define CF(p) reinterpret_cast<std::complex<float>*>(p)
#define CCF(p) reinterpret_cast<const std::complex<float>*>(p)

extern "C" {

int or_apply_gate_c128(double* v, int n, int k, const int* pos, const double* U, int nt) {
  return apply_gate<double>(CD(v), n, k, pos, CCD(U), nt);
}
int or_apply_gate_c64(float* v, int n, int k, const int* pos, const float* U, int nt) {
  return apply_gate<float>(CF(v), n, k, pos, CCF(U), nt);
}
int or_apply_gate_add_c128(const double* v, double* vout, int n, int k, const int* pos, const double* U, int nt) {
  return apply_gate_add<double>(CCD(v), CD(vout), n, k, pos, CCD(U), nt);
}
int or_apply_gate_add_c64(const float* v, float* vout, int n, int k, const int* pos, const float* U, int nt) {
  return apply_gate_add<float>(CCF(v), CF(vout), n, k, pos, CCF(U), nt);
}
// out[0..1] = (re, im) of sum vc^dagger M v; vc may be NULL (one-state form).
int or_expect_c128(const double* v, const double* vc, int n, int k, const int* pos, const double* M, double* out,
                   int nt) {
  return expect<double, double>(CCD(v), vc ? CCD(vc) : nullptr, n, k, pos, CCD(M),
                                reinterpret_cast<std::complex<double>*>(out), nt);
}
// FP32 states, FP32 accumulation: the reference's own ComplexF32 behaviour.
int or_expect_c64(const float* v, const float* vc, int n, int k, const int* pos, const float* M, float* out, int nt) {
  return expect<float, float>(CCF(v), vc ? CCF(vc) : nullptr, n, k, pos, CCF(M),
                              reinterpret_cast<std::complex<float>*>(out), nt);
}
int or_dm_apply_gate_c128(double* rho, int n, int k, const int* pos, const double* U, int nt) {
  return dm_apply_gate<double>(CD(rho), n, k, pos, CCD(U), nt);
}
int or_dm_ptrace_c128(const double* rho, int n, int m, const int* sites, double* out) {
  return dm_ptrace<double>(CCD(rho), n, m, sites, CD(out));
}
int or_sv_ptrace_c128(const double* psi, int n, int m, const int* sites, double* out) {
  return sv_ptrace<double>(CCD(psi), n, m, sites, CD(out));
}
int or_dm_probs_c128(const double* rho, int n, double* out) { return dm_probs<double>(CCD(rho), n, out); }
double or_dm_prob_zero_c128(const double* rho, int n, int q) { return dm_prob_zero<double>(CCD(rho), n, q); }
int or_max_threads(void) { return (int)std::thread::hardware_concurrency(); }

}  // extern "C"
