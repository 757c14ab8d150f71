// expectation(H, psi), expectation(phi, H, psi) and H * psi on the device.
//
// Reference: hamiltonian/expecs/expecs.jl:12-78 (one pass per position key,
// accumulation in eltype(psi)), expec_threaded.jl / expec_threaded_2.jl (the
// loops), apply_qterms/apply_qterms.jl:13-28 and short_range_threaded.jl
// (vout += M_key psi per key).
//
// Pauli sums take one pass over the state for the whole operator: terms are
// grouped by their X/Y flip mask x; for output index i each group reads the
// partner amplitude psi[i ^ x] once and multiplies it by the group's summed
// phase f_x(i) = sum_t c_t i^{|x & z_t|} (-1)^{|(i ^ x) & z_t|}.  All sums are
// FP64 (also for FP32 states) and reduced in a fixed order.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>

#include "engine.h"
#include "subspace.cuh"
#include "tile_plan.cuh"

namespace vqc {


constexpr int kMaxTermsPerLaunch = 2048;

// Prepared operator: groups + terms, uploaded to h->opbuf.
struct PauliPlan {
  std::vector<DevGroup> groups;
  std::vector<DevTerm> terms;
};

int plan_pauli(int nq, const vqc_pauli* t, int nt, bool apply_hermitian_part, PauliPlan& p) {
  if (nt < 0 || (nt > 0 && !t)) return fail(VQC_ERR_ARG, "bad Pauli term array");
  const uint64_t lim = nq >= 64 ? ~0ull : ((1ull << nq) - 1);
  std::map<uint64_t, std::vector<int>> by_x;
  for (int i = 0; i < nt; ++i) {
    if ((t[i].xmask & ~lim) || (t[i].zmask & ~lim)) return fail(VQC_ERR_ARG, "Pauli term acts outside the register");
    by_x[t[i].xmask].push_back(i);
  }
  for (auto& kv : by_x) {
    DevGroup g{kv.first, (int)p.terms.size(), (int)kv.second.size()};
    for (int i : kv.second) {
      const int ny = __builtin_popcountll(t[i].xmask & t[i].zmask) & 3;
      const cd ph[4] = {cd(1, 0), cd(0, 1), cd(-1, 0), cd(0, -1)};
      cd c = cd(t[i].coeff_re, t[i].coeff_im) * ph[ny];
      // (H + H^dagger): a Pauli string is Hermitian, so its coefficient becomes 2 Re(c).
      cd d = apply_hermitian_part ? cd(2 * t[i].coeff_re, 0) * ph[ny] : c;
      p.terms.push_back(DevTerm{t[i].zmask, make_double2(c.real(), c.imag()), make_double2(d.real(), d.imag())});
    }
    p.groups.push_back(g);
  }
  return VQC_OK;
}

// One pass: optionally out = H' psi, and sum conj(bra_i) (H psi)_i.
template <class R, bool WRITE, bool ACC>
__global__ void __launch_bounds__(kRedThreads)
    k_pauli(const cplx<R>* __restrict__ bra, const cplx<R>* __restrict__ ket, cplx<R>* __restrict__ out, int64_t N,
            const DevGroup* __restrict__ groups, int ng, const DevTerm* __restrict__ terms, int nt, Scratch s,
            double* res) {
  extern __shared__ unsigned char smem[];
  DevGroup* sg = reinterpret_cast<DevGroup*>(smem);
  DevTerm* st = reinterpret_cast<DevTerm*>(smem + sizeof(DevGroup) * ng);
  for (int i = threadIdx.x; i < ng; i += blockDim.x) sg[i] = groups[i];
  for (int i = threadIdx.x; i < nt; i += blockDim.x) st[i] = terms[i];
  __syncthreads();
  double acc[2] = {0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += stride) {
    double2 hv = make_double2(0, 0), ov = make_double2(0, 0);
    for (int gi = 0; gi < ng; ++gi) {
      const DevGroup g = sg[gi];
      const int64_t j = i ^ (int64_t)g.x;
      if (!VQC_DCHECK(j, N)) continue;
      const double2 kv = to_d2(ket[j]);
      double2 f = make_double2(0, 0), fd = make_double2(0, 0);
      for (int q = g.start; q < g.start + g.count; ++q) {
        const double sgn = (__popcll((unsigned long long)j & st[q].z) & 1) ? -1.0 : 1.0;
        if (ACC) {
          f.x = fma(sgn, st[q].c.x, f.x);
          f.y = fma(sgn, st[q].c.y, f.y);
        }
        if (WRITE) {
          fd.x = fma(sgn, st[q].d.x, fd.x);
          fd.y = fma(sgn, st[q].d.y, fd.y);
        }
      }
      if (ACC) hv = cfma(f, kv, hv);
      if (WRITE) ov = cfma(fd, kv, ov);
    }
    if (WRITE) out[i] = mkc<R>((R)ov.x, (R)ov.y);
    if (ACC) {
      const double2 b = to_d2(bra[i]);
      acc[0] = fma(b.x, hv.x, fma(b.y, hv.y, acc[0]));
      acc[1] = fma(b.x, hv.y, fma(-b.y, hv.x, acc[1]));
    }
  }
  if (ACC) grid_reduce<2>(acc, s, res);
}

// Four consecutive outputs per thread, i = 4k + a (a = 0..3).  The partners
// of group x are the four amplitudes at 4k ^ (x & ~3), permuted by x & 3.
// A term's sign (-1)^{|j & z|} splits into its high bits (the same for the
// four partners) and its low-bit class z & 3, so every term is evaluated
// once per four outputs into class sums F[cls]; a 4-point Walsh-Hadamard
// transform of F gives the group's phase at each partner's low bits b:
//   f(b) = sum_cls (-1)^{|b & cls|} F[cls].
// Terms arrive sorted by class, group g's class c in [cs[g][c], cs[g][c+1]).
// SEP: separate coefficients d for the written operator (complex Pauli
// coefficients with the Hermitian part requested); otherwise the written
// operator is dfac * (the expectation operator).
struct DevGroup4 {
  uint64_t x;
  int cs[5];
  int pad;
};

// The quad kernel computes in the state's precision (FP32 phases and
// products for FP32 states, whose written output is FP32); the expectation
// itself is accumulated in FP64.  The class sums F of real Pauli-sum
// coefficients such as 1 and 0.5 are exact in either precision.
template <class R>
struct PTerm {
  uint64_t z;
  cplx<R> c, d;
};
template <int AX, class V>
__device__ __forceinline__ void pauli4_add(V (&hv)[4], const V (&W)[4], const V (&kv)[4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) hv[a] = cfma(W[a ^ AX], kv[a ^ AX], hv[a]);
}
template <int AX, class V>
__device__ __forceinline__ void pauli4_add1(V (&hv)[4], const V& f, const V (&kv)[4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) hv[a] = cfma(f, kv[a ^ AX], hv[a]);
}
template <class V>
__device__ __forceinline__ void pauli4_wh(const V (&F)[4], V (&W)[4]) {
  V s01, d01, s23, d23;
  s01.x = F[0].x + F[1].x, s01.y = F[0].y + F[1].y, d01.x = F[0].x - F[1].x, d01.y = F[0].y - F[1].y;
  s23.x = F[2].x + F[3].x, s23.y = F[2].y + F[3].y, d23.x = F[2].x - F[3].x, d23.y = F[2].y - F[3].y;
  W[0].x = s01.x + s23.x, W[0].y = s01.y + s23.y;
  W[1].x = d01.x + d23.x, W[1].y = d01.y + d23.y;
  W[2].x = s01.x - s23.x, W[2].y = s01.y - s23.y;
  W[3].x = d01.x - d23.x, W[3].y = d01.y - d23.y;
}
template <class R>
__device__ __forceinline__ void load4(const cplx<R>* p, cplx<R> (&kv)[4]) {
  if constexpr (sizeof(R) == 4) {
    const float4 a = *reinterpret_cast<const float4*>(p), b = *reinterpret_cast<const float4*>(p + 2);
    kv[0] = make_float2(a.x, a.y), kv[1] = make_float2(a.z, a.w);
    kv[2] = make_float2(b.x, b.y), kv[3] = make_float2(b.z, b.w);
  } else {
#pragma unroll
    for (int b = 0; b < 4; ++b) kv[b] = p[b];
  }
}

template <class R, bool WRITE, bool ACC, bool SEP>
__global__ void __launch_bounds__(kRedThreads)
    k_pauli4(const cplx<R>* __restrict__ bra, const cplx<R>* __restrict__ ket, cplx<R>* __restrict__ out, int64_t N,
             const DevGroup4* __restrict__ groups, int ng, const DevTerm* __restrict__ terms, int nt, double dfac,
             Scratch s, double* res) {
  using V = cplx<R>;
  extern __shared__ unsigned char smem[];
  DevGroup4* sg = reinterpret_cast<DevGroup4*>(smem);
  PTerm<R>* st = reinterpret_cast<PTerm<R>*>(smem + sizeof(DevGroup4) * ng);
  for (int i = threadIdx.x; i < ng; i += blockDim.x) sg[i] = groups[i];
  for (int i = threadIdx.x; i < nt; i += blockDim.x) {
    const DevTerm t = terms[i];
    st[i] = PTerm<R>{t.z, mkc<R>((R)t.c.x, (R)t.c.y), mkc<R>((R)t.d.x, (R)t.d.y)};
  }
  __syncthreads();
  double acc[2] = {0, 0};
  const V zero = mkc<R>(R(0), R(0));
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, nq4 = N >> 2;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < nq4; k += stride) {
    const int64_t i0 = k << 2;
    V hv[4], ov[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) hv[a] = ov[a] = zero;
    for (int gi = 0; gi < ng; ++gi) {
      const DevGroup4& g = sg[gi];
      const int64_t jb = i0 ^ (int64_t)(g.x & ~3ull);
      if (!VQC_DCHECK(jb + 3, N)) continue;
      V kv[4];
      load4<R>(ket + jb, kv);
      if (g.cs[1] == g.cs[4]) {
        // every term of the group in class 0 (no Z on the two lowest qubits): the
        // same phase at all four partners, W[b] = F[0] (uniform over the grid)
        V f = zero, fd = zero;
        for (int q = g.cs[0]; q < g.cs[1]; ++q) {
          const uint64_t m = (uint64_t)jb & st[q].z;
          const bool odd = (__popc((unsigned)m ^ (unsigned)(m >> 32)) & 1) != 0;
          const V cc = st[q].c;
          f.x += odd ? -cc.x : cc.x;
          f.y += odd ? -cc.y : cc.y;
          if (SEP) {
            const V dd = st[q].d;
            fd.x += odd ? -dd.x : dd.x;
            fd.y += odd ? -dd.y : dd.y;
          }
        }
        switch ((int)(g.x & 3)) {  // (compile-time register indices)
          case 0: pauli4_add1<0>(hv, f, kv); if (SEP) pauli4_add1<0>(ov, fd, kv); break;
          case 1: pauli4_add1<1>(hv, f, kv); if (SEP) pauli4_add1<1>(ov, fd, kv); break;
          case 2: pauli4_add1<2>(hv, f, kv); if (SEP) pauli4_add1<2>(ov, fd, kv); break;
          default: pauli4_add1<3>(hv, f, kv); if (SEP) pauli4_add1<3>(ov, fd, kv); break;
        }
        continue;
      }
      V F[4], Fd[4];
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        F[c] = Fd[c] = zero;
        for (int q = g.cs[c]; q < g.cs[c + 1]; ++q) {
          const uint64_t m = (uint64_t)jb & st[q].z;
          const bool odd = (__popc((unsigned)m ^ (unsigned)(m >> 32)) & 1) != 0;
          const V cc = st[q].c;
          F[c].x += odd ? -cc.x : cc.x;
          F[c].y += odd ? -cc.y : cc.y;
          if (SEP) {
            const V dd = st[q].d;
            Fd[c].x += odd ? -dd.x : dd.x;
            Fd[c].y += odd ? -dd.y : dd.y;
          }
        }
      }
      V W[4], Wd[4];
      pauli4_wh(F, W);
      if (SEP) pauli4_wh(Fd, Wd);
      switch ((int)(g.x & 3)) {
        case 0: pauli4_add<0>(hv, W, kv); if (SEP) pauli4_add<0>(ov, Wd, kv); break;
        case 1: pauli4_add<1>(hv, W, kv); if (SEP) pauli4_add<1>(ov, Wd, kv); break;
        case 2: pauli4_add<2>(hv, W, kv); if (SEP) pauli4_add<2>(ov, Wd, kv); break;
        default: pauli4_add<3>(hv, W, kv); if (SEP) pauli4_add<3>(ov, Wd, kv); break;
      }
    }
    if (WRITE) {
      const R df = (R)dfac;  // 1 or 2
#pragma unroll
      for (int a = 0; a < 4; ++a) out[i0 + a] = SEP ? ov[a] : mkc<R>(df * hv[a].x, df * hv[a].y);
    }
    if (ACC) {
      V b[4];
      load4<R>(bra + i0, b);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const double2 bb = to_d2(b[a]), hh = to_d2(hv[a]);
        acc[0] = fma(bb.x, hh.x, fma(bb.y, hh.y, acc[0]));
        acc[1] = fma(bb.x, hh.y, fma(-bb.y, hh.x, acc[1]));
      }
    }
  }
  if (ACC) grid_reduce<2>(acc, s, res);
}

// Phase tables over 6-bit windows of the index.  The quad kernel above
// evaluates every term of every group at every quad (a 64-bit mask, a
// parity, a sign, two adds); here that work is done once, on the host.  A
// group's phase at partner index j is
//   f(j) = sum_w T_w[(j >> s_w) & 63] + sum_{t in no window} c_t (-1)^{|j & z_t|},
//   T_w[u] = sum_{t in w} c_t (-1)^{|u & (z_t >> s_w)|},
// where window w holds the terms whose whole z support lies in the bits
// [s_w, s_w + 6) (the tables are summed in FP64 on the host and stored in the
// state's precision; terms without Z have a constant phase, folded into a
// table).  A window starting at bit 0 gives the four partners of a quad four
// phases (entries u .. u+3, u a multiple of 4); a window starting at bit 2 or
// above gives one phase for all four.  For the XXZ chain each flip-mask group
// is one window, the diagonal group five.
constexpr int kWinBits = 6, kWinSize = 1 << kWinBits;
static bool env_on(const char* name, bool dflt) {
  const char* v = std::getenv(name);
  return v && *v ? std::atoi(v) != 0 : dflt;
}
constexpr size_t kWinMaxTableBytes = 96 * 1024;
struct DevGroupW {
  uint64_t x;
  int wbeg, wend;  // windows [wbeg, wend); window wbeg starts at bit 0 when low0
  int tbeg, tend;  // terms in no window: signs evaluated directly
  int low0;
  int rlow;  // 1: a term in no window has Z on qubit 0 or 1 (the four partners' phases differ)
};

// Traversal: with thl > 0 the linear quad counter t maps to the quad index
// k whose bits [0, tlo) are t's lowest bits (coalesced lanes), bits
// [ths, ths + thl) (the top of the index) its next thl bits, and bits
// [tlo, ths) the rest: every combination of the top bits is in flight at once,
// so flip masks on those bits find their partners among the amplitudes being
// read.  ADD: out accumulates (out += df H psi) instead of being overwritten.
__device__ __forceinline__ int64_t pauli_trav(int64_t t, int tlo, int ths, int thl) {
  if (thl == 0) return t;
  const int64_t lo = t & ((int64_t(1) << tlo) - 1), hi = (t >> tlo) & ((int64_t(1) << thl) - 1);
  return lo | (hi << ths) | ((t >> (tlo + thl)) << tlo);
}

template <class R, bool WRITE, bool ACC, bool ADD>
__global__ void __launch_bounds__(kRedThreads)
    k_pauli_win(const cplx<R>* __restrict__ bra, const cplx<R>* __restrict__ ket, cplx<R>* __restrict__ out,
                int64_t N, const DevGroupW* __restrict__ groups, int ng, const int* __restrict__ shifts,
                const cplx<R>* __restrict__ tables, int nw, const DevTerm* __restrict__ terms, int nt, double dfac,
                int tlo, int ths, int thl, Scratch s, double* res) {
  using V = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem[];
  V* stab = reinterpret_cast<V*>(smem);
  DevGroupW* sg = reinterpret_cast<DevGroupW*>(smem + sizeof(V) * (size_t)nw * kWinSize);
  int* ssh = reinterpret_cast<int*>(sg + ng);
  PTerm<R>* st = reinterpret_cast<PTerm<R>*>(ssh + ((nw + 3) & ~3));
  for (int i = threadIdx.x; i < nw * kWinSize; i += blockDim.x) stab[i] = tables[i];
  for (int i = threadIdx.x; i < ng; i += blockDim.x) sg[i] = groups[i];
  for (int i = threadIdx.x; i < nw; i += blockDim.x) ssh[i] = shifts[i];
  for (int i = threadIdx.x; i < nt; i += blockDim.x) {
    const DevTerm t = terms[i];
    st[i] = PTerm<R>{t.z, mkc<R>((R)t.c.x, (R)t.c.y), mkc<R>((R)t.c.x, (R)t.c.y)};
  }
  __syncthreads();
  double acc[2] = {0, 0};
  const V zero = mkc<R>(R(0), R(0));
  const int64_t stride = (int64_t)gridDim.x * blockDim.x, nq4 = N >> 2;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < nq4; t += stride) {
    const int64_t i0 = pauli_trav(t, tlo, ths, thl) << 2;
    V hv[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) hv[a] = zero;
    for (int gi = 0; gi < ng; ++gi) {
      const DevGroupW& g = sg[gi];
      const int64_t jb = i0 ^ (int64_t)(g.x & ~3ull);
      if (!VQC_DCHECK(jb + 3, N)) continue;
      V kv[4];
      load4<R>(ket + jb, kv);
      int w = g.wbeg;
      V f = zero;
      V W[4];
      const bool four = g.low0 || g.rlow;
      if (g.low0) {
        const V* t = stab + (size_t)w * kWinSize + (jb & (kWinSize - 1));
#pragma unroll
        for (int b = 0; b < 4; ++b) W[b] = t[b];
        ++w;
      } else {
#pragma unroll
        for (int b = 0; b < 4; ++b) W[b] = zero;
      }
      for (; w < g.wend; ++w) {
        const V t = stab[(size_t)w * kWinSize + ((jb >> ssh[w]) & (kWinSize - 1))];
        f.x += t.x;
        f.y += t.y;
      }
      for (int q = g.tbeg; q < g.tend; ++q) {
        const uint64_t m = (uint64_t)jb & st[q].z;
        const int hb = (__popc((unsigned)m ^ (unsigned)(m >> 32)) & 1);
        const V cc = st[q].c;
        if ((st[q].z & 3) == 0) {  // the same phase at the four partners
          f.x += hb ? -cc.x : cc.x;
          f.y += hb ? -cc.y : cc.y;
          continue;
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const bool odd = (hb ^ (__popc((unsigned)(b & st[q].z)) & 1)) != 0;
          W[b].x += odd ? -cc.x : cc.x;
          W[b].y += odd ? -cc.y : cc.y;
        }
      }
      if (four) {
#pragma unroll
        for (int b = 0; b < 4; ++b) W[b].x += f.x, W[b].y += f.y;
        switch ((int)(g.x & 3)) {  // (compile-time register indices)
          case 0: pauli4_add<0>(hv, W, kv); break;
          case 1: pauli4_add<1>(hv, W, kv); break;
          case 2: pauli4_add<2>(hv, W, kv); break;
          default: pauli4_add<3>(hv, W, kv); break;
        }
      } else {
        switch ((int)(g.x & 3)) {
          case 0: pauli4_add1<0>(hv, f, kv); break;
          case 1: pauli4_add1<1>(hv, f, kv); break;
          case 2: pauli4_add1<2>(hv, f, kv); break;
          default: pauli4_add1<3>(hv, f, kv); break;
        }
      }
    }
    if (WRITE) {
      const R df = (R)dfac;  // 1 or 2
      V o[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) o[a] = mkc<R>(df * hv[a].x, df * hv[a].y);
      if (ADD) {
        V prev[4];
        load4<R>(out + i0, prev);
#pragma unroll
        for (int a = 0; a < 4; ++a) o[a].x += prev[a].x, o[a].y += prev[a].y;
      }
      if constexpr (sizeof(R) == 4) {
        *reinterpret_cast<float4*>(out + i0) = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
        *reinterpret_cast<float4*>(out + i0 + 2) = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
      } else {
#pragma unroll
        for (int a = 0; a < 4; ++a) out[i0 + a] = o[a];
      }
    }
    if (ACC) {
      V b[4];
      load4<R>(bra + i0, b);
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        const double2 bb = to_d2(b[a]), hh = to_d2(hv[a]);
        acc[0] = fma(bb.x, hh.x, fma(bb.y, hh.y, acc[0]));
        acc[1] = fma(bb.x, hh.y, fma(-bb.y, hh.x, acc[1]));
      }
    }
  }
  if (ACC) grid_reduce<2>(acc, s, res);
}

// Adds the second launch's sums (res[2..3]) to the first's (res[0..1]).
__global__ void k_add_pair(double* res) {
  if (threadIdx.x < 2) res[threadIdx.x] += res[2 + threadIdx.x];
}

// ----------------------------------------------------------------------------- tile passes
// Pauli sums on states far larger than L2.  One pass streams the state once
// in tiles of 2^M amplitudes over a chosen set of M qubits (the lowest CLOW
// qubits always among them: 128-byte runs), staged in shared memory; a group
// whose flip mask lies inside the tile's qubits reads its partners there
// instead of from DRAM.  The groups are cut into passes on the host (a first
// pass over the lowest M qubits, then passes over the high qubits that the
// remaining flip masks use); a group no pass covers reads its partners from
// global memory.  Later passes add into the written output (ADD).  REAL: every
// phase of the operator is real (real Pauli-sum coefficients with an even
// number of Y per term), so a phase times an amplitude takes two FMAs.
constexpr int kPTThreads = 512;
constexpr int kPTHiBits = 9;  // tile bits above the always-resident low qubits
template <class R>
struct PTCfg;
template <>
struct PTCfg<float> {
  static constexpr int M = 13, CLOW = 4;  // 64 KiB tile
};
template <>
struct PTCfg<double> {
  static constexpr int M = 12, CLOW = 3;  // 64 KiB tile
};
struct DevPTPass {
  uint64_t nontile_mask;  // global qubits enumerated by the tile counter
  int64_t ntiles;
};

// Shared-memory layout of a tile pass (host and device compute it alike).
template <class R>
struct PTLayout {
  size_t stab, st, sg, shi, sxt, ssh, total;
  __host__ __device__ PTLayout(int nw, int nt, int ng) {
    constexpr size_t V = sizeof(cplx<R>);
    stab = V << PTCfg<R>::M;
    st = stab + (size_t)nw * kWinSize * V;
    sg = (st + sizeof(PTerm<R>) * (size_t)nt + 15) & ~size_t(15);
    shi = sg + sizeof(DevGroupW) * (size_t)ng;
    sxt = shi + sizeof(int64_t) * (size_t(1) << kPTHiBits);
    ssh = sxt + sizeof(int) * (size_t)ng;
    total = (ssh + sizeof(int) * (size_t)nw + 15) & ~size_t(15);
  }
};

// The tile in shared memory as 16-byte planes: a quad's four amplitudes are
// one 16-byte element in each of 2 (FP32) or 4 (FP64) planes of NQ elements,
// so the lanes of a warp reading consecutive quads (or a permutation of them)
// touch consecutive 16-byte words: no bank conflicts.
template <class V, int NQ>
__device__ __forceinline__ void tile_ld4(const V* t, int q, V (&kv)[4]) {
  const float4* f = reinterpret_cast<const float4*>(t);
  if constexpr (sizeof(V) == 8) {
    const float4 a = f[q], b = f[NQ + q];
    kv[0] = make_float2(a.x, a.y), kv[1] = make_float2(a.z, a.w);
    kv[2] = make_float2(b.x, b.y), kv[3] = make_float2(b.z, b.w);
  } else {
#pragma unroll
    for (int a = 0; a < 4; ++a) kv[a] = t[a * NQ + q];
  }
}
template <class V, int NQ>
__device__ __forceinline__ void tile_st4(V* t, int q, const V (&kv)[4]) {
  float4* f = reinterpret_cast<float4*>(t);
  if constexpr (sizeof(V) == 8) {
    f[q] = make_float4(kv[0].x, kv[0].y, kv[1].x, kv[1].y);
    f[NQ + q] = make_float4(kv[2].x, kv[2].y, kv[3].x, kv[3].y);
  } else {
#pragma unroll
    for (int a = 0; a < 4; ++a) t[a * NQ + q] = kv[a];
  }
}

// hv += W[b] kv[b] over the four partners b = a ^ AX, real phases (in .x).
template <int AX, class V>
__device__ __forceinline__ void pauli4_add_re(V (&hv)[4], const V (&W)[4], const V (&kv)[4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    hv[a].x = fma(W[a ^ AX].x, kv[a ^ AX].x, hv[a].x);
    hv[a].y = fma(W[a ^ AX].x, kv[a ^ AX].y, hv[a].y);
  }
}
template <int AX, class V, class S>
__device__ __forceinline__ void pauli4_add1_re(V (&hv)[4], S f, const V (&kv)[4]) {
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    hv[a].x = fma(f, kv[a ^ AX].x, hv[a].x);
    hv[a].y = fma(f, kv[a ^ AX].y, hv[a].y);
  }
}

template <class R, bool WRITE, bool ACC, bool ADD, bool REAL>
__global__ void __launch_bounds__(kPTThreads, 2)
    k_pauli_tile(const cplx<R>* __restrict__ bra, const cplx<R>* __restrict__ ket, cplx<R>* __restrict__ out,
                 int64_t N, const DevPTPass pass, const DevGroupW* __restrict__ groups, const int* __restrict__ gxt,
                 int ng, const int64_t* __restrict__ hioff, const int* __restrict__ shifts,
                 const cplx<R>* __restrict__ tables, int nw, const DevTerm* __restrict__ terms, int nt, double dfac,
                 Scratch s, double* res) {
  using V = cplx<R>;
  constexpr int M = PTCfg<R>::M, CLOW = PTCfg<R>::CLOW, T = 1 << M, QPT = (T >> 2) / kPTThreads;
  static_assert(M - CLOW == kPTHiBits, "tile layout");
  extern __shared__ __align__(16) unsigned char smem[];
  const PTLayout<R> L(nw, nt, ng);
  V* tile = reinterpret_cast<V*>(smem);
  V* stab = reinterpret_cast<V*>(smem + L.stab);
  PTerm<R>* st = reinterpret_cast<PTerm<R>*>(smem + L.st);
  DevGroupW* sg = reinterpret_cast<DevGroupW*>(smem + L.sg);
  int64_t* shi = reinterpret_cast<int64_t*>(smem + L.shi);
  int* sxt = reinterpret_cast<int*>(smem + L.sxt);
  int* ssh = reinterpret_cast<int*>(smem + L.ssh);
  __shared__ uint64_t s_base, s_inc;
  for (int i = threadIdx.x; i < nw * kWinSize; i += kPTThreads) stab[i] = tables[i];
  for (int i = threadIdx.x; i < nt; i += kPTThreads) {
    const DevTerm t = terms[i];
    st[i] = PTerm<R>{t.z, mkc<R>((R)t.c.x, (R)t.c.y), mkc<R>((R)t.c.x, (R)t.c.y)};
  }
  for (int i = threadIdx.x; i < ng; i += kPTThreads) sg[i] = groups[i], sxt[i] = gxt[i];
  for (int i = threadIdx.x; i < (1 << kPTHiBits); i += kPTThreads) shi[i] = hioff[i];
  for (int i = threadIdx.x; i < nw; i += kPTThreads) ssh[i] = shifts[i];
  if (threadIdx.x == 0) {
    // the first tile's base (tile index blockIdx.x spread over the non-tile
    // qubits) and the increment for gridDim.x tiles
    uint64_t mm = pass.nontile_mask, b0 = 0, inc = 0;
    uint64_t t = blockIdx.x, g = gridDim.x;
    while (mm) {
      const uint64_t low = mm & (~mm + 1);
      if (t & 1) b0 |= low;
      if (g & 1) inc |= low;
      t >>= 1;
      g >>= 1;
      mm ^= low;
    }
    s_base = b0;
    s_inc = inc;
  }
  __syncthreads();
  const uint64_t ntm = pass.nontile_mask, inc = s_inc;
  uint64_t base = s_base;
  const V zero = mkc<R>(R(0), R(0));
  double acc[2] = {0, 0};
  for (int64_t tl = blockIdx.x; tl < pass.ntiles; tl += gridDim.x) {
    // the thread's quads: tile quads threadIdx.x + k * kPTThreads
#pragma unroll
    for (int k = 0; k < QPT; ++k) {
      const int u = (threadIdx.x + k * kPTThreads) << 2;
      const int64_t gqk = (int64_t)base + shi[u >> CLOW] + (u & ((1 << CLOW) - 1));
      V kv[4];
      if (!VQC_DCHECK(gqk + 3, N)) continue;
      load4<R>(ket + gqk, kv);
      tile_st4<V, (T >> 2)>(tile, u >> 2, kv);
    }
    __syncthreads();
    if (tl + gridDim.x < pass.ntiles) {
      // the next tile's amplitudes (and output words) into L2 while this one is computed
      const uint64_t nb = ((base | ~ntm) + inc) & ntm;
#pragma unroll
      for (int k = 0; k < QPT; ++k) {
        const int u = (threadIdx.x + k * kPTThreads) << 2;
        const int64_t g = (int64_t)nb + shi[u >> CLOW] + (u & ((1 << CLOW) - 1));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(ket + g));
        if (ADD) asm volatile("prefetch.global.L2 [%0];" ::"l"(out + g));
      }
    }
    // one quad at a time (four accumulators: the group loop's registers stay few)
#pragma unroll 1
    for (int k = 0; k < QPT; ++k) {
      const int u = (threadIdx.x + k * kPTThreads) << 2;
      const int64_t gqk = (int64_t)base + shi[u >> CLOW] + (u & ((1 << CLOW) - 1));
      if (!VQC_DCHECK(gqk + 3, N)) continue;
      V hv[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) hv[a] = zero;
      for (int gi = 0; gi < ng; ++gi) {
        const DevGroupW g = sg[gi];
        const int xt = sxt[gi];
        const int64_t jb = gqk ^ (int64_t)(g.x & ~3ull);
        V kv[4];
        if (xt >= 0) {
          const int ub = (u ^ xt) & ~3;
          if (!VQC_DCHECK(ub + 3, T)) continue;
          tile_ld4<V, (T >> 2)>(tile, ub >> 2, kv);
        } else {
          if (!VQC_DCHECK(jb + 3, N)) continue;
          load4<R>(ket + jb, kv);
        }
        int w = g.wbeg;
        V f = zero, W[4];
        if (g.low0) {
          const V* t = stab + (size_t)w * kWinSize + (jb & (kWinSize - 1));
#pragma unroll
          for (int b = 0; b < 4; ++b) W[b] = t[b];
          ++w;
        } else {
#pragma unroll
          for (int b = 0; b < 4; ++b) W[b] = zero;
        }
        for (; w < g.wend; ++w) {
          const V t = stab[(size_t)w * kWinSize + ((jb >> ssh[w]) & (kWinSize - 1))];
          f.x += t.x;
          if (!REAL) f.y += t.y;
        }
        for (int q = g.tbeg; q < g.tend; ++q) {
          const uint64_t m = (uint64_t)jb & st[q].z;
          const int hb = (__popc((unsigned)m ^ (unsigned)(m >> 32)) & 1);
          const V cc = st[q].c;
          if ((st[q].z & 3) == 0) {
            f.x += hb ? -cc.x : cc.x;
            if (!REAL) f.y += hb ? -cc.y : cc.y;
            continue;
          }
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const bool odd = (hb ^ (__popc((unsigned)(b & st[q].z)) & 1)) != 0;
            W[b].x += odd ? -cc.x : cc.x;
            if (!REAL) W[b].y += odd ? -cc.y : cc.y;
          }
        }
        const int ax = (int)(g.x & 3);
        if (g.low0 || g.rlow) {
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            W[b].x += f.x;
            if (!REAL) W[b].y += f.y;
          }
          if (REAL) {
            switch (ax) {
              case 0: pauli4_add_re<0>(hv, W, kv); break;
              case 1: pauli4_add_re<1>(hv, W, kv); break;
              case 2: pauli4_add_re<2>(hv, W, kv); break;
              default: pauli4_add_re<3>(hv, W, kv); break;
            }
          } else {
            switch (ax) {
              case 0: pauli4_add<0>(hv, W, kv); break;
              case 1: pauli4_add<1>(hv, W, kv); break;
              case 2: pauli4_add<2>(hv, W, kv); break;
              default: pauli4_add<3>(hv, W, kv); break;
            }
          }
        } else if (REAL) {
          switch (ax) {
            case 0: pauli4_add1_re<0>(hv, f.x, kv); break;
            case 1: pauli4_add1_re<1>(hv, f.x, kv); break;
            case 2: pauli4_add1_re<2>(hv, f.x, kv); break;
            default: pauli4_add1_re<3>(hv, f.x, kv); break;
          }
        } else {
          switch (ax) {
            case 0: pauli4_add1<0>(hv, f, kv); break;
            case 1: pauli4_add1<1>(hv, f, kv); break;
            case 2: pauli4_add1<2>(hv, f, kv); break;
            default: pauli4_add1<3>(hv, f, kv); break;
          }
        }
      }
      if (WRITE) {
        const R df = (R)dfac;  // 1 or 2
        V o[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) o[a] = mkc<R>(df * hv[a].x, df * hv[a].y);
        if (ADD) {
          V prev[4];
          load4<R>(out + gqk, prev);
#pragma unroll
          for (int a = 0; a < 4; ++a) o[a].x += prev[a].x, o[a].y += prev[a].y;
        }
        if constexpr (sizeof(R) == 4) {
          *reinterpret_cast<float4*>(out + gqk) = make_float4(o[0].x, o[0].y, o[1].x, o[1].y);
          *reinterpret_cast<float4*>(out + gqk + 2) = make_float4(o[2].x, o[2].y, o[3].x, o[3].y);
        } else {
#pragma unroll
          for (int a = 0; a < 4; ++a) out[gqk + a] = o[a];
        }
      }
      if (ACC) {
        V b[4];
        if (bra == ket) {
          tile_ld4<V, (T >> 2)>(tile, u >> 2, b);
        } else {
          load4<R>(bra + gqk, b);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const double2 bb = to_d2(b[a]), hh = to_d2(hv[a]);
          acc[0] = fma(bb.x, hh.x, fma(bb.y, hh.y, acc[0]));
          acc[1] = fma(bb.x, hh.y, fma(-bb.y, hh.x, acc[1]));
        }
      }
    }
    base = ((base | ~ntm) + inc) & ntm;
    __syncthreads();  // every read of this tile is done before the next one is stored
  }
  if (ACC) grid_reduce<2, kPTThreads>(acc, s, res);
}

// res[0..1] += the sums of the later passes, res[2p..2p+1] for p = 1..npass-1.
__global__ void k_add_passes(double* res, int npass) {
  if (threadIdx.x < 2)
    for (int p = 1; p < npass; ++p) res[threadIdx.x] += res[2 * p + threadIdx.x];
}

// Window tables of a prepared operator (terms grouped by flip mask; the
// expectation's coefficients c).  Returns false when the tables would not fit
// the kernel's shared memory (the quad kernel runs instead).
struct PauliWin {
  std::vector<DevGroupW> groups;
  std::vector<int> shifts;
  std::vector<cd> tables;  // nw * 64
  std::vector<DevTerm> rest;
};
static bool build_windows(const std::vector<DevGroup>& groups, const std::vector<DevTerm>& terms, size_t amp_bytes,
                          PauliWin& pw) {
  for (const DevGroup& g : groups) {
    std::vector<int> idx;
    for (int t = g.start; t < g.start + g.count; ++t) idx.push_back(t);
    auto lo_of = [&](int t) { return terms[t].z ? __builtin_ctzll(terms[t].z) : 0; };
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return lo_of(a) < lo_of(b); });
    struct Win {
      int s;
      std::vector<int> ts;
    };
    std::vector<Win> wins;
    cd c0(0);
    std::vector<DevTerm> rest;
    for (int t : idx) {
      const uint64_t z = terms[t].z;
      if (!z) {
        c0 += cd(terms[t].c.x, terms[t].c.y);
        continue;
      }
      const int lo = __builtin_ctzll(z), hi = 63 - __builtin_clzll(z);
      Win* w = nullptr;
      for (Win& x : wins)
        if (x.s <= lo && hi < x.s + kWinBits) w = &x;
      if (!w) {
        int sh = -1;
        if (hi < kWinBits)
          sh = 0;
        else if (lo >= 2 && hi - lo < kWinBits)
          sh = lo;
        if (sh < 0) {
          rest.push_back(terms[t]);
          continue;
        }
        wins.push_back(Win{sh, {}});
        w = &wins.back();
      }
      w->ts.push_back(t);
    }
    // a table pays for its lookup only when it folds several terms: windows of
    // one or two terms are evaluated term by term (one parity each)
    std::vector<Win> keep;
    for (Win& w : wins) {
      if ((int)w.ts.size() >= 3) {
        keep.push_back(std::move(w));
      } else {
        for (int t : w.ts) rest.push_back(terms[t]);
      }
    }
    wins.swap(keep);
    if (c0 != cd(0) && wins.empty()) {
      DevTerm ct{};
      ct.z = 0;
      ct.c = make_double2(c0.real(), c0.imag());
      ct.d = ct.c;
      rest.push_back(ct);
      c0 = cd(0);
    }
    std::vector<std::vector<cd>> tabs;
    for (const Win& w : wins) {
      std::vector<cd> tab(kWinSize, cd(0));
      for (int t : w.ts) {
        const cd c(terms[t].c.x, terms[t].c.y);
        const uint64_t zl = terms[t].z >> w.s;
        for (int u = 0; u < kWinSize; ++u) tab[u] += (__builtin_popcountll((uint64_t)u & zl) & 1) ? -c : c;
      }
      tabs.push_back(std::move(tab));
    }
    if (c0 != cd(0))
      for (cd& v : tabs[0]) v += c0;
    // the window at bit 0 (if any) first
    std::vector<int> order(wins.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return (wins[a].s == 0) > (wins[b].s == 0); });
    DevGroupW d{};
    d.x = g.x;
    d.wbeg = (int)pw.shifts.size();
    for (int i : order) {
      pw.shifts.push_back(wins[i].s);
      pw.tables.insert(pw.tables.end(), tabs[i].begin(), tabs[i].end());
    }
    d.wend = (int)pw.shifts.size();
    d.low0 = !wins.empty() && wins[order[0]].s == 0;
    d.tbeg = (int)pw.rest.size();
    pw.rest.insert(pw.rest.end(), rest.begin(), rest.end());
    d.tend = (int)pw.rest.size();
    d.rlow = 0;
    for (const DevTerm& t : rest)
      if (t.z & 3) d.rlow = 1;
    pw.groups.push_back(d);
  }
  return pw.tables.size() * amp_bytes <= kWinMaxTableBytes;
}

// tr(H rho) for a Pauli sum on a density matrix (expecs_dm.jl:19-30; the
// reference sums tr(M_key rho_key) per position key, expec_dm_serial.jl).
// With P|j> = c' (-1)^{|j & z|} |j ^ x> (the state-vector kernels' phase
// convention), tr(P rho) = sum_k c' (-1)^{|k & z|} rho[k, k ^ x]: one entry
// per row and flip mask, read at k + N (k ^ x) of the column-major storage.
template <class R>
__global__ void __launch_bounds__(kRedThreads)
    k_pauli_dm(const cplx<R>* __restrict__ rho, int64_t N, const DevGroup* __restrict__ groups, int ng,
               const DevTerm* __restrict__ terms, int nt, Scratch s, double* res) {
  extern __shared__ unsigned char smem[];
  DevGroup* sg = reinterpret_cast<DevGroup*>(smem);
  DevTerm* st = reinterpret_cast<DevTerm*>(smem + sizeof(DevGroup) * ng);
  for (int i = threadIdx.x; i < ng; i += blockDim.x) sg[i] = groups[i];
  for (int i = threadIdx.x; i < nt; i += blockDim.x) st[i] = terms[i];
  __syncthreads();
  double acc[2] = {0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < N; k += stride) {
    for (int gi = 0; gi < ng; ++gi) {
      const DevGroup g = sg[gi];
      const double2 v = to_d2(rho[k + N * (k ^ (int64_t)g.x)]);
      double2 f = make_double2(0, 0);
      for (int q = g.start; q < g.start + g.count; ++q) {
        const bool odd = (__popcll((unsigned long long)k & st[q].z) & 1) != 0;
        f.x += odd ? -st[q].c.x : st[q].c.x;
        f.y += odd ? -st[q].c.y : st[q].c.y;
      }
      acc[0] = fma(f.x, v.x, fma(-f.y, v.y, acc[0]));
      acc[1] = fma(f.x, v.y, fma(f.y, v.x, acc[1]));
    }
  }
  grid_reduce<2>(acc, s, res);
}

template <class R>
__global__ void k_axpy(cplx<R>* y, const cplx<R>* x, int64_t N) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N; i += (int64_t)gridDim.x * blockDim.x) {
    cplx<R> a = y[i], b = x[i];
    y[i] = mkc<R>(a.x + b.x, a.y + b.y);
  }
}

int axpy_device(vqc_state h, void* y, const void* x) {
  const int g = launch_grid(h->device, h->size());
  if (h->dtype == VQC_C64)
    k_axpy<float><<<g, 256, 0, h->stream>>>((float2*)y, (const float2*)x, h->size());
  else
    k_axpy<double><<<g, 256, 0, h->stream>>>((double2*)y, (const double2*)x, h->size());
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

// Tile passes of a prepared operator (see k_pauli_tile): the groups are
// reordered by pass; pass p runs groups [gbeg[p], gbeg[p+1]).
constexpr int kMaxPTPasses = 3;
constexpr int kPTMinQubits = 18;
constexpr int kPTNearBits = 5;  // flip masks below bit M + 5 find their partners in L2 in pass 0
struct PTPlan {
  std::vector<DevPTPass> passes;
  std::vector<int> gbeg;
  std::vector<int> xt;           // per (reordered) group: tile-space flip mask, or -1: partner from global memory
  std::vector<int64_t> hioff;    // per pass: global offset of each tile high-bit pattern (2^kPTHiBits entries)
};
static void plan_pauli_tiles(int nq, int M, int clow, bool write, std::vector<DevGroupW>& groups, PTPlan& pt) {
  const uint64_t all = nq >= 64 ? ~0ull : ((1ull << nq) - 1), lowm = (1ull << clow) - 1;
  const int nh = M - clow;
  std::vector<uint64_t> tmask{((1ull << M) - 1) & all};
  std::vector<int> pass_of(groups.size(), -1);
  for (size_t i = 0; i < groups.size(); ++i)
    if (!(groups[i].x & ~tmask[0])) pass_of[i] = 0;
  // a further pass covers the high qubits the remaining far flip masks use;
  // it streams the state once more, so it must take several groups
  const int min_local = write ? 3 : 2;
  while ((int)tmask.size() < kMaxPTPasses) {
    uint64_t U = 0;
    int nfar = 0;
    for (size_t i = 0; i < groups.size(); ++i)
      if (pass_of[i] < 0 && 63 - __builtin_clzll(groups[i].x) >= M + kPTNearBits) {
        U |= groups[i].x & ~lowm;
        ++nfar;
      }
    if (!nfar) break;
    uint64_t H = 0;
    if (__builtin_popcountll(U) <= nh) {
      H = U;
      for (int q = nq - 1; q >= clow && __builtin_popcountll(H) < nh; --q) H |= 1ull << q;
    } else {
      for (int q = 63; q >= clow && __builtin_popcountll(H) < nh; --q)
        if (U >> q & 1) H |= 1ull << q;
    }
    const uint64_t tm = lowm | H;
    int nloc = 0;
    for (size_t i = 0; i < groups.size(); ++i)
      if (pass_of[i] < 0 && !(groups[i].x & ~tm)) ++nloc;
    if (nloc < min_local) break;
    for (size_t i = 0; i < groups.size(); ++i)
      if (pass_of[i] < 0 && !(groups[i].x & ~tm)) pass_of[i] = (int)tmask.size();
    tmask.push_back(tm);
  }
  for (int& p : pass_of)
    if (p < 0) p = 0;  // partners from global memory in the first pass
  std::vector<DevGroupW> reordered;
  pt.gbeg.assign(1, 0);
  for (size_t p = 0; p < tmask.size(); ++p) {
    // tile bit b -> global qubit
    int tq[64];
    int nb = 0;
    for (int q = 0; q < 64; ++q)
      if (tmask[p] >> q & 1) tq[nb++] = q;
    for (size_t i = 0; i < groups.size(); ++i) {
      if (pass_of[i] != (int)p) continue;
      const uint64_t x = groups[i].x;
      int xt = -1;
      if (!(x & ~tmask[p])) {
        xt = 0;
        for (int b = 0; b < nb; ++b)
          if (x >> tq[b] & 1) xt |= 1 << b;
      }
      reordered.push_back(groups[i]);
      pt.xt.push_back(xt);
    }
    pt.gbeg.push_back((int)reordered.size());
    for (int h = 0; h < (1 << kPTHiBits); ++h) {
      int64_t off = 0;
      for (int i = 0; i < nh; ++i)
        if (h >> i & 1) off |= int64_t(1) << tq[clow + i];
      pt.hioff.push_back(off);
    }
    DevPTPass dp;
    dp.nontile_mask = all & ~tmask[p];
    dp.ntiles = int64_t(1) << (nq - M);
    pt.passes.push_back(dp);
  }
  groups.swap(reordered);
}

template <class R, bool WRITE, bool ACC, bool ADD, bool REAL>
static int pt_launch1(vqc_state h, const void* bra, const void* ket, void* out, const DevPTPass& pass,
                      const DevGroupW* g, const int* xt, int ng, const int64_t* hioff, const int* shifts,
                      const void* tables, int nw, const DevTerm* terms, int nt, double dfac, double* res) {
  auto k = k_pauli_tile<R, WRITE, ACC, ADD, REAL>;
  const size_t smem = PTLayout<R>(nw, nt, ng).total;
  VQC_CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<int64_t>(pass.ntiles, (int64_t)device_info(h->device).sms * 2);
  k<<<grid, kPTThreads, smem, h->stream>>>((const cplx<R>*)bra, (const cplx<R>*)ket, (cplx<R>*)out, h->size(), pass,
                                           g, xt, ng, hioff, shifts, (const cplx<R>*)tables, nw, terms, nt, dfac,
                                           h->scr, res);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}
template <class R, bool REAL>
static int pt_launch(vqc_state h, bool write, bool acc, bool add, const void* bra, const void* ket, void* out,
                     const DevPTPass& pass, const DevGroupW* g, const int* xt, int ng, const int64_t* hioff,
                     const int* shifts, const void* tables, int nw, const DevTerm* terms, int nt, double dfac,
                     double* res) {
#define VQC_PT(W, A, D) \
  pt_launch1<R, W, A, D, REAL>(h, bra, ket, out, pass, g, xt, ng, hioff, shifts, tables, nw, terms, nt, dfac, res)
  if (!write) return VQC_PT(false, true, false);
  if (acc) return add ? VQC_PT(true, true, true) : VQC_PT(true, true, false);
  return add ? VQC_PT(true, false, true) : VQC_PT(true, false, false);
#undef VQC_PT
}

// ----------------------------------------------------------------------------- compiled tile passes
// k_pauli_tile decodes every group at run time (descriptor and term loads, a
// loop per group, a switch on the partner permutation).  On states of
// 2^kPTJitMinQubits amplitudes and more each pass is compiled once per
// operator structure (NVRTC, cached by source): the groups unrolled, flip
// masks, Z masks, tile offsets and table shifts as constants, the coefficients
// of the terms outside the window tables a kernel parameter (new coefficient
// values reuse the kernel); the window tables stay in shared memory.
constexpr int kPTJitMinQubits = 20;
constexpr size_t kPTJitMaxCoefBytes = 30000;  // kernel-parameter space

static int parity64(uint64_t m) { return __builtin_popcountll(m) & 1; }

// Block shape of the compiled passes: 512 threads, two CTAs per SM, or 256
// threads, three CTAs (VQC_PAULI_NT=256; measured slower at 2^26 FP32
// amplitudes: 1.09 against 0.965 ms per Pauli step).
struct PTJitShape {
  int threads, per_sm;
};
static PTJitShape pt_jit_shape() {
  const char* v = std::getenv("VQC_PAULI_NT");
  if (v && *v && std::atoi(v) == 256) return {256, 3};
  return {512, 2};
}

// Source of one compiled pass; coef receives the parameter values in the
// order the source reads them.
static std::string pt_jit_source(bool f32, bool write, bool acc, bool add, bool real, int nw,
                                 const DevGroupW* groups, const int* xts, int ng, const PauliWin& pw,
                                 std::vector<double>& coef, const PTJitShape& shape) {
  const int M = f32 ? PTCfg<float>::M : PTCfg<double>::M, CLOW = f32 ? PTCfg<float>::CLOW : PTCfg<double>::CLOW;
  const char* R = f32 ? "float" : "double";
  std::ostringstream os;
  coef.clear();
  std::ostringstream body;
  for (int gi = 0; gi < ng; ++gi) {
    const DevGroupW& g = groups[gi];
    const uint64_t XQ = g.x & ~3ull;
    const int AX = (int)(g.x & 3);
    const bool four = g.low0 || g.rlow;
    body << "      {  // flip mask 0x" << std::hex << g.x << std::dec << "\n";
    if (xts[gi] >= 0)
      body << "        V k[4];\n        tld4(tile, (u ^ " << xts[gi] << ") >> 2, k);\n";
    else
      body << "        V k[4];\n        ld4(ket + (g ^ " << (long long)XQ << "ll), k);\n";
    body << "        R fx = 0" << (real ? "" : ", fy = 0") << ";\n";
    if (four) body << "        R Wx[4] = {0, 0, 0, 0}" << (real ? "" : ", Wy[4] = {0, 0, 0, 0}") << ";\n";
    int w = g.wbeg;
    if (g.low0) {
      body << "        { const V* t = stab + " << w * kWinSize << " + (((unsigned long long)g ^ " << XQ
           << "ull) & 63);\n          for (int b = 0; b < 4; ++b) { Wx[b] += t[b].x;" << (real ? "" : " Wy[b] += t[b].y;")
           << " } }\n";
      ++w;
    }
    for (; w < g.wend; ++w)
      body << "        { const V t = stab[" << w * kWinSize << " + ((((unsigned long long)g ^ " << XQ << "ull) >> "
           << pw.shifts[w] << ") & 63)]; fx += t.x;" << (real ? "" : " fy += t.y;") << " }\n";
    for (int q = g.tbeg; q < g.tend; ++q) {
      const DevTerm& t = pw.rest[q];
      const uint64_t zh = t.z & ~3ull, zl = t.z & 3;
      const int cs = parity64(XQ & zh);
      const int ci = (int)coef.size();
      coef.push_back(t.c.x);
      if (!real) coef.push_back(t.c.y);
      std::string o;
      if (zh == 0)
        o = cs ? "true" : "false";
      else
        o = std::string("(par((unsigned long long)g & ") + std::to_string((unsigned long long)zh) + "ull)" +
            (cs ? " ^ 1)" : ")") + " != 0";
      body << "        { const bool o = " << o << ";\n";
      body << "          const R ex = o ? -coef.c[" << ci << "] : coef.c[" << ci << "];\n";
      if (!real) body << "          const R ey = o ? -coef.c[" << ci + 1 << "] : coef.c[" << ci + 1 << "];\n";
      if (zl == 0) {
        body << "          fx += ex;" << (real ? "" : " fy += ey;") << " }\n";
      } else {
        body << "         ";
        for (int b = 0; b < 4; ++b) {
          const bool sb = parity64((uint64_t)b & zl);
          body << " Wx[" << b << "] " << (sb ? "-=" : "+=") << " ex;";
          if (!real) body << " Wy[" << b << "] " << (sb ? "-=" : "+=") << " ey;";
        }
        body << " }\n";
      }
    }
    // output a takes the partner b = a ^ AX with the phase at b
    for (int a = 0; a < 4; ++a) {
      const int b = a ^ AX;
      const std::string cx = four ? "(Wx[" + std::to_string(b) + "] + fx)" : "fx";
      const std::string cy = four ? "(Wy[" + std::to_string(b) + "] + fy)" : "fy";
      if (real) {
        body << "        h[" << a << "].x = FMA(" << cx << ", k[" << b << "].x, h[" << a << "].x);"
             << " h[" << a << "].y = FMA(" << cx << ", k[" << b << "].y, h[" << a << "].y);\n";
      } else {
        body << "        { const R cx = " << cx << ", cy = " << cy << ";\n"
             << "          h[" << a << "].x = FMA(cx, k[" << b << "].x, FMA(-cy, k[" << b << "].y, h[" << a << "].x));\n"
             << "          h[" << a << "].y = FMA(cx, k[" << b << "].y, FMA(cy, k[" << b << "].x, h[" << a << "].y)); }\n";
      }
    }
    body << "      }\n";
  }
  const int nc = std::max<int>(1, (int)coef.size());
  os << "typedef " << R << " R;\ntypedef " << (f32 ? "float2" : "double2") << " V;\n"
     << "struct Scratch { double* partials; unsigned* counter; double* result; int max_blocks; };\n"
     << "struct PassT { unsigned long long nontile_mask; long long ntiles; };\n"
     << "struct Coef { R c[" << nc << "]; };\n"
     << "#define FMA " << (f32 ? "__fmaf_rn" : "__fma_rn") << "\n"
     << "__device__ __forceinline__ int par(unsigned long long m) {\n"
     << "  return (__popc((unsigned)m) ^ __popc((unsigned)(m >> 32))) & 1;\n}\n";
  if (f32)
    os << "__device__ __forceinline__ void ld4(const V* p, V (&k)[4]) {\n"
       << "  const float4 a = *reinterpret_cast<const float4*>(p), b = *reinterpret_cast<const float4*>(p + 2);\n"
       << "  k[0] = make_float2(a.x, a.y); k[1] = make_float2(a.z, a.w); k[2] = make_float2(b.x, b.y); "
          "k[3] = make_float2(b.z, b.w);\n}\n"
       << "__device__ __forceinline__ void st4(V* p, const V (&k)[4]) {\n"
       << "  *reinterpret_cast<float4*>(p) = make_float4(k[0].x, k[0].y, k[1].x, k[1].y);\n"
       << "  *reinterpret_cast<float4*>(p + 2) = make_float4(k[2].x, k[2].y, k[3].x, k[3].y);\n}\n";
  else
    os << "__device__ __forceinline__ void ld4(const V* p, V (&k)[4]) { for (int a = 0; a < 4; ++a) k[a] = p[a]; }\n"
       << "__device__ __forceinline__ void st4(V* p, const V (&k)[4]) { for (int a = 0; a < 4; ++a) p[a] = k[a]; }\n";
  // the tile as 16-byte planes (quad q: one element per plane), bank-conflict free
  const int nq4 = 1 << (M - 2);
  if (f32)
    os << "__device__ __forceinline__ void tld4(const V* t, int q, V (&k)[4]) {\n"
       << "  const float4 a = reinterpret_cast<const float4*>(t)[q], b = reinterpret_cast<const float4*>(t)[" << nq4
       << " + q];\n"
       << "  k[0] = make_float2(a.x, a.y); k[1] = make_float2(a.z, a.w); k[2] = make_float2(b.x, b.y); "
          "k[3] = make_float2(b.z, b.w);\n}\n"
       << "__device__ __forceinline__ void tst4(V* t, int q, const V (&k)[4]) {\n"
       << "  reinterpret_cast<float4*>(t)[q] = make_float4(k[0].x, k[0].y, k[1].x, k[1].y);\n"
       << "  reinterpret_cast<float4*>(t)[" << nq4 << " + q] = make_float4(k[2].x, k[2].y, k[3].x, k[3].y);\n}\n";
  else
    os << "__device__ __forceinline__ void tld4(const V* t, int q, V (&k)[4]) { for (int a = 0; a < 4; ++a) k[a] = t[a * "
       << nq4 << " + q]; }\n"
       << "__device__ __forceinline__ void tst4(V* t, int q, const V (&k)[4]) { for (int a = 0; a < 4; ++a) t[a * " << nq4
       << " + q] = k[a]; }\n";
  os << "extern \"C\" __global__ void __launch_bounds__(" << shape.threads << ", " << shape.per_sm << ")\n"
     << "vqc_pauli(const V* __restrict__ bra, const V* __restrict__ ket, V* __restrict__ out, const PassT pass,\n"
     << "          const long long* __restrict__ hioff, const V* __restrict__ tables, double dfac, Scratch s,\n"
     << "          double* res, const __grid_constant__ Coef coef) {\n"
     << "  constexpr int M = " << M << ", CLOW = " << CLOW << ", T = 1 << M, NT = " << shape.threads
     << ", QPT = (T >> 2) / NT, NW = " << nw << ";\n"
     << "  extern __shared__ __align__(16) unsigned char smem[];\n"
     << "  V* tile = reinterpret_cast<V*>(smem);\n  V* stab = tile + T;\n"
     << "  long long* shi = reinterpret_cast<long long*>(stab + NW * 64);\n"
     << "  __shared__ unsigned long long s_base, s_inc;\n"
     << "  __shared__ double sred[NT / 32][2];\n  __shared__ bool s_last;\n"
     << "  for (int i = threadIdx.x; i < NW * 64; i += NT) stab[i] = tables[i];\n"
     << "  for (int i = threadIdx.x; i < " << (1 << kPTHiBits) << "; i += NT) shi[i] = hioff[i];\n"
     << "  if (threadIdx.x == 0) {\n"
     << "    unsigned long long mm = pass.nontile_mask, b0 = 0, inc = 0, t = blockIdx.x, gd = gridDim.x;\n"
     << "    while (mm) {\n      const unsigned long long low = mm & (~mm + 1);\n"
     << "      if (t & 1) b0 |= low;\n      if (gd & 1) inc |= low;\n"
     << "      t >>= 1; gd >>= 1; mm ^= low;\n    }\n    s_base = b0; s_inc = inc;\n  }\n"
     << "  __syncthreads();\n"
     << "  const unsigned long long ntm = pass.nontile_mask, inc = s_inc;\n"
     << "  unsigned long long base = s_base;\n"
     << "  double acc0 = 0, acc1 = 0;\n"
     << "  for (long long tl = blockIdx.x; tl < pass.ntiles; tl += gridDim.x) {\n"
     << "#pragma unroll\n    for (int kq = 0; kq < QPT; ++kq) {\n"
     << "      const int u = (threadIdx.x + kq * NT) << 2;\n"
     << "      const long long g = (long long)base + shi[u >> CLOW] + (u & ((1 << CLOW) - 1));\n"
     << "      V k[4];\n      ld4(ket + g, k);\n      tst4(tile, u >> 2, k);\n    }\n"
     << "    __syncthreads();\n"
     << "    if (tl + gridDim.x < pass.ntiles) {\n"
     << "      const unsigned long long nb = ((base | ~ntm) + inc) & ntm;\n"
     << "#pragma unroll\n      for (int kq = 0; kq < QPT; ++kq) {\n"
     << "        const int u = (threadIdx.x + kq * NT) << 2;\n"
     << "        const long long g = (long long)nb + shi[u >> CLOW] + (u & ((1 << CLOW) - 1));\n"
     << "        asm volatile(\"prefetch.global.L2 [%0];\" ::\"l\"(ket + g));\n"
     << (add ? "        asm volatile(\"prefetch.global.L2 [%0];\" ::\"l\"(out + g));\n" : "")
     << "      }\n    }\n"
     << "#pragma unroll 1\n    for (int kq = 0; kq < QPT; ++kq) {\n"
     << "      const int u = (threadIdx.x + kq * NT) << 2;\n"
     << "      const long long g = (long long)base + shi[u >> CLOW] + (u & ((1 << CLOW) - 1));\n"
     << "      V h[4];\n      for (int a = 0; a < 4; ++a) h[a].x = h[a].y = 0;\n"
     << body.str();
  if (write) {
    os << "      {\n        const R df = (R)dfac;\n        V o[4];\n"
       << "        for (int a = 0; a < 4; ++a) { o[a].x = df * h[a].x; o[a].y = df * h[a].y; }\n";
    if (add)
      os << "        V pv[4];\n        ld4(out + g, pv);\n"
         << "        for (int a = 0; a < 4; ++a) { o[a].x += pv[a].x; o[a].y += pv[a].y; }\n";
    os << "        st4(out + g, o);\n      }\n";
  }
  if (acc)
    os << "      {\n        V bv[4];\n        if (bra == ket) tld4(tile, u >> 2, bv); else ld4(bra + g, bv);\n"
       << "        for (int a = 0; a < 4; ++a) {\n"
       << "          const double bx = bv[a].x, by = bv[a].y, hx = h[a].x, hy = h[a].y;\n"
       << "          acc0 = __fma_rn(bx, hx, __fma_rn(by, hy, acc0));\n"
       << "          acc1 = __fma_rn(bx, hy, __fma_rn(-by, hx, acc1));\n"
       << "        }\n      }\n";
  os << "    }\n    base = ((base | ~ntm) + inc) & ntm;\n    __syncthreads();\n  }\n";
  if (acc) {
    // the deterministic grid reduction: block sums in warp order, then the
    // last block adds the block partials in block order
    os << "  {\n    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;\n"
       << "    double v0 = acc0, v1 = acc1;\n"
       << "    for (int o = 16; o > 0; o >>= 1) { v0 += __shfl_xor_sync(0xffffffffu, v0, o);"
          " v1 += __shfl_xor_sync(0xffffffffu, v1, o); }\n"
       << "    if (lane == 0) { sred[warp][0] = v0; sred[warp][1] = v1; }\n    __syncthreads();\n"
       << "    if (threadIdx.x < 2) {\n      double v = 0;\n"
       << "      for (int w = 0; w < NT / 32; ++w) v += sred[w][threadIdx.x];\n"
       << "      s.partials[(unsigned long long)blockIdx.x * " << kMaxAcc << " + threadIdx.x] = v;\n    }\n"
       << "    __threadfence();\n    __syncthreads();\n"
       << "    if (threadIdx.x == 0) s_last = (atomicAdd(s.counter, 1u) == gridDim.x - 1);\n"
       << "    __syncthreads();\n    if (!s_last) return;\n    __threadfence();\n"
       << "    for (int i = 0; i < 2; ++i) {\n      double v = 0;\n"
       << "      for (int b = threadIdx.x; b < (int)gridDim.x; b += NT) v += __ldcg(&s.partials[(unsigned long long)b * "
       << kMaxAcc << " + i]);\n"
       << "      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);\n"
       << "      __syncthreads();\n      if (lane == 0) sred[warp][0] = v;\n      __syncthreads();\n"
       << "      if (threadIdx.x == 0) {\n        double t = 0;\n"
       << "        for (int w = 0; w < NT / 32; ++w) t += sred[w][0];\n        res[i] = t;\n      }\n    }\n"
       << "    if (threadIdx.x == 0) *s.counter = 0;\n  }\n";
  }
  os << "}\n";
  return os.str();
}

// Launches a compiled pass (kernel from jit_kernels, name vqc_pauli).
static int pt_jit_launch(vqc_state h, const void* kernel, bool f32, const void* bra, const void* ket, void* out,
                         const DevPTPass& pass, const int64_t* hioff, const void* tables, int nw, double dfac,
                         double* res, const std::vector<double>& coef, const PTJitShape& shape) {
  const size_t amp = f32 ? 8 : 16;
  const size_t smem = (amp << (f32 ? PTCfg<float>::M : PTCfg<double>::M)) + (size_t)nw * kWinSize * amp +
                      sizeof(int64_t) * (size_t(1) << kPTHiBits);
  VQC_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int grid = (int)std::min<int64_t>(pass.ntiles, (int64_t)device_info(h->device).sms * shape.per_sm);
  std::vector<unsigned char> cb(std::max<size_t>(1, coef.size()) * (f32 ? 4 : 8), 0);
  for (size_t i = 0; i < coef.size(); ++i) {
    if (f32) {
      const float v = (float)coef[i];
      std::memcpy(cb.data() + 4 * i, &v, 4);
    } else {
      std::memcpy(cb.data() + 8 * i, &coef[i], 8);
    }
  }
  Scratch s = h->scr;
  void* args[] = {(void*)&bra, (void*)&ket, (void*)&out, (void*)&pass, (void*)&hioff, (void*)&tables,
                  (void*)&dfac, (void*)&s, (void*)&res, (void*)cb.data()};
  VQC_CK(cudaLaunchKernel(kernel, dim3(grid), dim3(shape.threads), args, smem, h->stream));
  return VQC_OK;
}

// Runs the Pauli kernel in chunks of at most kMaxTermsPerLaunch terms; the
// expectation (if any) is summed on the host in FP64 over chunks.
int pauli_run(vqc_state h, const void* bra, const void* ket, void* out, const vqc_pauli* terms, int nterms,
              bool write, bool acc, bool hermitian_part, double* result, bool* deferred = nullptr) {
  if (deferred) *deferred = false;
  double tot[2] = {0, 0};
  bool first = true;
  int start = 0;
  do {
    const int cnt = std::min(kMaxTermsPerLaunch, nterms - start);
    PauliPlan p;
    int rc = plan_pauli(h->nq, terms + start, cnt, hermitian_part, p);
    if (rc) return rc;
    if (p.groups.empty()) {
      // empty operator: H psi = 0
      if (write && first) VQC_CK(cudaMemsetAsync(out, 0, h->size() * h->amp_bytes(), h->stream));
      break;
    }
    // quad kernels (n >= 2): window tables when one coefficient set serves the
    // expectation and the written operator and the tables fit; otherwise the
    // terms of each group sorted by their low-bit class
    const bool quad = h->nq >= 2;
    bool sep = false;
    {
      const double f = hermitian_part ? 2.0 : 1.0;
      for (const DevTerm& t : p.terms)
        if (t.d.x != f * t.c.x || t.d.y != f * t.c.y) sep = true;
    }
    PauliWin pw;
    const bool win = quad && !sep && build_windows(p.groups, p.terms, h->amp_bytes(), pw);
    // tile passes (k_pauli_tile) for states of 2^kPTMinQubits amplitudes and
    // more whose operator has window tables (VQC_PAULI_TILE=0: one pass with
    // every partner read from global memory)
    PTPlan pt;
    bool tiled = false, real = false;
    if (win && h->nq >= kPTMinQubits && env_on("VQC_PAULI_TILE", true)) {
      const bool f32 = h->amp_bytes() == 8;
      const size_t need = f32 ? PTLayout<float>((int)pw.shifts.size(), (int)pw.rest.size(), (int)pw.groups.size()).total
                              : PTLayout<double>((int)pw.shifts.size(), (int)pw.rest.size(), (int)pw.groups.size()).total;
      if (need <= (size_t)device_info(h->device).max_smem_optin) {
        tiled = true;
        plan_pauli_tiles(h->nq, f32 ? PTCfg<float>::M : PTCfg<double>::M, f32 ? PTCfg<float>::CLOW : PTCfg<double>::CLOW,
                         write, pw.groups, pt);
        real = true;
        for (const cd& v : pw.tables)
          if (v.imag() != 0) real = false;
        for (const DevTerm& t : pw.rest)
          if (t.c.y != 0) real = false;
      }
    }
    // VQC_PAULI_SPLIT=1: groups whose flip masks reach beyond the amplitudes one
    // wave of the grid covers (the XXZ chain's top pairs on a state larger than
    // L2) run in a second launch whose traversal puts the top bits in the fast
    // dimension, so their partner reads hit amplitudes read at the same time.
    // It reads 2.76 GB instead of 3.69 GB at 2^26 FP32 amplitudes but takes
    // longer on B200 (1.70 against 1.62 ms: the first launch is issue-bound),
    // so one launch is the default.
    const int grid = reduction_grid(h->device, h->size());
    int nlow = (int)pw.groups.size(), tlo = 0, ths = 0, thl = 0;
    if (win && !tiled && h->nq >= 20 && env_on("VQC_PAULI_SPLIT", false)) {
      const int nq4 = h->nq - 2, tlo_ = 5;
      int wave = 0;
      while ((int64_t(2) << wave) <= (int64_t)grid * kRedThreads) ++wave;  // quad bits one wave covers
      std::stable_partition(pw.groups.begin(), pw.groups.end(), [&](const DevGroupW& g) {
        return (g.x >> 2) < (uint64_t(1) << wave);
      });
      uint64_t hx = 0;
      nlow = 0;
      for (const DevGroupW& g : pw.groups) {
        if ((g.x >> 2) < (uint64_t(1) << wave))
          ++nlow;
        else
          hx |= g.x >> 2;
      }
      if (hx) {
        const int lowbit = __builtin_ctzll(hx);
        if (lowbit >= tlo_ && nq4 - lowbit + tlo_ <= wave) {
          tlo = tlo_;
          ths = lowbit;
          thl = nq4 - lowbit;
        } else {
          nlow = (int)pw.groups.size();  // no traversal fits: one launch
        }
      }
    }
    std::vector<DevGroup4> g4;
    if (quad && !win) {
      std::vector<DevTerm> sorted;
      for (const DevGroup& g : p.groups) {
        DevGroup4 q{};
        q.x = g.x;
        for (int c = 0; c < 4; ++c) {
          q.cs[c] = (int)sorted.size();
          for (int t = g.start; t < g.start + g.count; ++t)
            if ((int)(p.terms[t].z & 3) == c) sorted.push_back(p.terms[t]);
        }
        q.cs[4] = (int)sorted.size();
        g4.push_back(q);
      }
      p.terms.swap(sorted);
    }
    // device image: [window tables][groups][shifts][terms in no window] for the
    // window kernel, [groups][terms] otherwise
    const size_t amp = h->amp_bytes();
    const size_t wtb = win ? pw.tables.size() * amp : 0,
                 gb = win ? sizeof(DevGroupW) * pw.groups.size()
                          : (quad ? sizeof(DevGroup4) * g4.size() : sizeof(DevGroup) * p.groups.size()),
                 shb = win ? sizeof(int) * ((pw.shifts.size() + 3) & ~size_t(3)) : 0,
                 tb = sizeof(DevTerm) * (win ? pw.rest.size() : p.terms.size());
    // tile passes: [flip masks in tile space][high-bit offset tables] after the rest
    const size_t xtb = tiled ? ((sizeof(int) * pt.xt.size() + 15) & ~size_t(15)) : 0,
                 hob = tiled ? sizeof(int64_t) * pt.hioff.size() : 0;
    std::vector<unsigned char> buf(wtb + gb + shb + tb + xtb + hob, 0);
    if (tiled) {
      std::memcpy(buf.data() + wtb + gb + shb + tb, pt.xt.data(), sizeof(int) * pt.xt.size());
      std::memcpy(buf.data() + wtb + gb + shb + tb + xtb, pt.hioff.data(), hob);
    }
    if (win) {
      for (size_t i = 0; i < pw.tables.size(); ++i) {
        if (amp == 8) {
          const float2 v = make_float2((float)pw.tables[i].real(), (float)pw.tables[i].imag());
          std::memcpy(buf.data() + i * amp, &v, amp);
        } else {
          const double2 v = make_double2(pw.tables[i].real(), pw.tables[i].imag());
          std::memcpy(buf.data() + i * amp, &v, amp);
        }
      }
      std::memcpy(buf.data() + wtb, pw.groups.data(), gb);
      if (!pw.shifts.empty()) std::memcpy(buf.data() + wtb + gb, pw.shifts.data(), sizeof(int) * pw.shifts.size());
      if (tb) std::memcpy(buf.data() + wtb + gb + shb, pw.rest.data(), tb);
    } else {
      std::memcpy(buf.data(), quad ? (const void*)g4.data() : (const void*)p.groups.data(), gb);
      std::memcpy(buf.data() + gb, p.terms.data(), tb);
    }
    if ((rc = upload_ops(h, buf.data(), buf.size()))) return rc;
    const unsigned char* ob = (const unsigned char*)h->opbuf;
    const DevGroup* dg = (const DevGroup*)(ob + wtb);
    const DevTerm* dt = (const DevTerm*)(ob + wtb + gb + shb);
    const int ng = (int)p.groups.size(), nt = (int)(win ? pw.rest.size() : p.terms.size());
    const int nw = (int)pw.shifts.size();
    const size_t smem = win ? wtb + gb + shb + pw.rest.size() * (amp == 8 ? sizeof(PTerm<float>) : sizeof(PTerm<double>))
                            : gb + tb;
    // a later chunk accumulates onto `out`: run it into a workspace and add
    void* target = out;
    if (write && !first) {  // the third workspace is never an operand of this call
      void* w3[3];
      if ((rc = workspace(h, 3, w3))) return rc;
      target = w3[2];
    }
    // compiled tile passes (nullptr: the generic tile kernel runs that pass)
    std::vector<const void*> ptk;
    std::vector<std::vector<double>> ptc;
    const PTJitShape pshape = pt_jit_shape();
    if (tiled && h->nq >= kPTJitMinQubits && jit_mode() != 0 && jit_available()) {
      const bool f32 = amp == 8;
      std::vector<std::string> srcs;
      for (size_t pp = 0; pp < pt.passes.size(); ++pp) {
        const int g0 = pt.gbeg[pp], ngp = pt.gbeg[pp + 1] - g0;
        std::vector<double> c;
        srcs.push_back(pt_jit_source(f32, write, acc, pp > 0, real, nw, pw.groups.data() + g0, pt.xt.data() + g0, ngp,
                                     pw, c, pshape));
        if (c.size() * (f32 ? 4 : 8) > kPTJitMaxCoefBytes) srcs.back().clear();
        ptc.push_back(std::move(c));
      }
      if ((rc = jit_kernels(srcs, ptk, "vqc_pauli"))) return rc;
    }
    ProfScope prof(h->stream, write ? "pauli_apply" : "pauli_expect",
                   (double)h->size() * h->amp_bytes() * (1 + (write ? 1 : 0) + (acc && bra != ket ? 1 : 0)));
#define VQC_PAULI_LAUNCH(R)                                                                                      \
  do {                                                                                                           \
    if (tiled) {                                                                                                 \
      const DevGroupW* gw = (const DevGroupW*)(ob + wtb);                                                        \
      const int* xts = (const int*)(ob + wtb + gb + shb + tb);                                                   \
      const int64_t* hio = (const int64_t*)(ob + wtb + gb + shb + tb + xtb);                                     \
      const int np = (int)pt.passes.size();                                                                      \
      for (int pp = 0; pp < np; ++pp) {                                                                          \
        const int g0 = pt.gbeg[pp], ngp = pt.gbeg[pp + 1] - g0;                                                  \
        if (pp < (int)ptk.size() && ptk[pp])                                                                     \
          rc = pt_jit_launch(h, ptk[pp], sizeof(R) == 4, bra, ket, target, pt.passes[pp],                        \
                             hio + ((size_t)pp << kPTHiBits), ob, nw, hermitian_part ? 2.0 : 1.0,                \
                             h->scr.result + 2 * pp, ptc[pp], pshape);                                           \
        else                                                                                                     \
          rc = (real ? pt_launch<R, true> : pt_launch<R, false>)(                                                \
              h, write, acc, pp > 0, bra, ket, target, pt.passes[pp], gw + g0, xts + g0, ngp,                    \
              hio + ((size_t)pp << kPTHiBits), (const int*)(ob + wtb + gb), ob, nw, dt, nt,                      \
              hermitian_part ? 2.0 : 1.0, h->scr.result + 2 * pp);                                               \
        if (rc) return rc;                                                                                       \
      }                                                                                                          \
      if (acc && np > 1) k_add_passes<<<1, 32, 0, h->stream>>>(h->scr.result, np);                              \
    } else if (win) {                                                                                            \
      const DevGroupW* gw = (const DevGroupW*)(ob + wtb);                                                        \
      const int nhigh = (int)pw.groups.size() - nlow;                                                            \
      auto k1 = write ? (acc ? k_pauli_win<R, true, true, false> : k_pauli_win<R, true, false, false>)           \
                      : k_pauli_win<R, false, true, false>;                                                      \
      auto k2 = write ? (acc ? k_pauli_win<R, true, true, true> : k_pauli_win<R, true, false, true>)             \
                      : k_pauli_win<R, false, true, true>;                                                       \
      if (smem > 48 * 1024) {                                                                                    \
        VQC_CK(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));                \
        VQC_CK(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));                \
      }                                                                                                          \
      k1<<<grid, kRedThreads, smem, h->stream>>>((const cplx<R>*)bra, (const cplx<R>*)ket, (cplx<R>*)target,     \
                                                  h->size(), gw, nlow, (const int*)(ob + wtb + gb),              \
                                                  (const cplx<R>*)ob, nw, dt, nt, hermitian_part ? 2.0 : 1.0,   \
                                                  0, 0, 0, h->scr, h->scr.result);                               \
      if (nhigh > 0) {                                                                                           \
        VQC_CK(cudaGetLastError());                                                                              \
        k2<<<grid, kRedThreads, smem, h->stream>>>((const cplx<R>*)bra, (const cplx<R>*)ket, (cplx<R>*)target,   \
                                                    h->size(), gw + nlow, nhigh, (const int*)(ob + wtb + gb),    \
                                                    (const cplx<R>*)ob, nw, dt, nt, hermitian_part ? 2.0 : 1.0, \
                                                    tlo, ths, thl, h->scr, h->scr.result + 2);                   \
        if (acc) {                                                                                               \
          VQC_CK(cudaGetLastError());                                                                            \
          k_add_pair<<<1, 32, 0, h->stream>>>(h->scr.result);                                                    \
        }                                                                                                        \
      }                                                                                                          \
    } else if (quad) {                                                                                           \
      auto kfun = write ? (acc ? (sep ? k_pauli4<R, true, true, true> : k_pauli4<R, true, true, false>)          \
                               : (sep ? k_pauli4<R, true, false, true> : k_pauli4<R, true, false, false>))       \
                        : k_pauli4<R, false, true, false>;                                                       \
      if (smem > 48 * 1024) VQC_CK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
      kfun<<<grid, kRedThreads, smem, h->stream>>>((const cplx<R>*)bra, (const cplx<R>*)ket, (cplx<R>*)target,   \
                                                    h->size(), (const DevGroup4*)h->opbuf, ng, dt, nt,           \
                                                    hermitian_part ? 2.0 : 1.0, h->scr, h->scr.result);          \
    } else {                                                                                                     \
      auto kfun = write ? (acc ? k_pauli<R, true, true> : k_pauli<R, true, false>)                               \
                        : k_pauli<R, false, true>;                                                               \
      if (smem > 48 * 1024) VQC_CK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
      kfun<<<grid, kRedThreads, smem, h->stream>>>((const cplx<R>*)bra, (const cplx<R>*)ket, (cplx<R>*)target,   \
                                                    h->size(), dg, ng, dt, nt, h->scr, h->scr.result);           \
    }                                                                                                            \
  } while (0)
    if (h->dtype == VQC_C64)
      VQC_PAULI_LAUNCH(float);
    else
      VQC_PAULI_LAUNCH(double);
#undef VQC_PAULI_LAUNCH
    VQC_CK(cudaGetLastError());
    if (write && !first) {
      if ((rc = axpy_device(h, out, target))) return rc;
    }
    if (acc) {
      if (deferred && first && start + cnt >= nterms) {
        // one chunk: copy the sums to the handle's reserved pinned slot
        // without waiting; the caller reads them after its next synchronisation
        VQC_CK(cudaMemcpyAsync(h->h_result + kDeferredSlot, h->scr.result, 2 * sizeof(double),
                               cudaMemcpyDeviceToHost, h->stream));
        *deferred = true;
      } else {
        if ((rc = fetch_result(h, 2))) return rc;
        tot[0] += h->h_result[0];
        tot[1] += h->h_result[1];
      }
    }
    first = false;
    start += cnt;
  } while (start < nterms);
  if (result && !(deferred && *deferred)) {
    result[0] = tot[0];
    result[1] = tot[1];
  }
  return VQC_OK;
}

// ----------------------------------------------------------------------------- dense keys
template <int MS>
struct DenseArgs {
  int64_t ngroups;
  int64_t mask[6];
  int k;
  int64_t off[MS];
  double2 M[MS * MS];
};

template <class R, int MS>
__global__ void __launch_bounds__(kRedThreads)
    k_expect_dense(const cplx<R>* __restrict__ bra, const cplx<R>* __restrict__ ket,
                   const __grid_constant__ DenseArgs<MS> a, Scratch s, double* res) {
  double acc[2] = {0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.ngroups; g += stride) {
    const int64_t base = group_base(g, a.k, a.mask);
    double2 x[MS];
#pragma unroll
    for (int c = 0; c < MS; ++c) x[c] = to_d2(ket[base + a.off[c]]);
#pragma unroll
    for (int r = 0; r < MS; ++r) {
      double2 row = make_double2(0, 0);
#pragma unroll
      for (int c = 0; c < MS; ++c) row = cfma(a.M[r * MS + c], x[c], row);
      const double2 b = to_d2(bra[base + a.off[r]]);
      acc[0] = fma(b.x, row.x, fma(b.y, row.y, acc[0]));
      acc[1] = fma(b.x, row.y, fma(-b.y, row.x, acc[1]));
    }
  }
  grid_reduce<2>(acc, s, res);
}

template <class R, int MS>
__global__ void __launch_bounds__(256)
    k_apply_dense_add(const cplx<R>* __restrict__ ket, cplx<R>* __restrict__ out, const __grid_constant__ DenseArgs<MS> a) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.ngroups; g += stride) {
    const int64_t base = group_base(g, a.k, a.mask);
    double2 x[MS];
#pragma unroll
    for (int c = 0; c < MS; ++c) x[c] = to_d2(ket[base + a.off[c]]);
#pragma unroll
    for (int r = 0; r < MS; ++r) {
      double2 row = to_d2(out[base + a.off[r]]);
#pragma unroll
      for (int c = 0; c < MS; ++c) row = cfma(a.M[r * MS + c], x[c], row);
      out[base + a.off[r]] = mkc<R>((R)row.x, (R)row.y);
    }
  }
}

template <int MS>
static void fill_dense(int nq, int k, const int* sp, const std::vector<cd>& M, DenseArgs<MS>& a) {
  a.ngroups = mask_of(k, sp, nq, a.mask);
  for (int j = k + 1; j < 6; ++j) a.mask[j] = 0;
  a.k = k;
  for (int j = 0; j < MS; ++j) a.off[j] = offset_of(j, k, sp);
  for (int i = 0; i < MS * MS; ++i) a.M[i] = make_double2(M[i].real(), M[i].imag());
}

template <int MS>
static int expect_dense_ms(vqc_state h, const void* bra, const void* ket, int k, const int* sp,
                           const std::vector<cd>& M, double* res) {
  DenseArgs<MS> a;
  fill_dense<MS>(h->nq, k, sp, M, a);
  const int grid = reduction_grid(h->device, a.ngroups);
  ProfScope prof(h->stream, "expect_dense", (double)h->size() * h->amp_bytes() * (bra == ket ? 1 : 2));
  if (h->dtype == VQC_C64)
    k_expect_dense<float, MS><<<grid, kRedThreads, 0, h->stream>>>((const float2*)bra, (const float2*)ket, a, h->scr, res);
  else
    k_expect_dense<double, MS><<<grid, kRedThreads, 0, h->stream>>>((const double2*)bra, (const double2*)ket, a, h->scr,
                                                                    res);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

// sum conj(bra) M ket over the key's groups into res[0..1] (device).
int expect_dense_device(vqc_state h, const void* bra, const void* ket, int k, const int* sp, const std::vector<cd>& M,
                        double* res) {
  switch (k) {
    case 1: return expect_dense_ms<2>(h, bra, ket, k, sp, M, res);
    case 2: return expect_dense_ms<4>(h, bra, ket, k, sp, M, res);
    case 3: return expect_dense_ms<8>(h, bra, ket, k, sp, M, res);
    case 4: return expect_dense_ms<16>(h, bra, ket, k, sp, M, res);
    default: return expect_dense_ms<32>(h, bra, ket, k, sp, M, res);
  }
}

template <int MS>
static int apply_dense_ms(vqc_state h, const void* ket, void* out, int k, const int* sp, const std::vector<cd>& M) {
  DenseArgs<MS> a;
  fill_dense<MS>(h->nq, k, sp, M, a);
  const int grid = launch_grid(h->device, a.ngroups);
  if (h->dtype == VQC_C64)
    k_apply_dense_add<float, MS><<<grid, 256, 0, h->stream>>>((const float2*)ket, (float2*)out, a);
  else
    k_apply_dense_add<double, MS><<<grid, 256, 0, h->stream>>>((const double2*)ket, (double2*)out, a);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

}  // namespace vqc

using namespace vqc;

extern "C" {

int vqc_dm_expect_pauli(vqc_state rho, const vqc_pauli* terms, int nterms, double* out) {
  int rc = enter(rho);
  if (rc) return rc;
  if (!out) return fail(VQC_ERR_ARG, "null output");
  if (!rho->n_dm) return fail(VQC_ERR_ARG, "not a density matrix");
  std::lock_guard<std::mutex> lk(rho->mu);
  double tot[2] = {0, 0};
  int start = 0;
  do {
    const int cnt = std::min(kMaxTermsPerLaunch, nterms - start);
    PauliPlan p;
    if ((rc = plan_pauli(rho->n_dm, terms + start, cnt, false, p))) return rc;
    if (p.groups.empty()) break;
    const size_t gb = sizeof(DevGroup) * p.groups.size(), tb = sizeof(DevTerm) * p.terms.size();
    std::vector<unsigned char> buf(gb + tb);
    std::memcpy(buf.data(), p.groups.data(), gb);
    std::memcpy(buf.data() + gb, p.terms.data(), tb);
    if ((rc = upload_ops(rho, buf.data(), buf.size()))) return rc;
    const DevGroup* dg = (const DevGroup*)rho->opbuf;
    const DevTerm* dt = (const DevTerm*)((unsigned char*)rho->opbuf + gb);
    const int64_t N = int64_t(1) << rho->n_dm;
    const int grid = reduction_grid(rho->device, N);
    const size_t smem = gb + tb;
    ProfScope prof(rho->stream, "dm_pauli_expect", (double)N * p.groups.size() * rho->amp_bytes());
    if (rho->dtype == VQC_C64) {
      if (smem > 48 * 1024)
        VQC_CK(cudaFuncSetAttribute(k_pauli_dm<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_pauli_dm<float><<<grid, kRedThreads, smem, rho->stream>>>((const float2*)rho->d, N, dg, (int)p.groups.size(),
                                                                 dt, (int)p.terms.size(), rho->scr, rho->scr.result);
    } else {
      if (smem > 48 * 1024)
        VQC_CK(cudaFuncSetAttribute(k_pauli_dm<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      k_pauli_dm<double><<<grid, kRedThreads, smem, rho->stream>>>((const double2*)rho->d, N, dg,
                                                                   (int)p.groups.size(), dt, (int)p.terms.size(),
                                                                   rho->scr, rho->scr.result);
    }
    VQC_CK(cudaGetLastError());
    if ((rc = fetch_result(rho, 2))) return rc;
    tot[0] += rho->h_result[0];
    tot[1] += rho->h_result[1];
    start += cnt;
  } while (start < nterms);
  out[0] = tot[0];
  out[1] = tot[1];
  return VQC_OK;
}

int vqc_expect_pauli(vqc_state psi, const vqc_pauli* terms, int nterms, double* out) {
  int rc = enter(psi);
  if (rc) return rc;
  if (!out) return fail(VQC_ERR_ARG, "null output");
  std::lock_guard<std::mutex> lk(psi->mu);
  return pauli_run(psi, psi->d, psi->d, nullptr, terms, nterms, false, true, false, out);
}

int vqc_expect_pauli2(vqc_state phi, vqc_state psi, const vqc_pauli* terms, int nterms, double* out) {
  int rc = enter(psi);
  if (rc) return rc;
  if (!phi || !out || phi->nq != psi->nq || phi->dtype != psi->dtype || phi->device != psi->device)
    return fail(VQC_ERR_ARG, "expectation: states differ in size, dtype or device");
  std::lock_guard<std::mutex> lk(psi->mu);
  if ((rc = stream_after(psi, phi))) return rc;
  return pauli_run(psi, phi->d, psi->d, nullptr, terms, nterms, false, true, false, out);
}

int vqc_apply_pauli(vqc_state psi, vqc_state out, const vqc_pauli* terms, int nterms) {
  int rc = enter(psi);
  if (rc) return rc;
  if (!out || out == psi || out->nq != psi->nq || out->dtype != psi->dtype || out->device != psi->device)
    return fail(VQC_ERR_ARG, "apply: output must be a distinct state of the same size, dtype and device");
  std::lock_guard<std::mutex> lk(psi->mu);
  if ((rc = stream_after(psi, out))) return rc;
  if ((rc = pauli_run(psi, nullptr, psi->d, out->d, terms, nterms, true, false, false, nullptr))) return rc;
  return stream_after(out, psi);
}

int vqc_expect_dense(vqc_state phi, vqc_state psi, int k, const int* pos, const double* mat, double* out) {
  int rc = enter(psi);
  if (rc) return rc;
  if (!out) return fail(VQC_ERR_ARG, "null output");
  if (phi && (phi->nq != psi->nq || phi->dtype != psi->dtype || phi->device != psi->device))
    return fail(VQC_ERR_ARG, "expectation: states differ in size, dtype or device");
  std::lock_guard<std::mutex> lk(psi->mu);
  int sp[5];
  std::vector<cd> M;
  if ((rc = order_matrix(psi->nq, k, pos, mat, sp, M))) return rc;
  if (phi && (rc = stream_after(psi, phi))) return rc;
  if ((rc = expect_dense_device(psi, phi ? phi->d : psi->d, psi->d, k, sp, M, psi->scr.result))) return rc;
  if ((rc = fetch_result(psi, 2))) return rc;
  out[0] = psi->h_result[0];
  out[1] = psi->h_result[1];
  return VQC_OK;
}

int vqc_apply_dense_add(vqc_state psi, vqc_state out, int k, const int* pos, const double* mat) {
  int rc = enter(psi);
  if (rc) return rc;
  if (!out || out == psi || out->nq != psi->nq || out->dtype != psi->dtype || out->device != psi->device)
    return fail(VQC_ERR_ARG, "apply: output must be a distinct state of the same size, dtype and device");
  std::lock_guard<std::mutex> lk(psi->mu);
  int sp[5];
  std::vector<cd> M;
  if ((rc = order_matrix(psi->nq, k, pos, mat, sp, M))) return rc;
  if ((rc = stream_after(psi, out))) return rc;
  switch (k) {
    case 1: rc = apply_dense_ms<2>(psi, psi->d, out->d, k, sp, M); break;
    case 2: rc = apply_dense_ms<4>(psi, psi->d, out->d, k, sp, M); break;
    case 3: rc = apply_dense_ms<8>(psi, psi->d, out->d, k, sp, M); break;
    case 4: rc = apply_dense_ms<16>(psi, psi->d, out->d, k, sp, M); break;
    default: rc = apply_dense_ms<32>(psi, psi->d, out->d, k, sp, M); break;
  }
  if (rc) return rc;
  return stream_after(out, psi);
}

}  // extern "C"

namespace vqc {

// ----------------------------------------------------------------------------- serving support
int serve_pauli_image(int nq, const vqc_pauli* terms, int nterms, bool hermitian_part, std::vector<unsigned char>& img,
                      int& ng, int& nt) {
  if (nterms > kMaxTermsPerLaunch) return fail(VQC_ERR_UNSUPPORTED, "serving takes at most 2048 Pauli terms");
  PauliPlan p;
  int rc = plan_pauli(nq, terms, nterms, hermitian_part, p);
  if (rc) return rc;
  ng = (int)p.groups.size();
  nt = (int)p.terms.size();
  const size_t gb = sizeof(DevGroup) * p.groups.size(), tb = sizeof(DevTerm) * p.terms.size();
  img.resize(gb + tb);
  if (gb) std::memcpy(img.data(), p.groups.data(), gb);
  if (tb) std::memcpy(img.data() + gb, p.terms.data(), tb);
  return VQC_OK;
}

// One Pauli pass each over many states: item blockIdx.y, indices strided over
// blockIdx.x; per-CTA FP64 partial sums of conj(psi) H psi in fixed order.
template <class R, bool WRITE>
__global__ void __launch_bounds__(kRedThreads) k_pauli_batch(const PauliItem* __restrict__ items) {
  extern __shared__ unsigned char smem[];
  __shared__ double red[kRedThreads / 32][2];
  const PauliItem it = items[blockIdx.y];
  if ((int64_t)blockIdx.x * blockDim.x >= it.N) return;  // beyond this state: no partial written
  DevGroup* sg = reinterpret_cast<DevGroup*>(smem);
  DevTerm* st = reinterpret_cast<DevTerm*>(smem + sizeof(DevGroup) * it.ng);
  for (int i = threadIdx.x; i < it.ng; i += blockDim.x) sg[i] = it.groups[i];
  for (int i = threadIdx.x; i < it.nt; i += blockDim.x) st[i] = it.terms[i];
  __syncthreads();
  const cplx<R>* ket = (const cplx<R>*)it.ket;
  cplx<R>* out = (cplx<R>*)it.out;
  double acc[2] = {0, 0};
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < it.N; i += stride) {
    double2 hv = make_double2(0, 0), ov = make_double2(0, 0);
    for (int gi = 0; gi < it.ng; ++gi) {
      const DevGroup g = sg[gi];
      const int64_t j = i ^ (int64_t)g.x;
      const double2 kv = to_d2(ket[j]);
      double2 f = make_double2(0, 0), fd = make_double2(0, 0);
      for (int q = g.start; q < g.start + g.count; ++q) {
        const double sgn = (__popcll((unsigned long long)j & st[q].z) & 1) ? -1.0 : 1.0;
        f.x = fma(sgn, st[q].c.x, f.x);
        f.y = fma(sgn, st[q].c.y, f.y);
        if (WRITE) {
          fd.x = fma(sgn, st[q].d.x, fd.x);
          fd.y = fma(sgn, st[q].d.y, fd.y);
        }
      }
      hv = cfma(f, kv, hv);
      if (WRITE) ov = cfma(fd, kv, ov);
    }
    if (WRITE) out[i] = mkc<R>((R)ov.x, (R)ov.y);
    const double2 b = to_d2(ket[i]);
    acc[0] = fma(b.x, hv.x, fma(b.y, hv.y, acc[0]));
    acc[1] = fma(b.x, hv.y, fma(-b.y, hv.x, acc[1]));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < 2; ++c) {
    double v = acc[c];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[warp][c] = v;
  }
  __syncthreads();
  if (threadIdx.x < 2) {
    double v = 0;
    for (int w = 0; w < kRedThreads / 32; ++w) v += red[w][threadIdx.x];
    it.partials[blockIdx.x * 2 + threadIdx.x] = v;
  }
}

__global__ void __launch_bounds__(32) k_pauli_reduce_batch(const PauliRed* __restrict__ items) {
  const PauliRed it = items[blockIdx.x];
  if (threadIdx.x < 2) {
    double v = 0;
    for (int b = 0; b < it.nblocks; ++b) v += it.partials[b * 2 + threadIdx.x];
    it.out[threadIdx.x] = v;
  }
}

int serve_launch_pauli(int dtype, bool write, const PauliItem* d_items, int nitems, int gridx, size_t smem,
                       cudaStream_t stream) {
  if (nitems == 0) return VQC_OK;
  ProfScope prof(stream, "serve_pauli", 0);
#define VQC_PB(R, W)                                                                                        \
  do {                                                                                                      \
    auto kf = k_pauli_batch<R, W>;                                                                          \
    if (smem > 48 * 1024) VQC_CK(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    kf<<<dim3(gridx, nitems), kRedThreads, smem, stream>>>(d_items);                                        \
  } while (0)
  if (dtype == VQC_C64) {
    if (write) VQC_PB(float, true); else VQC_PB(float, false);
  } else {
    if (write) VQC_PB(double, true); else VQC_PB(double, false);
  }
#undef VQC_PB
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

int serve_launch_pauli_reduce(const PauliRed* d_items, int nitems, cudaStream_t stream) {
  if (nitems == 0) return VQC_OK;
  k_pauli_reduce_batch<<<nitems, 32, 0, stream>>>(d_items);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

}  // namespace vqc

// ----------------------------------------------------------------------------- allocation-free expectation
// Some callers of this library cannot allocate device memory: a host
// application that hands over a pre-sized arena and forbids cudaMalloc/cudaFree
// after start-up (allocation there can stall other streams, fail under memory
// pressure, or break a fixed memory plan), or code that must not touch the
// allocator while other work is in flight.  For them, ⟨psi|H|psi⟩ of a state in
// the caller's own device buffer runs here with all of its scratch (the Pauli
// tables, the per-block partial sums, the last-block counter and the result)
// in one static device array.  Every GPU that loads the library holds this
// array until the process exits.
namespace vqc {

constexpr int kNoAllocMaxTerms = 1024;    // Pauli terms per call at most
constexpr int kNoAllocMaxBlocks = 296;    // reduction grid at most
constexpr size_t kNoAllocTableBytes = kNoAllocMaxTerms * (sizeof(DevTerm) + sizeof(DevGroup));
constexpr size_t kNoAllocPartialBytes = (size_t)kNoAllocMaxBlocks * kMaxAcc * sizeof(double);
constexpr size_t kNoAllocBytes = kNoAllocTableBytes + kNoAllocPartialBytes + 1024;  // + counter and result

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Device address of the static scratch array, looked up once per device with
// that device current (the array's name is only a host-side stand-in).
static unsigned char* noalloc_scratch_ptr(int device) {
  static std::mutex mu;
  static unsigned char* ptrs[64] = {nullptr};
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!ptrs[device]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess) return nullptr;
    ptrs[device] = (unsigned char*)p;
  }
  return ptrs[device];
}

}  // namespace vqc

extern "C" int vqc_expect_pauli_noalloc(const void* state, int nqubits, int dtype, const vqc_pauli* terms,
                                        int nterms, void* stream, double* out) {
  using namespace vqc;
  if (!state || !out) return fail(VQC_ERR_ARG, "null state or output");
  if (dtype != VQC_C64 && dtype != VQC_C128) return fail(VQC_ERR_ARG, "dtype must be VQC_C64 or VQC_C128");
  if (nqubits < 1 || nqubits > 40) return fail(VQC_ERR_ARG, "number of qubits must be in 1..40");
  if (nterms < 0 || (nterms > 0 && !terms)) return fail(VQC_ERR_ARG, "bad Pauli term array");
  if (nterms > kNoAllocMaxTerms)
    return fail(VQC_ERR_ARG, "the allocation-free expectation takes at most 1024 Pauli terms per call");
  int device = 0;
  VQC_CK(cudaGetDevice(&device));
  {
    // the state must be device (or managed) memory of the current device: a
    // host pointer or another GPU's buffer would fault the kernel
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, state) != cudaSuccess) {
      cudaGetLastError();
      return fail(VQC_ERR_ARG, "state is not a CUDA device pointer");
    }
    if ((pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) || pa.device != device)
      return fail(VQC_ERR_ARG, "state must be device memory of the current device");
  }
  unsigned char* base = noalloc_scratch_ptr(device);
  if (!base) return fail(VQC_ERR_CUDA, "cudaGetSymbolAddress of the static scratch array failed");
  cudaStream_t st = (cudaStream_t)stream;
  if (nterms == 0) {
    out[0] = out[1] = 0;
    return VQC_OK;
  }
  // group the terms by flip mask into a fixed-size table (no heap use)
  const uint64_t lim = nqubits >= 64 ? ~0ull : ((1ull << nqubits) - 1);
  // host tables in thread-local storage (not on the caller's stack, which
  // may be small for the threads of such hosts)
  static thread_local int order[kNoAllocMaxTerms];
  for (int i = 0; i < nterms; ++i) {
    if ((terms[i].xmask & ~lim) || (terms[i].zmask & ~lim)) return fail(VQC_ERR_ARG, "Pauli term acts outside the register");
    int j = i;
    for (; j > 0 && terms[order[j - 1]].xmask > terms[i].xmask; --j) order[j] = order[j - 1];
    order[j] = i;
  }
  // [groups][terms]: the terms are first written after room for nterms groups,
  // then moved down behind the ng groups actually used
  alignas(16) static thread_local unsigned char table[kNoAllocTableBytes];
  DevGroup* groups = reinterpret_cast<DevGroup*>(table);
  DevTerm* dt = reinterpret_cast<DevTerm*>(table + sizeof(DevGroup) * nterms);
  int ng = 0;
  for (int a = 0; a < nterms; ++a) {
    const vqc_pauli& t = terms[order[a]];
    if (ng == 0 || groups[ng - 1].x != t.xmask) groups[ng++] = DevGroup{t.xmask, a, 0};
    ++groups[ng - 1].count;
    const int ny = __builtin_popcountll(t.xmask & t.zmask) & 3;
    const cd ph[4] = {cd(1, 0), cd(0, 1), cd(-1, 0), cd(0, -1)};
    const cd c = cd(t.coeff_re, t.coeff_im) * ph[ny];
    dt[a] = DevTerm{t.zmask, make_double2(c.real(), c.imag()), make_double2(c.real(), c.imag())};
  }
  const size_t gb = sizeof(DevGroup) * ng, tb = sizeof(DevTerm) * nterms;
  std::memmove(table + gb, dt, tb);
  unsigned char* d_table = base;
  Scratch scr;
  scr.partials = reinterpret_cast<double*>(base + kNoAllocTableBytes);
  scr.counter = reinterpret_cast<unsigned*>(base + kNoAllocTableBytes + kNoAllocPartialBytes);
  scr.result = reinterpret_cast<double*>(base + kNoAllocTableBytes + kNoAllocPartialBytes + 256);
  scr.max_blocks = kNoAllocMaxBlocks;
  // the table (pageable source: staged before the call returns) and a zero counter
  VQC_CK(cudaMemcpyAsync(d_table, table, gb + tb, cudaMemcpyHostToDevice, st));
  VQC_CK(cudaMemsetAsync(scr.counter, 0, sizeof(unsigned), st));
  const int64_t N = int64_t(1) << nqubits;
  const int grid = std::min(reduction_grid(device, N), kNoAllocMaxBlocks);
  const size_t smem = gb + tb;
#define VQC_NOALLOC_LAUNCH(R)                                                                                    \
  do {                                                                                                           \
    auto kfun = k_pauli<R, false, true>;                                                                         \
    if (smem > 48 * 1024) VQC_CK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)); \
    kfun<<<grid, kRedThreads, smem, st>>>((const cplx<R>*)state, (const cplx<R>*)state, nullptr, N,              \
                                          (const DevGroup*)d_table, ng, (const DevTerm*)(d_table + gb), nterms, scr, \
                                          scr.result);                                                           \
  } while (0)
  if (dtype == VQC_C64)
    VQC_NOALLOC_LAUNCH(float);
  else
    VQC_NOALLOC_LAUNCH(double);
#undef VQC_NOALLOC_LAUNCH
  VQC_CK(cudaGetLastError());
  VQC_CK(cudaMemcpyAsync(out, scr.result, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
  VQC_CK(cudaStreamSynchronize(st));
  return VQC_OK;
}
