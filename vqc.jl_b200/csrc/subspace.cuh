// Launch arguments of the per-gate "active subspace" kernels: one thread per
// group of 2^k amplitudes that share every non-target bit, touching only the
// active indices of the gate (see GateSpec in engine.h).
#pragma once

#include "engine.h"

namespace vqc {

template <class R, int MS>
struct SubArgs {
  int64_t namp;  // amplitudes of the state (the debug build's index limit)
  int64_t ngroups;
  int64_t mask[6];
  int k;
  int ns;
  int64_t off[MS];      // offset of active amplitude a within its group
  int64_t src_off[MS];  // kMono: offset of the amplitude that lands on a
  cplx<R> U[MS * MS];   // kDense: ns x ns (row stride MS); kDiag/kMono: U[a]
};

// Group base index: the mask-interleave formula of
// applygates/generic/threaded_long_range.jl:3-55 generalised to k bits.
__device__ __forceinline__ int64_t group_base(int64_t g, int k, const int64_t* mask) {
  int64_t b = 0;
#pragma unroll
  for (int j = 0; j < 6; ++j)
    if (j <= k) b |= (g << j) & mask[j];
  return b;
}

template <class R, int MS>
void fill_sub_args(const GateSpec& g, int nq, SubArgs<R, MS>& a) {
  a.namp = int64_t(1) << nq;
  a.ngroups = mask_of(g.k, g.sp, nq, a.mask);
  for (int j = g.k + 1; j < 6; ++j) a.mask[j] = 0;
  a.k = g.k;
  a.ns = g.ns;
  for (int s = 0; s < MS; ++s) {
    a.off[s] = s < g.ns ? offset_of(g.S[s], g.k, g.sp) : 0;
    a.src_off[s] = (s < g.ns && g.mode == kMono) ? offset_of(g.S[g.mono_src[s]], g.k, g.sp) : 0;
  }
  for (int i = 0; i < MS * MS; ++i) a.U[i] = mkc<R>(R(0), R(0));
  for (int r = 0; r < g.ns; ++r) {
    if (g.mode == kDense) {
      for (int c = 0; c < g.ns; ++c) {
        cd u = g.US[r * g.ns + c];
        a.U[r * MS + c] = mkc<R>((R)u.real(), (R)u.imag());
      }
    } else {
      cd u = g.mode == kDiag ? g.US[r * g.ns + r] : g.US[r * g.ns + g.mono_src[r]];
      a.U[r] = mkc<R>((R)u.real(), (R)u.imag());
    }
  }
}

inline int ms_of(int ns) {
  int m = 1;
  while (m < ns) m <<= 1;
  return m;
}

}  // namespace vqc
