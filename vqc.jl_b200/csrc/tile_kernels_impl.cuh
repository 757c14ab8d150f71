// Device code of the fused tile engine: the op bodies of the classic tile
// kernel (FP64, and FP32 passes that are interpreted) and the tile kernels
// k_tile / k_tile_batch.  The kernels are instantiated in the tile_inst_*.cu
// translation units (compiled in parallel); the planner in fused.cu sees only
// their declarations (tile_kernels.cuh).
#pragma once

#include <type_traits>

#include "engine.h"
#include "subspace.cuh"
#include "tile_plan.cuh"
#include "tile_f32.cuh"

namespace vqc {

// ----------------------------------------------------------------------------- device helpers
template <class R>
struct Swz;
template <>
struct Swz<float> {  // 8-byte amplitudes: half-warps must hit 16 distinct 8-byte bank pairs
  __device__ static __forceinline__ uint32_t f(uint32_t t) { return t ^ ((t >> 4) & 15u); }
};
template <>
struct Swz<double> {  // 16-byte amplitudes: quarter-warps must hit 8 distinct 16-byte bank quads
  __device__ static __forceinline__ uint32_t f(uint32_t t) { return t ^ (((t >> 3) ^ (t >> 6)) & 7u); }
};

__device__ __forceinline__ int64_t dep64(int64_t v, uint64_t mask) {
  int64_t r = 0;
  while (mask) {
    const uint64_t low = mask & (~mask + 1);
    if (v & 1) r |= (int64_t)low;
    v >>= 1;
    mask ^= low;
  }
  return r;
}
__device__ __forceinline__ uint32_t dep32(uint32_t v, uint32_t mask) {
  uint32_t r = 0;
  while (mask) {
    const uint32_t low = mask & (~mask + 1);
    if (v & 1) r |= low;
    v >>= 1;
    mask ^= low;
  }
  return r;
}

template <class C>
__device__ __forceinline__ C ldpool(const C* p) {
  return *p;
}

template <class R>
__device__ __forceinline__ void acc_pair(R (&a)[8], cplx<R> l0, cplx<R> l1, cplx<R> p0, cplx<R> p1) {
  // A00 += conj(l0) p0, A01 += conj(l0) p1, A10 += conj(l1) p0, A11 += conj(l1) p1
  a[0] = fma(l0.x, p0.x, fma(l0.y, p0.y, a[0]));
  a[1] = fma(l0.x, p0.y, fma(-l0.y, p0.x, a[1]));
  a[2] = fma(l0.x, p1.x, fma(l0.y, p1.y, a[2]));
  a[3] = fma(l0.x, p1.y, fma(-l0.y, p1.x, a[3]));
  a[4] = fma(l1.x, p0.x, fma(l1.y, p0.y, a[4]));
  a[5] = fma(l1.x, p0.y, fma(-l1.y, p0.x, a[5]));
  a[6] = fma(l1.x, p1.x, fma(l1.y, p1.y, a[6]));
  a[7] = fma(l1.x, p1.y, fma(-l1.y, p1.x, a[7]));
}

// Warp reduce-scatter of 8 values (FP64): afterwards lane L with L % 4 == 0
// holds the warp total of value L / 4.
__device__ __forceinline__ double warp_reduce8(const double (&x)[8]) {
  const int lane = threadIdx.x & 31;
  double y[4], z[2];
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const double keep = b4 ? x[i + 4] : x[i], send = b4 ? x[i] : x[i + 4];
    y[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const double keep = b3 ? y[i + 2] : y[i], send = b3 ? y[i] : y[i + 2];
    z[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  double u = (b2 ? z[1] : z[0]) + __shfl_xor_sync(0xffffffffu, b2 ? z[0] : z[1], 4);
  u += __shfl_xor_sync(0xffffffffu, u, 2);
  u += __shfl_xor_sync(0xffffffffu, u, 1);
  return u;
}

template <class R>
__device__ __forceinline__ void flush_acc(const R (&a)[8], double* sacc, int slot, int nwarps) {
  double x[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) x[i] = (double)a[i];
  const double u = warp_reduce8(x);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if ((lane & 3) == 0) sacc[((size_t)slot * nwarps + warp) * 8 + (lane >> 2)] += u;
}

// one-qubit op on register slot RR, both states in ADJ mode

template <int FORM, class C>
__device__ __forceinline__ void u1_apply(C& x0, C& x1, C u00, C u01, C u10, C u11) {
  const C a = x0, b = x1;
  if (FORM == kFormGen) {
    x0 = cfma(u01, b, cmul(u00, a));
    x1 = cfma(u11, b, cmul(u10, a));
  } else if (FORM == kFormRI) {  // u00 = p, u01 = i q, u10 = i r, u11 = s (p, q, r, s real)
    x0.x = fma(u00.x, a.x, -u01.y * b.y);
    x0.y = fma(u00.x, a.y, u01.y * b.x);
    x1.x = fma(u11.x, b.x, -u10.y * a.y);
    x1.y = fma(u11.x, b.y, u10.y * a.x);
  } else if (FORM == kFormReal) {
    x0.x = fma(u00.x, a.x, u01.x * b.x);
    x0.y = fma(u00.x, a.y, u01.x * b.y);
    x1.x = fma(u10.x, a.x, u11.x * b.x);
    x1.y = fma(u10.x, a.y, u11.x * b.y);
  } else if (FORM == kFormDiag) {
    x0 = cmul(u00, a);
    x1 = cmul(u11, b);
  } else {  // swap
    x0 = b;
    x1 = a;
  }
}

template <int RR, bool ADJ, bool CTL, int FORM, class R>
__device__ __forceinline__ void op_u1(cplx<R> (&v)[16], cplx<R> (&w)[16], const cplx<R>* U, uint32_t cm, uint32_t cv,
                                      uint32_t tthr, const uint32_t* dep, bool acc, int acck, double* sacc, int slot,
                                      int nwarps) {
  {
    const cplx<R> u00 = ldpool(U), u01 = ldpool(U + 1), u10 = ldpool(U + 2), u11 = ldpool(U + 3);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int j0 = ((p >> RR) << (RR + 1)) | (p & ((1 << RR) - 1)), j1 = j0 | (1 << RR);
      if (!CTL || ((tthr | dep[j0]) & cm) == cv) {
        u1_apply<FORM>(v[j0], v[j1], u00, u01, u10, u11);
        if (ADJ) u1_apply<FORM>(w[j0], w[j1], u00, u01, u10, u11);
      }
    }
  }
  if (ADJ && acc) {
    // A[a][b] += conj(lam_a) psi_b over the pairs (after the uncompute); only
    // the entries the parameters' D matrices touch
    R a[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = R(0);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
      const int j0 = ((p >> RR) << (RR + 1)) | (p & ((1 << RR) - 1)), j1 = j0 | (1 << RR);
      if (!CTL || ((tthr | dep[j0]) & cm) == cv) {
        const cplx<R> l0 = w[j0], l1 = w[j1], p0 = v[j0], p1 = v[j1];
        if (acck != kAccOff) {
          a[0] = fma(l0.x, p0.x, fma(l0.y, p0.y, a[0]));
          a[1] = fma(l0.x, p0.y, fma(-l0.y, p0.x, a[1]));
          a[6] = fma(l1.x, p1.x, fma(l1.y, p1.y, a[6]));
          a[7] = fma(l1.x, p1.y, fma(-l1.y, p1.x, a[7]));
        }
        if (acck != kAccDiag) {
          a[2] = fma(l0.x, p1.x, fma(l0.y, p1.y, a[2]));
          a[3] = fma(l0.x, p1.y, fma(-l0.y, p1.x, a[3]));
          a[4] = fma(l1.x, p0.x, fma(l1.y, p0.y, a[4]));
          a[5] = fma(l1.x, p0.y, fma(-l1.y, p0.x, a[5]));
        }
      }
    }
    flush_acc<R>(a, sacc, slot, nwarps);
  }
}

// two-qubit op on register slots (RA < RB), matrix bit 0 <-> RA
template <class C>
__device__ __forceinline__ void u2_quad(C& x0, C& x1, C& x2, C& x3, const C* U) {
  const C x[4] = {x0, x1, x2, x3};
  C o[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    o[r] = cmul(ldpool(U + 4 * r), x[0]);
#pragma unroll
    for (int c = 1; c < 4; ++c) o[r] = cfma(ldpool(U + 4 * r + c), x[c], o[r]);
  }
  x0 = o[0];
  x1 = o[1];
  x2 = o[2];
  x3 = o[3];
}

template <int RA, int RB, bool ADJ, class R>
__device__ __forceinline__ void op_u2(cplx<R> (&v)[16], cplx<R> (&w)[16], const cplx<R>* U, uint32_t cm, uint32_t cv,
                                      uint32_t tthr, const uint32_t* dep) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    int j = q;
    j = ((j >> RA) << (RA + 1)) | (j & ((1 << RA) - 1));
    j = ((j >> RB) << (RB + 1)) | (j & ((1 << RB) - 1));
    const int i0 = j, i1 = j | (1 << RA), i2 = j | (1 << RB), i3 = j | (1 << RA) | (1 << RB);
    if (((tthr | dep[i0]) & cm) == cv) {
      u2_quad(v[i0], v[i1], v[i2], v[i3], U);
      if (ADJ) u2_quad(w[i0], w[i1], w[i2], w[i3], U);
    }
  }
}

template <int RR, bool ADJ, bool CTL, class R>
__device__ __forceinline__ void dispatch_form(int form, cplx<R> (&v)[16], cplx<R> (&w)[16], const cplx<R>* U,
                                              uint32_t cm, uint32_t cv, uint32_t tthr, const uint32_t* dep, bool acc,
                                              int acck, double* sacc, int slot, int nwarps) {
  if (ADJ) {  // reverse sweep: the general and RX-like (CRX) forms
    if (form == kFormRI)
      op_u1<RR, ADJ, CTL, kFormRI, R>(v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps);
    else
      op_u1<RR, ADJ, CTL, kFormGen, R>(v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps);
    return;
  }
  // forward: every form runs as the general one (a per-op form switch cost
  // more than it saved in the single-state kernel)
  (void)form;
  op_u1<RR, ADJ, CTL, kFormGen, R>(v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps);
}

template <bool ADJ, class R>
__device__ __forceinline__ void dispatch_u1(int r, bool ctl, int form, cplx<R> (&v)[16], cplx<R> (&w)[16],
                                            const cplx<R>* U, uint32_t cm, uint32_t cv, uint32_t tthr,
                                            const uint32_t* dep, bool acc, int acck, double* sacc, int slot,
                                            int nwarps) {
  switch (r + (ctl ? 4 : 0)) {
    case 0: dispatch_form<0, ADJ, false, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
    case 1: dispatch_form<1, ADJ, false, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
    case 2: dispatch_form<2, ADJ, false, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
    case 3: dispatch_form<3, ADJ, false, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
    case 4: dispatch_form<0, ADJ, true, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
    case 5: dispatch_form<1, ADJ, true, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
    case 6: dispatch_form<2, ADJ, true, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
    default: dispatch_form<3, ADJ, true, R>(form, v, w, U, cm, cv, tthr, dep, acc, acck, sacc, slot, nwarps); break;
  }
}

template <bool ADJ, class R>
__device__ __forceinline__ void dispatch_u2(int ra, int rb, cplx<R> (&v)[16], cplx<R> (&w)[16], const cplx<R>* U,
                                            uint32_t cm, uint32_t cv, uint32_t tthr, const uint32_t* dep) {
  switch (ra * 4 + rb) {
    case 1: op_u2<0, 1, ADJ, R>(v, w, U, cm, cv, tthr, dep); break;
    case 2: op_u2<0, 2, ADJ, R>(v, w, U, cm, cv, tthr, dep); break;
    case 3: op_u2<0, 3, ADJ, R>(v, w, U, cm, cv, tthr, dep); break;
    case 6: op_u2<1, 2, ADJ, R>(v, w, U, cm, cv, tthr, dep); break;
    case 7: op_u2<1, 3, ADJ, R>(v, w, U, cm, cv, tthr, dep); break;
    default: op_u2<2, 3, ADJ, R>(v, w, U, cm, cv, tthr, dep); break;
  }
}

// The tile kernel: one launch per pass, persistent over the tiles.
// Resident CTAs per SM the register budget is sized for.
#ifndef VQC_MINB_F32_FWD
#define VQC_MINB_F32_FWD 3
#endif
#ifndef VQC_MINB_F32_ADJ
#define VQC_MINB_F32_ADJ 2
#endif
template <class R, bool ADJ, bool PACKED>
struct MinBlocks {
  static constexpr int value = 2;
};
template <bool ADJ>
struct MinBlocks<float, ADJ, true> {
  static constexpr int value = ADJ ? VQC_MINB_F32_ADJ : VQC_MINB_F32_FWD;
};

// GEN = false: a pass made of one-qubit ops only (the common case of
// parameterised circuits), compiled without the two-qubit and diagonal paths.
template <class R, int M, bool ADJ, bool GEN = true>
__device__ __forceinline__ void tile_body(cplx<R>* __restrict__ psi, cplx<R>* __restrict__ lam,
                                          const DevPass* __restrict__ pass, const DevStage* __restrict__ stages,
                                          const DevOp* __restrict__ ops, const cplx<R>* __restrict__ pool,
                                          double* __restrict__ partials, int ncta) {
  constexpr int NT = 1 << (M - kRegBits), T = 1 << M, NW = NT / 32;
  using C = cplx<R>;
  extern __shared__ __align__(16) unsigned char smem[];
  C* sp = reinterpret_cast<C*>(smem);
  C* sl = sp + (ADJ ? T : 0);
  double* sacc = reinterpret_cast<double*>(smem + tile_bytes<R, M, ADJ>());
  __shared__ DevPass P;
  if (threadIdx.x == 0) P = *pass;
  __syncthreads();
  const int nslots = ADJ ? P.nslots : 0;
  for (int i = threadIdx.x; i < nslots * NW * 8; i += NT) sacc[i] = 0;
  {
    // stage this pass's descriptors in shared memory (16-byte words)
    unsigned char* dst = smem + tile_bytes<R, M, ADJ>() + (size_t)nslots * NW * 8 * sizeof(double);
    const int nst = P.stage_end - P.stage_begin;
    const size_t b1 = sizeof(DevStage) * nst, b2 = sizeof(DevOp) * P.nops, b3 = sizeof(C) * P.npool;
    const int4* s1 = reinterpret_cast<const int4*>(stages + P.stage_begin);
    const int4* s2 = reinterpret_cast<const int4*>(ops);
    const int4* s3 = reinterpret_cast<const int4*>(pool);
    int4* d1 = reinterpret_cast<int4*>(dst);
    int4* d2 = reinterpret_cast<int4*>(dst + b1);
    int4* d3 = reinterpret_cast<int4*>(dst + b1 + b2);
    for (size_t i = threadIdx.x; i < b1 / 16; i += NT) d1[i] = __ldg(s1 + i);
    for (size_t i = threadIdx.x; i < b2 / 16; i += NT) d2[i] = __ldg(s2 + i);
    for (size_t i = threadIdx.x; i < (b3 + 15) / 16; i += NT) d3[i] = __ldg(s3 + i);
    stages = reinterpret_cast<const DevStage*>(dst) - P.stage_begin;
    ops = reinterpret_cast<const DevOp*>(dst + b1);
    pool = reinterpret_cast<const C*>(dst + b1 + b2);
    __syncthreads();
  }
  C v[16], w[16];
  const int s_first = P.stage_begin, s_last = P.stage_end - 1;
  [[maybe_unused]] const int64_t namp = P.ntiles << M;  // the debug build's index limits
  [[maybe_unused]] constexpr int64_t tsize = int64_t(1) << M;
  for (int64_t tile = blockIdx.x; tile < P.ntiles; tile += ncta) {
    const int64_t base = dep64(tile, P.nontile_mask);
    for (int s = s_first; s <= s_last; ++s) {
      const DevStage* S = stages + s;
      const uint32_t* dep = S->dep;  // shared memory
      const uint32_t tthr = dep32(threadIdx.x, (S->thr_mask));
      if (s == s_first) {
        // HBM -> registers directly in this stage's layout
        const int64_t g0 = base + dep64(threadIdx.x, (S->gthr_mask));
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int64_t gi = g0 + (S->gdep[j]);
          if (!VQC_DCHECK(gi, namp)) continue;
          v[j] = psi[gi];
          if (ADJ) w[j] = lam[gi];
        }
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const uint32_t t = Swz<R>::f(tthr | dep[j]);
          if (!VQC_DCHECK(t, tsize)) continue;
          v[j] = sp[t];
          if (ADJ) w[j] = sl[t];
        }
      }
      const int ob = (S->op_begin), oe = (S->op_end);
      for (int o = ob; o < oe; ++o) {
        const DevOp* op = ops + o;
        const int4 hd = *reinterpret_cast<const int4*>(op);
        const int code = hd.x, type = code & 15;
        if (code & kCodeGCtl) {  // a control on a non-tile qubit: uniform over the tile
          if ((base & (int64_t)(op->gmask)) != (int64_t)(op->gval)) continue;
        }
        const uint32_t cm = (uint32_t)hd.z, cv = (uint32_t)hd.w;
        const C* U = pool + hd.y;
        if (!GEN || type == kOpU1) {
          const bool acc = ADJ && (code & kCodeAcc);
          dispatch_u1<ADJ, R>((code >> 4) & 3, code & kCodeCtl, (code >> 11) & 7, v, w, U, cm, cv, tthr, dep, acc,
                              (code >> 14) & 3, sacc, acc ? (op->slot) : 0, NW);
        } else if (!GEN) {
        } else if (type == kOpU2) {
          dispatch_u2<ADJ, R>((code >> 4) & 3, (code >> 6) & 3, v, w, U, cm, cv, tthr, dep);
        } else {
          // diagonal: phase index from the op's qubits (tile bits per amplitude, others per tile)
          const int nd = (op->nd);
          uint32_t gidx = 0;
          int db[5];
#pragma unroll
          for (int i = 0; i < 5; ++i) {
            db[i] = i < nd ? (op->dbit[i]) : -1;
            if (i < nd && db[i] < 0) gidx |= (uint32_t)((base >> (op->dglob[i])) & 1) << i;
          }
          if (type == kOpDiag) {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const uint32_t t = tthr | dep[j];
              uint32_t idx = gidx;
#pragma unroll
              for (int i = 0; i < 5; ++i)
                if (db[i] >= 0) idx |= ((t >> db[i]) & 1u) << i;
              const C d = ldpool(U + idx);
              v[j] = cmul(d, v[j]);
              if (ADJ) w[j] = cmul(d, w[j]);
            }
          } else if (ADJ) {
            // kOpAccD: bins of conj(lam) psi over the op's (at most 2) qubits
            R a[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = R(0);
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              const uint32_t t = tthr | dep[j];
              uint32_t idx = gidx;
#pragma unroll
              for (int i = 0; i < 2; ++i)
                if (db[i] >= 0) idx |= ((t >> db[i]) & 1u) << i;
              const C l = w[j], p = v[j];
              const R re = fma(l.x, p.x, l.y * p.y), im = fma(l.x, p.y, -l.y * p.x);
#pragma unroll
              for (int b = 0; b < 4; ++b)
                if (idx == (uint32_t)b) {
                  a[2 * b] += re;
                  a[2 * b + 1] += im;
                }
            }
            flush_acc<R>(a, sacc, (op->slot), NW);
          }
        }
      }
      if (s == s_last) {
        // registers -> HBM directly from this stage's layout
        const int64_t g0 = base + dep64(threadIdx.x, (S->gthr_mask));
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int64_t gi = g0 + (S->gdep[j]);
          if (!VQC_DCHECK(gi, namp)) continue;
          psi[gi] = v[j];
          if (ADJ) lam[gi] = w[j];
        }
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const uint32_t t = Swz<R>::f(tthr | dep[j]);
          if (!VQC_DCHECK(t, tsize)) continue;
          sp[t] = v[j];
          if (ADJ) sl[t] = w[j];
        }
      }
      __syncthreads();  // also orders this tile's last shared reads before the next tile's writes
    }
  }
  if (ADJ && nslots > 0) {
    __syncthreads();
    for (int i = threadIdx.x; i < nslots * 8; i += NT) {
      const int slot = i >> 3, val = i & 7;
      double s = 0;
      for (int wp = 0; wp < NW; ++wp) s += sacc[((size_t)slot * NW + wp) * 8 + val];
      partials[((size_t)blockIdx.x * nslots + slot) * 8 + val] = s;
    }
  }
}

// One pass of one state.  PACKED: the FP32 packed body (tile_f32.cuh) on a
// plan laid out for it (lane bit in every stage, DevStageF); it is the
// interpreted form of the run-time compiled passes and runs only where a
// compiled kernel is missing.  Otherwise the body above (FP64, and FP32
// passes that are interpreted: the serving loop, small states).
template <class R, int M, bool ADJ, bool GEN, bool PACKED>
__device__ __forceinline__ void tile_run(cplx<R>* psi, cplx<R>* lam, const DevPass* pass, const void* stages,
                                         const DevOp* ops, const cplx<R>* pool, double* partials, int ncta) {
  if constexpr (PACKED && std::is_same<R, float>::value)
    f32t::tile_body<M, ADJ, GEN>(psi, lam, pass, (const DevStageF*)stages, ops, pool, partials, ncta);
  else
    tile_body<R, M, ADJ, GEN>(psi, lam, pass, (const DevStage*)stages, ops, pool, partials, ncta);
}

template <class R, int M, bool ADJ, bool GEN, bool PACKED>
__global__ void __launch_bounds__(1 << (M - kRegBits), MinBlocks<R, ADJ, PACKED>::value)
    k_tile(cplx<R>* psi, cplx<R>* lam, const DevPass* pass, const void* stages, const DevOp* ops,
           const cplx<R>* pool, double* partials) {
  tile_run<R, M, ADJ, GEN, PACKED>(psi, lam, pass, stages, ops, pool, partials, gridDim.x);
}

template <class R, int M, bool ADJ>
__global__ void __launch_bounds__(1 << (M - kRegBits), MinBlocks<R, ADJ, false>::value)
    k_tile_batch(const TileItem* __restrict__ items) {
  const TileItem it = items[blockIdx.y];
  if ((int)blockIdx.x >= it.ncta) return;
  tile_run<R, M, ADJ, true, false>((cplx<R>*)it.psi, (cplx<R>*)it.lam, it.pass, it.stages, it.ops,
                                   (const cplx<R>*)it.pool, it.partials, it.ncta);
}

}  // namespace vqc

// Explicit instantiation of the tile kernels of one element type, M and mode.
#define VQC_INST_TILE(R, M, ADJ, GEN, PACKED)                                                               \
  template __global__ void vqc::k_tile<R, M, ADJ, GEN, PACKED>(vqc::cplx<R>*, vqc::cplx<R>*, const vqc::DevPass*, \
                                                               const void*, const vqc::DevOp*, const vqc::cplx<R>*, \
                                                               double*);
#define VQC_INST_BATCH(R, M, ADJ) template __global__ void vqc::k_tile_batch<R, M, ADJ>(const vqc::TileItem*);
