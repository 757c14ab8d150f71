// The FP32 tile body of the fused engine, written for sm_100's packed
// two-lane FP32 arithmetic (fma/mul .f32x2: one instruction issue for two
// FMAs).
//
// Register layout.  A thread holds 16 amplitudes of its tile, j = l + 2m:
// l is tile bit 0 (always qubit 0, the "lane" bit) and m runs over the
// stage's three other register bits.  Pair m is two 64-bit registers
//     v[m].r = (re(l=0), re(l=1)),   v[m].i = (im(l=0), im(l=1)),
// the operands of the packed instructions as they are.  A one-qubit op on a
// non-lane register bit combines whole pairs (two amplitude pairs per packed
// instruction); an op on the lane bit combines the two lanes of one pair
// (with a lane swap).  Controls on register bits are compile-time variants
// (a single control at |1>) or a 16-bit mask of the enabled amplitudes;
// controls on thread bits are one test per op, on non-tile qubits one test
// per tile.
//
// Shared memory holds the tile as 16-byte pairs (v[m].r, v[m].i), XOR-
// swizzled over the pair index so that 16-byte accesses of 8 consecutive
// lanes land in 8 different bank groups (the planner picks register bits
// that keep the lowest three thread bits in distinct swizzle classes).  The
// swizzle is linear over XOR, so a pair's address is (thread part) ^ (pair
// part), both tabulated per stage on the host.  Global memory keeps the
// interleaved complex layout; the first and last stage of a pass convert.
#pragma once

#include "tile_dev.cuh"

namespace vqc {
namespace f32t {

// ----------------------------------------------------------------------------- packed arithmetic
// A packed value is one 64-bit register pair: low half = lane 0, high half =
// lane 1.  The state lives in these pairs so that the packed instructions
// take their operands without repacking.
typedef unsigned long long u64;
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {  // a * b + c, lane-wise
  u64 d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}
__device__ __forceinline__ u64 mul2(u64 a, u64 b) {
  u64 d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ float lo(u64 a) { return __uint_as_float((unsigned)a); }
__device__ __forceinline__ float hi(u64 a) { return __uint_as_float((unsigned)(a >> 32)); }
__device__ __forceinline__ u64 mk(float l, float h) {
  return (u64)__float_as_uint(l) | ((u64)__float_as_uint(h) << 32);
}
__device__ __forceinline__ u64 swp(u64 a) { return (a >> 32) | (a << 32); }
__device__ __forceinline__ u64 neg2(u64 a) { return a ^ 0x8000000080000000ull; }

// Pair m of the thread's amplitudes: r = (re lane 0, re lane 1), i = (im lane 0, im lane 1).
struct Pk {
  u64 r, i;
};

// amplitude j = lane + 2m of the thread's 2 NP (j compile-time after unrolling)
template <int NP>
__device__ __forceinline__ float2 amp(const Pk (&v)[NP], int j) {
  const Pk& q = v[j >> 1];
  return (j & 1) ? make_float2(hi(q.r), hi(q.i)) : make_float2(lo(q.r), lo(q.i));
}
template <int NP>
__device__ __forceinline__ void set_amp(Pk (&v)[NP], int j, float2 a) {
  Pk& q = v[j >> 1];
  if (j & 1) {
    q.r = mk(lo(q.r), a.x);
    q.i = mk(lo(q.i), a.y);
  } else {
    q.r = mk(a.x, hi(q.r));
    q.i = mk(a.y, hi(q.i));
  }
}

// complex products on float2 (U2 and diagonal ops)
__device__ __forceinline__ float2 ccmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 ccfma(float2 a, float2 b, float2 acc) {
  acc.x = fmaf(a.x, b.x, acc.x);
  acc.x = fmaf(-a.y, b.y, acc.x);
  acc.y = fmaf(a.x, b.y, acc.y);
  acc.y = fmaf(a.y, b.x, acc.y);
  return acc;
}

// Pair-space swizzle (pair index = tile index >> 1, at most 11 bits).
__host__ __device__ __forceinline__ uint32_t swz_pair(uint32_t p) {
  return p ^ ((p >> 3) & 7u) ^ ((p >> 6) & 7u) ^ ((p >> 9) & 7u);
}

// ----------------------------------------------------------------------------- one-qubit forms
// Coefficient layouts in the matrix pool (float2 entries, each op's block
// 16-byte aligned).  "free": the op's target is a non-lane register bit and
// every entry is a coefficient duplicated into both lanes; "lane": the target
// is the lane bit and entry = (row-0 coefficient, row-1 coefficient).
//   form      free layout                                          lane layout
//   general   u00r u00i -u00i u01r u01i -u01i u10r u10i -u10i       (u00r,u11r) (u01r,u10r) (u00i,u11i)
//             u11r u11i -u11i                                      (-u00i,-u11i) (u01i,u10i) (-u01i,-u10i)
//   RI        p q -q s r -r   (u00 = p, u01 = i q, u10 = i r, u11 = s) (p,s) (-q,-r) (q,r)
//   real      a00 a01 a10 a11                                      (a00,a11) (a01,a10)
//   diagonal  d0r d0i -d0i d1r d1i -d1i                            (d0r,d1r) (d0i,d1i) (-d0i,-d1i)
//   swap      (none)                                               (none)
constexpr int kPoolFree[5] = {12, 6, 4, 6, 0};
constexpr int kPoolLane[5] = {6, 3, 2, 3, 0};

// Every free layout stores an imaginary part next to its negation, so conj(U)
// (CJ: the reverse sweep holds the cotangent conjugated) is U with the two
// exchanged: a compile-time permutation of the coefficient indices.
template <bool CJ>
struct FreeIx {
  static constexpr int i1 = CJ ? 2 : 1, i2 = CJ ? 1 : 2, i4 = CJ ? 5 : 4, i5 = CJ ? 4 : 5, i7 = CJ ? 8 : 7,
                       i8 = CJ ? 7 : 8, i10 = CJ ? 11 : 10, i11 = CJ ? 10 : 11;
};

// Two pairs at once: (A, B) = amplitudes with target bit 0 / 1, both lanes.
template <int FORM, bool CJ = false>
__device__ __forceinline__ void free_apply(Pk& A, Pk& B, const u64* c) {
  using I = FreeIx<CJ>;
  const u64 ar = A.r, ai = A.i, br = B.r, bi = B.i;
  if (FORM == kFormGen) {
    A.r = fma2(c[0], ar, fma2(c[I::i2], ai, fma2(c[3], br, mul2(c[I::i5], bi))));
    A.i = fma2(c[0], ai, fma2(c[I::i1], ar, fma2(c[3], bi, mul2(c[I::i4], br))));
    B.r = fma2(c[6], ar, fma2(c[I::i8], ai, fma2(c[9], br, mul2(c[I::i11], bi))));
    B.i = fma2(c[6], ai, fma2(c[I::i7], ar, fma2(c[9], bi, mul2(c[I::i10], br))));
  } else if (FORM == kFormRI) {
    A.r = fma2(c[0], ar, mul2(c[I::i2], bi));
    A.i = fma2(c[0], ai, mul2(c[I::i1], br));
    B.r = fma2(c[3], br, mul2(c[I::i5], ai));
    B.i = fma2(c[3], bi, mul2(c[I::i4], ar));
  } else if (FORM == kFormReal) {
    A.r = fma2(c[0], ar, mul2(c[1], br));
    A.i = fma2(c[0], ai, mul2(c[1], bi));
    B.r = fma2(c[2], ar, mul2(c[3], br));
    B.i = fma2(c[2], ai, mul2(c[3], bi));
  } else if (FORM == kFormDiag) {
    A.r = fma2(c[0], ar, mul2(c[I::i2], ai));
    A.i = fma2(c[0], ai, mul2(c[I::i1], ar));
    B.r = fma2(c[3], br, mul2(c[I::i5], bi));
    B.i = fma2(c[3], bi, mul2(c[I::i4], br));
  } else {
    const Pk t = A;
    A = B;
    B = t;
  }
}

// One lane of two pairs (the pair of that lane), free layout, scalar.
template <int FORM, int LANE, bool CJ = false>
__device__ __forceinline__ void scalar_apply(Pk& A, Pk& B, const u64* c) {
  using I = FreeIx<CJ>;
  const float Ar = LANE ? hi(A.r) : lo(A.r), Ai = LANE ? hi(A.i) : lo(A.i);
  const float Br = LANE ? hi(B.r) : lo(B.r), Bi = LANE ? hi(B.i) : lo(B.i);
  float ar, ai, br, bi;
  if (FORM == kFormGen) {
    ar = fmaf(lo(c[0]), Ar, fmaf(lo(c[I::i2]), Ai, fmaf(lo(c[3]), Br, lo(c[I::i5]) * Bi)));
    ai = fmaf(lo(c[0]), Ai, fmaf(lo(c[I::i1]), Ar, fmaf(lo(c[3]), Bi, lo(c[I::i4]) * Br)));
    br = fmaf(lo(c[6]), Ar, fmaf(lo(c[I::i8]), Ai, fmaf(lo(c[9]), Br, lo(c[I::i11]) * Bi)));
    bi = fmaf(lo(c[6]), Ai, fmaf(lo(c[I::i7]), Ar, fmaf(lo(c[9]), Bi, lo(c[I::i10]) * Br)));
  } else if (FORM == kFormRI) {
    ar = fmaf(lo(c[0]), Ar, lo(c[I::i2]) * Bi);
    ai = fmaf(lo(c[0]), Ai, lo(c[I::i1]) * Br);
    br = fmaf(lo(c[3]), Br, lo(c[I::i5]) * Ai);
    bi = fmaf(lo(c[3]), Bi, lo(c[I::i4]) * Ar);
  } else if (FORM == kFormReal) {
    ar = fmaf(lo(c[0]), Ar, lo(c[1]) * Br);
    ai = fmaf(lo(c[0]), Ai, lo(c[1]) * Bi);
    br = fmaf(lo(c[2]), Ar, lo(c[3]) * Br);
    bi = fmaf(lo(c[2]), Ai, lo(c[3]) * Bi);
  } else if (FORM == kFormDiag) {
    ar = fmaf(lo(c[0]), Ar, lo(c[I::i2]) * Ai);
    ai = fmaf(lo(c[0]), Ai, lo(c[I::i1]) * Ar);
    br = fmaf(lo(c[3]), Br, lo(c[I::i5]) * Bi);
    bi = fmaf(lo(c[3]), Bi, lo(c[I::i4]) * Br);
  } else {
    ar = Br, ai = Bi, br = Ar, bi = Ai;
  }
  if (LANE) {
    A.r = mk(lo(A.r), ar), A.i = mk(lo(A.i), ai), B.r = mk(lo(B.r), br), B.i = mk(lo(B.i), bi);
  } else {
    A.r = mk(ar, hi(A.r)), A.i = mk(ai, hi(A.i)), B.r = mk(br, hi(B.r)), B.i = mk(bi, hi(B.i));
  }
}

// The pair inside one register pair set (target = lane bit), lane layout;
// CJ: conj(U) (the negated imaginary parts exchanged with the plain ones).
template <int FORM, bool CJ = false>
__device__ __forceinline__ void lane_apply(Pk& V, const u64* c) {
  const u64 pr = V.r, pi = V.i;
  if (FORM == kFormGen) {
    constexpr int g2 = CJ ? 3 : 2, g3 = CJ ? 2 : 3, g4 = CJ ? 5 : 4, g5 = CJ ? 4 : 5;
    const u64 qr = swp(pr), qi = swp(pi);
    V.r = fma2(c[0], pr, fma2(c[1], qr, fma2(c[g3], pi, mul2(c[g5], qi))));
    V.i = fma2(c[0], pi, fma2(c[1], qi, fma2(c[g2], pr, mul2(c[g4], qr))));
  } else if (FORM == kFormRI) {
    constexpr int r1 = CJ ? 2 : 1, r2 = CJ ? 1 : 2;
    V.r = fma2(c[0], pr, mul2(c[r1], swp(pi)));
    V.i = fma2(c[0], pi, mul2(c[r2], swp(pr)));
  } else if (FORM == kFormReal) {
    V.r = fma2(c[0], pr, mul2(c[1], swp(pr)));
    V.i = fma2(c[0], pi, mul2(c[1], swp(pi)));
  } else if (FORM == kFormDiag) {
    constexpr int d1 = CJ ? 2 : 1, d2 = CJ ? 1 : 2;
    V.r = fma2(c[0], pr, mul2(c[d2], pi));
    V.i = fma2(c[0], pi, mul2(c[d1], pr));
  } else {
    V.r = swp(pr);
    V.i = swp(pi);
  }
}

// j-bit layout of the 2 NP amplitudes: bit 0 = lane, bits 1.. = free slots
// (NP = 8: three, NP = 16: four).  TB: target j-bit.  CB: single register
// control (j-bit, at |1>), or -1.
template <int TB, int CB, int FORM, bool ADJ, int NP>
__device__ __forceinline__ void u1_static(Pk (&v)[NP], Pk (&w)[NP], const u64* c) {
  if constexpr (TB == 0) {
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      if (CB > 0 && !((m >> (CB - 1)) & 1)) continue;
      lane_apply<FORM>(v[m], c);
      if (ADJ) lane_apply<FORM, true>(w[m], c);
    }
  } else {
    constexpr int T = TB - 1;
#pragma unroll
    for (int g = 0; g < NP / 2; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      if (CB > 0 && !((m0 >> (CB - 1)) & 1)) continue;
      if (CB == 0) {  // lane control: lane 1 only
        scalar_apply<FORM, 1>(v[m0], v[m1], c);
        if (ADJ) scalar_apply<FORM, 1, true>(w[m0], w[m1], c);
      } else {
        free_apply<FORM>(v[m0], v[m1], c);
        if (ADJ) free_apply<FORM, true>(w[m0], w[m1], c);
      }
    }
  }
}

// Register controls given as a mask over the pair representatives (bit j set:
// amplitude j, target bit clear, satisfies the register controls).
template <int TB, int FORM, bool ADJ, int NP>
__device__ __forceinline__ void u1_masked(Pk (&v)[NP], Pk (&w)[NP], const u64* c, uint32_t rmask) {
  if constexpr (TB == 0) {
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      if (!((rmask >> (2 * m)) & 1)) continue;
      lane_apply<FORM>(v[m], c);
      if (ADJ) lane_apply<FORM, true>(w[m], c);
    }
  } else {
    constexpr int T = TB - 1;
#pragma unroll
    for (int g = 0; g < NP / 2; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      if ((rmask >> (2 * m0)) & 1) {
        scalar_apply<FORM, 0>(v[m0], v[m1], c);
        if (ADJ) scalar_apply<FORM, 0, true>(w[m0], w[m1], c);
      }
      if ((rmask >> (2 * m0 + 1)) & 1) {
        scalar_apply<FORM, 1>(v[m0], v[m1], c);
        if (ADJ) scalar_apply<FORM, 1, true>(w[m0], w[m1], c);
      }
    }
  }
}

// ----------------------------------------------------------------------------- reduced-matrix accumulation
// A[a][b] += conj(lam_a) psi_b over the op's pairs, after the uncompute.  The
// reverse sweep holds the cotangent conjugated (M = conj(lam), loaded and
// stored conjugated at HBM), so A[a][b] = sum M_a psi_b: Re = Mr Pr - Mi Pi,
// Im = Mr Pi + Mi Pr.  A thread's partials s[8] = (A00r, A00i, A01r, A01i,
// A10r, A10i, A11r, A11i).
template <int KIND>
__device__ __forceinline__ void acc_free(u64 (&a)[8], const Pk& M0, const Pk& M1, const Pk& P0, const Pk& P1) {
  const u64 n0i = neg2(M0.i), n1i = neg2(M1.i);
  if (KIND != kAccOff) {
    a[0] = fma2(M0.r, P0.r, fma2(n0i, P0.i, a[0]));
    a[1] = fma2(M0.r, P0.i, fma2(M0.i, P0.r, a[1]));
    a[6] = fma2(M1.r, P1.r, fma2(n1i, P1.i, a[6]));
    a[7] = fma2(M1.r, P1.i, fma2(M1.i, P1.r, a[7]));
  }
  if (KIND != kAccDiag) {
    a[2] = fma2(M0.r, P1.r, fma2(n0i, P1.i, a[2]));
    a[3] = fma2(M0.r, P1.i, fma2(M0.i, P1.r, a[3]));
    a[4] = fma2(M1.r, P0.r, fma2(n1i, P0.i, a[4]));
    a[5] = fma2(M1.r, P0.i, fma2(M1.i, P0.r, a[5]));
  }
}
template <int KIND, int LANE>
__device__ __forceinline__ void acc_scalar(float (&s)[8], const Pk& M0, const Pk& M1, const Pk& P0, const Pk& P1) {
  const float m0r = LANE ? hi(M0.r) : lo(M0.r), m0i = LANE ? hi(M0.i) : lo(M0.i);
  const float m1r = LANE ? hi(M1.r) : lo(M1.r), m1i = LANE ? hi(M1.i) : lo(M1.i);
  const float p0r = LANE ? hi(P0.r) : lo(P0.r), p0i = LANE ? hi(P0.i) : lo(P0.i);
  const float p1r = LANE ? hi(P1.r) : lo(P1.r), p1i = LANE ? hi(P1.i) : lo(P1.i);
  if (KIND != kAccOff) {
    s[0] = fmaf(m0r, p0r, fmaf(-m0i, p0i, s[0]));
    s[1] = fmaf(m0r, p0i, fmaf(m0i, p0r, s[1]));
    s[6] = fmaf(m1r, p1r, fmaf(-m1i, p1i, s[6]));
    s[7] = fmaf(m1r, p1i, fmaf(m1i, p1r, s[7]));
  }
  if (KIND != kAccDiag) {
    s[2] = fmaf(m0r, p1r, fmaf(-m0i, p1i, s[2]));
    s[3] = fmaf(m0r, p1i, fmaf(m0i, p1r, s[3]));
    s[4] = fmaf(m1r, p0r, fmaf(-m1i, p0i, s[4]));
    s[5] = fmaf(m1r, p0i, fmaf(m1i, p0r, s[5]));
  }
}
// lane target: c0 = (A00r, A11r), c1 = (A00i, A11i), c2 = (A01r, A10r), c3 = (A01i, A10i)
template <int KIND>
__device__ __forceinline__ void acc_lane(u64 (&c)[4], const Pk& M, const Pk& P) {
  const u64 ni = neg2(M.i);
  if (KIND != kAccOff) {
    c[0] = fma2(M.r, P.r, fma2(ni, P.i, c[0]));
    c[1] = fma2(M.r, P.i, fma2(M.i, P.r, c[1]));
  }
  if (KIND != kAccDiag) {
    const u64 qr = swp(P.r), qi = swp(P.i);
    c[2] = fma2(M.r, qr, fma2(ni, qi, c[2]));
    c[3] = fma2(M.r, qi, fma2(M.i, qr, c[3]));
  }
}
// Anti-Hermitian projection (KIND & kAccAH): when every matrix D the op's
// partials contract with is anti-Hermitian (D = U^dagger dU/dtheta of a
// unitary family), Re sum_ab D_ab A_ab = -Im D00 s0 - Im D11 s1 + Re D01 s2
// - Im D01 s3 needs only s = (Im A00, Im A11, Re A01 - Re A10, Im A01 + Im A10):
// three quarters of the products and half the values to reduce.  With the
// conjugated cotangent every one of them is a plain sum of products:
//   s0 = sum M0r P0i + M0i P0r,  s1 = sum M1r P1i + M1i P1r,
//   s2 = sum (M0r P1r + M1i P0i) - sum (M0i P1i + M1r P0r),
//   s3 = sum M0r P1i + M0i P1r + M1r P0i + M1i P0r.
template <int KIND>
__device__ __forceinline__ void acch_free(u64 (&a)[5], const Pk& M0, const Pk& M1, const Pk& P0, const Pk& P1) {
  if ((KIND & 3) != kAccOff) {
    a[0] = fma2(M0.r, P0.i, fma2(M0.i, P0.r, a[0]));
    a[1] = fma2(M1.r, P1.i, fma2(M1.i, P1.r, a[1]));
  }
  if ((KIND & 3) != kAccDiag) {
    a[2] = fma2(M0.r, P1.r, fma2(M1.i, P0.i, a[2]));
    a[3] = fma2(M0.i, P1.i, fma2(M1.r, P0.r, a[3]));
    a[4] = fma2(M0.r, P1.i, fma2(M0.i, P1.r, fma2(M1.r, P0.i, fma2(M1.i, P0.r, a[4]))));
  }
}
template <int KIND, int LANE>
__device__ __forceinline__ void acch_scalar(float (&s)[8], const Pk& M0, const Pk& M1, const Pk& P0, const Pk& P1) {
  const float m0r = LANE ? hi(M0.r) : lo(M0.r), m0i = LANE ? hi(M0.i) : lo(M0.i);
  const float m1r = LANE ? hi(M1.r) : lo(M1.r), m1i = LANE ? hi(M1.i) : lo(M1.i);
  const float p0r = LANE ? hi(P0.r) : lo(P0.r), p0i = LANE ? hi(P0.i) : lo(P0.i);
  const float p1r = LANE ? hi(P1.r) : lo(P1.r), p1i = LANE ? hi(P1.i) : lo(P1.i);
  if ((KIND & 3) != kAccOff) {
    s[0] = fmaf(m0r, p0i, fmaf(m0i, p0r, s[0]));
    s[1] = fmaf(m1r, p1i, fmaf(m1i, p1r, s[1]));
  }
  if ((KIND & 3) != kAccDiag) {
    s[2] = fmaf(m0r, p1r, fmaf(-m0i, p1i, fmaf(-m1r, p0r, fmaf(m1i, p0i, s[2]))));
    s[3] = fmaf(m0r, p1i, fmaf(m0i, p1r, fmaf(m1r, p0i, fmaf(m1i, p0r, s[3]))));
  }
}
// lane target: c0 = (Im A00, Im A11); (Re A01, Re A10) = c1 - c2 with
// c1 = Mr Qr, c2 = Mi Qi (Q = the lane-swapped P); c3 = (Im A01, Im A10)
template <int KIND>
__device__ __forceinline__ void acch_lane(u64 (&c)[4], const Pk& M, const Pk& P) {
  if ((KIND & 3) != kAccOff) c[0] = fma2(M.r, P.i, fma2(M.i, P.r, c[0]));
  if ((KIND & 3) != kAccDiag) {
    const u64 qr = swp(P.r), qi = swp(P.i);
    c[1] = fma2(M.r, qr, c[1]);
    c[2] = fma2(M.i, qi, c[2]);
    c[3] = fma2(M.r, qi, fma2(M.i, qr, c[3]));
  }
}
__device__ __forceinline__ void packh_free(const u64 (&a)[5], float (&s)[8]) {
  s[0] = lo(a[0]) + hi(a[0]);
  s[1] = lo(a[1]) + hi(a[1]);
  s[2] = (lo(a[2]) + hi(a[2])) - (lo(a[3]) + hi(a[3]));
  s[3] = lo(a[4]) + hi(a[4]);
}
__device__ __forceinline__ void packh_lane(const u64 (&c)[4], float (&s)[8]) {
  s[0] = lo(c[0]), s[1] = hi(c[0]), s[2] = (lo(c[1]) - lo(c[2])) - (hi(c[1]) - hi(c[2])), s[3] = lo(c[3]) + hi(c[3]);
}
__device__ __forceinline__ void pack_free(const u64 (&a)[8], float (&s)[8]) {
#pragma unroll
  for (int i = 0; i < 8; ++i) s[i] = lo(a[i]) + hi(a[i]);
}
__device__ __forceinline__ void pack_lane(const u64 (&c)[4], float (&s)[8]) {
  s[0] = lo(c[0]), s[1] = lo(c[1]), s[2] = lo(c[2]), s[3] = lo(c[3]);
  s[4] = hi(c[2]), s[5] = hi(c[3]), s[6] = hi(c[0]), s[7] = hi(c[1]);
}

// Thread partials -> the warp's slot row in shared memory.  A warp
// reduce-scatter of the 8 values in FP32 (each warp partial sums at most 256
// products: 32 lanes x 8 amplitude pairs); the warp partials are added in
// FP64 into the warp's slot row, and every later level (warps, CTAs, the
// grid) is FP64.  Afterwards lane L with L % 4 == 0 holds the warp total of
// value L / 4.  Every lane of the warp must call it.
__device__ __forceinline__ void flush8(const float (&s)[8], double* sacc, int slot, int nwarps) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
  float y[4], z[2];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const float keep = b4 ? s[i + 4] : s[i], send = b4 ? s[i] : s[i + 4];
    y[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float keep = b3 ? y[i + 2] : y[i], send = b3 ? y[i] : y[i + 2];
    z[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
  }
  float u = (b2 ? z[1] : z[0]) + __shfl_xor_sync(0xffffffffu, b2 ? z[0] : z[1], 4);
  u += __shfl_xor_sync(0xffffffffu, u, 2);
  u += __shfl_xor_sync(0xffffffffu, u, 1);
  if ((lane & 3) == 0) sacc[((unsigned long long)slot * nwarps + warp) * 8 + (lane >> 2)] += (double)u;
}

// The first four values only (an anti-Hermitian projection); lane L with
// L % 8 == 0 holds the warp total of value L / 8 afterwards.
__device__ __forceinline__ void flush4(const float (&s)[8], double* sacc, int slot, int nwarps) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool b4 = lane & 16, b3 = lane & 8;
  float y[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const float keep = b4 ? s[i + 2] : s[i], send = b4 ? s[i] : s[i + 2];
    y[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
  }
  float u = (b3 ? y[1] : y[0]) + __shfl_xor_sync(0xffffffffu, b3 ? y[0] : y[1], 8);
  u += __shfl_xor_sync(0xffffffffu, u, 4);
  u += __shfl_xor_sync(0xffffffffu, u, 2);
  u += __shfl_xor_sync(0xffffffffu, u, 1);
  if ((lane & 7) == 0) sacc[((unsigned long long)slot * nwarps + warp) * 8 + (lane >> 3)] += (double)u;
}

template <int TB, int CB, int KIND>
__device__ __forceinline__ void acc_static(const Pk (&v)[8], const Pk (&w)[8], float (&s8)[8]) {
  if constexpr ((KIND & kAccAH) && TB == 0) {
    u64 c[4] = {0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if (CB > 0 && !((m >> (CB - 1)) & 1)) continue;
      acch_lane<KIND>(c, w[m], v[m]);
    }
    packh_lane(c, s8);
  } else if constexpr ((KIND & kAccAH) && CB == 0) {
    constexpr int T = TB - 1;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      acch_scalar<KIND, 1>(s8, w[m0], w[m1], v[m0], v[m1]);
    }
  } else if constexpr (KIND & kAccAH) {
    constexpr int T = TB - 1;
    u64 a[5] = {0, 0, 0, 0, 0};
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      if (CB > 0 && !((m0 >> (CB - 1)) & 1)) continue;
      acch_free<KIND>(a, w[m0], w[m1], v[m0], v[m1]);
    }
    packh_free(a, s8);
  } else if constexpr (TB == 0) {
    u64 c[4] = {0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      if (CB > 0 && !((m >> (CB - 1)) & 1)) continue;
      acc_lane<KIND>(c, w[m], v[m]);
    }
    pack_lane(c, s8);
  } else if constexpr (CB == 0) {  // lane control: lane 1 only
    constexpr int T = TB - 1;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      acc_scalar<KIND, 1>(s8, w[m0], w[m1], v[m0], v[m1]);
    }
  } else {
    constexpr int T = TB - 1;
    u64 a[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      if (CB > 0 && !((m0 >> (CB - 1)) & 1)) continue;
      acc_free<KIND>(a, w[m0], w[m1], v[m0], v[m1]);
    }
    pack_free(a, s8);
  }
}
template <int TB, int KIND>
__device__ __forceinline__ void acc_masked(const Pk (&v)[8], const Pk (&w)[8], uint32_t rmask, float (&s8)[8]) {
  if constexpr ((KIND & kAccAH) && TB == 0) {
    u64 c[4] = {0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < 8; ++m)
      if ((rmask >> (2 * m)) & 1) acch_lane<KIND>(c, w[m], v[m]);
    packh_lane(c, s8);
  } else if constexpr (KIND & kAccAH) {
    constexpr int T = TB - 1;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      if ((rmask >> (2 * m0)) & 1) acch_scalar<KIND, 0>(s8, w[m0], w[m1], v[m0], v[m1]);
      if ((rmask >> (2 * m0 + 1)) & 1) acch_scalar<KIND, 1>(s8, w[m0], w[m1], v[m0], v[m1]);
    }
  } else if constexpr (TB == 0) {
    u64 c[4] = {0, 0, 0, 0};
#pragma unroll
    for (int m = 0; m < 8; ++m)
      if ((rmask >> (2 * m)) & 1) acc_lane<KIND>(c, w[m], v[m]);
    pack_lane(c, s8);
  } else {
    constexpr int T = TB - 1;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      const int m0 = ((g >> T) << (T + 1)) | (g & ((1 << T) - 1)), m1 = m0 | (1 << T);
      if ((rmask >> (2 * m0)) & 1) acc_scalar<KIND, 0>(s8, w[m0], w[m1], v[m0], v[m1]);
      if ((rmask >> (2 * m0 + 1)) & 1) acc_scalar<KIND, 1>(s8, w[m0], w[m1], v[m0], v[m1]);
    }
  }
}

// ----------------------------------------------------------------------------- dispatch
template <int TB, int CB, bool ADJ>
__device__ __forceinline__ void u1_form(int form, Pk (&v)[8], Pk (&w)[8], const u64* c) {
  switch (form) {
    case kFormRI: u1_static<TB, CB, kFormRI, ADJ>(v, w, c); break;
    case kFormReal: u1_static<TB, CB, kFormReal, ADJ>(v, w, c); break;
    case kFormDiag: u1_static<TB, CB, kFormDiag, ADJ>(v, w, c); break;
    case kFormSwap: u1_static<TB, CB, kFormSwap, ADJ>(v, w, c); break;
    default: u1_static<TB, CB, kFormGen, ADJ>(v, w, c); break;
  }
}
template <int TB, bool ADJ>
__device__ __forceinline__ void u1_form_masked(int form, Pk (&v)[8], Pk (&w)[8], const u64* c, uint32_t rmask) {
  switch (form) {
    case kFormRI: u1_masked<TB, kFormRI, ADJ>(v, w, c, rmask); break;
    case kFormReal: u1_masked<TB, kFormReal, ADJ>(v, w, c, rmask); break;
    case kFormDiag: u1_masked<TB, kFormDiag, ADJ>(v, w, c, rmask); break;
    case kFormSwap: u1_masked<TB, kFormSwap, ADJ>(v, w, c, rmask); break;
    default: u1_masked<TB, kFormGen, ADJ>(v, w, c, rmask); break;
  }
}
template <int TB, int CB>
__device__ __forceinline__ void acc_kind(int kind, const Pk (&v)[8], const Pk (&w)[8], float (&s8)[8]) {
  switch (kind) {
    case kAccOff: acc_static<TB, CB, kAccOff>(v, w, s8); break;
    case kAccDiag: acc_static<TB, CB, kAccDiag>(v, w, s8); break;
    case kAccAH | kAccFull: acc_static<TB, CB, kAccAH | kAccFull>(v, w, s8); break;
    case kAccAH | kAccOff: acc_static<TB, CB, kAccAH | kAccOff>(v, w, s8); break;
    case kAccAH | kAccDiag: acc_static<TB, CB, kAccAH | kAccDiag>(v, w, s8); break;
    default: acc_static<TB, CB, kAccFull>(v, w, s8); break;
  }
}
template <int TB>
__device__ __forceinline__ void acc_kind_masked(int kind, const Pk (&v)[8], const Pk (&w)[8], uint32_t rmask,
                                                float (&s8)[8]) {
  switch (kind) {
    case kAccOff: acc_masked<TB, kAccOff>(v, w, rmask, s8); break;
    case kAccDiag: acc_masked<TB, kAccDiag>(v, w, rmask, s8); break;
    case kAccAH | kAccFull: acc_masked<TB, kAccAH | kAccFull>(v, w, rmask, s8); break;
    case kAccAH | kAccOff: acc_masked<TB, kAccAH | kAccOff>(v, w, rmask, s8); break;
    case kAccAH | kAccDiag: acc_masked<TB, kAccAH | kAccDiag>(v, w, rmask, s8); break;
    default: acc_masked<TB, kAccFull>(v, w, rmask, s8); break;
  }
}

// rctl: 0 = no register control, 1..4 = one control on j-bit rctl-1 at |1>,
// 7 = controls given by rmask.  With acc, s8 receives this thread's partials
// of the reduced matrix (the caller reduces them over the warp).
template <int TB, bool ADJ>
__device__ __forceinline__ void u1_target(int rctl, int form, bool acc, int kind, uint32_t rmask, Pk (&v)[8],
                                          Pk (&w)[8], const u64* c, float (&s8)[8]) {
#define VQC_U1_CB(CBV)                                 \
  {                                                    \
    u1_form<TB, CBV, ADJ>(form, v, w, c);              \
    if (ADJ && acc) acc_kind<TB, CBV>(kind, v, w, s8); \
  }
  switch (rctl) {
    case 0: VQC_U1_CB(-1) break;
    case 1: VQC_U1_CB(TB == 0 ? -1 : 0) break;  // (TB == 0 never has a lane control)
    case 2: VQC_U1_CB(TB == 1 ? -1 : 1) break;
    case 3: VQC_U1_CB(TB == 2 ? -1 : 2) break;
    case 4: VQC_U1_CB(TB == 3 ? -1 : 3) break;
    default:
      u1_form_masked<TB, ADJ>(form, v, w, c, rmask);
      if (ADJ && acc) acc_kind_masked<TB>(kind, v, w, rmask, s8);
      break;
  }
#undef VQC_U1_CB
}

// Two target j-bits JA < JB: dense 4x4 (bit 0 <-> JA) on each quad whose base
// amplitude is enabled in rmask.
template <int JA, int JB, bool ADJ, int NP>
__device__ __forceinline__ void u2_op(Pk (&v)[NP], Pk (&w)[NP], const float2* U, uint32_t rmask) {
#pragma unroll
  for (int q = 0; q < NP / 2; ++q) {
    int j = q;
    j = ((j >> JA) << (JA + 1)) | (j & ((1 << JA) - 1));
    j = ((j >> JB) << (JB + 1)) | (j & ((1 << JB) - 1));
    if (!((rmask >> j) & 1)) continue;
    const int idx[4] = {j, j | (1 << JA), j | (1 << JB), j | (1 << JA) | (1 << JB)};
#pragma unroll
    for (int st = 0; st < (ADJ ? 2 : 1); ++st) {
      Pk(&s)[NP] = st ? w : v;
      float2 x[4], o[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) x[i] = amp(s, idx[i]);
#pragma unroll
      for (int r = 0; r < 4; ++r) {  // the cotangent (st == 1, held conjugated) with conj(U)
        const float sg = st ? -1.f : 1.f;
        const float2 u0 = U[4 * r];
        o[r] = ccmul(make_float2(u0.x, sg * u0.y), x[0]);
#pragma unroll
        for (int cc = 1; cc < 4; ++cc) {
          const float2 u = U[4 * r + cc];
          o[r] = ccfma(make_float2(u.x, sg * u.y), x[cc], o[r]);
        }
      }
#pragma unroll
      for (int i = 0; i < 4; ++i) set_amp(s, idx[i], o[i]);
    }
  }
}
template <bool ADJ>
__device__ __forceinline__ void u2_dispatch(int ja, int jb, Pk (&v)[8], Pk (&w)[8], const float2* U, uint32_t rmask) {
  switch (ja * 4 + jb) {
    case 1: u2_op<0, 1, ADJ>(v, w, U, rmask); break;
    case 2: u2_op<0, 2, ADJ>(v, w, U, rmask); break;
    case 3: u2_op<0, 3, ADJ>(v, w, U, rmask); break;
    case 6: u2_op<1, 2, ADJ>(v, w, U, rmask); break;
    case 7: u2_op<1, 3, ADJ>(v, w, U, rmask); break;
    default: u2_op<2, 3, ADJ>(v, w, U, rmask); break;
  }
}

// ----------------------------------------------------------------------------- diagonal ops
// Diagonal (phase) op: phase index from the op's qubits, tile bits per
// amplitude and non-tile qubits per tile.
template <bool ADJ, int NP>
__device__ __forceinline__ void diag_op(Pk (&v)[NP], Pk (&w)[NP], const DevOp* op, const float2* c, uint32_t tthr,
                                        const uint32_t* dep, uint64_t base) {
  const int nd = op->nd;
  uint32_t gidx = 0;
  int db[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    db[i] = i < nd ? op->dbit[i] : -1;
    if (i < nd && db[i] < 0) gidx |= (uint32_t)((base >> op->dglob[i]) & 1) << i;
  }
#pragma unroll
  for (int j = 0; j < 2 * NP; ++j) {
    const uint32_t t = tthr | dep[j];
    uint32_t idx = gidx;
#pragma unroll
    for (int i = 0; i < 5; ++i)
      if (db[i] >= 0) idx |= ((t >> db[i]) & 1u) << i;
    const float2 d = c[idx];
    set_amp(v, j, ccmul(d, amp(v, j)));
    if (ADJ) set_amp(w, j, ccmul(make_float2(d.x, -d.y), amp(w, j)));  // the conjugated cotangent
  }
}
// Bins of conj(lam) psi over a diagonal op's (at most 2) qubits -> s8.
__device__ __forceinline__ void accd_op(const Pk (&v)[8], const Pk (&w)[8], const DevOp* op, uint32_t tthr,
                                        const uint32_t* dep, uint64_t base, float (&s8)[8]) {
  const int nd = op->nd;
  uint32_t gidx = 0;
  int db[2];
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    db[i] = i < nd ? op->dbit[i] : -1;
    if (i < nd && db[i] < 0) gidx |= (uint32_t)((base >> op->dglob[i]) & 1) << i;
  }
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const uint32_t t = tthr | dep[j];
    uint32_t idx = gidx;
#pragma unroll
    for (int i = 0; i < 2; ++i)
      if (db[i] >= 0) idx |= ((t >> db[i]) & 1u) << i;
    const float2 m = amp(w, j), p = amp(v, j);  // m = conj(lam)
    const float re = fmaf(m.x, p.x, -m.y * p.y), im = fmaf(m.x, p.y, m.y * p.x);
#pragma unroll
    for (int b = 0; b < 4; ++b)
      if (idx == (uint32_t)b) {
        s8[2 * b] += re;
        s8[2 * b + 1] += im;
      }
  }
}

// ----------------------------------------------------------------------------- the tile loop
// Per-CTA context of a pass: the state pointers, the staged descriptors in
// shared memory, and the tile counter in the deposited (non-tile bit) space,
// base(t + ncta) = ((base | ~mask) + inc) & mask.
template <int M, bool ADJ, int RB = kRegBits>
struct TileCtx {
  static constexpr int NT = 1 << (M - RB), NW = NT / 32, NPAIR = 1 << (M - 1);
  float2* psi;
  float2* lam;
  ulonglong2* sp;
  ulonglong2* sl;
  ulonglong2* spb;  // the second tile buffer of the asynchronous forward passes (NBUF = 2)
  double* sacc;
  const DevStageF* stages;
  const DevOp* ops;
  const float2* pool;
  const DevPass* P;  // shared copy
  uint64_t base;
  int ntiles_here, tlo, thi;
};

// Stages the pass's descriptors, zeroes the accumulation slots and sets up
// the tile counter.  Every thread of the CTA calls it.  NBUF = 2 puts a
// second tile buffer in front of the usual layout (the asynchronous forward
// passes copy the next tile into it while the current one is computed).
template <int M, bool ADJ, int NBUF = 1, int RB = kRegBits>
__device__ __forceinline__ void tile_setup(TileCtx<M, ADJ, RB>& x, float2* psi, float2* lam, const DevPass* pass,
                                           const DevStageF* stages, const DevOp* ops, const float2* pool, int ncta,
                                           DevPass& P, uint64_t& s_inc, uint64_t& s_base0, bool stage_pool = true) {
  constexpr int NT = TileCtx<M, ADJ, RB>::NT, NW = TileCtx<M, ADJ, RB>::NW, NPAIR = TileCtx<M, ADJ, RB>::NPAIR;
  extern __shared__ __align__(16) unsigned char smem_all[];
  unsigned char* smem = smem_all + (NBUF - 1) * (unsigned long long)NPAIR * 16;
  if (threadIdx.x == 0) P = *pass;
  __syncthreads();
  const int nslots = ADJ ? P.nslots : 0;
  x.spb = reinterpret_cast<ulonglong2*>(smem_all);
  x.sp = reinterpret_cast<ulonglong2*>(smem);
  x.sl = x.sp + (ADJ ? NPAIR : 0);
  x.sacc = reinterpret_cast<double*>(smem + tile_bytes_f32<M, ADJ>());
  for (int i = threadIdx.x; i < nslots * NW * 8; i += NT) x.sacc[i] = 0;
  {
    // the pass's descriptors -> shared memory (16-byte words)
    unsigned char* dst = smem + tile_bytes_f32<M, ADJ>() + (unsigned long long)nslots * NW * 8 * sizeof(double);
    const int nst = P.stage_end - P.stage_begin;
    const unsigned long long b1 = sizeof(DevStageF) * nst, b2 = sizeof(DevOp) * P.nops,
                             b3 = sizeof(float2) * P.npool;
    const int4* s1 = reinterpret_cast<const int4*>(stages + P.stage_begin);
    const int4* s2 = reinterpret_cast<const int4*>(ops);
    const int4* s3 = reinterpret_cast<const int4*>(pool);
    int4* d1 = reinterpret_cast<int4*>(dst);
    int4* d2 = reinterpret_cast<int4*>(dst + b1);
    int4* d3 = reinterpret_cast<int4*>(dst + b1 + b2);
    for (unsigned i = threadIdx.x; i < b1 / 16; i += NT) d1[i] = __ldg(s1 + i);
    for (unsigned i = threadIdx.x; i < b2 / 16; i += NT) d2[i] = __ldg(s2 + i);
    if (stage_pool)
      for (unsigned i = threadIdx.x; i < (b3 + 15) / 16; i += NT) d3[i] = __ldg(s3 + i);
    x.stages = reinterpret_cast<const DevStageF*>(dst) - P.stage_begin;
    x.ops = reinterpret_cast<const DevOp*>(dst + b1);
    x.pool = reinterpret_cast<const float2*>(dst + b1 + b2);
  }
  if (threadIdx.x == 0) {
    uint64_t mm = P.nontile_mask, b0 = 0, inc = 0;
    int64_t t = blockIdx.x, s = ncta;
    while (mm) {
      const uint64_t low = mm & (~mm + 1);
      if (t & 1) b0 |= low;
      if (s & 1) inc |= low;
      t >>= 1;
      s >>= 1;
      mm ^= low;
    }
    s_inc = inc;
    s_base0 = b0;
  }
  __syncthreads();
  x.psi = psi;
  x.lam = lam;
  x.P = &P;
  x.base = s_base0;
  const int64_t rem = P.ntiles - (int64_t)blockIdx.x;
  x.ntiles_here = rem > 0 ? (int)((rem - 1) / ncta + 1) : 0;  // this CTA's tiles
  x.tlo = threadIdx.x & 15;
  x.thi = threadIdx.x >> 4;
}

// A stage's registers: from HBM (the pass's first stage) or shared memory.
template <int M, bool ADJ>
__device__ __forceinline__ void stage_load(const TileCtx<M, ADJ>& x, const DevStageF* S, bool first, Pk (&v)[8],
                                           Pk (&w)[8]) {
  if (first) {
    const int64_t g0 = (int64_t)x.base + S->gthr[0][x.tlo] + S->gthr[1][x.thi];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int64_t gi = g0 + S->gdep[m];
      if (!VQC_DCHECK(gi + 1, x.P->ntiles << M)) continue;
      const float4 t = *reinterpret_cast<const float4*>(x.psi + gi);
      v[m].r = mk(t.x, t.z);
      v[m].i = mk(t.y, t.w);
      if (ADJ) {  // the cotangent is held conjugated
        const float4 u = *reinterpret_cast<const float4*>(x.lam + gi);
        w[m].r = mk(u.x, u.z);
        w[m].i = mk(-u.y, -u.w);
      }
    }
  } else {
    const uint32_t sw = S->swt[0][x.tlo] ^ S->swt[1][x.thi];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint32_t a = sw ^ S->swm[m];
      if (!VQC_DCHECK(a, (TileCtx<M, ADJ>::NPAIR))) continue;
      const ulonglong2 t = x.sp[a];
      v[m].r = t.x;
      v[m].i = t.y;
      if (ADJ) {
        const ulonglong2 u = x.sl[a];
        w[m].r = u.x;
        w[m].i = u.y;
      }
    }
  }
}
// ... and back (HBM after the pass's last stage), then the CTA barrier.
template <int M, bool ADJ>
__device__ __forceinline__ void stage_store(const TileCtx<M, ADJ>& x, const DevStageF* S, bool last, const Pk (&v)[8],
                                            const Pk (&w)[8]) {
  if (last) {
    const int64_t g0 = (int64_t)x.base + S->gthr[0][x.tlo] + S->gthr[1][x.thi];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int64_t gi = g0 + S->gdep[m];
      if (!VQC_DCHECK(gi + 1, x.P->ntiles << M)) continue;
      *reinterpret_cast<float4*>(x.psi + gi) = make_float4(lo(v[m].r), lo(v[m].i), hi(v[m].r), hi(v[m].i));
      if (ADJ)  // conjugated back
        *reinterpret_cast<float4*>(x.lam + gi) = make_float4(lo(w[m].r), -lo(w[m].i), hi(w[m].r), -hi(w[m].i));
    }
  } else {
    const uint32_t sw = S->swt[0][x.tlo] ^ S->swt[1][x.thi];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const uint32_t a = sw ^ S->swm[m];
      if (!VQC_DCHECK(a, (TileCtx<M, ADJ>::NPAIR))) continue;
      x.sp[a] = make_ulonglong2(v[m].r, v[m].i);
      if (ADJ) x.sl[a] = make_ulonglong2(w[m].r, w[m].i);
    }
  }
  __syncthreads();  // also orders this tile's last shared reads before the next tile's writes
}
// The same with the stage's pair offsets as compile-time constants (the
// compiled pass kernels): no dependent descriptor loads before the data.
template <int M, bool ADJ, int RB, int NP>
__device__ __forceinline__ void stage_load_k(const TileCtx<M, ADJ, RB>& x, const DevStageF* S, bool first,
                                             Pk (&v)[NP], Pk (&w)[NP], const uint32_t (&swm)[NP],
                                             const int64_t (&gdep)[NP]) {
  static_assert(NP == (1 << (RB - 1)), "register pairs");
  if (first) {
    const int64_t g0 = (int64_t)x.base + S->gthr[0][x.tlo] + S->gthr[1][x.thi];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      const int64_t gi = g0 + gdep[m];
      if (!VQC_DCHECK(gi + 1, x.P->ntiles << M)) continue;
      const float4 t = *reinterpret_cast<const float4*>(x.psi + gi);
      v[m].r = mk(t.x, t.z);
      v[m].i = mk(t.y, t.w);
      if (ADJ) {  // the cotangent is held conjugated
        const float4 u = *reinterpret_cast<const float4*>(x.lam + gi);
        w[m].r = mk(u.x, u.z);
        w[m].i = mk(-u.y, -u.w);
      }
    }
  } else {
    const uint32_t sw = S->swt[0][x.tlo] ^ S->swt[1][x.thi];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      const uint32_t a = sw ^ swm[m];
      if (!VQC_DCHECK(a, (TileCtx<M, ADJ, RB>::NPAIR))) continue;
      const ulonglong2 t = x.sp[a];
      v[m].r = t.x;
      v[m].i = t.y;
      if (ADJ) {
        const ulonglong2 u = x.sl[a];
        w[m].r = u.x;
        w[m].i = u.y;
      }
    }
  }
}
// cta = false: the next stage (or the next tile's first stage) maps the warp
// index to the same tile bits as this one, so every pair a thread reads next
// was stored by its own warp and a warp barrier orders the exchange (a thread
// stores only the pairs it loaded, so no other warp's reads are overtaken).
template <int M, bool ADJ, int RB, int NP>
__device__ __forceinline__ void stage_store_k(const TileCtx<M, ADJ, RB>& x, const DevStageF* S, bool last,
                                              const Pk (&v)[NP], const Pk (&w)[NP], const uint32_t (&swm)[NP],
                                              const int64_t (&gdep)[NP], bool cta = true) {
  if (last) {
    const int64_t g0 = (int64_t)x.base + S->gthr[0][x.tlo] + S->gthr[1][x.thi];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      const int64_t gi = g0 + gdep[m];
      if (!VQC_DCHECK(gi + 1, x.P->ntiles << M)) continue;
      *reinterpret_cast<float4*>(x.psi + gi) = make_float4(lo(v[m].r), lo(v[m].i), hi(v[m].r), hi(v[m].i));
      if (ADJ)  // conjugated back
        *reinterpret_cast<float4*>(x.lam + gi) = make_float4(lo(w[m].r), -lo(w[m].i), hi(w[m].r), -hi(w[m].i));
    }
  } else {
    const uint32_t sw = S->swt[0][x.tlo] ^ S->swt[1][x.thi];
#pragma unroll
    for (int m = 0; m < NP; ++m) {
      const uint32_t a = sw ^ swm[m];
      if (!VQC_DCHECK(a, (TileCtx<M, ADJ, RB>::NPAIR))) continue;
      x.sp[a] = make_ulonglong2(v[m].r, v[m].i);
      if (ADJ) x.sl[a] = make_ulonglong2(w[m].r, w[m].i);
    }
  }
  if (cta)
    __syncthreads();
  else
    __syncwarp();
}

// ----------------------------------------------------------------------------- asynchronous tile copies
// Forward passes: the next tile's first-stage pairs are copied into a second
// shared buffer with cp.async (16 bytes per pair, as stored in HBM: two
// interleaved complex amplitudes) while the current tile is computed, so the
// HBM transfer overlaps the arithmetic instead of following it.
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
template <int M, bool ADJ>
__device__ __forceinline__ uint64_t tile_base_after(const TileCtx<M, ADJ>& x, uint64_t s_inc) {
  return ((x.base | ~x.P->nontile_mask) + s_inc) & x.P->nontile_mask;
}
// The first stage's pairs of the tile at `base` into `buf`, at the stage's
// swizzled pair indices; one commit group per tile.
template <int M>
__device__ __forceinline__ void tile_copy_async(const TileCtx<M, false>& x, const DevStageF* S, uint64_t base,
                                                ulonglong2* buf, const uint32_t (&swm)[8], const int64_t (&gdep)[8]) {
  const int64_t g0 = (int64_t)base + S->gthr[0][x.tlo] + S->gthr[1][x.thi];
  const uint32_t sw = S->swt[0][x.tlo] ^ S->swt[1][x.thi];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const int64_t gi = g0 + gdep[m];
    const uint32_t a = sw ^ swm[m];
    if (!VQC_DCHECK(gi + 1, x.P->ntiles << M) || !VQC_DCHECK(a, (TileCtx<M, false>::NPAIR))) continue;
    cp_async16(buf + a, x.psi + gi);
  }
  cp_async_commit();
}
// The first stage's registers from that copy (interleaved -> packed pairs).
template <int M>
__device__ __forceinline__ void stage_load_raw(const TileCtx<M, false>& x, const DevStageF* S, const ulonglong2* buf,
                                               Pk (&v)[8], const uint32_t (&swm)[8]) {
  const uint32_t sw = S->swt[0][x.tlo] ^ S->swt[1][x.thi];
#pragma unroll
  for (int m = 0; m < 8; ++m) {
    const uint32_t a = sw ^ swm[m];
    if (!VQC_DCHECK(a, (TileCtx<M, false>::NPAIR))) continue;
    const float4 t = reinterpret_cast<const float4*>(buf)[a];
    v[m].r = mk(t.x, t.z);
    v[m].i = mk(t.y, t.w);
  }
}

// L2 prefetch of the next tile's first-stage pairs (no shared memory, no
// registers held): the next tile's loads then come from L2.
template <int M, bool ADJ, int RB, int NP>
__device__ __forceinline__ void prefetch_next_l2(const TileCtx<M, ADJ, RB>& x, const DevStageF* S, uint64_t s_inc,
                                                 const int64_t (&gdep)[NP]) {
  const uint64_t next = ((x.base | ~x.P->nontile_mask) + s_inc) & x.P->nontile_mask;
  const int64_t g0 = (int64_t)next + S->gthr[0][x.tlo] + S->gthr[1][x.thi];
#pragma unroll
  for (int m = 0; m < NP; ++m) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(x.psi + g0 + gdep[m]));
    if (ADJ) asm volatile("prefetch.global.L2 [%0];" ::"l"(x.lam + g0 + gdep[m]));
  }
}

template <int M, bool ADJ, int RB>
__device__ __forceinline__ void tile_next(TileCtx<M, ADJ, RB>& x, uint64_t s_inc) {
  x.base = ((x.base | ~x.P->nontile_mask) + s_inc) & x.P->nontile_mask;
}
// Per-warp slot rows -> this CTA's partials row (fixed order).
template <int M, bool ADJ, int RB>
__device__ __forceinline__ void tile_finish(const TileCtx<M, ADJ, RB>& x, double* partials) {
  constexpr int NT = TileCtx<M, ADJ, RB>::NT, NW = TileCtx<M, ADJ, RB>::NW;
  const int nslots = ADJ ? x.P->nslots : 0;
  if (ADJ && nslots > 0) {
    __syncthreads();
    for (int i = threadIdx.x; i < nslots * 8; i += NT) {
      const int slot = i >> 3, val = i & 7;
      double s = 0;
      for (int wp = 0; wp < NW; ++wp) s += x.sacc[((unsigned long long)slot * NW + wp) * 8 + val];
      partials[((unsigned long long)blockIdx.x * nslots + slot) * 8 + val] = s;
    }
  }
}

// The interpreter: every op decoded at run time (any pass, any batch).
template <int M, bool ADJ, bool GEN>
__device__ __forceinline__ void interp_ops(const TileCtx<M, ADJ>& x, const DevStageF* S, Pk (&v)[8], Pk (&w)[8]) {
  constexpr int NW = TileCtx<M, ADJ>::NW;
  const uint32_t tthr = S->thr[0][x.tlo] | S->thr[1][x.thi];
  const int ob = S->op_begin, oe = S->op_end;
  for (int o = ob; o < oe; ++o) {
    const DevOp* op = x.ops + o;
    const int4 hd = *reinterpret_cast<const int4*>(op);
    const int code = hd.x, type = code & 15;
    if (code & kCodeGCtl) {  // a control on a non-tile qubit: uniform over the tile
      if ((x.base & op->gmask) != op->gval) continue;
    }
    // controls on thread bits: one test per op (may differ between the lanes
    // of a warp: the warp-wide reduction below runs outside it)
    const bool run = !(code & kCodeCtl) || (tthr & (uint32_t)hd.z) == (uint32_t)hd.w;
    const float2* c = x.pool + hd.y;
    const u64* c2 = reinterpret_cast<const u64*>(c);
    if (!GEN || type == kOpU1) {
      const bool acc = ADJ && (code & kCodeAcc);
      if (!run && !acc) continue;
      const int tb = (code >> 4) & 3, rctl = (code >> 16) & 7, form = (code >> 11) & 7, kind = acc_kind_of(code);
      const uint32_t rmask = (uint32_t)op->rmask;
      float s8[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) s8[i] = 0.f;
      if (run) {
        switch (tb) {
          case 0: u1_target<0, ADJ>(rctl, form, acc, kind, rmask, v, w, c2, s8); break;
          case 1: u1_target<1, ADJ>(rctl, form, acc, kind, rmask, v, w, c2, s8); break;
          case 2: u1_target<2, ADJ>(rctl, form, acc, kind, rmask, v, w, c2, s8); break;
          default: u1_target<3, ADJ>(rctl, form, acc, kind, rmask, v, w, c2, s8); break;
        }
      }
      if (ADJ && acc) {
        if (kind & kAccAH)
          flush4(s8, x.sacc, op->slot, NW);
        else
          flush8(s8, x.sacc, op->slot, NW);
      }
    } else if (!run && type != kOpAccD) {  // (diagonal ops carry no controls; AccD always reduces)
    } else if (type == kOpU2) {
      u2_dispatch<ADJ>((code >> 4) & 3, (code >> 6) & 3, v, w, c, (uint32_t)op->rmask);
    } else if (type == kOpDiag) {
      diag_op<ADJ>(v, w, op, c, tthr, S->dep, x.base);
    } else if (ADJ) {
      float s8[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) s8[i] = 0.f;
      accd_op(v, w, op, tthr, S->dep, x.base, s8);
      flush8(s8, x.sacc, op->slot, NW);
    }
  }
}

template <int M, bool ADJ, bool GEN>
__device__ __forceinline__ void tile_body(float2* __restrict__ psi, float2* __restrict__ lam,
                                          const DevPass* __restrict__ pass, const DevStageF* __restrict__ stages,
                                          const DevOp* __restrict__ ops, const float2* __restrict__ pool,
                                          double* __restrict__ partials, int ncta) {
  __shared__ DevPass P;
  __shared__ uint64_t s_inc, s_base0;
  TileCtx<M, ADJ> x;
  tile_setup<M, ADJ>(x, psi, lam, pass, stages, ops, pool, ncta, P, s_inc, s_base0);
  Pk v[8], w[8];
  for (int it = 0; it < x.ntiles_here; ++it) {
    const int s_first = P.stage_begin, s_last = P.stage_end - 1;
    for (int s = s_first; s <= s_last; ++s) {
      const DevStageF* S = x.stages + s;
      stage_load<M, ADJ>(x, S, s == s_first, v, w);
      interp_ops<M, ADJ, GEN>(x, S, v, w);
      stage_store<M, ADJ>(x, S, s == s_last, v, w);
    }
    tile_next<M, ADJ>(x, s_inc);
  }
  tile_finish<M, ADJ>(x, partials);
}

}  // namespace f32t
}  // namespace vqc
