// Device-side descriptors of the tile engine: the pass, stage and op
// records the tile kernels read.  Self-contained (no host headers) so that the
// run-time compiled pass kernels can include it as well.
#pragma once

#ifdef __CUDACC_RTC__
typedef unsigned long long uint64_t;
typedef long long int64_t;
typedef unsigned int uint32_t;
typedef int int32_t;
#else
#include <cstdint>
#endif

// Index checks of the debug build (common.cuh); the run-time compiled pass
// kernels and the release build see the constant true.
#ifndef VQC_DCHECK
#define VQC_DCHECK(i, lim) true
#endif

namespace vqc {

constexpr int kRegBits = 4;  // 16 amplitudes per thread
constexpr int kMaxSlots = 64;
constexpr int kMaxOpsPerPass = 192;  // bounds the pass's descriptors staged in shared memory
enum { kOpU1 = 1, kOpU2 = 2, kOpDiag = 3, kOpAccD = 4 };

struct DevPass {
  uint64_t nontile_mask;  // global bits enumerated by the tile counter
  int64_t ntiles;
  int32_t stage_begin, stage_end;
  int32_t nslots;
  int32_t nops;           // ops of this pass (copied to shared memory with the stages)
  int32_t npool;          // matrix pool entries of this pass
  int32_t pad;
};

struct alignas(16) DevStage {
  uint32_t dep[16];    // tile index of register slot j (OR with the thread part)
  int64_t gdep[16];    // global offset of register slot j
  uint64_t gthr_mask;  // global qubits of the thread's tile bits
  uint32_t thr_mask;   // tile bits held by the thread index, ascending
  int32_t op_begin, op_end, pad;
};

// A stage of the FP32 (packed) tile body: tile bit 0 is always a register
// bit (the lane bit inside each float4 pair), plus three free register bits
// (16 amplitudes per thread), or four in the wide forward passes (32).
// Per-thread quantities are split into two tables indexed by the thread
// index's low and high nibble (thread bits are at most 8).
constexpr int kWideRegBits = 5;  // wide compiled forward passes: 32 amplitudes per thread
struct alignas(16) DevStageF {
  int64_t gdep[16];      // global amplitude offset of register pair m (lane 0)
  int64_t gthr[2][16];   // global offset of the thread's tile bits: [0][tid & 15] + [1][tid >> 4]
  uint32_t thr[2][16];   // tile index of the thread's bits: [0][tid & 15] | [1][tid >> 4]
  uint32_t swt[2][16];   // swizzled pair index of the thread's bits: [0][..] ^ [1][..]
  uint32_t swm[16];      // swizzled pair index of register pair m
  uint32_t dep[32];      // tile index of register amplitude j = lane + 2m
  int32_t op_begin, op_end, pad0, pad1;
};

// code: bits 0-3 op type, 4-5 r0, 6-7 r1, 8 tile-bit controls, 9 non-tile
// controls, 10 accumulate, 20-21 the third bits of r0 / r1.  The first 16 bytes are read as one vector load.
// In the FP32 body, r0/r1 are j-bits (0 = lane bit, 1..3 or 1..4 = free
// register bits), cmask/cval hold only the controls on thread bits, and the
// controls on register bits are bits 16-18 (0: none, 1..5: one control on
// j-bit value-1 at |1>, 7: the amplitudes enabled in rmask).
struct alignas(16) DevOp {
  int32_t code;
  int32_t mat;     // pool offset (complex elements)
  uint32_t cmask, cval;  // controls on tile bits
  uint64_t gmask, gval;  // controls on non-tile qubits
  int32_t slot;    // accumulation slot or -1
  int32_t nd;      // diagonal ops: number of qubits
  int32_t dbit[5];  // tile bit of diagonal qubit i, or -1
  int32_t dglob[5]; // global qubit of diagonal qubit i when not a tile bit
  int32_t rmask;    // FP32 body: register amplitudes (pair representatives) the controls enable
};
constexpr int kCodeCtl = 1 << 8, kCodeGCtl = 1 << 9, kCodeAcc = 1 << 10;
// r0 / r1 as 3-bit j-bits (the wide FP32 body has j-bits 0..4): bits 4-5 and
// 6-7 hold the low two bits, bits 20 and 21 the third.
__host__ __device__ constexpr int op_r0(int code) { return ((code >> 4) & 3) | (((code >> 20) & 1) << 2); }
__host__ __device__ constexpr int op_r1(int code) { return ((code >> 6) & 3) | (((code >> 21) & 1) << 2); }
__host__ __device__ constexpr int op_r_bits(int r0, int r1) {
  return ((r0 & 3) << 4) | ((r1 & 3) << 6) | ((r0 >> 2) << 20) | ((r1 >> 2) << 21);
}
// bits 11-13: one-qubit matrix form; bits 14-15: reduced-matrix entries
// accumulated; bits 16-18: register control; bit 19: anti-Hermitian projection
constexpr int kCodeAH = 1 << 19;
// One-qubit matrix forms (read off the matrix on the host): general complex;
// "RI" = real diagonal and imaginary off-diagonal (RX-like); real (RY-like);
// diagonal (RZ / phase); the exact swap [[0,1],[1,0]] (X, the CNOT/Toffoli target).
enum { kFormGen = 0, kFormRI = 1, kFormReal = 2, kFormDiag = 3, kFormSwap = 4 };
// Reduced-matrix entries a parameter's D touches: all four, off-diagonal,
// diagonal; kAccAH added (FP32 body) when every D is anti-Hermitian and only
// (Im A00, Im A11, Re A01 - Re A10, Im A01 + Im A10) are accumulated.
enum { kAccFull = 0, kAccOff = 1, kAccDiag = 2, kAccAH = 4 };
__host__ __device__ constexpr int acc_kind_of(int code) {
  return ((code >> 14) & 3) | ((code & kCodeAH) ? kAccAH : 0);
}

// One pass each of many states in one launch (the serving path): request
// blockIdx.y, its tiles strided over its own `ncta` CTAs (fixed per request,
// so its sums are grouped the same way whatever it is batched with); CTAs
// beyond ncta leave at once.
struct TileItem {
  void* psi;
  void* lam;
  const DevPass* pass;
  const void* stages;  // DevStage (FP64) or DevStageF (FP32)
  const DevOp* ops;
  const void* pool;
  double* partials;  // [ncta][nslots][8]
  int64_t ntiles;
  int ncta;
  int pad;
};

// Shared-memory bytes of the FP32 tile(s) of one pass.
template <int M, bool ADJ>
__host__ __device__ constexpr unsigned long long tile_bytes_f32() {
  return (ADJ ? 2ull : 1ull) * (1ull << M) * 8ull;
}

}  // namespace vqc
