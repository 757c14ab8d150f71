// The fused tile engine: apply!(::QCircuit, state) (generic.jl:26-31) and the
// reverse sweep of the circuit pullback (circuitdiff.jl:61-75) with many gates
// per HBM round trip.
//
// The reference runs one full pass over the state per gate.  Here a host
// planner groups the gates into *passes*.  A pass picks a set Q of M "tile"
// qubits (always including the lowest qubits, so every tile is made of
// contiguous runs of amplitudes); every CTA loads whole tiles (the 2^M
// amplitudes that share all non-tile bits) into shared memory, applies every
// gate of the pass to them, and writes them back: one HBM read + write per
// pass instead of per gate.
//   * a gate whose matrix acts on one or two target qubits (after stripping
//     control qubits, read off the matrix) is applied in registers: each
//     thread holds 16 amplitudes spanning 4 tile bits ("register bits"), and
//     the pass is cut into *stages*, each with one register-bit set;
//     between stages the tile goes through shared memory (XOR-swizzled, so
//     the 16-byte / 8-byte accesses are free of bank conflicts);
//   * controls on tile bits are tested per amplitude, controls on non-tile
//     qubits once per tile;
//   * diagonal gates (CZ, CPHASE, ...) act on any qubits, tile or not;
//   * consecutive one-qubit gates on the same qubit are merged into one 2x2.
// In the reverse sweep (ADJ) each op applies U^dagger to both the cotangent
// and the state and accumulates the reduced matrix
//   A[a][b] = sum conj(lambda_a) psi_b   over the op's target pairs
// (per thread over its 8 pairs in the state's precision, then in FP64 across
// the warp, the CTA and the grid, in a fixed order); the host contracts A
// with D_j = B^dagger dB/dtheta_j of each parameter j of the (merged) block.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <thread>
#include <type_traits>

#include "engine.h"
#include "subspace.cuh"
#include "tile_f32.cuh"
#include "tile_kernels.cuh"
#include "tile_plan.cuh"

namespace vqc {

// The tile kernels themselves live in tile_kernels_impl.cuh (tile_inst_*.cu).

// Sums the per-CTA partials of many passes over their grids in a fixed order:
// one item per pass (blockIdx.y), block x = slot (defined with the serving
// support below).
__global__ void __launch_bounds__(256) k_reduce_slots_batch(const RedItem* __restrict__ items);

// ----------------------------------------------------------------------------- host planner
// A gate in planner form: one op, or "standalone" (kept as a GateSpec).
struct PItem {
  bool standalone = false;
  int gate = -1;  // index in the caller's gate list
  FOp op;
};

static inline int popc64(uint64_t x) { return __builtin_popcountll(x); }

// Reads a gate's structure off its (sorted, possibly daggered) matrix.
// Returns false when the gate cannot be fused (3+ target qubits).
static bool to_fop(const GateSpec& g, FOp& f) {
  const int k = g.k, d = 1 << k;
  f = FOp();
  for (int b = 0; b < k; ++b) f.qubits |= 1ull << g.sp[b];
  if (g.ns == 0) {  // identity
    f.kind = kOpDiag;
    f.nd = 0;
    f.mat = {cd(1)};
    return true;
  }
  if (k == 1) {  // one-qubit gates (diagonal ones too) run in registers and merge
    f.kind = kOpU1;
    f.tq[0] = g.sp[0];
    f.mat = g.U;
    return true;
  }
  if (g.mode == kDiag) {
    f.kind = kOpDiag;
    f.nd = k;
    for (int b = 0; b < k; ++b) f.dq[b] = g.sp[b];
    f.mat.resize(d);
    for (int j = 0; j < d; ++j) f.mat[j] = g.U[(size_t)j * d + j];
    return true;
  }
  // controls: bits constant over the active set
  int ctrl_bits = 0, cval_bits = 0;
  for (int b = 0; b < k; ++b) {
    bool all1 = true, all0 = true;
    for (int s = 0; s < g.ns; ++s) {
      if (g.S[s] >> b & 1)
        all0 = false;
      else
        all1 = false;
    }
    if (all1 || all0) {
      ctrl_bits |= 1 << b;
      if (all1) cval_bits |= 1 << b;
    }
  }
  int tb[5], nt = 0;
  for (int b = 0; b < k; ++b)
    if (!(ctrl_bits >> b & 1)) tb[nt++] = b;
  if (nt == 0 || nt > 2) return false;
  for (int b = 0; b < k; ++b)
    if (ctrl_bits >> b & 1) {
      f.cmask |= 1ull << g.sp[b];
      if (cval_bits >> b & 1) f.cval |= 1ull << g.sp[b];
    }
  f.kind = nt == 1 ? kOpU1 : kOpU2;
  for (int i = 0; i < nt; ++i) f.tq[i] = g.sp[tb[i]];
  const int dn = 1 << nt;
  f.mat.assign((size_t)dn * dn, cd(0));
  auto full = [&](int a) {  // target-subspace index -> gate index
    int j = cval_bits;
    for (int i = 0; i < nt; ++i)
      if (a >> i & 1) j |= 1 << tb[i];
    return j;
  };
  for (int a = 0; a < dn; ++a)
    for (int c = 0; c < dn; ++c) f.mat[(size_t)a * dn + c] = g.U[(size_t)full(a) * d + full(c)];
  return true;
}

// Restriction of a full sorted-order k-qubit matrix to the op's target subspace.
static std::vector<cd> restrict_to(const GateSpec& g, const FOp& f, const std::vector<cd>& D) {
  const int k = g.k, d = 1 << k;
  int cval_bits = 0, tb[2], nt = 0;
  for (int b = 0; b < k; ++b) {
    const uint64_t q = 1ull << g.sp[b];
    if (f.cmask & q) {
      if (f.cval & q) cval_bits |= 1 << b;
    } else {
      tb[nt++] = b;
    }
  }
  const int dn = 1 << nt;
  std::vector<cd> R((size_t)dn * dn);
  auto full = [&](int a) {
    int j = cval_bits;
    for (int i = 0; i < nt; ++i)
      if (a >> i & 1) j |= 1 << tb[i];
    return j;
  };
  for (int a = 0; a < dn; ++a)
    for (int c = 0; c < dn; ++c) R[(size_t)a * dn + c] = D[(size_t)full(a) * d + full(c)];
  return R;
}

static void mat2_mul(const std::vector<cd>& A, const std::vector<cd>& B, std::vector<cd>& C) {  // C = A B
  C.assign(4, cd(0));
  for (int r = 0; r < 2; ++r)
    for (int c = 0; c < 2; ++c) C[r * 2 + c] = A[r * 2] * B[c] + A[r * 2 + 1] * B[2 + c];
}
static std::vector<cd> mat2_dag(const std::vector<cd>& A) {
  return {std::conj(A[0]), std::conj(A[2]), std::conj(A[1]), std::conj(A[3])};
}

struct PlanStage {
  std::vector<int> rs;   // tile-bit indices (ascending)
  std::vector<int> ops;  // indices into PlanPass::ops
};
struct PlanPass {
  bool standalone = false;
  int gate = -1;                 // standalone: the caller's gate
  std::vector<int> tile_q;       // M global qubits, ascending
  std::vector<FOp> ops;
  std::vector<PlanStage> stages;
  int nslots = 0;
};

struct TileConfig {
  int M;      // tile bits
  int clow;   // always-resident low qubits
};

static TileConfig tile_config(int dtype, int n) {
  // 2^12 FP32 or 2^11 FP64 amplitudes per tile (32 KiB per state), smaller
  // tiles for smaller states; the lowest 4 (FP32) / 3 (FP64) qubits are always
  // tile qubits so that a tile is made of 128-byte runs (11-qubit FP32 tiles
  // for the reverse sweep measured slower: more passes at the same pass cost;
  // 3 always-resident FP32 qubits give 10 % fewer passes at 1.4x the reverse
  // pass time, 11.6 vs 12.6 gradients/s at n = 26)
  const int M = std::min(dtype == VQC_C64 ? 12 : 11, n);
  return {M, std::min(dtype == VQC_C64 ? 4 : 3, M)};
}
constexpr int kMinTileBits = 9;  // 32 threads x 16 amplitudes

// Greedy pass formation (see the file comment).  items are in execution order.
static void plan_passes(int n, const TileConfig& tc, bool adj, std::vector<PItem>& items, std::vector<PlanPass>& out) {
  const int M = tc.M;
  std::vector<char> done(items.size(), 0);
  size_t first = 0;
  while (true) {
    while (first < items.size() && done[first]) ++first;
    if (first >= items.size()) break;
    if (items[first].standalone) {
      PlanPass p;
      p.standalone = true;
      p.gate = items[first].gate;
      out.push_back(std::move(p));
      done[first] = 1;
      continue;
    }
    PlanPass p;
    uint64_t Q = 0;
    for (int q = 0; q < std::min(tc.clow, n); ++q) Q |= 1ull << q;
    uint64_t blocked = 0;
    std::vector<int> last_on(n, -1);  // last op index in p.ops touching qubit q
    for (size_t i = first; i < items.size(); ++i) {
      if (done[i]) continue;
      PItem& it = items[i];
      const uint64_t qs = it.op.qubits;
      if (it.standalone) {  // runs after this pass: its qubits stay blocked
        blocked |= qs;
        continue;
      }
      if (qs & blocked) {
        blocked |= qs;
        continue;
      }
      FOp& f = it.op;
      uint64_t need = 0;
      if (f.kind == kOpU1) need = 1ull << f.tq[0];
      if (f.kind == kOpU2) need = (1ull << f.tq[0]) | (1ull << f.tq[1]);
      const bool fits = popc64(Q | need) <= M;
      const bool slot_ok = (!(adj && f.acc) || p.nslots < kMaxSlots) && (int)p.ops.size() < kMaxOpsPerPass;
      if (!fits || !slot_ok) {
        blocked |= qs;
        continue;
      }
      Q |= need;
      done[i] = 1;
      // merge consecutive uncontrolled one-qubit ops on the same qubit
      if (f.kind == kOpU1 && f.cmask == 0) {
        const int prev = last_on[f.tq[0]];
        if (prev >= 0) {
          FOp& g = p.ops[prev];
          if (g.kind == kOpU1 && g.cmask == 0 && g.tq[0] == f.tq[0]) {
            // g applied first, then f: merged = f.mat * g.mat
            std::vector<cd> merged;
            mat2_mul(f.mat, g.mat, merged);
            if (adj) {
              // g's gradients were taken at g's output side = f's input: move them
              // to the block input (f is applied after g, so D -> F^dag D F)
              const std::vector<cd> Fd = mat2_dag(f.mat);
              for (PGrad& pg : g.grads) {
                std::vector<cd> t1, t2;
                // in the reverse sweep the op matrices are U^dagger: f.mat = U_f^dagger,
                // the block input lies after f, and D_g moves by conjugation with f.mat^dagger
                mat2_mul(pg.D, Fd, t1);
                mat2_mul(f.mat, t1, t2);
                pg.D = t2;
              }
              for (PGrad& pg : f.grads) g.grads.push_back(pg);
              if (f.acc && !g.acc) {
                g.acc = true;
                ++p.nslots;
              }
            }
            g.mat = merged;
            continue;
          }
        }
      }
      if (adj && f.acc) ++p.nslots;
      p.ops.push_back(f);
      for (int q = 0; q < n; ++q)
        if (qs >> q & 1) last_on[q] = (int)p.ops.size() - 1;
    }
    // fill the tile with the lowest remaining qubits
    for (int q = 0; q < n && popc64(Q) < M; ++q) Q |= 1ull << q;
    for (int q = 0; q < n; ++q)
      if (Q >> q & 1) p.tile_q.push_back(q);
    out.push_back(std::move(p));
  }
}

// Conflict check of a register-bit set for the shared-memory swizzle.
// FP64: 16-byte amplitudes, quarter-warps over the tile swizzle Swz<double>;
// FP32: 8-byte amplitudes, half-warps over Swz<float>.  Packed FP32: 16-byte
// pairs, the lowest three thread bits (tile bits outside rs, ascending) must
// fall in distinct classes of the pair swizzle, class = (tile bit - 1) mod 3.
static bool rs_conflict_free(const std::vector<int>& rs, int M, int dtype, bool packed) {
  if (packed) {
    int seen = 0, k = 0;
    for (int b = 1; b < M && k < 3; ++b) {
      if (std::find(rs.begin(), rs.end(), b) != rs.end()) continue;
      const int res = (b - 1) % 3;
      if (seen >> res & 1) return false;
      seen |= 1 << res;
      ++k;
    }
    return true;
  }
  std::vector<int> lanes;
  for (int b = 0; b < M && (int)lanes.size() < (dtype == VQC_C64 ? 4 : 3); ++b)
    if (std::find(rs.begin(), rs.end(), b) == rs.end()) lanes.push_back(b);
  int seen = 0;
  for (int b : lanes) {
    int res;
    if (dtype == VQC_C64)
      res = b < 4 ? b : (b < 8 ? b - 4 : -1);
    else
      res = b < 3 ? b : (b < 9 ? (b - 3) % 3 : -1);
    if (res < 0 || (seen >> res & 1)) return false;
    seen |= 1 << res;
  }
  return true;
}

// Cuts a pass into stages: runs of ops whose target bits fit the register
// set (4 tile bits; for FP32 tile bit 0 is always one of them, the lane bit
// of the packed layout).  The free bits left over are filled preferring the
// stage's control bits (register controls are compile-time cases in the FP32
// body), then a bank-conflict-free layout.
static void plan_stages(PlanPass& p, int M, int dtype, bool packed, int rb = kRegBits) {
  const bool lane0 = packed;
  p.stages.clear();
  std::map<int, int> tbit;  // global qubit -> tile bit
  for (int b = 0; b < (int)p.tile_q.size(); ++b) tbit[p.tile_q[b]] = b;
  std::vector<int> pending(p.ops.size());
  for (size_t i = 0; i < pending.size(); ++i) pending[i] = (int)i;
  while (!pending.empty()) {
    PlanStage st;
    uint64_t blocked = 0;
    std::vector<int> rest;
    std::vector<int> rs;
    if (lane0) rs.push_back(0);
    for (int oi : pending) {
      const FOp& f = p.ops[oi];
      if (f.qubits & blocked) {
        blocked |= f.qubits;
        rest.push_back(oi);
        continue;
      }
      std::vector<int> need;
      if (f.kind == kOpU1) need = {tbit[f.tq[0]]};
      if (f.kind == kOpU2) need = {tbit[f.tq[0]], tbit[f.tq[1]]};
      std::vector<int> u = rs;
      for (int b : need)
        if (std::find(u.begin(), u.end(), b) == u.end()) u.push_back(b);
      if ((int)u.size() <= rb) {
        rs = u;
        st.ops.push_back(oi);
      } else {
        blocked |= f.qubits;
        rest.push_back(oi);
      }
    }
    // fill the register set to 4 bits: control bits of the stage's ops first
    std::vector<int> cand;
    for (int oi : st.ops) {
      const FOp& f = p.ops[oi];
      for (int q = 0; q < 64; ++q)
        if ((f.cmask >> q & 1) && tbit.count(q)) {
          const int b = tbit[q];
          if (std::find(rs.begin(), rs.end(), b) == rs.end() && std::find(cand.begin(), cand.end(), b) == cand.end())
            cand.push_back(b);
        }
    }
    for (int b = 0; b < M; ++b)
      if (std::find(rs.begin(), rs.end(), b) == rs.end() && std::find(cand.begin(), cand.end(), b) == cand.end())
        cand.push_back(b);
    const int need_more = rb - (int)rs.size();
    std::vector<int> best;
    bool found = false;
    const int nc = std::min((int)cand.size(), 10);
    for (int mask = 0; mask < (1 << nc) && !found; ++mask) {
      if (popc64((uint64_t)mask) != need_more) continue;
      std::vector<int> t = rs;
      for (int i = 0; i < nc; ++i)
        if (mask >> i & 1) t.push_back(cand[i]);
      std::sort(t.begin(), t.end());
      if (best.empty()) best = t;
      if (rs_conflict_free(t, M, dtype, packed)) {
        best = t;
        found = true;
      }
    }
    if (!found) prof_note("plan_stages_bank_conflicted", 1);
    st.rs = best;
    p.stages.push_back(st);
    pending = rest;
  }
}

// ----------------------------------------------------------------------------- execution
struct Device {
  std::vector<unsigned char> buf;
  template <class T>
  size_t put(const T* p, size_t n) {
    size_t off = (buf.size() + 15) & ~size_t(15);
    buf.resize(off + sizeof(T) * n);
    std::memcpy(buf.data() + off, p, sizeof(T) * n);
    return off;
  }
};

template <class R, int M, bool ADJ>
static size_t pass_smem(const PassShape& ps) {
  constexpr int NT = 1 << (M - kRegBits);
  const size_t npool = (size_t)ps.npool * sizeof(cplx<R>);
  return tile_bytes<R, M, ADJ>() + (ADJ ? (size_t)ps.nslots * (NT / 32) * 8 * sizeof(double) : 0) +
         (ps.packed ? sizeof(DevStageF) : sizeof(DevStage)) * ps.nstages + sizeof(DevOp) * ps.nops +
         ((npool + 15) & ~size_t(15));
}

// The tile kernel of a pass shape.
template <class R, int M, bool ADJ>
static auto tile_kernel(const PassShape& ps) -> decltype(&k_tile<R, M, ADJ, true, false>) {
  if constexpr (std::is_same<R, float>::value)
    if (ps.packed) return ps.general ? k_tile<R, M, ADJ, true, true> : k_tile<R, M, ADJ, false, true>;
  return ps.general ? k_tile<R, M, ADJ, true, false> : k_tile<R, M, ADJ, false, false>;
}

template <class R, int M, bool ADJ>
static int tile_grid(int device, const PassShape& ps) {
  constexpr int NT = 1 << (M - kRegBits);
  const size_t smem = pass_smem<R, M, ADJ>(ps);
  auto kfun = tile_kernel<R, M, ADJ>(ps);
  cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfun, NT, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
  return device_info(device).sms * per_sm;
}

template <class R, int M, bool ADJ>
static int launch_tile(vqc_state h, void* psi, void* lam, const DevPass* dp, const void* ds, const DevOp* dops,
                       const void* pool, double* partials, int grid, const PassShape& ps, double flops) {
  constexpr int NT = 1 << (M - kRegBits);
  const size_t smem = pass_smem<R, M, ADJ>(ps);
  auto kfun = tile_kernel<R, M, ADJ>(ps);
  VQC_CK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024)));
  ProfScope prof(h->stream, ADJ ? "tile_adjoint" : "tile_forward",
                 (double)(ADJ ? 4 : 2) * h->size() * sizeof(cplx<R>), flops);
  kfun<<<grid, NT, smem, h->stream>>>((cplx<R>*)psi, (cplx<R>*)lam, dp, ds, dops, (const cplx<R>*)pool, partials);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

int standalone_adjoint(vqc_state h, void* lam, void* y, const GateSpec& gs, bool acc, double* out);

// The structure class of a one-qubit matrix (exact zeros: the matrices are
// built from closed forms, so structural zeros are exact).
static int u1_form(const std::vector<cd>& m) {
  const cd u00 = m[0], u01 = m[1], u10 = m[2], u11 = m[3];
  if (u00 == cd(0) && u11 == cd(0) && u01 == cd(1) && u10 == cd(1)) return kFormSwap;
  if (u01 == cd(0) && u10 == cd(0)) return kFormDiag;
  if (u00.imag() == 0 && u01.imag() == 0 && u10.imag() == 0 && u11.imag() == 0) return kFormReal;
  if (u00.imag() == 0 && u11.imag() == 0 && u01.real() == 0 && u10.real() == 0) return kFormRI;
  return kFormGen;
}

// Which entries of the reduced matrix the op's parameters need.
static int acc_kind(const FOp& f) {
  bool diag = false, off = false;
  for (const PGrad& pg : f.grads) {
    if (pg.D.size() < 4) return kAccFull;
    if (pg.D[0] != cd(0) || pg.D[3] != cd(0)) diag = true;
    if (pg.D[1] != cd(0) || pg.D[2] != cd(0)) off = true;
  }
  if (diag && !off) return kAccDiag;
  if (off && !diag) return kAccOff;
  return kAccFull;
}
// Every D of the op anti-Hermitian (as U^dagger dU/dtheta of a unitary family
// is): the FP32 body then accumulates the four-value projection (kAccAH).
static bool acc_anti_hermitian(const FOp& f) {
  for (const PGrad& pg : f.grads) {
    if (pg.D.size() != 4) return false;
    double scale = 0;
    for (const cd& d : pg.D) scale = std::max(scale, std::abs(d));
    const double eps = 1e-12 * scale;
    if (std::abs(pg.D[0].real()) > eps || std::abs(pg.D[3].real()) > eps ||
        std::abs(pg.D[1] + std::conj(pg.D[2])) > eps)
      return false;
  }
  return !f.grads.empty();
}

// FMA-pipe lane operations (fused multiply-adds, multiplies, adds) of one pass
// over the whole state of n qubits, as the tile bodies implement its ops: a
// one-qubit op costs per amplitude pair and state 16 (general form), 8
// (RX-like, real, diagonal) or 0 (swap), and in the reverse sweep its
// reduced-matrix accumulation 16 / 8 per pair (12 / 8 / 4 for the FP32
// anti-Hermitian projection); a two-qubit op 64 per amplitude quad and state;
// a diagonal op 4 per amplitude and state (6 more for its accumulation).
// Controls scale by the fraction of amplitudes they enable.  The classic body
// runs every forward one-qubit op in the general form, and in the reverse
// sweep the RX-like form or the general one.  The numerator of the compute
// roofline (vqc_fma_peak is the denominator).
static double pass_fma_ops(const PlanPass& p, int n, bool adj, bool packed) {
  const double pairs = std::ldexp(1.0, n - 1), amps = std::ldexp(1.0, n);
  const int nst = adj ? 2 : 1;
  static const int per_pair[5] = {16, 8, 8, 8, 0};  // by kForm*
  double ops = 0;
  for (const FOp& f : p.ops) {
    const double act = std::ldexp(1.0, -popc64(f.cmask));
    if (f.kind == kOpU1) {
      int form = u1_form(f.mat);
      if (!packed) form = adj ? (form == kFormRI ? kFormRI : kFormGen) : kFormGen;
      double o = (double)per_pair[form] * nst;
      if (adj && f.acc) {
        const int k = acc_kind(f);
        if (packed && acc_anti_hermitian(f))
          o += k == kAccFull ? 12 : (k == kAccOff ? 8 : 4);
        else
          o += k == kAccFull ? 16 : 8;
      }
      ops += o * pairs * act;
    } else if (f.kind == kOpU2) {
      ops += 64.0 * nst * (amps / 4) * act;
    } else if (f.kind == kOpDiag) {
      ops += 4.0 * nst * amps + (adj && f.acc ? 6.0 * amps : 0.0);
    }
  }
  return ops;
}

// One stage of the FP32 (packed) tile body: its DevStageF tables, its ops
// (j-bit targets, register controls as compile-time cases or a mask, the
// coefficient layouts of tile_f32.cuh) and their pool blocks.
static void stage_f32(const PlanPass& p, const PlanStage& st, int M, int n, uint64_t tile_mask,
                      std::map<int, int>& tbit, bool adj, int& slot, int row, std::vector<DevStageF>& ds,
                      std::vector<DevOp>& dops, std::vector<float2>& pool, size_t pool_begin,
                      std::vector<AccRef>* accs, int rb) {
  DevStageF s{};
  const std::vector<int>& rs = st.rs;  // ascending, rs[0] = tile bit 0
  const int na = 1 << rb, np = na / 2;  // register amplitudes, pairs
  uint32_t rsmask = 0;
  for (int b : rs) rsmask |= 1u << b;
  uint32_t dep[32];
  for (int j = 0; j < na; ++j) {
    uint32_t t = 0;
    for (int i = 0; i < rb; ++i)
      if (j >> i & 1) t |= 1u << rs[i];
    dep[j] = t;
    s.dep[j] = t;
  }
  std::vector<int> thr;
  for (int b = 0; b < M; ++b)
    if (!(rsmask >> b & 1)) thr.push_back(b);
  auto gq = [&](uint32_t t) {
    int64_t g = 0;
    for (int b = 0; b < M; ++b)
      if (t >> b & 1) g |= int64_t(1) << p.tile_q[b];
    return g;
  };
  for (int k = 0; k < 2; ++k)
    for (int nib = 0; nib < 16; ++nib) {
      uint32_t t = 0;
      for (int i = 0; i < 4; ++i)
        if ((nib >> i & 1) && 4 * k + i < (int)thr.size()) t |= 1u << thr[4 * k + i];
      s.thr[k][nib] = t;
      s.swt[k][nib] = f32t::swz_pair(t >> 1);
      s.gthr[k][nib] = gq(t);
    }
  for (int m = 0; m < np; ++m) {
    s.swm[m] = f32t::swz_pair(dep[2 * m] >> 1);
    s.gdep[m] = gq(dep[2 * m]);
  }
  auto jbit = [&](int b) { return (int)(std::find(rs.begin(), rs.end(), b) - rs.begin()); };
  auto put = [&](double a, double b) { pool.push_back(make_float2((float)a, (float)b)); };
  auto dup = [&](double a) { put(a, a); };
  s.op_begin = (int)dops.size();
  for (int oi : st.ops) {
    const FOp& f = p.ops[oi];
    DevOp o{};
    o.code = f.kind;
    o.slot = -1;
    std::vector<std::pair<int, int>> rc;  // register controls: (j-bit, value)
    for (int q = 0; q < n; ++q) {
      if (!(f.cmask >> q & 1)) continue;
      const int v = (int)(f.cval >> q & 1);
      if (tile_mask >> q & 1) {
        const int b = tbit[q];
        if (rsmask >> b & 1) {
          rc.push_back({jbit(b), v});
        } else {
          o.cmask |= 1u << b;
          if (v) o.cval |= 1u << b;
        }
      } else {
        o.gmask |= 1ull << q;
        if (v) o.gval |= 1ull << q;
      }
    }
    uint32_t rmask = 0;
    for (int j = 0; j < na; ++j) {
      bool ok = true;
      for (auto& c : rc) ok = ok && ((j >> c.first & 1) == c.second);
      if (ok) rmask |= 1u << j;
    }
    o.rmask = (int32_t)rmask;
    int rctl = 0;
    if (!rc.empty()) rctl = (rc.size() == 1 && rc[0].second == 1) ? rc[0].first + 1 : 7;
    if (o.cmask) o.code |= kCodeCtl;
    if (o.gmask) o.code |= kCodeGCtl;
    while (pool.size() % 2) put(0, 0);  // each op's block starts on 16 bytes
    o.mat = (int)(pool.size() - pool_begin);
    if (f.kind == kOpU1) {
      const int tb = jbit(tbit[f.tq[0]]), form = u1_form(f.mat);
      o.code |= op_r_bits(tb, 0) | (form << 11) | (rctl << 16);
      if (adj && f.acc) o.code |= (acc_kind(f) << 14) | (acc_anti_hermitian(f) ? kCodeAH : 0);
      const cd u00 = f.mat[0], u01 = f.mat[1], u10 = f.mat[2], u11 = f.mat[3];
      if (tb != 0) {
        switch (form) {
          case kFormGen:
            for (const cd& u : {u00, u01, u10, u11}) {
              dup(u.real());
              dup(u.imag());
              dup(-u.imag());
            }
            break;
          case kFormRI:
            dup(u00.real()), dup(u01.imag()), dup(-u01.imag()), dup(u11.real()), dup(u10.imag()), dup(-u10.imag());
            break;
          case kFormReal: dup(u00.real()), dup(u01.real()), dup(u10.real()), dup(u11.real()); break;
          case kFormDiag:
            dup(u00.real()), dup(u00.imag()), dup(-u00.imag()), dup(u11.real()), dup(u11.imag()), dup(-u11.imag());
            break;
          default: break;
        }
      } else {
        switch (form) {
          case kFormGen:
            put(u00.real(), u11.real()), put(u01.real(), u10.real()), put(u00.imag(), u11.imag());
            put(-u00.imag(), -u11.imag()), put(u01.imag(), u10.imag()), put(-u01.imag(), -u10.imag());
            break;
          case kFormRI: put(u00.real(), u11.real()), put(-u01.imag(), -u10.imag()), put(u01.imag(), u10.imag()); break;
          case kFormReal: put(u00.real(), u11.real()), put(u01.real(), u10.real()); break;
          case kFormDiag:
            put(u00.real(), u11.real()), put(u00.imag(), u11.imag()), put(-u00.imag(), -u11.imag());
            break;
          default: break;
        }
      }
    } else {
      if (f.kind == kOpU2) o.code |= op_r_bits(jbit(tbit[f.tq[0]]), jbit(tbit[f.tq[1]]));
      for (const cd& c : f.mat) put(c.real(), c.imag());
    }
    o.nd = f.nd;
    for (int i = 0; i < 5; ++i) {
      o.dbit[i] = -1;
      o.dglob[i] = 0;
      if (i < f.nd) {
        if (tile_mask >> f.dq[i] & 1)
          o.dbit[i] = tbit[f.dq[i]];
        else
          o.dglob[i] = f.dq[i];
      }
    }
    if (adj && f.acc) {
      o.slot = slot++;
      if (f.kind == kOpDiag) {
        // the accumulation runs as its own op right after the diagonal
        dops.push_back(o);
        DevOp a = o;
        a.code = (a.code & ~15) | kOpAccD;
        dops.push_back(a);
        if (accs) accs->push_back(AccRef{row + o.slot, f});
        continue;
      }
      if (accs) accs->push_back(AccRef{row + o.slot, f, (o.code & kCodeAH) != 0});
      o.code |= kCodeAcc;
    }
    dops.push_back(o);
  }
  s.op_end = (int)dops.size();
  ds.push_back(s);
}

template <class R, int M, bool ADJ>
static void serialize_plan(int n, int dtype, std::vector<PlanPass>& passes, SerialPlan& sp, std::vector<AccRef>* accs,
                           bool packed = false, int rb = kRegBits) {
  Device d;
  std::vector<cplx<R>> pool;
  std::vector<PassLoc>& locs = sp.locs;
  locs.assign(passes.size(), PassLoc());
  int row = 0;
  for (size_t pi = 0; pi < passes.size(); ++pi) {
    PlanPass& p = passes[pi];
    if (p.standalone) {
      locs[pi].standalone = true;
      locs[pi].gate = p.gate;
      continue;
    }
    plan_stages(p, M, dtype, packed, rb);
    std::vector<DevStage> ds;
    std::vector<DevOp> dops;
    std::map<int, int> tbit;
    for (int b = 0; b < M; ++b) tbit[p.tile_q[b]] = b;
    uint64_t tile_mask = 0;
    for (int q : p.tile_q) tile_mask |= 1ull << q;
    int slot = 0;
    while ((pool.size() * sizeof(cplx<R>)) % 16) pool.push_back(mkc<R>(R(0), R(0)));
    const size_t pool_begin = pool.size();
    std::vector<DevStageF> dsf;
    for (const PlanStage& st : p.stages) {
      if constexpr (std::is_same<R, float>::value) {
        if (packed) {
          stage_f32(p, st, M, n, tile_mask, tbit, ADJ, slot, row, dsf, dops, pool, pool_begin, accs, rb);
          continue;
        }
      }
      DevStage s{};
      uint32_t rsmask = 0;
      for (int b : st.rs) rsmask |= 1u << b;
      for (int j = 0; j < 16; ++j) {
        uint32_t t = 0;
        for (int i = 0; i < kRegBits; ++i)
          if (j >> i & 1) t |= 1u << st.rs[i];
        s.dep[j] = t;
      }
      s.thr_mask = ((1u << M) - 1) & ~rsmask;
      s.gthr_mask = 0;
      for (int b = 0; b < M; ++b)
        if (s.thr_mask >> b & 1) s.gthr_mask |= 1ull << p.tile_q[b];
      for (int j = 0; j < 16; ++j) {
        int64_t g = 0;
        for (int b = 0; b < M; ++b)
          if (s.dep[j] >> b & 1) g |= int64_t(1) << p.tile_q[b];
        s.gdep[j] = g;
      }
      s.op_begin = (int)dops.size();
      for (int oi : st.ops) {
        const FOp& f = p.ops[oi];
        DevOp o{};
        o.code = f.kind;
        o.slot = -1;
        auto slot_of = [&](int b) { return (int)(std::find(st.rs.begin(), st.rs.end(), b) - st.rs.begin()); };
        if (f.kind == kOpU1) {
          o.code |= slot_of(tbit[f.tq[0]]) << 4;
          o.code |= u1_form(f.mat) << 11;
          if (ADJ && f.acc) o.code |= acc_kind(f) << 14;
        }
        if (f.kind == kOpU2) o.code |= (slot_of(tbit[f.tq[0]]) << 4) | (slot_of(tbit[f.tq[1]]) << 6);
        for (int q = 0; q < n; ++q) {
          if (!(f.cmask >> q & 1)) continue;
          const bool v = f.cval >> q & 1;
          if (tile_mask >> q & 1) {
            o.cmask |= 1u << tbit[q];
            if (v) o.cval |= 1u << tbit[q];
          } else {
            o.gmask |= 1ull << q;
            if (v) o.gval |= 1ull << q;
          }
        }
        if (o.cmask) o.code |= kCodeCtl;
        if (o.gmask) o.code |= kCodeGCtl;
        o.mat = (int)(pool.size() - pool_begin);
        for (const cd& c : f.mat) pool.push_back(mkc<R>((R)c.real(), (R)c.imag()));
        o.nd = f.nd;
        for (int i = 0; i < 5; ++i) {
          o.dbit[i] = -1;
          o.dglob[i] = 0;
          if (i < f.nd) {
            if (tile_mask >> f.dq[i] & 1)
              o.dbit[i] = tbit[f.dq[i]];
            else
              o.dglob[i] = f.dq[i];
          }
        }
        if (ADJ && f.acc) {
          o.slot = slot++;
          if (f.kind == kOpDiag) {
            // the accumulation runs as its own op right after the diagonal
            dops.push_back(o);
            DevOp a = o;
            a.code = (a.code & ~15) | kOpAccD;
            dops.push_back(a);
            if (accs) accs->push_back(AccRef{row + o.slot, f});
            continue;
          }
          if (accs) accs->push_back(AccRef{row + o.slot, f});
          o.code |= kCodeAcc;
        }
        dops.push_back(o);
      }
      s.op_end = (int)dops.size();
      ds.push_back(s);
    }
    p.nslots = slot;
    DevPass P{};
    P.nontile_mask = ((n >= 64) ? ~0ull : ((1ull << n) - 1)) & ~tile_mask;
    P.ntiles = int64_t(1) << (n - M);
    locs[pi].ntiles = P.ntiles;
    P.nslots = slot;
    P.nops = (int)dops.size();
    P.npool = (int)(pool.size() - pool_begin);
    locs[pi].pool_begin = pool_begin;
    locs[pi].shape.nslots = ADJ ? slot : 0;
    locs[pi].shape.nstages = (int)p.stages.size();
    locs[pi].shape.nops = P.nops;
    locs[pi].shape.npool = P.npool;
    locs[pi].shape.general = false;
    for (const DevOp& o : dops)
      if ((o.code & 15) != kOpU1) locs[pi].shape.general = true;
    locs[pi].row0 = row;
    row += slot;
    locs[pi].nslots = slot;
    locs[pi].fma_ops = pass_fma_ops(p, n, ADJ, packed);
    // stage indices are local to this pass's stage array
    P.stage_begin = 0;
    P.stage_end = (int)p.stages.size();
    locs[pi].pass = d.put(&P, 1);
    if (packed)
      locs[pi].stages = d.put(dsf.data(), dsf.size());
    else
      locs[pi].stages = d.put(ds.data(), ds.size());
    locs[pi].shape.packed = packed;
    // op indices in stages are local to this pass's op array
    locs[pi].ops = d.put(dops.data(), std::max<size_t>(dops.size(), 1));
  }
  for (int i = 0; i < 4; ++i) pool.push_back(mkc<R>(R(0), R(0)));  // the staging copy reads whole 16-byte words
  sp.pool_off = d.put(pool.data(), pool.size());
  sp.rows = row;
  sp.buf.swap(d.buf);
}

static void note_plan(bool adj, const std::vector<PlanPass>& passes) {
  long long np = 0, ns = 0, no = 0, nsa = 0;
  for (auto& p : passes) {
    if (p.standalone) {
      ++nsa;
      continue;
    }
    ++np;
    ns += (long long)p.stages.size();
    no += (long long)p.ops.size();
  }
  prof_note(adj ? "plan_adjoint_passes" : "plan_forward_passes", np);
  prof_note(adj ? "plan_adjoint_stages" : "plan_forward_stages", ns);
  prof_note(adj ? "plan_adjoint_ops" : "plan_forward_ops", no);
  prof_note("plan_standalone_gates", nsa);
}

template <int M, bool ADJ>
static int jit_grid(int device, const void* k, const PassShape& ps, int rb = kRegBits) {
  const int NT = 1 << (M - rb);
  const size_t smem = pass_smem<float, M, ADJ>(ps) + jit_extra_smem(ADJ, M, rb);
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, NT, smem) != cudaSuccess || per_sm < 1) {
    cudaGetLastError();
    per_sm = 1;
  }
  return device_info(device).sms * per_sm;
}

template <int M, bool ADJ>
static int launch_tile_jit(vqc_state h, const void* k, void* psi, void* lam, const DevPass* dp, const void* ds,
                           const DevOp* dops, const void* pool, double* partials, int grid, const PassShape& ps,
                           const void* host_pool, double flops, int rb = kRegBits) {
  const int NT = 1 << (M - rb);
  const size_t smem = pass_smem<float, M, ADJ>(ps) + jit_extra_smem(ADJ, M, rb);
  VQC_CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024)));
  ProfScope prof(h->stream, ADJ ? "tile_adjoint" : "tile_forward", (double)(ADJ ? 4 : 2) * h->size() * sizeof(float2),
                 flops);
  // the last parameter is the pass's matrix pool by value (host copy)
  void* args[] = {&psi, &lam, (void*)&dp, (void*)&ds, (void*)&dops, (void*)&pool, &partials, const_cast<void*>(host_pool)};
  VQC_CK(cudaLaunchKernel(k, dim3(grid), dim3(NT), args, smem, h->stream));
  return VQC_OK;
}

// JIT tile passes for FP32 states of at least 2^18 amplitudes (VQC_JIT=auto),
// all FP32 tile passes (on), none (off).
static bool use_jit(const vqc_state h) {
  const int mode = jit_mode();
  return h->dtype == VQC_C64 && (mode == 1 || (mode == 2 && h->nq >= 18)) && jit_available();
}
// The packed FP32 plan layout: for the compiled passes, or forced with
// VQC_JIT=interp (the packed interpreter, the compiled kernels' fallback).
static bool use_packed(const vqc_state h) { return h->dtype == VQC_C64 && (use_jit(h) || jit_mode() == 3); }
// VQC_JIT_WIDE=1: compiled forward passes with 32 amplitudes per thread (four
// free register bits per stage: 3.0 instead of 3.8 stages per pass on the
// headline circuit).  Off by default: measured slower at 2^26 amplitudes
// (0.40 against 0.355 ms per pass: five 128-thread CTAs per SM at 96
// registers, with spills), and NVRTC takes 15-140 s per such pass (1-2 s at
// 16 amplitudes), in its optimizer, not in ptxas.
static bool wide_forward() {
  const char* v = std::getenv("VQC_JIT_WIDE");
  return v && *v && std::atoi(v) != 0;
}

// An upper bound of one pass's serialised bytes (serialize_plan): at most one
// stage per op, two op records per op, 32 matrix entries (+ alignment) per op.
template <class R>
static size_t op_bytes_bound(const PlanPass& p) {
  const size_t nops = p.ops.size() + 1;
  return 3 * 16 + sizeof(DevPass) + nops * std::max(sizeof(DevStageF), sizeof(DevStage)) + 2 * nops * sizeof(DevOp) +
         (34 * nops + 8) * sizeof(cplx<R>);
}

// op_used != nullptr: the pass descriptors go to the op buffer at op_off
// (reserved by the caller) and *op_used receives their size, so that later
// chunks of one sweep can be uploaded while these passes run.
template <class R, int M, bool ADJ>
static int run_plan(vqc_state h, void* psi, void* lam, std::vector<PlanPass>& passes, const std::vector<GateSpec>& specs,
                    std::vector<AccRef>* accs, double* rows_dev, size_t op_off = 0, size_t* op_used = nullptr) {
  const int n = h->nq;
  SerialPlan sp;
  const bool packed = use_packed(h);
  // wide compiled forward passes (VQC_JIT_WIDE=1): 32 amplitudes per thread,
  // four free register bits per stage; the generic kernels take 16
  int rb = (!ADJ && packed && use_jit(h) && wide_forward()) ? kWideRegBits : kRegBits;
  const size_t accs0 = accs ? accs->size() : 0;
  serialize_plan<R, M, ADJ>(n, h->dtype, passes, sp, accs, packed, rb);
  note_plan(ADJ, passes);
  // run-time specialised kernels (FP32), one per pass structure
  std::vector<const void*> jk(passes.size(), nullptr);
  if constexpr (std::is_same<R, float>::value) {
    if (packed && use_jit(h)) {
      auto compile = [&]() {
        std::vector<JitPassRef> refs(passes.size());
        for (size_t pi = 0; pi < passes.size(); ++pi)
          if (!sp.locs[pi].standalone)
            refs[pi] = JitPassRef{(const DevStageF*)(sp.buf.data() + sp.locs[pi].stages), sp.locs[pi].shape.nstages,
                                  (const DevOp*)(sp.buf.data() + sp.locs[pi].ops), sp.locs[pi].shape.npool};
        jit_pass_kernels(M, ADJ, refs, jk, false, true, rb);
      };
      compile();
      if (rb != kRegBits) {
        // a wide pass without a kernel (beyond the parameter space, or a failed
        // compile) has no generic kernel: plan the whole sweep at 16 amplitudes
        bool missing = false;
        for (size_t pi = 0; pi < passes.size(); ++pi) missing = missing || (!sp.locs[pi].standalone && !jk[pi]);
        if (missing) {
          rb = kRegBits;
          sp = SerialPlan();
          if (accs) accs->resize(accs0);
          serialize_plan<R, M, ADJ>(n, h->dtype, passes, sp, accs, packed, rb);
          jk.assign(passes.size(), nullptr);
          compile();
        }
      }
    }
  }
  const std::vector<PassLoc>& locs = sp.locs;
  const size_t pool_off = sp.pool_off;
  std::vector<int> grids(passes.size(), 0);
  for (size_t pi = 0; pi < passes.size(); ++pi) {
    if (locs[pi].standalone) continue;
    int g = 0;
    if constexpr (std::is_same<R, float>::value)
      if (jk[pi]) g = jit_grid<M, ADJ>(h->device, jk[pi], locs[pi].shape, rb);
    if (!g) g = tile_grid<R, M, ADJ>(h->device, locs[pi].shape);
    grids[pi] = (int)std::min<int64_t>(g, locs[pi].ntiles);
  }
  // partial sums scratch: one row of 8 doubles per (CTA, slot) of every pass,
  // summed over the CTAs by one launch after the sweep (the same fixed order
  // per slot as a reduction after each pass)
  std::vector<size_t> poff(passes.size(), 0);
  size_t need = 0;
  int max_slots = 0;
  for (size_t pi = 0; pi < passes.size(); ++pi)
    if (!locs[pi].standalone && locs[pi].nslots > 0) {
      poff[pi] = need / sizeof(double);
      need += (size_t)grids[pi] * locs[pi].nslots * 8 * sizeof(double);
      max_slots = std::max(max_slots, locs[pi].nslots);
    }
  double* partials = nullptr;
  if (ADJ && need > 0) {
    if (need > h->fused_scratch_bytes) {
      if (h->fused_scratch) {
        VQC_CK(cudaStreamSynchronize(h->stream));
        VQC_CK(cudaFree(h->fused_scratch));
        h->fused_scratch = nullptr;
      }
      VQC_CK(cudaMalloc(&h->fused_scratch, need));
      h->fused_scratch_bytes = need;
    }
    partials = (double*)h->fused_scratch;
  }
  // the reduction items travel with the pass descriptors
  size_t red_off = 0, nred = 0;
  if (ADJ && need > 0) {
    std::vector<RedItem> red;
    for (size_t pi = 0; pi < passes.size(); ++pi)
      if (!locs[pi].standalone && locs[pi].nslots > 0)
        red.push_back(RedItem{partials + poff[pi], grids[pi], locs[pi].nslots, rows_dev + (size_t)locs[pi].row0 * 8});
    red_off = (sp.buf.size() + 15) & ~size_t(15);
    nred = red.size();
    sp.buf.resize(red_off + sizeof(RedItem) * nred);
    std::memcpy(sp.buf.data() + red_off, red.data(), sizeof(RedItem) * nred);
  }
  int rc = op_used ? upload_ops_at(h, op_off, sp.buf.data(), sp.buf.size()) : upload_ops(h, sp.buf.data(), sp.buf.size());
  if (rc) return rc;
  if (op_used) *op_used = sp.buf.size();
  const unsigned char* base = (const unsigned char*)h->opbuf + op_off;
  for (size_t pi = 0; pi < passes.size(); ++pi) {
    if (locs[pi].standalone) {
      const GateSpec& gs = specs[locs[pi].gate];
      if (ADJ) {
        if ((rc = standalone_adjoint(h, lam, psi, gs, false, nullptr))) return rc;
      } else {
        if ((rc = launch_gate(gs, psi, n, h->dtype, h->device, h->stream))) return rc;
      }
      continue;
    }
    const int grid = grids[pi];
    double* pp = partials ? partials + poff[pi] : nullptr;
    const DevPass* dp = (const DevPass*)(base + locs[pi].pass);
    const void* ds = (const void*)(base + locs[pi].stages);
    const DevOp* dops = (const DevOp*)(base + locs[pi].ops);
    const void* dpool = base + pool_off + locs[pi].pool_begin * sizeof(cplx<R>);
    if (jk[pi]) {
      if constexpr (std::is_same<R, float>::value)
        if ((rc = launch_tile_jit<M, ADJ>(h, jk[pi], psi, lam, dp, ds, dops, dpool, pp, grid,
                                          locs[pi].shape,
                                          sp.buf.data() + pool_off + locs[pi].pool_begin * sizeof(float2),
                                          2.0 * locs[pi].fma_ops, rb)))
          return rc;
    } else if ((rc = launch_tile<R, M, ADJ>(h, psi, lam, dp, ds, dops, dpool, pp, grid, locs[pi].shape,
                                            2.0 * locs[pi].fma_ops))) {
      return rc;
    }
  }
  if (nred > 0) {
    k_reduce_slots_batch<<<dim3(max_slots, (unsigned)nred), 256, 0, h->stream>>>((const RedItem*)(base + red_off));
    VQC_CK(cudaGetLastError());
  }
  return VQC_OK;
}

int fused_supported(vqc_state h) { return h->nq >= kMinTileBits && h->nq <= 40; }

template <class R, int M>
static int forward_impl(vqc_state h, const vqc_gate* gates, int ngates, const double* mats) {
  std::vector<GateSpec> specs(ngates);
  std::vector<PItem> items(ngates);
  // gate analysis, on up to four host threads for long circuits (it precedes
  // the first launch: the device waits for it)
  auto analyze = [&](int i0, int i1) {
    for (int i = i0; i < i1; ++i) {
      if (analyze_gate(h->nq, gates[i].nq, gates[i].pos, mats + gates[i].mat, false, specs[i])) return i;
      items[i].gate = i;
      items[i].standalone = !to_fop(specs[i], items[i].op);
    }
    return -1;
  };
  const int nth = ngates >= 1024 ? (int)std::min(4u, std::max(1u, std::thread::hardware_concurrency())) : 1;
  std::vector<int> bad(nth, -1);
  std::vector<std::thread> pool;
  for (int t = 1; t < nth; ++t)
    pool.emplace_back([&, t] { bad[t] = analyze((int)((int64_t)ngates * t / nth), (int)((int64_t)ngates * (t + 1) / nth)); });
  bad[0] = analyze(0, (int)((int64_t)ngates / nth));
  for (auto& th : pool) th.join();
  for (int t = 0; t < nth; ++t)
    if (bad[t] >= 0)  // again on this thread, for its error message
      return analyze_gate(h->nq, gates[bad[t]].nq, gates[bad[t]].pos, mats + gates[bad[t]].mat, false, specs[bad[t]]);
  std::vector<PlanPass> passes;
  plan_passes(h->nq, tile_config(h->dtype, h->nq), false, items, passes);
  const char* pc = std::getenv("VQC_PLAN_CHUNKS");  // 0: one serialisation for the whole sweep
  if (passes.size() < 4 || (pc && *pc && std::atoi(pc) == 0))
    return run_plan<R, M, false>(h, h->d, nullptr, passes, specs, nullptr, nullptr);
  // Serialised and launched in chunks of 1, 2, 4, ... passes: the host plans
  // the next chunk while the device runs the previous ones, instead of the
  // device waiting for the whole sweep's descriptors (about 1.5 ms for 2,000
  // gates).  Each chunk's descriptors get their own region of the op buffer.
  size_t bound = 256;
  for (const PlanPass& p : passes) bound += op_bytes_bound<R>(p);
  int rc = reserve_ops(h, bound);
  if (rc) return rc;
  size_t off = 0, take = 1;
  for (size_t first = 0; first < passes.size(); first += take, take *= 2) {
    const size_t last = std::min(passes.size(), first + take);
    std::vector<PlanPass> chunk(std::make_move_iterator(passes.begin() + first),
                                std::make_move_iterator(passes.begin() + last));
    size_t used = 0;
    if ((rc = run_plan<R, M, false>(h, h->d, nullptr, chunk, specs, nullptr, nullptr, off, &used))) return rc;
    off = (off + used + 255) & ~size_t(255);
  }
  return VQC_OK;
}

int apply_circuit_fused(vqc_state h, const vqc_gate* gates, int ngates, const double* mats) {
  if (!fused_supported(h)) {
    for (int i = 0; i < ngates; ++i) {
      int rc = apply_gate_raw(h, gates[i].nq, gates[i].pos, mats + gates[i].mat);
      if (rc) return rc;
    }
    return VQC_OK;
  }
  switch (tile_config(h->dtype, h->nq).M + (h->dtype == VQC_C64 ? 0 : 100)) {
    case 12: return forward_impl<float, 12>(h, gates, ngates, mats);
    case 11: return forward_impl<float, 11>(h, gates, ngates, mats);
    case 10: return forward_impl<float, 10>(h, gates, ngates, mats);
    case 9: return forward_impl<float, 9>(h, gates, ngates, mats);
    case 111: return forward_impl<double, 11>(h, gates, ngates, mats);
    case 110: return forward_impl<double, 10>(h, gates, ngates, mats);
    default: return forward_impl<double, 9>(h, gates, ngates, mats);
  }
}

// Reverse sweep on the tile engine.  grads[j] receive the partials.  Gates
// the tile engine cannot take (3+ targets, or 2 targets with parameters) run
// through the per-gate adjoint path.
int per_gate_params_grad(vqc_state h, void* lam, void* y, const GateSpec& gs, const std::vector<ParamInfo>& ps,
                         double* grads);

// The reverse sweep's op list: gates last to first (specs hold U^dagger),
// with the reduced-matrix accumulation on every op that carries parameters.
static std::vector<PItem> reverse_items(const std::vector<GateSpec>& specs,
                                        const std::vector<std::vector<ParamInfo>>& params) {
  const int ng = (int)specs.size();
  std::vector<PItem> items;
  items.reserve(ng);
  for (int i = ng - 1; i >= 0; --i) {
    PItem it;
    it.gate = i;
    const GateSpec& gs = specs[i];
    bool ok = to_fop(gs, it.op);
    if (ok && !params[i].empty()) {
      FOp& f = it.op;
      if (f.kind == kOpU1) {
        f.acc = true;
        for (const ParamInfo& pi : params[i]) f.grads.push_back(PGrad{pi.index, restrict_to(gs, f, pi.D)});
      } else if (f.kind == kOpDiag && f.nd <= 2 && f.nd >= 1) {
        f.acc = true;
        const int d = 1 << gs.k;
        for (const ParamInfo& pi : params[i]) {
          PGrad pg{pi.index, {}};
          for (int j = 0; j < d; ++j) pg.D.push_back(pi.D[(size_t)j * d + j]);
          f.grads.push_back(pg);
        }
      } else {
        ok = false;
      }
    }
    it.standalone = !ok;
    items.push_back(std::move(it));
  }
  return items;
}

template <class R, int M>
static int reverse_impl(vqc_state h, void* lam, void* y, const std::vector<GateSpec>& specs,
                        const std::vector<std::vector<ParamInfo>>& params, double* grads) {
  std::vector<PItem> items = reverse_items(specs, params);
  std::vector<PlanPass> passes;
  plan_passes(h->nq, tile_config(h->dtype, h->nq), true, items, passes);
  // standalone gates with parameters: split their passes out so the per-gate
  // path can evaluate the partials right after the uncompute
  std::vector<AccRef> accs;
  int total_rows = 0;
  for (auto& p : passes)
    if (!p.standalone) {
      int s = 0;
      for (auto& f : p.ops) s += f.acc ? 1 : 0;
      total_rows += s;
    }
  if ((size_t)total_rows * 8 > h->accbuf_rows * 32) {
    if (h->accbuf) {
      VQC_CK(cudaStreamSynchronize(h->stream));
      VQC_CK(cudaFree(h->accbuf));
      h->accbuf = nullptr;
    }
    const size_t rows32 = ((size_t)total_rows * 8 + 31) / 32 + 1;
    VQC_CK(cudaMalloc(&h->accbuf, sizeof(double) * 32 * rows32));
    h->accbuf_rows = rows32;
  }
  // run pass by pass so that standalone gates with parameters see the right states
  std::vector<PlanPass> one(1);
  int row_base = 0;
  for (size_t pi = 0; pi < passes.size(); ++pi) {
    if (passes[pi].standalone) {
      const int gi = passes[pi].gate;
      const GateSpec& gs = specs[gi];
      if (params[gi].empty()) {
        int rc = standalone_adjoint(h, lam, y, gs, false, nullptr);
        if (rc) return rc;
      } else {
        int rc = per_gate_params_grad(h, lam, y, gs, params[gi], grads);
        if (rc) return rc;
      }
      continue;
    }
    // group consecutive tile passes into one upload
    size_t pj = pi;
    std::vector<PlanPass> group;
    while (pj < passes.size() && !passes[pj].standalone) group.push_back(std::move(passes[pj++]));
    std::vector<AccRef> gaccs;
    int rc = run_plan<R, M, true>(h, y, lam, group, specs, &gaccs, h->accbuf + (size_t)row_base * 8);
    if (rc) return rc;
    for (auto& a : gaccs) {
      a.row += row_base;
      accs.push_back(std::move(a));
    }
    for (auto& g : group) row_base += g.nslots;
    pi = pj - 1;
  }
  // contract A with the D matrices
  std::vector<double> A((size_t)std::max(row_base, 1) * 8);
  if (row_base > 0)
    VQC_CK(cudaMemcpyAsync(A.data(), h->accbuf, sizeof(double) * 8 * row_base, cudaMemcpyDeviceToHost, h->stream));
  VQC_CK(cudaStreamSynchronize(h->stream));
  contract_grads(accs, A.data(), grads);
  return VQC_OK;
}

int reverse_sweep_fused(vqc_state h, void* lam, void* y, const std::vector<GateSpec>& specs,
                        const std::vector<std::vector<ParamInfo>>& params, double* grads) {
  switch (tile_config(h->dtype, h->nq).M + (h->dtype == VQC_C64 ? 0 : 100)) {
    case 12: return reverse_impl<float, 12>(h, lam, y, specs, params, grads);
    case 11: return reverse_impl<float, 11>(h, lam, y, specs, params, grads);
    case 10: return reverse_impl<float, 10>(h, lam, y, specs, params, grads);
    case 9: return reverse_impl<float, 9>(h, lam, y, specs, params, grads);
    case 111: return reverse_impl<double, 11>(h, lam, y, specs, params, grads);
    case 110: return reverse_impl<double, 10>(h, lam, y, specs, params, grads);
    default: return reverse_impl<double, 9>(h, lam, y, specs, params, grads);
  }
}

}  // namespace vqc

namespace vqc {

// g_j = Re sum_ab D_j[a][b] A[a][b] for every parameter of every accumulating op
// (U1: D is 2x2 row-major and A[a][b] sits at 2a+b; AccD: diagonal bins in order).
void contract_grads(const std::vector<AccRef>& accs, const double* A, double* grads) {
  for (const AccRef& a : accs) {
    const double* r = &A[(size_t)a.row * 8];
    if (a.ah) {
      // r = (Im A00, Im A11, Re A01 - Re A10, Im A01 + Im A10), D anti-Hermitian
      for (const PGrad& pg : a.op.grads)
        grads[pg.param] = -pg.D[0].imag() * r[0] - pg.D[3].imag() * r[1] + pg.D[1].real() * r[2] -
                          pg.D[1].imag() * r[3];
      continue;
    }
    const cd Av[4] = {cd(r[0], r[1]), cd(r[2], r[3]), cd(r[4], r[5]), cd(r[6], r[7])};
    for (const PGrad& pg : a.op.grads) {
      double g = 0;
      for (size_t i = 0; i < pg.D.size() && i < 4; ++i) g += (pg.D[i] * Av[i]).real();
      grads[pg.param] = g;
    }
  }
}

// ----------------------------------------------------------------------------- serving support
__global__ void __launch_bounds__(256) k_reduce_slots_batch(const RedItem* __restrict__ items) {
  __shared__ double sm[8][8];
  const RedItem it = items[blockIdx.y];
  const int slot = blockIdx.x, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (slot >= it.nslots) return;
  for (int val = 0; val < 8; ++val) {
    double s = 0;
    for (int b = threadIdx.x; b < it.nblocks; b += blockDim.x)
      s += it.partials[((size_t)b * it.nslots + slot) * 8 + val];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) sm[warp][val] = s;
  }
  __syncthreads();
  if (threadIdx.x < 8) {
    double s = 0;
    for (int wp = 0; wp < (int)(blockDim.x >> 5); ++wp) s += sm[wp][threadIdx.x];
    it.out[(size_t)slot * 8 + threadIdx.x] = s;
  }
}

template <class R, int M>
static int build_plan_tm(int n, int dtype, const std::vector<GateSpec>& fspecs, const std::vector<GateSpec>& rspecs,
                         const std::vector<std::vector<ParamInfo>>& params, bool want_grad, bool packed,
                         ReqPlan& rp) {
  const TileConfig tc = tile_config(dtype, n);
  auto shape_max = [packed](const SerialPlan& sp) {
    PassShape m;
    m.packed = packed;
    for (const PassLoc& l : sp.locs) {
      m.nslots = std::max(m.nslots, l.shape.nslots);
      m.nstages = std::max(m.nstages, l.shape.nstages);
      m.nops = std::max(m.nops, l.shape.nops);
      m.npool = std::max(m.npool, l.shape.npool);
    }
    return m;
  };
  std::vector<PItem> items(fspecs.size());
  for (size_t i = 0; i < fspecs.size(); ++i) {
    items[i].gate = (int)i;
    items[i].standalone = !to_fop(fspecs[i], items[i].op);
  }
  std::vector<PlanPass> passes;
  plan_passes(n, tc, false, items, passes);
  for (const PlanPass& p : passes)
    if (p.standalone) return fail(VQC_ERR_UNSUPPORTED, "serving takes gates with at most two target qubits");
  serialize_plan<R, M, false>(n, dtype, passes, rp.fwd, nullptr, packed);
  rp.fwd_max = shape_max(rp.fwd);
  if (want_grad) {
    std::vector<PItem> ritems = reverse_items(rspecs, params);
    std::vector<PlanPass> rpasses;
    plan_passes(n, tc, true, ritems, rpasses);
    for (const PlanPass& p : rpasses)
      if (p.standalone)
        return fail(VQC_ERR_UNSUPPORTED, "serving takes parameterised gates with one target qubit (or diagonal)");
    serialize_plan<R, M, true>(n, dtype, rpasses, rp.adj, &rp.accs, packed);
    rp.adj_max = shape_max(rp.adj);
  }
  rp.M = M;
  rp.ntiles = int64_t(1) << (n - M);
  return VQC_OK;
}

static int build_plan_any(int n, int dtype, const std::vector<GateSpec>& fspecs, const std::vector<GateSpec>& rspecs,
                          const std::vector<std::vector<ParamInfo>>& params, bool want_grad, bool packed,
                          ReqPlan& rp) {
  switch (tile_config(dtype, n).M + (dtype == VQC_C64 ? 0 : 100)) {
    case 12: return build_plan_tm<float, 12>(n, dtype, fspecs, rspecs, params, want_grad, packed, rp);
    case 11: return build_plan_tm<float, 11>(n, dtype, fspecs, rspecs, params, want_grad, packed, rp);
    case 10: return build_plan_tm<float, 10>(n, dtype, fspecs, rspecs, params, want_grad, packed, rp);
    case 9: return build_plan_tm<float, 9>(n, dtype, fspecs, rspecs, params, want_grad, packed, rp);
    case 111: return build_plan_tm<double, 11>(n, dtype, fspecs, rspecs, params, want_grad, false, rp);
    case 110: return build_plan_tm<double, 10>(n, dtype, fspecs, rspecs, params, want_grad, false, rp);
    default: return build_plan_tm<double, 9>(n, dtype, fspecs, rspecs, params, want_grad, false, rp);
  }
}

// The compiled batch kernels of a packed plan's passes (false when one has
// none); compile = false only looks them up.
static bool plan_kernels(int M, bool adj, const SerialPlan& sp, std::vector<const void*>& ks, bool compile) {
  std::vector<JitPassRef> refs(sp.locs.size());
  for (size_t i = 0; i < sp.locs.size(); ++i)
    refs[i] = JitPassRef{(const DevStageF*)(sp.buf.data() + sp.locs[i].stages), sp.locs[i].shape.nstages,
                         (const DevOp*)(sp.buf.data() + sp.locs[i].ops), sp.locs[i].shape.npool};
  if (jit_pass_kernels(M, adj, refs, ks, true, compile)) return false;
  for (const void* k : ks)
    if (!k) return false;
  return true;
}

// Serving compiles the passes of requests of at least 2^18 amplitudes (where
// the device time of a mix concentrates); smaller requests share the generic
// kernel's single launch per step kind.
constexpr int kServeJitMinQubits = 18;

int serve_build_plan(int n, int dtype, const std::vector<GateSpec>& fspecs, const std::vector<GateSpec>& rspecs,
                     const std::vector<std::vector<ParamInfo>>& params, bool want_grad, bool compiled, ReqPlan& rp,
                     ReqPlan* to_compile) {
  if (n < kMinTileBits || n > 40) return fail(VQC_ERR_UNSUPPORTED, "serving takes 9 to 40 qubits");
  if (compiled && dtype == VQC_C64 && n >= kServeJitMinQubits && jit_available()) {
    int rc = build_plan_any(n, dtype, fspecs, rspecs, params, want_grad, true, rp);
    if (rc) return rc;
    if (plan_kernels(rp.M, false, rp.fwd, rp.fwd_k, false) &&
        (!want_grad || plan_kernels(rp.M, true, rp.adj, rp.adj_k, false)))
      return VQC_OK;
    // not compiled yet: this request runs the classic plan on the generic kernel
    if (to_compile) *to_compile = std::move(rp);
    rp = ReqPlan();
  }
  return build_plan_any(n, dtype, fspecs, rspecs, params, want_grad, false, rp);
}

void serve_compile_plan(const ReqPlan& packed, bool want_grad) {
  std::vector<const void*> ks;
  plan_kernels(packed.M, false, packed.fwd, ks, true);
  if (want_grad) plan_kernels(packed.M, true, packed.adj, ks, true);
}

// Shared memory of a compiled FP32 pass of shape ps (the formula of pass_smem).
static size_t jit_pass_smem(int M, bool adj, const PassShape& ps) {
  const size_t nt = size_t(1) << (M - kRegBits);
  const size_t npool = (size_t)ps.npool * sizeof(float2);
  return (adj ? 2 : 1) * (size_t(1) << M) * sizeof(float2) + (adj ? (size_t)ps.nslots * (nt / 32) * 8 * sizeof(double) : 0) +
         sizeof(DevStageF) * ps.nstages + sizeof(DevOp) * ps.nops + ((npool + 15) & ~size_t(15));
}

int serve_jit_gridx(int M, bool adj, const std::vector<const void*>& ks, const SerialPlan& sp, int64_t ntiles,
                    int device) {
  int per_sm = 1 << 20;
  for (size_t i = 0; i < ks.size(); ++i) {
    const size_t smem = jit_pass_smem(M, adj, sp.locs[i].shape);
    cudaFuncSetAttribute(ks[i], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024));
    int b = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, ks[i], 1 << (M - kRegBits), smem) != cudaSuccess || b < 1) {
      cudaGetLastError();
      b = 1;
    }
    per_sm = std::min(per_sm, b);
  }
  if (ks.empty()) per_sm = 1;
  return (int)std::max<int64_t>(1, std::min<int64_t>(ntiles, (int64_t)device_info(device).sms * per_sm));
}

int serve_launch_jit(int M, bool adj, const void* kernel, const TileItem* d_items, int nitems, int gridx,
                     const PassShape& maxs, cudaStream_t stream) {
  const size_t smem = jit_pass_smem(M, adj, maxs);
  VQC_CK(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)std::max<size_t>(smem, 48 * 1024)));
  ProfScope prof(stream, adj ? "serve_tile_adjoint" : "serve_tile_forward", 0);
  void* args[] = {(void*)&d_items};
  VQC_CK(cudaLaunchKernel(kernel, dim3(gridx, nitems), dim3(1 << (M - kRegBits)), args, smem, stream));
  return VQC_OK;
}

template <class R, int M, bool ADJ>
static int grid_x_tm(const PassShape& maxs, int64_t max_ntiles, int device) {
  return (int)std::max<int64_t>(1, std::min<int64_t>(max_ntiles, tile_grid<R, M, ADJ>(device, maxs)));
}

template <class R, int M, bool ADJ>
static int launch_batch_tm(const TileItem* d_items, int nitems, int gridx, const PassShape& maxs,
                           cudaStream_t stream) {
  constexpr int NT = 1 << (M - kRegBits);
  const size_t smem = pass_smem<R, M, ADJ>(maxs);
  auto kfun = k_tile_batch<R, M, ADJ>;
  VQC_CK(cudaFuncSetAttribute(kfun, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 48 * 1024)));
  ProfScope prof(stream, ADJ ? "serve_tile_adjoint" : "serve_tile_forward", 0);
  kfun<<<dim3(gridx, nitems), NT, smem, stream>>>(d_items);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

#define VQC_TILE_SWITCH(FN, ...)                                         \
  switch (M + (dtype == VQC_C64 ? 0 : 100) + (adj ? 1000 : 0)) {          \
    case 12: return FN<float, 12, false>(__VA_ARGS__);                    \
    case 11: return FN<float, 11, false>(__VA_ARGS__);                    \
    case 10: return FN<float, 10, false>(__VA_ARGS__);                    \
    case 9: return FN<float, 9, false>(__VA_ARGS__);                      \
    case 1012: return FN<float, 12, true>(__VA_ARGS__);                   \
    case 1011: return FN<float, 11, true>(__VA_ARGS__);                   \
    case 1010: return FN<float, 10, true>(__VA_ARGS__);                   \
    case 1009: return FN<float, 9, true>(__VA_ARGS__);                    \
    case 111: return FN<double, 11, false>(__VA_ARGS__);                  \
    case 110: return FN<double, 10, false>(__VA_ARGS__);                  \
    case 109: return FN<double, 9, false>(__VA_ARGS__);                   \
    case 1111: return FN<double, 11, true>(__VA_ARGS__);                  \
    case 1110: return FN<double, 10, true>(__VA_ARGS__);                  \
    case 1109: return FN<double, 9, true>(__VA_ARGS__);                   \
    default: return fail(VQC_ERR_ARG, "no tile kernel for this size");   \
  }

int serve_tile_gridx(int dtype, int M, bool adj, const PassShape& maxs, int64_t max_ntiles, int device) {
  VQC_TILE_SWITCH(grid_x_tm, maxs, max_ntiles, device)
}

int serve_launch_tiles(int dtype, int M, bool adj, const TileItem* d_items, int nitems, int gridx,
                       const PassShape& maxs, cudaStream_t stream) {
  VQC_TILE_SWITCH(launch_batch_tm, d_items, nitems, gridx, maxs, stream)
}
#undef VQC_TILE_SWITCH

int serve_launch_reduce(const RedItem* d_items, int nitems, int maxslots, cudaStream_t stream) {
  if (nitems == 0 || maxslots == 0) return VQC_OK;
  k_reduce_slots_batch<<<dim3(maxslots, nitems), 256, 0, stream>>>(d_items);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

}  // namespace vqc
