// Host-side gate analysis shared by the gate, gradient and density-matrix
// paths of libvqcb200.
#pragma once

#include <complex>
#include <vector>

#include "common.cuh"

namespace vqc {

using cd = std::complex<double>;

// A gate reduced to the part of the state it changes.
//
// The reference dispatches on the gate's Julia type to specialised kernels
// (applygates/specific/*.jl: CZ touches a quarter of the amplitudes, CNOT
// half, ...) and sends every other gate through the dense k-qubit loops.
// Here the structure is read off the matrix instead: an index j of the
// 2^k-dimensional gate space is *inactive* when row j and column j of U are
// the unit vector e_j; only the active indices S are loaded, multiplied by
// U restricted to S and stored back.  CZ gives |S| = 1, CNOT and CRX |S| = 2,
// Toffoli |S| = 2, FREDKIN |S| = 2, a dense 1-qubit gate |S| = 2.
struct GateSpec {
  int k = 0;
  int sp[5] = {0, 0, 0, 0, 0};  // sorted positions
  std::vector<cd> U;            // 2^k x 2^k, bit b <-> sp[b]
  int ns = 0;                   // |S|
  int S[32];                    // active indices, ascending
  int mode = 0;                 // kDense / kDiag / kMono on U[S][S]
  std::vector<cd> US;           // ns x ns
  int mono_src[32];             // kMono: out_a = US[a][mono_src[a]] * in_{mono_src[a]}
};
constexpr int kDense = 0, kDiag = 1, kMono = 2;

// Validates positions (distinct, in [0, n)), k in 1..5, orders the gate and
// finds its active subspace.  dagger: analyse U^dagger instead of U.
int analyze_gate(int n, int k, const int* pos, const double* mat, bool dagger, GateSpec& g);
// Sorted-order matrix of an arbitrary operator (no unitarity assumed).
int order_matrix(int n, int k, const int* pos, const double* mat, int* sp, std::vector<cd>& M);

// One circuit parameter in the reverse sweep: D = U^dagger dU/dtheta (or
// G^dagger for generator-kind parameters), sorted order, 2^k x 2^k.
struct ParamInfo {
  int index;  // position in the caller's params array
  std::vector<cd> D;
};

int prepare_reverse(int nq, const vqc_gate* gates, int ngates, const double* mats, const vqc_param* params,
                    int nparams, std::vector<GateSpec>& specs, std::vector<std::vector<ParamInfo>>& per_gate);

// Applies an analysed gate to a 2^nq vector on `stream` (dtype VQC_C64/C128).
int launch_gate(const GateSpec& g, void* v, int nq, int dtype, int device, cudaStream_t stream);

// Applies a gate given as (k, pos, mat) to h (state vector semantics on all
// of h's stored qubits).
int apply_gate_raw(vqc_state h, int k, const int* pos, const double* mat);

// Density-matrix form: rho <- U rho U^dagger on the n_dm-qubit matrix held in h.
int dm_apply_gate_raw(vqc_state h, int k, const int* pos, const double* mat);

// The fused tile engine (fused.cu).  Plans the gates into passes and runs them.
int apply_circuit_fused(vqc_state h, const vqc_gate* gates, int ngates, const double* mats);

inline int64_t mask_of(int k, const int* sp, int nq, int64_t* mask) {
  const int64_t L = int64_t(1) << nq;
  mask[0] = (int64_t(1) << sp[0]) - 1;
  for (int i = 1; i < k; ++i) mask[i] = ((int64_t(1) << sp[i]) - 1) ^ ((int64_t(2) << sp[i - 1]) - 1);
  mask[k] = (L - 1) ^ ((int64_t(2) << sp[k - 1]) - 1);
  return L >> k;
}

inline int64_t offset_of(int j, int k, const int* sp) {
  int64_t o = 0;
  for (int b = 0; b < k; ++b)
    if (j >> b & 1) o += int64_t(1) << sp[b];
  return o;
}

}  // namespace vqc
