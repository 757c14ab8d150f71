// Adjoint-mode circuit gradients: the Zygote adjoint of *(circuit, psi)
// (circuitdiff.jl:2-8, back_propagate :23-32, back_propagate_util :61-75)
// and of expectation(H, psi) (expecdiff.jl:30-33, 68).
//
// Reverse sweep, per gate (last to first), as the reference does:
//   delta <- U^dagger delta,  y <- U^dagger y          (uncompute, no storage)
//   grad_j = Re <delta_out | dU/dtheta_j | y_in>
//          = Re sum_ab D_j[a,b] A[a,b],  D_j = U^dagger dU/dtheta_j,
//            A[a,b] = sum over groups of conj(delta_a) y_b   (after the uncompute)
// The reference evaluates one two-state expectation pass per parameter
// (real(expectation(y, dG, delta)), circuitdiff.jl:29).  Here the uncompute of
// both states and the reduced matrix A are one pass: A is accumulated in FP64
// over the gate's active subspace (D_j vanishes outside it), reduced on the
// device in a fixed order, and the per-parameter contractions with D_j run on
// the host in FP64.
#include <algorithm>
#include <cstring>

#include "engine.h"
#include "subspace.cuh"

namespace vqc {

int pauli_run(vqc_state h, const void* bra, const void* ket, void* out, const vqc_pauli* terms, int nterms,
              bool write, bool acc, bool hermitian_part, double* result, bool* deferred = nullptr);
int expect_dense_device(vqc_state h, const void* bra, const void* ket, int k, const int* sp, const std::vector<cd>& M,
                        double* res);
int apply_circuit_raw(vqc_state h, const vqc_gate* gates, int ngates, const double* mats, bool dm, int fuse);

constexpr int kAccMaxS = 4;  // A is reduced in one pass for |S| <= 4

// lam, psi <- U^dagger (a.U holds U^dagger restricted to S); with ACC,
// out (device) receives A[a][b] = sum conj(lam_a) psi_b as (re, im) pairs.
template <class R, int MS, bool ACC>
__global__ void __launch_bounds__(kRedThreads)
    k_adjoint_sub(cplx<R>* __restrict__ lam, cplx<R>* __restrict__ psi, const __grid_constant__ SubArgs<R, MS> a,
                  Scratch s, double* out) {
  double acc[ACC ? 2 * MS * MS : 1];
#pragma unroll
  for (int i = 0; i < (ACC ? 2 * MS * MS : 1); ++i) acc[i] = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < a.ngroups; g += stride) {
    const int64_t base = group_base(g, a.k, a.mask);
    cplx<R> xl[MS], xp[MS], yl[MS], yp[MS];
#pragma unroll
    for (int s = 0; s < MS; ++s)
      if (s < a.ns) {
        if (!VQC_DCHECK(base + a.off[s], a.namp)) {
          xl[s] = xp[s] = mkc<R>(R(0), R(0));
          continue;
        }
        xl[s] = lam[base + a.off[s]];
        xp[s] = psi[base + a.off[s]];
      }
#pragma unroll
    for (int r = 0; r < MS; ++r) {
      if (r < a.ns) {
        cplx<R> al = mkc<R>(R(0), R(0)), ap = al;
#pragma unroll
        for (int c = 0; c < MS; ++c)
          if (c < a.ns) {
            al = cfma(a.U[r * MS + c], xl[c], al);
            ap = cfma(a.U[r * MS + c], xp[c], ap);
          }
        yl[r] = al;
        yp[r] = ap;
        if (!VQC_DCHECK(base + a.off[r], a.namp)) continue;
        lam[base + a.off[r]] = al;
        psi[base + a.off[r]] = ap;
      }
    }
    if (ACC) {
#pragma unroll
      for (int r = 0; r < MS; ++r) {
        if (r < a.ns) {
          const double2 l = to_d2(yl[r]);
#pragma unroll
          for (int c = 0; c < MS; ++c)
            if (c < a.ns) {
              const double2 p = to_d2(yp[c]);
              double* q = &acc[2 * (r * MS + c)];
              q[0] = fma(l.x, p.x, fma(l.y, p.y, q[0]));
              q[1] = fma(l.x, p.y, fma(-l.y, p.x, q[1]));
            }
        }
      }
    }
  }
  if (ACC) grid_reduce<(ACC ? 2 * MS * MS : 1)>(acc, s, out);
}

template <class R, int MS>
static int launch_adj(const GateSpec& gd, vqc_state h, void* lam, void* psi, bool acc, double* out) {
  SubArgs<R, MS> a;
  fill_sub_args<R, MS>(gd, h->nq, a);
  if (gd.mode != kDense) {  // the kernel is written for the dense form: expand
    for (int i = 0; i < MS * MS; ++i) a.U[i] = mkc<R>(R(0), R(0));
    for (int r = 0; r < gd.ns; ++r)
      for (int c = 0; c < gd.ns; ++c) {
        cd u = gd.US[r * gd.ns + c];
        a.U[r * MS + c] = mkc<R>((R)u.real(), (R)u.imag());
      }
  }
  const int grid = acc ? reduction_grid(h->device, a.ngroups) : launch_grid(h->device, a.ngroups);
  ProfScope prof(h->stream, "adjoint_gate", 4.0 * a.ngroups * gd.ns * sizeof(cplx<R>));
  if constexpr (MS <= kAccMaxS) {
    if (acc) {
      k_adjoint_sub<R, MS, true><<<grid, kRedThreads, 0, h->stream>>>((cplx<R>*)lam, (cplx<R>*)psi, a, h->scr, out);
      VQC_CK(cudaGetLastError());
      return VQC_OK;
    }
  }
  k_adjoint_sub<R, MS, false><<<grid, kRedThreads, 0, h->stream>>>((cplx<R>*)lam, (cplx<R>*)psi, a, h->scr, out);
  VQC_CK(cudaGetLastError());
  return VQC_OK;
}

template <class R>
static int launch_adj_r(const GateSpec& gd, vqc_state h, void* lam, void* psi, bool acc, double* out) {
  switch (ms_of(gd.ns)) {
    case 1: return launch_adj<R, 1>(gd, h, lam, psi, acc, out);
    case 2: return launch_adj<R, 2>(gd, h, lam, psi, acc, out);
    case 4: return launch_adj<R, 4>(gd, h, lam, psi, acc, out);
    case 8: return launch_adj<R, 8>(gd, h, lam, psi, false, out);
    case 16: return launch_adj<R, 16>(gd, h, lam, psi, false, out);
    default: return launch_adj<R, 32>(gd, h, lam, psi, false, out);
  }
}

int fused_supported(vqc_state h);
int reverse_sweep_fused(vqc_state h, void* lam, void* y, const std::vector<GateSpec>& specs,
                        const std::vector<std::vector<ParamInfo>>& params, double* grads);

// lam, y <- U^dagger (gd holds U^dagger); with acc, out receives A (|S| <= 4).
int standalone_adjoint(vqc_state h, void* lam, void* y, const GateSpec& gd, bool acc, double* out) {
  if (gd.ns == 0) return VQC_OK;
  return h->dtype == VQC_C64 ? launch_adj_r<float>(gd, h, lam, y, acc, out)
                             : launch_adj_r<double>(gd, h, lam, y, acc, out);
}

// One gate of the reverse sweep with its parameters' partials, evaluated at
// once (used for gates the tile engine does not take).
int per_gate_params_grad(vqc_state h, void* lam, void* y, const GateSpec& gs, const std::vector<ParamInfo>& ps,
                         double* grads) {
  const int d = 1 << gs.k;
  if (gs.ns > 0 && gs.ns <= kAccMaxS) {
    int rc = standalone_adjoint(h, lam, y, gs, true, h->scr.result);
    if (rc) return rc;
    if ((rc = fetch_result(h, 2 * kAccMaxS * kAccMaxS))) return rc;
    const int MS = ms_of(gs.ns);
    for (const ParamInfo& pi : ps) {
      double g = 0;
      for (int r = 0; r < gs.ns; ++r)
        for (int c = 0; c < gs.ns; ++c) {
          const cd Dv = pi.D[(size_t)gs.S[r] * d + gs.S[c]];
          const cd Av(h->h_result[2 * (r * MS + c)], h->h_result[2 * (r * MS + c) + 1]);
          g += (Dv * Av).real();
        }
      grads[pi.index] = g;
    }
    return VQC_OK;
  }
  int rc = standalone_adjoint(h, lam, y, gs, false, nullptr);
  if (rc) return rc;
  for (const ParamInfo& pi : ps) {
    if ((rc = expect_dense_device(h, lam, y, gs.k, gs.sp, pi.D, h->scr.result))) return rc;
    if ((rc = fetch_result(h, 2))) return rc;
    grads[pi.index] = h->h_result[0];
  }
  return VQC_OK;
}

// The analysed gates of a circuit for its reverse sweep (U^dagger) and, per
// gate, its parameters with D = U^dagger dU/dtheta (or G^dagger).
int prepare_reverse(int nq, const vqc_gate* gates, int ngates, const double* mats, const vqc_param* params,
                    int nparams, std::vector<GateSpec>& specs, std::vector<std::vector<ParamInfo>>& per_gate) {
  if (nparams < 0 || (nparams > 0 && !params)) return fail(VQC_ERR_ARG, "bad parameter arrays");
  per_gate.assign(ngates, {});
  for (int j = 0; j < nparams; ++j) {
    const int gi = params[j].gate;
    if (gi < 0 || gi >= ngates) return fail(VQC_ERR_ARG, "parameter refers to a gate out of range");
    per_gate[gi].push_back(ParamInfo{j, {}});
  }
  specs.assign(ngates, GateSpec());
  for (int i = 0; i < ngates; ++i) {
    const vqc_gate& gt = gates[i];
    int rc = analyze_gate(nq, gt.nq, gt.pos, mats + gt.mat, true, specs[i]);
    if (rc) return rc;
    const GateSpec& gs = specs[i];
    const int d = 1 << gs.k;
    for (ParamInfo& pi : per_gate[i]) {
      int sp[5];
      std::vector<cd> dU;
      const vqc_param& pr = params[pi.index];
      if (pr.kind != VQC_PARAM_DERIVATIVE && pr.kind != VQC_PARAM_GENERATOR)
        return fail(VQC_ERR_ARG, "unknown parameter kind");
      if ((rc = order_matrix(nq, gt.nq, gt.pos, mats + pr.dmat, sp, dU))) return rc;
      pi.D.assign((size_t)d * d, cd(0));
      if (pr.kind == VQC_PARAM_GENERATOR) {
        // grad = Re <y_in|G|delta_in> = Re sum_ab conj(G_ba) A[a][b]: D = G^dagger
        for (int r = 0; r < d; ++r)
          for (int c = 0; c < d; ++c) pi.D[(size_t)r * d + c] = std::conj(dU[(size_t)c * d + r]);
        continue;
      }
      // D_j = U^dagger dU_j (gs.U holds U^dagger)
      for (int r = 0; r < d; ++r)
        for (int c = 0; c < d; ++c) {
          cd acc = 0;
          for (int m = 0; m < d; ++m) acc += gs.U[(size_t)r * d + m] * dU[(size_t)m * d + c];
          pi.D[(size_t)r * d + c] = acc;
        }
    }
  }
  return VQC_OK;
}

// The reverse sweep over lam (cotangent) and y (state): both are overwritten
// with their values at the circuit input; grads[j] receive the partials.
static int reverse_sweep(vqc_state h, void* lam, void* y, const vqc_gate* gates, int ngates, const double* mats,
                         const vqc_param* params, int nparams, double* grads, bool fuse) {
  if (nparams > 0 && !grads) return fail(VQC_ERR_ARG, "bad parameter arrays");
  std::vector<GateSpec> specs;
  std::vector<std::vector<ParamInfo>> per_gate;
  int rc0 = prepare_reverse(h->nq, gates, ngates, mats, params, nparams, specs, per_gate);
  if (rc0) return rc0;
  if (fuse && fused_supported(h)) return reverse_sweep_fused(h, lam, y, specs, per_gate, grads);
  for (int i = ngates - 1; i >= 0; --i) {
    int rc = per_gate[i].empty() ? standalone_adjoint(h, lam, y, specs[i], false, nullptr)
                                 : per_gate_params_grad(h, lam, y, specs[i], per_gate[i], grads);
    if (rc) return rc;
  }
  VQC_CK(cudaStreamSynchronize(h->stream));
  return VQC_OK;
}

}  // namespace vqc

using namespace vqc;

extern "C" {

int vqc_adjoint_grad(vqc_state psi0, const vqc_gate* gates, int ngates, const double* mats, const vqc_param* params,
                     int nparams, const vqc_pauli* terms, int nterms, double* energy, double* grads) {
  int rc = enter(psi0);
  if (rc) return rc;
  if (psi0->n_dm) return fail(VQC_ERR_ARG, "adjoint gradient of a density matrix is not on this path");
  if (!energy) return fail(VQC_ERR_ARG, "null energy output");
  if (ngates < 0 || (ngates > 0 && (!gates || !mats))) return fail(VQC_ERR_ARG, "bad circuit arrays");
  std::lock_guard<std::mutex> lk(psi0->mu);
  void* w[2];
  if ((rc = workspace(psi0, 2, w))) return rc;
  void* y = w[0];
  void* lam = w[1];
  VQC_CK(cudaMemcpyAsync(y, psi0->d, psi0->size() * psi0->amp_bytes(), cudaMemcpyDeviceToDevice, psi0->stream));
  // forward: y = circuit * psi0 (run on a view of psi0's handle whose buffer is y)
  void* keep = psi0->d;
  psi0->d = y;
  rc = apply_circuit_raw(psi0, gates, ngates, mats, false, 1);
  psi0->d = keep;
  if (rc) return rc;
  // E = <y|H|y>; cotangent lam = (conj(z) H + z H^dagger) y with z = 1.  E
  // arrives after the reverse sweep, so that its planning on the host runs
  // while the device is still busy with the forward passes.
  bool deferred = false;
  if ((rc = pauli_run(psi0, y, y, lam, terms, nterms, true, true, true, energy, &deferred))) return rc;
  if ((rc = reverse_sweep(psi0, lam, y, gates, ngates, mats, params, nparams, grads, true))) return rc;
  if (deferred) {
    VQC_CK(cudaStreamSynchronize(psi0->stream));
    energy[0] = psi0->h_result[kDeferredSlot];
    energy[1] = psi0->h_result[kDeferredSlot + 1];
  }
  return VQC_OK;
}

int vqc_circuit_backward(vqc_state y, vqc_state delta, const vqc_gate* gates, int ngates, const double* mats,
                         const vqc_param* params, int nparams, double* grads) {
  int rc = enter(y);
  if (rc) return rc;
  if (!delta || delta == y || delta->nq != y->nq || delta->dtype != y->dtype || delta->device != y->device ||
      y->n_dm || delta->n_dm)
    return fail(VQC_ERR_ARG, "backward: y and delta must be distinct state vectors of one size, dtype and device");
  if (ngates < 0 || (ngates > 0 && (!gates || !mats))) return fail(VQC_ERR_ARG, "bad circuit arrays");
  std::lock_guard<std::mutex> lk(y->mu);
  if ((rc = stream_after(y, delta))) return rc;
  if ((rc = reverse_sweep(y, delta->d, y->d, gates, ngates, mats, params, nparams, grads, true))) return rc;
  return stream_after(delta, y);
}

}  // extern "C"
