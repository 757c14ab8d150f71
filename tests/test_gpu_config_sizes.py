"""Parity at the benchmark configurations' own sizes, against the oracle on
the host cores (same inputs, same gates):

  * 30 qubits in ComplexF64 and ComplexF32 (16 GiB / 8 GiB on the device):
    one layer of U3 on every qubit, the CZ brickwork and a Toffoli on a
    high-stride triple (controls on qubit 1 and qubit 29, target qubit 30),
    through the fused tile passes and one gate at a time; the oracle applies
    the same gates to |0...0> with all host threads (generic.jl:26-31,
    threaded_short_range.jl, threaded_long_range.jl);
  * the 13-qubit density matrix (1 GiB ComplexF64): seeded random pure state,
    8 layers of U3 on every qubit + CNOT ladder as rho <- U rho U^dagger,
    partial trace over qubits 10-13 and the basis probabilities
    (generic.jl:54-64, ptrace.jl:38-53, measure.jl:69-81);
  * 26 qubits, the gradient workload truncated to its first two layers (RX,
    RY, RZ on every qubit + CRX(i, i+1); XXZ energy, 75 terms) against the
    oracle's restatement of circuitdiff.jl:23-32 and expecdiff.jl:30-33.

Bounds as in helpers.py, asserted as stated: 1e-12 in FP64 (max-abs on
normalised states, relative on energies, norm-wise on gradients), 1e-5 in
FP32.  Host memory: at most two 16 GiB vectors at a time."""
import gc
import os

import numpy as np
import pytest

import vqcb200 as V
from helpers import max_abs, max_abs_chunked, rel, rel_scalar, tol
from oracle import oracle as O
from vqcb200 import workloads as W

pytestmark = pytest.mark.gpu
NTHREADS = os.cpu_count() or 1


def _layer_n30(n):
    spec = [s for s in W.u3_cz_toffoli_spec(n, 1, 2030) if s[0] != "toffoli"]
    spec.append(("toffoli", (1, n - 1, n), ()))  # controls 1 and n-1, target n: the highest stride
    return spec


def test_gates_n30_both_precisions():
    n = 30
    spec = _layer_n30(n)
    ref = O.apply_circuit(O.zero_state(n), O.from_spec(spec), nthreads=NTHREADS)
    for dtype in (np.complex128, np.complex64):
        for fuse in (True, False):
            s = V.StateVector(n, dtype=dtype)
            V.apply(W.to_circuit(spec), s, fuse=fuse)
            got = s.storage()
            del s
            err = max_abs_chunked(got, ref)
            del got
            gc.collect()
            assert err < tol(dtype), (dtype.__name__, fuse, err)


def test_density_matrix_n13_config():
    n, layers, seed = 13, 8, 1303
    rng = np.random.default_rng(seed)
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    spec = W.u3_cnot_spec(n, layers, seed)
    sites = [10, 11, 12, 13]
    ref = O.density_matrix(psi)
    O.dm_apply_circuit(ref, n, O.from_spec(spec), nthreads=NTHREADS)
    red_ref = O.dm_ptrace(ref, n, [s - 1 for s in sites])
    probs_ref = O.dm_probs(ref, n)
    for fuse in (True, False):
        rho = V.DensityMatrix(V.StateVector(psi))
        V.apply(W.to_circuit(spec), rho, fuse=fuse)
        assert max_abs_chunked(rho.data(), ref) < 1e-12, fuse
        red = V.partial_tr(rho, sites)
        assert red.shape == (1 << (n - len(sites)),) * 2
        assert max_abs(red.reshape(-1, order="F"), red_ref) < 1e-12, fuse
        assert max_abs(V.probabilities(rho), probs_ref) < 1e-12, fuse
        assert abs(rho.tr() - 1) < 1e-12
        del rho
        gc.collect()


def test_gradient_n26_truncated():
    n, layers = 26, 2
    rng = np.random.default_rng(2626)
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    spec = W.rxyz_crx_spec(n, layers, th)
    hspec = W.xxz_spec(n, 0.5)
    e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(hspec), O.zero_state(n),
                                         nthreads=NTHREADS)
    assert g_ref.shape == (layers * (4 * n - 1),)
    for dtype in (np.complex128, np.complex64):
        e, g = V.energy_and_gradient(W.to_operator(hspec), W.to_circuit(spec), V.StateVector(n, dtype=dtype))
        assert rel_scalar(e, e_ref) < tol(dtype), (dtype.__name__, e, e_ref)
        assert rel(g, g_ref) < tol(dtype), dtype.__name__
