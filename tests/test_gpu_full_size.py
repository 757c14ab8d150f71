"""The headline configuration at its full size: adjoint gradient at n = 26,
20 layers of (RX, RY, RZ on every qubit + CRX(i, i+1)), XXZ energy (75 Pauli
terms), FP32 amplitudes with FP64 accumulation.  The oracle would take minutes
per gradient here, so the checks are properties that do not depend on the size:
  * FP32 against the device's FP64 path: energy and every partial within 1e-5
    relative (norm-wise on the gradient vector);
  * central differences of the FP64 energy (h = 1e-4) at a few parameters
    against the adjoint partials: 1e-6 relative to max |g|;
  * the forward circuit is unitary: |psi_out| = 1 within 1e-5 in FP32;
  * the energy of a Hermitian operator is real: |Im E| <= 1e-6 |E|.
"""
import numpy as np
import pytest

import vqcb200 as V
from helpers import rel
from vqcb200 import workloads as W

pytestmark = pytest.mark.gpu

N, LAYERS = 26, 20


def _problem():
    rng = np.random.default_rng(2026)
    th = rng.uniform(0, 2 * np.pi, LAYERS * (4 * N - 1))
    return th, W.to_operator(W.xxz_spec(N, 0.5))


def test_full_size_gradient_properties():
    th, H = _problem()
    c = W.to_circuit(W.rxyz_crx_spec(N, LAYERS, th))
    e32, g32 = V.energy_and_gradient(H, c, V.StateVector(N, dtype=np.complex64))
    e64, g64 = V.energy_and_gradient(H, c, V.StateVector(N, dtype=np.complex128))
    assert g32.shape == g64.shape == (LAYERS * (4 * N - 1),)
    assert abs(e32 - e64) / abs(e64) < 1e-5
    assert rel(g32, g64) < 1e-5
    assert abs(e64.imag) <= 1e-6 * abs(e64)
    assert abs(e32.imag) <= 1e-6 * abs(e32)

    # central differences of the FP64 energy at a few parameters (first layer,
    # a CRX in the middle, the last rotation)
    h = 1e-4
    scale = np.abs(g64).max()
    for j in [0, LAYERS * (4 * N - 1) // 2, LAYERS * (4 * N - 1) - 1]:
        es = []
        for s in (1, -1):
            t = th.copy()
            t[j] += s * h
            psi = W.to_circuit(W.rxyz_crx_spec(N, LAYERS, t)) * V.StateVector(N, dtype=np.complex128)
            es.append(V.expectation(H, psi).real)
            del psi
        fd = (es[0] - es[1]) / (2 * h)
        assert abs(fd - g64[j]) < 1e-6 * scale + 1e-8, (j, fd, g64[j])

    # unitarity of the fused forward passes in FP32
    psi = c * V.StateVector(N, dtype=np.complex64)
    assert abs(psi.norm() - 1.0) < 1e-5
