"""ground_state and time_evolution (utility/groundstate.jl:4-25) on the
device against dense linear algebra (numpy eigh, scipy expm) on the same
operators: the reference's KrylovKit is not available, and the results are
mathematical quantities of the operator.  Tolerances: FP64 1e-8 on the
energy and the evolved state, FP32 1e-4."""
import numpy as np
import pytest
import scipy.linalg

import vqcb200 as V
from helpers import max_abs, rand_psi
from oracle import dense_np as D
from oracle import oracle as O
from vqcb200 import workloads as W

pytestmark = pytest.mark.gpu


def _dense(n, hspec):
    return D.pauli_sum_matrix(n, O.terms_from_spec(hspec))


@pytest.mark.parametrize("n", [6, 10])
def test_ground_state_xxz(n):
    hspec = W.xxz_spec(n, 0.5)
    H = W.to_operator(hspec)
    e, psi = V.ground_state(H, rng=3)
    w, U = np.linalg.eigh(_dense(n, hspec))
    assert abs(e - w[0]) < 1e-8 * max(1.0, abs(w[0]))
    # the eigenvector (degenerate-safe check: residual of H psi - e psi)
    v = psi.storage()
    r = _dense(n, hspec) @ v - e * v
    assert np.linalg.norm(r) < 1e-5


@pytest.mark.parametrize("dtype,bound", [(np.complex128, 1e-8), (np.complex64, 1e-4)])
@pytest.mark.parametrize("t", [-0.7j, 0.3, -2.5j])
def test_time_evolution_tfim(dtype, bound, t):
    n = 8
    hspec = W.tfim_spec(n, 0.9)
    H = W.to_operator(hspec)
    rng = np.random.default_rng(12)
    psi = rand_psi(rng, n)
    out = V.time_evolution(H, t, V.StateVector(psi.astype(dtype), dtype=dtype))
    want = scipy.linalg.expm(t * _dense(n, hspec)) @ psi
    assert max_abs(out.storage(), want) < bound * max(1.0, np.abs(want).max())
