"""GPU parity of measurement and post-selection (measure.jl, postselect.jl)
against the oracle's restatement, with the same seeded outcome draws.
Bounds: helpers.py (1e-12 FP64, 1e-5 FP32), asserted as stated against the
oracle run on the same FP32-rounded input."""
import numpy as np
import pytest

import vqcb200 as V
from helpers import as_input, max_abs, rand_psi, tol
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DTYPES = [np.complex128, np.complex64]


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [3, 11])
def test_measure_and_post_select_state(dtype, n):
    rng = np.random.default_rng(90 + n)
    psi = as_input(rand_psi(rng, n), dtype)
    for pos in (1, 2, n):
        q = pos - 1
        s = V.StateVector(psi.astype(dtype), dtype=dtype)
        assert abs(V.prob_zero(s, pos) - O.sv_prob_zero(psi, q)) < tol(dtype)
        for reset in (True, False):
            s = V.StateVector(psi.astype(dtype), dtype=dtype)
            i, p = V.measure_inplace(s, pos, auto_reset=reset, rng=np.random.default_rng(7 + pos))
            p0 = O.sv_prob_zero(psi, q)
            u = np.random.default_rng(7 + pos).random()
            ir, pr = (0, p0) if u < p0 else (1, 1 - p0)
            assert i == ir and abs(p - pr) < tol(dtype)
            assert max_abs(s.storage(), O.collapse(psi, q, ir, pr, reset)) < tol(dtype)
        s = V.StateVector(psi.astype(dtype), dtype=dtype)
        out, i, p = V.measure(s, pos, rng=np.random.default_rng(11))
        u = np.random.default_rng(11).random()
        p0 = O.sv_prob_zero(psi, q)
        ir, pr = (0, p0) if u < p0 else (1, 1 - p0)
        assert out.nqubits == n - 1 and i == ir
        assert max_abs(out.storage(), O.take_qubit(psi, q, ir) / np.sqrt(pr)) < tol(dtype)
        for value in (0, 1):
            pv = p0 if value == 0 else 1 - p0
            want = O.take_qubit(psi, q, value) / np.sqrt(pv)
            s = V.StateVector(psi.astype(dtype), dtype=dtype)
            out, nrm = V.post_select(s, pos, value)
            assert abs(nrm - np.sqrt(pv)) < tol(dtype) and max_abs(out.storage(), want) < tol(dtype)
            out, nrm = V.post_select(s, pos, value, keep=True)
            keep_want = O.collapse(psi, q, value, pv, False)
            assert max_abs(out.storage(), keep_want) < tol(dtype)
            nrm = V.post_select_inplace(s, pos, value)
            assert abs(nrm - np.sqrt(pv)) < tol(dtype) and max_abs(s.storage(), keep_want) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_measure_density_matrix(dtype):
    """measure!(rho, pos) (measure.jl:4-16, 69-81): p0 from the diagonal,
    rho <- m rho m^dagger."""
    rng = np.random.default_rng(95)
    n = 5
    psi = as_input(rand_psi(rng, n), dtype)
    rho = V.DensityMatrix(V.StateVector(psi.astype(dtype), dtype=dtype))
    V.apply(V.Depolarizing(2, 0.3), rho)
    ref = O.dm_apply_channel(O.density_matrix(psi), n, [1], V.Depolarizing(2, 0.3).kraus)
    for pos in (2, 5):
        p0 = O.dm_prob_zero(ref, n, pos - 1)
        assert abs(V.prob_zero(rho, pos) - p0) < tol(dtype)
        i, p = V.measure_inplace(rho, pos, auto_reset=True, rng=np.random.default_rng(pos))
        u = np.random.default_rng(pos).random()
        ir, pr = (0, p0) if u < p0 else (1, 1 - p0)
        assert i == ir and abs(p - pr) < tol(dtype)
        m = np.zeros((2, 2), dtype=complex)
        m[0, ir] = 1 / np.sqrt(pr)
        O.dm_apply_gate(ref, n, [pos - 1], m)
        assert max_abs(rho.data(), ref) < tol(dtype)
    assert abs(rho.tr() - 1) < tol(dtype)
