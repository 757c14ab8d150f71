"""GPU parity of the fused tile engine (passes of many gates per HBM round
trip) against the oracle: forward circuits and the fused reverse sweep, on
states large enough for the tile path (n >= 12), every gate structure the
planner distinguishes (dense 1q, diagonal, controlled 1q/2q with tile and
non-tile controls, dense 2q, non-fusable 3-5q), both precisions.
Bounds: helpers.py (1e-12 FP64, 1e-5 FP32), asserted as stated; FP32 results
are compared against the oracle run on the same FP32-rounded input."""
import numpy as np
import pytest

import vqcb200 as V
from helpers import as_input, max_abs, max_rel, rand_psi, rel, rel_scalar, tol
from oracle import gates_ref as GR
from oracle import oracle as O
from vqcb200 import workloads as W

pytestmark = pytest.mark.gpu
DTYPES = [np.complex128, np.complex64]


def random_mixed_circuit(rng, n, ngates, with_wide=True, params=True):
    """(product circuit, oracle gate list) with seeded random gates."""
    prod, ref = [], []
    for _ in range(ngates):
        kind = rng.integers(0, 15 if with_wide else 12)
        q = [int(x) + 1 for x in rng.choice(n, 5, replace=False)]
        t = float(rng.uniform(0, 2 * np.pi))
        if kind == 0:
            g = V.U3Gate(q[0], t, 0.3 * t, -0.7, isparas=params)
        elif kind == 1:
            g = V.RzGate(q[0], t, isparas=params)
        elif kind == 2:
            g = V.RxGate(q[0], t, isparas=params)
        elif kind == 3:
            g = V.CNOTGate(q[0], q[1])
        elif kind == 4:
            g = V.CZGate(q[0], q[1])
        elif kind == 5:
            g = V.CRxGate(q[0], q[1], t, isparas=params)
        elif kind == 6:
            g = V.TOFFOLIGate(q[0], q[1], q[2])
        elif kind == 7:
            g = V.FREDKINGate(q[0], q[1], q[2])
        elif kind == 8:
            g = V.CPHASEGate(q[0], q[1], t, isparas=params)
        elif kind == 9:
            g = V.iSWAPGate(q[0], q[1])
        elif kind == 10:
            g = V.QuantumGate((q[0], q[1]), GR.random_unitary(2, rng))
        elif kind == 11:
            g = V.HGate(q[0])
        elif kind == 12:
            g = V.QuantumGate((q[0], q[1], q[2]), GR.random_unitary(3, rng))
        elif kind == 13:
            g = V.QuantumGate(tuple(q[:4]), GR.random_unitary(4, rng))
        else:
            g = V.CCPHASEGate(q[0], q[1], q[2], t, isparas=params)
        prod.append(g)
        ref.append(([p - 1 for p in g.positions], g.mat, g.derivatives()))
    return V.QCircuit(prod), ref


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [12, 14])
def test_fused_forward_mixed(dtype, n):
    rng = np.random.default_rng(1000 + n)
    c, ref = random_mixed_circuit(rng, n, 120)
    psi = rand_psi(rng, n)
    s = V.StateVector(psi.astype(dtype), dtype=dtype)
    V.apply(c, s, fuse=True)
    want = O.apply_circuit(as_input(psi, dtype), ref, nthreads=4)
    assert max_abs(s.storage(), want) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_equals_unfused_config_shapes(dtype):
    # the benchmark's circuit family at a small size: 4 layers RX/RY/RZ + CRX chain
    n, layers = 15, 4
    rng = np.random.default_rng(3)
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    c = W.to_circuit(W.rxyz_crx_spec(n, layers, th))
    a = V.StateVector(n, dtype=dtype)
    b = V.StateVector(n, dtype=dtype)
    V.apply(c, a, fuse=True)
    V.apply(c, b, fuse=False)
    ref = O.apply_circuit(O.zero_state(n), O.from_spec(W.rxyz_crx_spec(n, layers, th)), nthreads=4)
    assert max_abs(a.storage(), ref) < tol(dtype)
    assert max_abs(b.storage(), ref) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_u3_cz_toffoli(dtype):
    n, layers = 16, 5
    spec = W.u3_cz_toffoli_spec(n, layers, 77)
    s = V.StateVector(n, dtype=dtype)
    V.apply(W.to_circuit(spec), s)
    ref = O.apply_circuit(O.zero_state(n), O.from_spec(spec), nthreads=4)
    assert max_abs(s.storage(), ref) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_gradient_mixed_gates(dtype):
    """The fused reverse sweep (merged 1q blocks, controlled 1q with tile and
    non-tile controls, parameterised diagonal gates, standalone wide gates)
    against the oracle's restatement of circuitdiff.jl."""
    n = 13
    rng = np.random.default_rng(21)
    c, ref = random_mixed_circuit(rng, n, 90)
    psi0 = as_input(rand_psi(rng, n), dtype)
    target = as_input(rand_psi(rng, n), dtype)
    g_ref, d_ref = O.circuit_gradient(ref, psi0, target, nthreads=4)
    y = c * V.StateVector(psi0.astype(dtype), dtype=dtype)
    delta, g, yin = V.back_propagate(V.StateVector(target.astype(dtype), dtype=dtype), c, y)
    assert rel(g, g_ref) < tol(dtype)
    assert max_abs(yin.storage(), psi0) < tol(dtype)
    assert max_abs(delta.storage(), d_ref) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_energy_gradient_xxz(dtype):
    n, layers = 14, 3
    rng = np.random.default_rng(22)
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    spec = W.rxyz_crx_spec(n, layers, th)
    hspec = W.xxz_spec(n, 0.5)
    e, g = V.energy_and_gradient(W.to_operator(hspec), W.to_circuit(spec), V.StateVector(n, dtype=dtype))
    e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(hspec), O.zero_state(n), nthreads=8)
    assert rel_scalar(e, e_ref) < tol(dtype)
    assert rel(g, g_ref) < tol(dtype)


def test_fused_deterministic():
    n, layers = 14, 2
    rng = np.random.default_rng(23)
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    c = W.to_circuit(W.rxyz_crx_spec(n, layers, th))
    H = W.to_operator(W.xxz_spec(n, 0.5))
    r1 = V.energy_and_gradient(H, c, V.StateVector(n, dtype=np.complex64))
    r2 = V.energy_and_gradient(H, c, V.StateVector(n, dtype=np.complex64))
    assert r1[0] == r2[0]
    assert np.array_equal(r1[1], r2[1])


@pytest.mark.parametrize("dtype", DTYPES)
def test_fused_density_matrix_circuit(dtype):
    """rho <- U rho U^dagger through the tile engine (U on the row qubits and
    conj(U) on the column qubits as gates of the 2n-qubit vector)."""
    n, layers = 7, 3
    rng = np.random.default_rng(31)
    psi = rand_psi(rng, n)
    spec = W.u3_cnot_spec(n, layers, 5) + [("toffoli", (1, 4, 6), ()), ("cz", (2, 7), ()),
                                            ("crx", (5, 3), (0.7,))]
    rho = V.DensityMatrix(V.StateVector(psi.astype(dtype), dtype=dtype))
    V.apply(W.to_circuit(spec), rho)
    ref = O.density_matrix(as_input(psi, dtype))
    O.dm_apply_circuit(ref, n, O.from_spec(spec))
    assert max_abs(rho.data(), ref) < tol(dtype)
    red = V.partial_tr(rho, [6, 7])
    assert max_abs(red.reshape(-1, order="F"), O.dm_ptrace(ref, n, [5, 6])) < tol(dtype)
    assert max_abs(V.probabilities(rho), O.dm_probs(ref, n)) < tol(dtype)
    # fused and one-by-one agree
    rho2 = V.DensityMatrix(V.StateVector(psi.astype(dtype), dtype=dtype))
    V.apply(W.to_circuit(spec), rho2, fuse=False)
    assert max_abs(rho.data(), rho2.data()) < tol(dtype)
