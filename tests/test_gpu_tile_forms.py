"""GPU parity of the FP32 tile body's op variants against the oracle.

The FP32 body keeps qubit 0 inside each thread's packed registers (the lane
bit) and compiles one-qubit ops per matrix form (general, RX-like, real,
diagonal, swap), per target kind (lane bit or another register bit) and per
register control (none, one control at |1> on the lane bit or another
register bit, any other pattern through an amplitude mask); controls on
thread bits and on qubits outside the tile are tested at run time.  These
circuits put every form on qubit 0, on low, middle and high qubits, with
controls on each kind of bit, controls on |0>, two controls, dense two-qubit
gates and diagonal gates, at n = 14 (tile of 12 qubits, 2 qubits outside).  Each case runs
through the generic tile kernel (VQC_JIT=off), the kernels compiled at run
time for each pass structure (VQC_JIT=on) and their interpreted fallback on
the same packed plan (VQC_JIT=interp).
Bounds: helpers.py (FP32 1e-5 on normalised states and norm-wise on gradients,
FP64 1e-12), asserted as stated against the oracle run on the same FP32-rounded
input.
"""
import numpy as np
import pytest

import vqcb200 as V
from helpers import as_input, max_abs, rand_psi, rel, rel_scalar, tol
from oracle import gates_ref as GR
from oracle import oracle as O

pytestmark = pytest.mark.gpu
JIT = ["off", "on", "interp"]

N = 14
ONE_Q = [1, 2, 3, 7, 12, 14]  # 1-based: qubit 0 (lane bit), low, middle, high, outside the first tile
PAIRS = [(1, 2), (2, 1), (1, 9), (9, 1), (3, 4), (4, 3), (13, 2), (2, 13), (14, 1), (5, 12), (12, 5)]


def _ctrl0(V_):
    """|0><0| (x) V + |1><1| (x) I with the control on the gate's first position."""
    d = V_.shape[0]
    M = np.zeros((2 * d, 2 * d), dtype=complex)
    for a in range(d):
        M[2 * a + 1, 2 * a + 1] = 1
        for b in range(d):
            M[2 * a, 2 * b] = V_[a, b]
    return M


def _rx(t):
    c, s = np.cos(t / 2), np.sin(t / 2)
    return np.array([[c, -1j * s], [-1j * s, c]]), 0.5 * np.array([[-s, -1j * c], [-1j * c, -s]])


def one_qubit_gates(rng, q, params):
    t = float(rng.uniform(0, 2 * np.pi))
    return [
        V.U3Gate(q, t, 0.4 * t, -1.1, isparas=params),
        V.RxGate(q, t, isparas=params),
        V.RyGate(q, 0.7 * t, isparas=params),
        V.RzGate(q, 1.3 * t, isparas=params),
        V.XGate(q),
        V.HGate(q),
        V.SGate(q),
        V.YGate(q),
    ]


def controlled_gates(rng, c, t, params):
    th = float(rng.uniform(0, 2 * np.pi))
    U, dU = _rx(th)
    gs = [
        V.CRxGate(c, t, th, isparas=params),
        V.CRyGate(c, t, 0.5 * th, isparas=params),
        V.CNOTGate(c, t),
        V.CONTROLGate((c, t), GR.random_unitary(1, rng)),
        V.Gate((c, t), _ctrl0(U), (th,), params, [_ctrl0(dU) - _ctrl0(np.zeros((2, 2)))], name="C0Rx"),
    ]
    return gs


def build(rng, params):
    gates = []
    for q in ONE_Q:
        gates += one_qubit_gates(rng, q, params)
    for c, t in PAIRS:
        gates += controlled_gates(rng, c, t, params)
    # two controls: on register/thread bits, qubit 0, outside the tile
    gates += [V.TOFFOLIGate(1, 2, 3), V.TOFFOLIGate(2, 9, 1), V.TOFFOLIGate(13, 1, 5), V.TOFFOLIGate(4, 14, 2)]
    # dense two-qubit and diagonal gates
    for a, b in [(1, 2), (2, 1), (1, 10), (3, 12), (14, 2)]:
        gates.append(V.QuantumGate((a, b), GR.random_unitary(2, rng)))
    gates += [V.CPHASEGate(1, 2, 0.3, isparas=params), V.CZGate(1, 13), V.CCPHASEGate(1, 6, 14, 1.1, isparas=params)]
    order = rng.permutation(len(gates))
    return [gates[i] for i in order]


def to_ref(gates):
    return [([p - 1 for p in g.positions], g.mat, g.derivatives()) for g in gates]


@pytest.mark.parametrize("jit", JIT)
def test_f32_forms_forward(jit, monkeypatch):
    monkeypatch.setenv("VQC_JIT", jit)
    rng = np.random.default_rng(404)
    gates = build(rng, False) + build(rng, False)
    psi = rand_psi(rng, N)
    s = V.StateVector(psi.astype(np.complex64), dtype=np.complex64)
    V.apply(V.QCircuit(gates), s, fuse=True)
    want = O.apply_circuit(as_input(psi, np.complex64), to_ref(gates), nthreads=4)
    assert max_abs(s.storage(), want) < tol(np.complex64)


@pytest.mark.parametrize("jit", JIT)
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_f32_forms_gradient(dtype, jit, monkeypatch):
    monkeypatch.setenv("VQC_JIT", jit)
    rng = np.random.default_rng(405)
    gates = build(rng, True)
    c = V.QCircuit(gates)
    psi0 = as_input(rand_psi(rng, N), dtype)
    target = as_input(rand_psi(rng, N), dtype)
    g_ref, d_ref = O.circuit_gradient(to_ref(gates), psi0, target, nthreads=4)
    y = c * V.StateVector(psi0.astype(dtype), dtype=dtype)
    delta, g, yin = V.back_propagate(V.StateVector(target.astype(dtype), dtype=dtype), c, y)
    assert rel(g, g_ref) < tol(dtype)
    assert max_abs(yin.storage(), psi0) < tol(dtype)
    assert max_abs(delta.storage(), d_ref) < tol(dtype)


@pytest.mark.parametrize("jit", JIT)
@pytest.mark.parametrize("n", [9, 10, 11])
def test_f32_small_tiles(n, jit, monkeypatch):
    """Tiles of 9-11 qubits (fewer threads per tile, thread tables of < 8 bits)."""
    monkeypatch.setenv("VQC_JIT", jit)
    rng = np.random.default_rng(406 + n)
    gates = []
    for q in [1, 2, n // 2, n]:
        gates += one_qubit_gates(rng, q, True)
    for c, t in [(1, 2), (2, 1), (n, 1), (1, n), (3, n - 1)]:
        gates += controlled_gates(rng, c, t, True)
    gates.append(V.QuantumGate((1, n), GR.random_unitary(2, rng)))
    psi = as_input(rand_psi(rng, n), np.complex64)
    s = V.StateVector(psi.astype(np.complex64), dtype=np.complex64)
    V.apply(V.QCircuit(gates), s, fuse=True)
    want = O.apply_circuit(psi.copy(), to_ref(gates), nthreads=4)
    assert max_abs(s.storage(), want) < tol(np.complex64)
    target = as_input(rand_psi(rng, n), np.complex64)
    g_ref, _ = O.circuit_gradient(to_ref(gates), psi, target, nthreads=4)
    c = V.QCircuit(gates)
    y = c * V.StateVector(psi.astype(np.complex64), dtype=np.complex64)
    _, g, _ = V.back_propagate(V.StateVector(target.astype(np.complex64), dtype=np.complex64), c, y)
    assert rel(g, g_ref) < tol(np.complex64)


@pytest.mark.parametrize("jit", JIT)
def test_f32_headline_shape(jit, monkeypatch):
    """The benchmark's circuit family (RX, RY, RZ on every qubit + CRX chain,
    XXZ energy and gradient) at n = 18 through both kernel kinds."""
    monkeypatch.setenv("VQC_JIT", jit)
    from vqcb200 import workloads as W
    n, layers = 18, 3
    rng = np.random.default_rng(407)
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    spec = W.rxyz_crx_spec(n, layers, th)
    hspec = W.xxz_spec(n, 0.5)
    e, g = V.energy_and_gradient(W.to_operator(hspec), W.to_circuit(spec), V.StateVector(n, dtype=np.complex64))
    e64, g64 = V.energy_and_gradient(W.to_operator(hspec), W.to_circuit(spec), V.StateVector(n, dtype=np.complex128))
    assert rel_scalar(e, e64) < tol(np.complex64)
    assert rel(g, g64) < tol(np.complex64)


@pytest.mark.parametrize("jit", JIT)
def test_f32_partials_not_anti_hermitian(jit, monkeypatch):
    """Parameters whose D = U^dagger dU is not anti-Hermitian (dU supplied
    freely: full, diagonal-only and off-diagonal-only D, a gate mixing such a
    D with an anti-Hermitian one, and the same under a control on |0>) keep
    the full reduced-matrix accumulation; unitary families take the
    four-value anti-Hermitian projection.  Both against the oracle."""
    monkeypatch.setenv("VQC_JIT", jit)
    rng = np.random.default_rng(408)
    Z = np.zeros((2, 2))
    gates = []
    for q in ONE_Q:
        U = GR.random_unitary(1, rng)
        Dfull = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
        Ddiag = np.diag(rng.standard_normal(2))
        Doff = np.array([[0, 0.6], [0.6, 0]])
        Dah = -0.5j * np.array([[0, 1], [1, 0]])
        gates += [
            V.Gate((q,), U, (0.3,), True, [U @ Dfull], name="Dfull"),
            V.Gate((q,), U, (0.2,), True, [U @ Ddiag], name="Ddiag"),
            V.Gate((q,), U, (0.1,), True, [U @ Doff], name="Doff"),
            V.Gate((q,), U, (0.4, 0.5), True, [U @ Dah, U @ Doff], name="Dmixed"),
        ]
        gates += one_qubit_gates(rng, q, True)[:4]
    for c, t in PAIRS[:6]:
        U = GR.random_unitary(1, rng)
        Dfull = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
        gates.append(V.Gate((c, t), _ctrl0(U), (0.7,), True, [_ctrl0(U @ Dfull) - _ctrl0(Z)], name="C0Dfull"))
        gates += controlled_gates(rng, c, t, True)[:2]
    gates = [gates[i] for i in rng.permutation(len(gates))]
    c = V.QCircuit(gates)
    psi0 = as_input(rand_psi(rng, N), np.complex64)
    target = as_input(rand_psi(rng, N), np.complex64)
    g_ref, d_ref = O.circuit_gradient(to_ref(gates), psi0, target, nthreads=4)
    y = c * V.StateVector(psi0.astype(np.complex64), dtype=np.complex64)
    delta, g, _ = V.back_propagate(V.StateVector(target.astype(np.complex64), dtype=np.complex64), c, y)
    assert rel(g, g_ref) < tol(np.complex64)
    assert max_abs(delta.storage(), d_ref) < tol(np.complex64)
