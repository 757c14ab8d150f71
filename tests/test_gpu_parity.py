"""GPU parity tests: the sm_100a engine, called through the C ABI (via the
ctypes host mirror), against the CPU oracle and the golden fixtures, on the
same seeded inputs.  Tolerances: see helpers.py (1e-12 FP64, 1e-5 FP32)."""
import numpy as np
import pytest

import vqcb200 as V
from helpers import as_input, golden, max_abs, max_rel, rand_psi, rel, rel_scalar, tol
from oracle import gates_ref as GR
from oracle import oracle as O
from vqcb200 import workloads as W

pytestmark = pytest.mark.gpu
DTYPES = [np.complex128, np.complex64]


def sv(arr, dtype):
    return V.StateVector(np.asarray(arr, dtype=dtype), dtype=dtype)


# ----------------------------------------------------------------------------- gates
@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_gates(dtype):
    d = golden("gates_n7")
    for i in range(int(d["ncases"])):
        pos = [int(q) + 1 for q in d["pos%d" % i]]
        s = sv(d["psi"], dtype)
        V.apply(V.QuantumGate(pos, d["U%d" % i]), s)
        assert max_abs(s.storage(), d["out%d" % i]) < tol(dtype), (i, pos)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("k", [1, 2, 3])
def test_every_position_pattern(dtype, k):
    # test/check_gateop.jl:1-67: every target pattern, random unitaries
    rng = np.random.default_rng(100 + k)
    n = 9 if k < 3 else 7
    psi = rand_psi(rng, n)
    inp = as_input(psi, dtype)
    import itertools
    for pos in itertools.permutations(range(n), k):
        if k == 3 and rng.random() > 0.3:
            continue
        U = GR.random_unitary(k, rng)
        s = sv(psi, dtype)
        V.apply(V.QuantumGate([q + 1 for q in pos], U), s)
        ref = O.apply_gate(inp.copy(), list(pos), U)
        assert max_abs(s.storage(), ref) < tol(dtype), pos


@pytest.mark.parametrize("dtype", DTYPES)
def test_wide_gates_large_state(dtype):
    rng = np.random.default_rng(7)
    n = 20
    psi = rand_psi(rng, n)
    s = sv(psi, dtype)
    ref = as_input(psi, dtype)
    for k in (4, 5, 1, 2):
        pos = [int(q) for q in rng.choice(n, k, replace=False)]
        U = GR.random_unitary(k, rng)
        V.apply(V.QuantumGate([q + 1 for q in pos], U), s)
        O.apply_gate(ref, pos, U, nthreads=8)
    assert max_abs(s.storage(), ref) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_specialised_gates_and_adjoints(dtype):
    # test/check_gateop.jl:69-168: each specialised gate (and its adjoint)
    rng = np.random.default_rng(11)
    n = 8
    psi = rand_psi(rng, n)
    inp = as_input(psi, dtype)
    gs = [V.XGate(3), V.YGate(1), V.ZGate(8), V.HGate(5), V.SGate(2), V.TGate(7), V.PHASEGate(4, 0.7),
          V.CNOTGate(1, 2), V.CNOTGate(6, 3), V.CZGate(2, 8), V.CRxGate(5, 1, 0.4), V.CRyGate(2, 7, 1.1),
          V.CRzGate(8, 4, -0.3), V.CPHASEGate(3, 6, 0.9), V.SWAPGate(1, 8), V.iSWAPGate(4, 2),
          V.TOFFOLIGate(1, 5, 3), V.TOFFOLIGate(8, 2, 4), V.FREDKINGate(2, 6, 1), V.CCPHASEGate(7, 3, 5, 1.3),
          V.CONTROLGate((3, 4), GR.random_unitary(1, rng))]
    for g in gs:
        for gg in (g, g.adjoint()):
            s = sv(psi, dtype)
            V.apply(gg, s)
            ref = O.apply_gate(inp.copy(), [q - 1 for q in gg.positions], gg.mat)
            assert max_abs(s.storage(), ref) < tol(dtype), gg


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("fuse", [True, False])
def test_golden_circuit_u3_cz_toffoli(dtype, fuse):
    d = golden("u3_cz_toffoli_n10")
    spec = W.u3_cz_toffoli_spec(int(d["n"]), int(d["layers"]), int(d["seed"]))
    s = V.StateVector(int(d["n"]), dtype=dtype)
    V.apply(W.to_circuit(spec), s, fuse=fuse)
    assert max_abs(s.storage(), d["out"]) < tol(dtype)


def test_circuit_mul_copies():
    rng = np.random.default_rng(2)
    psi = V.StateVector(rand_psi(rng, 5))
    c = V.QCircuit([V.HGate(1), V.CNOTGate(1, 2)])
    before = psi.storage()
    out = c * psi
    assert np.array_equal(psi.storage(), before)
    assert max_abs(out.storage(), O.apply_circuit(before.copy(), [((0,), GR.h(0)[1]), ((0, 1), GR.cnot(0, 1)[1])])) < 1e-12


def test_gate_errors():
    s = V.StateVector(4)
    with pytest.raises(NotImplementedError):
        V.apply(V.QuantumGate(tuple(range(1, 7)), np.eye(64)), V.StateVector(6))
    with pytest.raises(ValueError):
        V.apply(V.XGate(5), s)
    with pytest.raises(ValueError):
        V.QuantumGate((1, 1), np.eye(4))
    # the C ABI itself rejects bad positions and k > 5
    import ctypes
    lib = V.load()
    pos = (ctypes.c_int * 2)(0, 0)
    m = np.eye(4, dtype=np.complex128).view(np.float64).ravel()
    assert lib.vqc_apply_gate(s.handle, 2, pos, m.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == -1
    pos6 = (ctypes.c_int * 6)(*range(6))
    s6 = V.StateVector(6)  # keep a reference: the handle lives as long as the object
    assert lib.vqc_apply_gate(s6.handle, 6, pos6, m.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == -4


def test_single_qubit_register():
    s = V.StateVector(1)
    V.apply(V.XGate(1), s)
    assert np.array_equal(s.storage(), np.array([0, 1], dtype=complex))


# ----------------------------------------------------------------------------- states
@pytest.mark.parametrize("dtype", DTYPES)
def test_state_basics(dtype):
    rng = np.random.default_rng(4)
    a, b = rand_psi(rng, 12), rand_psi(rng, 12)
    x, y = sv(a * 2, dtype), sv(b, dtype)
    ai, bi = as_input(a * 2, dtype), as_input(b, dtype)
    assert rel_scalar(x.norm(), np.linalg.norm(ai)) < tol(dtype)
    assert rel_scalar(x.dot(y), np.vdot(ai, bi)) < tol(dtype)
    z = x.copy()
    assert np.array_equal(z.storage(), x.storage())
    z.reset()
    e = np.zeros(1 << 12, dtype=dtype)
    e[0] = 1
    assert np.array_equal(z.storage(), e)
    w = x.astype(np.complex128 if dtype == np.complex64 else np.complex64)
    assert max_abs(w.storage(), x.storage()) < 1e-6


# ----------------------------------------------------------------------------- expectation
def _pauli_from_golden(d):
    ops = []
    for x, z, c in zip(d["xmask"], d["zmask"], d["coeff"]):
        spec = {}
        for q in range(int(d["n"])):
            b = ((int(x) >> q) & 1, (int(z) >> q) & 1)
            if b != (0, 0):
                spec[q + 1] = {(1, 0): "X", (0, 1): "Z", (1, 1): "Y"}[b]
        ops.append(V.QubitsTerm(spec, coeff=c))
    return V.QubitsOperator(*ops)


@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_pauli_sum(dtype):
    d = golden("pauli_sum_n9")
    H = _pauli_from_golden(d)
    s = sv(d["psi"], dtype)
    e = V.expectation(H, s)
    assert rel_scalar(e, d["energy"]) < tol(dtype)
    hp = V.apply_operator(H, s)
    assert max_rel(hp.storage(), d["hpsi"]) < tol(dtype)
    # two-state form <phi|H|psi>, against the oracle on the device's inputs
    rng = np.random.default_rng(8)
    phi = rand_psi(rng, int(d["n"]))
    terms = [O.make_term({q: "IXZY"[((int(x) >> q) & 1) | (((int(z) >> q) & 1) << 1)]
                          for q in range(int(d["n"])) if ((int(x) | int(z)) >> q) & 1}, complex(c))
             for x, z, c in zip(d["xmask"], d["zmask"], d["coeff"])]
    ref = O.expectation(terms, as_input(d["psi"], dtype), vc=as_input(phi, dtype))
    assert rel_scalar(V.expectation(sv(phi, dtype), H, s), ref) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_dense_key_expectation_and_apply(dtype):
    rng = np.random.default_rng(9)
    n = 10
    psi, phi = rand_psi(rng, n), rand_psi(rng, n)
    pin, fin = as_input(psi, dtype), as_input(phi, dtype)
    for k in range(1, 6):
        pos = [int(q) for q in rng.choice(n, k, replace=False)]
        M = GR.random_unitary(k, rng) + 0.2 * rng.standard_normal((1 << k, 1 << k))
        g = V.QuantumGate([q + 1 for q in pos], M)
        e1 = V.expectation(g, sv(psi, dtype))
        e2 = V.expectation(sv(phi, dtype), g, sv(psi, dtype))
        assert rel_scalar(e1, O.expect_dense(pin, pos, M)) < tol(dtype)
        assert rel_scalar(e2, O.expect_dense(pin, pos, M, vc=fin)) < tol(dtype)
        out = V.apply_operator(g, sv(psi, dtype))
        ref = np.zeros_like(pin)
        O.apply_gate_add(pin, ref, pos, M)
        assert max_rel(out.storage(), ref) < tol(dtype)


def test_non_pauli_operator_matches_key_matrices():
    # heisenberg-style sigma+ sigma- terms (spin_hamiltonians.jl:7-22) and a
    # general 2x2 operator: expanded to Pauli strings on the host, one pass on
    # the device; checked against the oracle's per-key dense matrices.
    rng = np.random.default_rng(12)
    n = 8
    psi = rand_psi(rng, n)
    A = rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))
    H = V.QubitsOperator(V.QubitsTerm({1: "+", 2: "-"}, coeff=2.0), V.QubitsTerm({1: "-", 2: "+"}, coeff=2.0),
                         V.QubitsTerm({3: A, 6: "Z"}, coeff=0.4 + 0.1j), V.QubitsTerm({}, coeff=0.25))
    oterms = [O.make_term({q - 1: (o if isinstance(o, str) else o) for q, o in zip(t.positions, t.ops)}, t.coeff)
              for t in H.terms]
    e = V.expectation(H, V.StateVector(psi))
    assert rel_scalar(e, O.expectation(oterms, psi)) < 1e-12
    out = V.apply_operator(H, V.StateVector(psi))
    assert max_rel(out.storage(), O.apply_operator(oterms, psi)) < 1e-12


# ----------------------------------------------------------------------------- gradients
@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_hea_tfim_gradient(dtype):
    d = golden("hea_tfim_n12")
    n = int(d["n"])
    c = W.to_circuit(W.hea_spec(n, int(d["layers"]), d["theta"]))
    H = W.to_operator(W.tfim_spec(n, float(d["g"])))
    e, g = V.energy_and_gradient(H, c, V.StateVector(n, dtype=dtype))
    assert rel_scalar(e, d["energy"]) < tol(dtype)
    assert rel(g, d["grads"]) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_rxyz_crx_xxz_gradient(dtype):
    d = golden("rxyz_crx_xxz_n8")
    n = int(d["n"])
    c = W.to_circuit(W.rxyz_crx_spec(n, int(d["layers"]), d["theta"]))
    H = W.to_operator(W.xxz_spec(n, 0.5))
    psi0 = V.StateVector(n, dtype=dtype)
    e, g = V.energy_and_gradient(H, c, psi0)
    assert rel_scalar(e, d["energy"]) < tol(dtype)
    assert rel(g, d["grads"]) < tol(dtype)
    # psi0 is not modified
    e0 = np.zeros(1 << n)
    e0[0] = 1
    assert np.array_equal(psi0.storage(), e0.astype(dtype))


def test_back_propagate_matches_oracle():
    # loss = real(dot(target, circuit * psi0)) (test/circuitgrad.jl:7-21): cotangent = target
    rng = np.random.default_rng(13)
    n, layers = 7, 3
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    spec = W.rxyz_crx_spec(n, layers, th)
    spec.insert(3, ("u3", (2,), (0.3, 1.2, -0.4)))
    c = W.to_circuit(spec)
    psi0 = rand_psi(rng, n)
    target = rand_psi(rng, n)
    gates = O.from_spec(spec)
    ref_g, ref_d = O.circuit_gradient(gates, psi0, target)
    y = c * V.StateVector(psi0)
    delta, g, yin = V.back_propagate(V.StateVector(target), c, y)
    assert rel(g, ref_g) < 1e-12
    assert max_abs(yin.storage(), psi0) < 1e-12
    assert max_abs(delta.storage(), ref_d) < 1e-12


def test_gradient_matches_finite_differences_on_device():
    rng = np.random.default_rng(14)
    n, layers = 6, 2
    th = rng.uniform(0, 2 * np.pi, layers * 2 * n)
    H = W.to_operator(W.tfim_spec(n, 0.9))
    e, g = V.energy_and_gradient(H, W.to_circuit(W.hea_spec(n, layers, th)), V.StateVector(n))
    h = 1e-4
    fd = []
    for j in range(th.size):
        vals = []
        for sgn in (1, -1):
            t2 = th.copy()
            t2[j] += sgn * h
            s = W.to_circuit(W.hea_spec(n, layers, t2)) * V.StateVector(n)
            vals.append(V.expectation(H, s).real)
        fd.append((vals[0] - vals[1]) / (2 * h))
    assert np.abs(g - np.array(fd)).max() < 1e-6


# ----------------------------------------------------------------------------- density matrices
@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_density_matrix(dtype):
    d = golden("dm_u3_cnot_n5")
    n = int(d["n"])
    rho = V.DensityMatrix(sv(d["psi"], dtype))
    V.apply(W.to_circuit(W.u3_cnot_spec(n, int(d["layers"]), int(d["seed"]))), rho)
    assert max_abs(rho.data(), d["rho"]) < tol(dtype)
    red = V.partial_tr(rho, [int(s) + 1 for s in d["sites"]])
    assert max_abs(red.reshape(-1, order="F"), d["ptrace"]) < tol(dtype)
    assert max_abs(V.probabilities(rho), d["probs"]) < tol(dtype)
    assert abs(rho.tr() - 1) < tol(dtype)


@pytest.mark.parametrize("sites", [[1, 2], [2, 5], [6, 3]])
def test_ptrace_state_vs_dm(sites):
    # test/check_utility.jl:3-13
    rng = np.random.default_rng(sum(sites))
    psi = rand_psi(rng, 6)
    rho = V.DensityMatrix(V.StateVector(psi))
    red = V.partial_tr(rho, sites)
    ref = O.sv_ptrace(psi, [s - 1 for s in sites])
    assert max_abs(red.reshape(-1, order="F"), ref) < 1e-12


def test_dm_three_qubit_gate_two_pass_path():
    rng = np.random.default_rng(15)
    n = 5
    psi = rand_psi(rng, n)
    U = GR.random_unitary(3, rng)
    rho = V.DensityMatrix(V.StateVector(psi))
    V.apply(V.QuantumGate((2, 5, 1), U), rho)
    ref = O.density_matrix(psi)
    O.dm_apply_gate(ref, n, [1, 4, 0], U)
    assert max_abs(rho.data(), ref) < 1e-12


def test_ptrace_errors_and_edges():
    rho = V.DensityMatrix(3)
    with pytest.raises(ValueError):
        V.partial_tr(rho, [1, 1])
    with pytest.raises(ValueError):
        V.partial_tr(rho, [4])
    assert abs(V.partial_tr(rho, [1, 2, 3]) - 1) < 1e-15
    red = V.partial_tr(rho, [2])
    assert red.shape == (4, 4) and abs(red[0, 0] - 1) < 1e-15
