"""GPU parity of quantum channels and Pauli-sum expectations on density
matrices (applygates/apply_qmaps.jl, hamiltonian/expecs_dm/expecs_dm.jl)
against the oracle's restatement, and the oracle against dense NumPy
(rho -> sum_i K_i rho K_i^dagger; tr(H rho)).
Bounds: helpers.py (1e-12 FP64, 1e-5 FP32), asserted as stated against the
oracle run on the same FP32-rounded input; density matrices after channels
and cotangent matrices (not normalised) are compared norm-wise."""
import numpy as np
import pytest

import vqcb200 as V
from helpers import as_input, max_abs, max_rel, rand_psi, rel, rel_scalar, tol
from oracle import dense_np as D
from oracle import gates_ref as GR
from oracle import oracle as O

pytestmark = pytest.mark.gpu
DTYPES = [np.complex128, np.complex64]


def _kraus2(rng):
    """A random 2-qubit channel: 3 Kraus operators, sum K^dagger K = I."""
    A = [rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)) for _ in range(3)]
    S = sum(a.conj().T @ a for a in A)
    w, U = np.linalg.eigh(S)
    inv_sqrt = U @ np.diag(w ** -0.5) @ U.conj().T
    return [a @ inv_sqrt for a in A]


def _dense_channel(rho_vec, n, pos, kraus):
    N = 1 << n
    R = rho_vec.reshape(N, N, order="F")
    out = sum(D.full_operator(n, pos, K) @ R @ D.full_operator(n, pos, K).conj().T for K in kraus)
    return out.reshape(-1, order="F")


@pytest.mark.parametrize("dtype", DTYPES)
def test_channels_on_density_matrix(dtype):
    rng = np.random.default_rng(52)
    n = 6
    psi = rand_psi(rng, n)
    rho = V.DensityMatrix(V.StateVector(psi.astype(dtype), dtype=dtype))
    ref = O.density_matrix(as_input(psi, dtype))
    maps = [V.Depolarizing(1, 0.1), V.AmplitudeDamping(4, 0.3), V.PhaseDamping(6, 0.25),
            V.QuantumMap((2, 5), _kraus2(rng)), V.QuantumMap((6, 1), _kraus2(rng))]
    for m in maps:
        V.apply(m, rho)
        O.dm_apply_channel(ref, n, [p - 1 for p in m.positions], m.kraus)
    assert max_abs(rho.data(), ref) < tol(dtype)
    assert abs(rho.tr() - 1) < tol(dtype)  # trace preserving
    # adjoint and inverse of the supermatrix
    m = V.QuantumMap((3, 2), _kraus2(rng))
    V.apply_dagger(m, rho)
    O.dm_apply_channel(ref, n, [2, 1], m.kraus, mode=1)
    assert max_rel(rho.data(), ref) < tol(dtype)
    m = V.AmplitudeDamping(3, 0.2)
    V.apply(m, rho)
    V.apply_inverse(m, rho)
    O.dm_apply_channel(ref, n, [2], m.kraus, mode=0)
    O.dm_apply_channel(ref, n, [2], m.kraus, mode=2)
    assert max_rel(rho.data(), ref) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_noisy_circuit_on_state(dtype):
    """A circuit with channels (the reference's noisy_circuit: a layer of
    Depolarizing after a variational circuit, test/check_noisy_grad.jl:3-9)
    applied to a StateVector gives a DensityMatrix (apply_qmaps.jl:16)."""
    rng = np.random.default_rng(53)
    n = 5
    gates = []
    for q in range(1, n + 1):
        gates.append(V.RyGate(q, float(rng.uniform(0, 6))))
    for q in range(1, n):
        gates.append(V.CNOTGate(q, q + 1))
    c = V.QCircuit(gates + [V.Depolarizing(q, 0.1) for q in range(1, n + 1)] + [V.HGate(2)])
    psi = rand_psi(rng, n)
    out = V.apply(c, V.StateVector(psi.astype(dtype), dtype=dtype))
    assert isinstance(out, V.DensityMatrix)
    ref = O.density_matrix(as_input(psi, dtype))
    for g in c:
        pos = [p - 1 for p in g.positions]
        if isinstance(g, V.QuantumMap):
            O.dm_apply_channel(ref, n, pos, g.kraus)
        else:
            O.dm_apply_gate(ref, n, pos, g.mat)
    assert max_abs(out.data(), ref) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("n", [3, 7, 10])
def test_dm_pauli_expectation(dtype, n):
    rng = np.random.default_rng(60 + n)
    psi = rand_psi(rng, n)
    rho = V.DensityMatrix(V.StateVector(psi.astype(dtype), dtype=dtype))
    V.apply(V.Depolarizing(1, 0.2), rho)
    ref = O.dm_apply_channel(O.density_matrix(as_input(psi, dtype)), n, [0], V.Depolarizing(1, 0.2).kraus)
    spec = [({1: "X", n: "Y"}, 0.36), ({1: "Z", 2: "Z"}, -0.8), ({2: "Y"}, 0.5 + 0.25j), ({n: "X", 1: "Z"}, 1.3),
            ({}, 0.1)]
    H = V.QubitsOperator(*[V.QubitsTerm(ops, coeff=c) for ops, c in spec])
    terms = [O.make_term({q - 1: o for q, o in ops.items()}, c) for ops, c in spec]
    got = V.expectation(H, rho)
    want = O.dm_expectation(terms, ref, n)
    assert rel_scalar(got, want) < tol(dtype)
    # a pure state: tr(H |psi><psi|) = <psi|H|psi>
    pure = V.DensityMatrix(V.StateVector(psi.astype(dtype), dtype=dtype))
    sv = V.expectation(H, V.StateVector(psi.astype(dtype), dtype=dtype))
    assert rel_scalar(V.expectation(H, pure), sv) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("loss", ["sum", "expectation"])
def test_noisy_dm_gradient(dtype, loss):
    """back_propagate for density matrices with channels (circuitdiff.jl:42-59)
    on the device against the oracle's restatement (which matches central
    differences, test_oracle.py), for the reference's two losses
    (check_noisy_grad.jl: real(sum(rho)) and real(expectation(H, rho)))."""
    rng = np.random.default_rng(81)
    n = 5
    gates = []
    for q in range(1, n + 1):
        gates.append(V.U3Gate(q, *rng.uniform(0, 6, 3), isparas=True))
    for q in range(1, n):
        gates.append(V.CRxGate(q, q + 1, float(rng.uniform(0, 6)), isparas=True))
    maps = [V.Depolarizing(q, 0.1) for q in range(1, n + 1)] + [V.QuantumMap((2, 4), _kraus2(rng))]
    items = gates[:n] + maps[:3] + gates[n:] + maps[3:] + [V.RzGate(3, 0.4, isparas=True)]
    c = V.QCircuit(items)
    N = 1 << n
    rho = V.apply(c, V.DensityMatrix(n, dtype=dtype))
    terms = [({1: "X", n: "Y"}, 0.36), ({2: "Z"}, 0.7), ({1: "Z", 3: "X"}, -0.5)]
    if loss == "sum":
        dmat = np.ones((N, N), dtype=complex)
    else:
        H = D.pauli_sum_matrix(n, [O.make_term({q - 1: o for q, o in ops.items()}, cf) for ops, cf in terms])
        dmat = H.conj().T
    delta = V.DensityMatrix(dmat.astype(dtype), dtype=dtype)
    ref_items = []
    for it in items:
        pos = [p - 1 for p in it.positions]
        if isinstance(it, V.QuantumMap):
            ref_items.append(("map", pos, it.kraus))
        else:
            ref_items.append(("gate", pos, it.mat, it.derivatives()))
    rho_ref = O.zero_state(2 * n)
    for it in ref_items:
        if it[0] == "map":
            rho_ref = O.dm_apply_channel(rho_ref, n, it[1], it[2])
        else:
            O.dm_apply_gate(rho_ref, n, it[1], it[2])
    assert max_abs(rho.data(), rho_ref) < tol(dtype)
    g_ref, d_ref, y_ref = O.dm_circuit_gradient(ref_items, rho_ref, as_input(dmat.reshape(-1, order="F"), dtype), n)
    d, g, y = V.back_propagate(delta, c, rho)
    assert rel(g, g_ref) < tol(dtype)
    assert max_rel(y.data(), y_ref) < tol(dtype)
    assert rel(d.data(), d_ref) < tol(dtype)


def _golden_noisy_items(d):
    """The fixture's noisy circuit, built from its parameters with the
    package's gate and channel constructors (item order as generated)."""
    n, th = int(d["n"]), d["theta"]
    items, k = [], 0
    for q in range(1, n + 1):
        items.append(V.U3Gate(q, float(th[k]), 0.3, -0.2, isparas=[True, False, False]))
        k += 1
    items.append(V.Depolarizing(2, 0.15))
    for q in range(1, n):
        items.append(V.CRxGate(q, q + 1, float(th[k]), isparas=True))
        k += 1
    items.append(V.QuantumMap((4, 1), list(d["kraus2"])))
    for q in range(1, n + 1):
        items.append(V.RyGate(q, float(th[k]), isparas=True))
        k += 1
    items.append(V.AmplitudeDamping(3, 0.25))
    return items


@pytest.mark.parametrize("dtype", DTYPES)
def test_golden_noisy_dm(dtype):
    """Committed fixture (oracle, checked against dense NumPy and central
    differences when generated): noisy circuit on a density matrix, tr(H rho)
    and the DM pullback (apply_qmaps.jl, expecs_dm.jl, circuitdiff.jl:42-75)."""
    from helpers import golden
    d = golden("noisy_dm_n4")
    n = int(d["n"])
    items = _golden_noisy_items(d)
    assert len(items) == int(d["nitems"])
    for i, it in enumerate(items):
        if int(d["kind%d" % i]) == 0:
            assert np.abs(it.mat - d["mat%d" % i]).max() < 1e-14
    rho = V.DensityMatrix(V.StateVector(d["psi"].astype(dtype), dtype=dtype))
    c = V.QCircuit(items)
    V.apply(c, rho)
    assert max_abs(rho.data(), d["rho"]) < tol(dtype)
    H = V.QubitsOperator(*[V.QubitsTerm({q + 1: "IXZY"[((int(x) >> q) & 1) | (((int(z) >> q) & 1) << 1)]
                                          for q in range(n) if ((int(x) | int(z)) >> q) & 1}, coeff=complex(cf))
                            for x, z, cf in zip(d["xmask"], d["zmask"], d["coeff"])])
    e = V.expectation(H, rho)
    assert rel_scalar(e, d["energy"]) < tol(dtype)
    terms = [O.make_term({q: "IXZY"[((int(x) >> q) & 1) | (((int(z) >> q) & 1) << 1)]
                          for q in range(n) if ((int(x) | int(z)) >> q) & 1}, complex(cf))
             for x, z, cf in zip(d["xmask"], d["zmask"], d["coeff"])]
    dmat = D.pauli_sum_matrix(n, terms).conj().T
    delta = V.DensityMatrix(dmat.astype(dtype), dtype=dtype)
    dd, g, _ = V.back_propagate(delta, c, rho)
    assert rel(g, d["grads"]) < tol(dtype)
    assert rel(dd.data(), d["delta_in"]) < tol(dtype)
