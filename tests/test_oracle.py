"""CPU tests of the oracle itself: it is pinned by the reference's own
relational and known-answer tests (restated here), by the independent dense
checker, and by the committed golden fixtures.  No GPU."""
import numpy as np
import pytest

from helpers import golden, max_abs, rand_psi
from oracle import dense_np as D
from oracle import gates_ref as GR
from oracle import oracle as O


def test_threaded_equals_serial():
    # test/check_gateop.jl:1-67: threaded apply! == apply_serial! for 1/2/3q
    rng = np.random.default_rng(1)
    n = 13
    psi = rand_psi(rng, n)
    for k in range(1, 6):
        for _ in range(3):
            pos = list(rng.choice(n, k, replace=False))
            U = GR.random_unitary(k, rng)
            a = O.apply_gate(psi.copy(), pos, U, nthreads=1)
            b = O.apply_gate(psi.copy(), pos, U, nthreads=7)
            assert np.array_equal(a, b)


@pytest.mark.parametrize("k", [1, 2, 3, 4, 5])
def test_gate_vs_dense(k):
    # test/check_high_qubit_gate.jl: kernels vs the dense matrix, permuted positions
    rng = np.random.default_rng(10 + k)
    n = 7
    psi = rand_psi(rng, n)
    for _ in range(6):
        pos = [int(q) for q in rng.choice(n, k, replace=False)]
        U = GR.random_unitary(k, rng)
        assert max_abs(O.apply_gate(psi.copy(), pos, U), D.apply(psi, pos, U)) < 1e-12
        M = GR.random_unitary(k, rng) + 0.3  # not unitary: expectation of an operator
        phi = rand_psi(rng, n)
        assert abs(O.expect_dense(psi, pos, M) - np.vdot(psi, D.apply(psi, pos, M))) < 1e-12
        assert abs(O.expect_dense(psi, pos, M, vc=phi) - np.vdot(phi, D.apply(psi, pos, M))) < 1e-12
        out = np.zeros_like(psi)
        O.apply_gate_add(psi, out, pos, M)
        assert max_abs(out, D.apply(psi, pos, M)) < 1e-12


def test_specialised_equal_dense_and_conventions():
    # test/check_gateop.jl:69-168 compares specialised gates with the dense
    # gate(ordered_positions, ordered_mat); here the conventions themselves:
    X, Z = GR.X, GR.Z
    _, U, _ = GR.cnot(0, 1)
    # control = first position: |c=1,t=0> (index 1) -> |c=1,t=1> (index 3)
    assert U[3, 1] == 1 and U[1, 3] == 1 and U[0, 0] == 1 and U[2, 2] == 1
    _, U, _ = GR.toffoli(0, 1, 2)
    assert U[7, 3] == 1 and U[3, 7] == 1
    _, U, _ = GR.fredkin(0, 1, 2)
    assert U[5, 3] == 1 and U[3, 5] == 1 and U[6, 6] == 1
    _, U, _ = GR.cz(0, 1)
    assert np.allclose(np.diag(U), [1, 1, 1, -1])
    # rotations are exp(-i t P / 2)
    _, U, (dU,) = GR.rx(0, 0.3)
    assert np.allclose(U, np.cos(0.15) * np.eye(2) - 1j * np.sin(0.15) * X)
    assert np.allclose(dU, -0.5j * X @ U)
    _, U, _ = GR.rz(0, 0.3)
    assert np.allclose(U, np.diag([np.exp(-0.15j), np.exp(0.15j)]))


def test_product_gate_library_matches_oracle_library():
    """The device path's closed-form gates equal the oracle's exponentials."""
    import vqcb200.gates as G
    rng = np.random.default_rng(3)
    for _ in range(5):
        t, p, l = rng.uniform(0, 2 * np.pi, 3)
        pairs = [
            (G.RxGate(1, t, True), GR.rx(0, t)), (G.RyGate(1, t, True), GR.ry(0, t)),
            (G.RzGate(1, t, True), GR.rz(0, t)), (G.U3Gate(1, t, p, l, True), GR.u3(0, t, p, l)),
            (G.PHASEGate(1, t, True), GR.phase(0, t)), (G.CRxGate(1, 2, t, True), GR.crx(0, 1, t)),
            (G.CRyGate(1, 2, t, True), GR.cry(0, 1, t)), (G.CRzGate(1, 2, t, True), GR.crz(0, 1, t)),
            (G.CPHASEGate(1, 2, t, True), GR.cphase(0, 1, t)), (G.CCPHASEGate(1, 2, 3, t, True), GR.ccphase(0, 1, 2, t)),
            (G.CNOTGate(1, 2), GR.cnot(0, 1)), (G.CZGate(1, 2), GR.cz(0, 1)), (G.SWAPGate(1, 2), GR.swap(0, 1)),
            (G.iSWAPGate(1, 2), GR.iswap(0, 1)), (G.TOFFOLIGate(1, 2, 3), GR.toffoli(0, 1, 2)),
            (G.FREDKINGate(1, 2, 3), GR.fredkin(0, 1, 2)), (G.HGate(1), GR.h(0)), (G.SGate(1), GR.s(0)),
            (G.TGate(1), GR.t(0)), (G.XGate(1), GR.x(0)), (G.YGate(1), GR.y(0)), (G.ZGate(1), GR.z(0)),
        ]
        for g, (_, U, dUs) in pairs:
            assert np.abs(g.mat - U).max() < 1e-13, g
            assert len(g.derivatives()) == len(dUs), g
            for a, b in zip(g.derivatives(), dUs):
                assert np.abs(a - b).max() < 1e-13, g


def test_lsb_first_encoding():
    # test/check_state_init.jl:2-14: onehot_encoding([1, 0]) == kron(ZERO, ONE)
    ZERO, ONE = np.array([1, 0], dtype=complex), np.array([0, 1], dtype=complex)
    v = O.zero_state(2)
    O.apply_gate(v, [0], GR.X)  # qubit 1 (1-based) flipped
    assert np.array_equal(v, np.kron(ZERO, ONE))
    v = O.zero_state(3)
    O.apply_gate(v, [2], GR.X)
    assert np.array_equal(v, np.kron(ONE, np.kron(ZERO, ZERO)))


@pytest.mark.parametrize("sites", [[0, 1], [1, 4], [5, 2]])
def test_ptrace_state_vs_density_matrix(sites):
    # test/check_utility.jl:3-13 (sites [1,2], [2,5], [6,3], 1-based)
    rng = np.random.default_rng(sum(sites))
    psi = rand_psi(rng, 6)
    rho = O.density_matrix(psi)
    assert max_abs(O.sv_ptrace(psi, sites), O.dm_ptrace(rho, 6, sites)) < 1e-13


def test_phase_estimation_known_answer():
    # test/algs.jl:1-40: with an exactly representable phase the QPE register
    # reads the phase's binary digits with probability 1.  Here on the density
    # matrix path, with the register's digits j read from the diagonal.
    L = 4
    j = [1, 0, 1, 1]
    phi = sum(b * 2.0 ** -(i + 1) for i, b in enumerate(j))
    n = L + 1
    H = GR.h(0)[1]
    U = np.array([[np.exp(2j * np.pi * phi), 0], [0, 1]])
    gates = [((i,), H) for i in range(L)]
    tmp = U
    for i in reversed(range(L)):
        gates.append(((i, L), GR.controlled(i, (L,), tmp)))
        tmp = tmp @ tmp
    # inverse QFT on qubits 0..L-1 (most significant digit on qubit 0)
    qft = []
    for i in range(L):
        qft.append(((i,), H))
        for m in range(i + 1, L):
            ph = np.exp(2j * np.pi / 2 ** (m - i + 1))
            qft.append(((m, i), GR.controlled(m, (i,), np.diag([1, ph]))))
    for a in range(L // 2):
        qft.append(((a, L - 1 - a), GR.swap(0, 1)[1]))
    for pos, M in reversed(qft):
        gates.append((pos, M.conj().T))
    rho = O.density_matrix(O.zero_state(n))
    O.dm_apply_circuit(rho, n, gates)
    probs = O.dm_probs(rho, n)
    # register qubit i (0-based) holds digit j[i]; the ancilla (qubit L) is |0>
    idx = sum(b << i for i, b in enumerate(j))
    assert abs(probs[idx] - 1) < 1e-12
    psi = O.apply_circuit(O.zero_state(n), [(p, M) for p, M in gates])
    assert abs(abs(psi[idx]) ** 2 - 1) < 1e-12


def test_golden_fixtures_reproduce():
    """The committed fixtures still match the oracle (guards both)."""
    import vqcb200.workloads as W
    d = golden("hea_tfim_n12")
    spec = W.hea_spec(int(d["n"]), int(d["layers"]), d["theta"])
    terms = O.terms_from_spec(W.tfim_spec(int(d["n"]), float(d["g"])))
    e, g = O.energy_and_gradient(O.from_spec(spec), terms, O.zero_state(int(d["n"])), nthreads=4)
    assert abs(e - d["energy"]) < 1e-12
    assert np.abs(g - d["grads"]).max() < 1e-12
    d = golden("gates_n7")
    for i in range(int(d["ncases"])):
        out = O.apply_gate(d["psi"].copy(), list(d["pos%d" % i]), d["U%d" % i])
        assert max_abs(out, d["out%d" % i]) < 1e-13
    d = golden("noisy_dm_n4")
    n = int(d["n"])
    items = []
    for i in range(int(d["nitems"])):
        pos = [int(p) for p in d["pos%d" % i]]
        if int(d["kind%d" % i]) == 1:
            items.append(("map", pos, list(d["kraus%d" % i])))
        else:
            items.append(("gate", pos, d["mat%d" % i], list(d["der%d" % i])))
    rho = O.density_matrix(d["psi"])
    for it in items:
        if it[0] == "map":
            rho = O.dm_apply_channel(rho, n, it[1], it[2])
        else:
            O.dm_apply_gate(rho, n, it[1], it[2])
    assert max_abs(rho, d["rho"]) < 1e-13
    terms = [O.make_term({q: o for q, o in enumerate("IXZY"[((int(x) >> q) & 1) | (((int(z) >> q) & 1) << 1)]
                                                     for q in range(n)) if o != "I"}, complex(c))
             for x, z, c in zip(d["xmask"], d["zmask"], d["coeff"])]
    assert abs(O.dm_expectation(terms, rho, n) - d["energy"]) < 1e-13
    H = D.pauli_sum_matrix(n, terms)
    g, d_in, _ = O.dm_circuit_gradient(items, rho, H.conj().T.reshape(-1, order="F").copy(), n)
    assert np.abs(g - d["grads"]).max() < 1e-12
    assert max_abs(d_in, d["delta_in"]) < 1e-12


def test_oracle_rejects_bad_positions():
    v = O.zero_state(3)
    with pytest.raises(ValueError):
        O.apply_gate(v, [0, 0], np.eye(4))
    with pytest.raises(ValueError):
        O.apply_gate(v, [3], np.eye(2))


def _kraus2_cpu(rng):
    """A random 2-qubit channel: 3 Kraus operators, sum K^dagger K = I."""
    A = [rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)) for _ in range(3)]
    S = sum(a.conj().T @ a for a in A)
    w, U = np.linalg.eigh(S)
    inv_sqrt = U @ np.diag(w ** -0.5) @ U.conj().T
    return [a @ inv_sqrt for a in A]


def test_oracle_channel_and_dm_expectation_vs_dense():
    """The oracle's restatements of apply_qmaps.jl (supermatrix as a gate on
    (pos, pos + n)) and expecs_dm.jl (tr(M_key rho_key) per key) against
    dense NumPy: rho -> sum_i K_i rho K_i^dagger and tr(H rho)."""
    import vqcb200 as V
    from oracle import dense_np as D
    rng = np.random.default_rng(51)
    n = 4
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    rho = O.density_matrix(psi / np.linalg.norm(psi))
    N = 1 << n
    for pos, kraus in [((1,), V.Depolarizing(2, 0.2).kraus), ((3, 0), _kraus2_cpu(rng))]:
        R = rho.reshape(N, N, order="F")
        want = sum(D.full_operator(n, pos, K) @ R @ D.full_operator(n, pos, K).conj().T for K in kraus)
        got = O.dm_apply_channel(rho.copy(), n, pos, kraus)
        assert np.abs(got - want.reshape(-1, order="F")).max() < 1e-13
        rho = got
    terms = [O.make_term({0: "X", 2: "Y"}, 0.3), O.make_term({1: "Z"}, -1.1), O.make_term({3: "X", 0: "Z"}, 0.7j),
             O.make_term({}, 0.25)]
    H = D.pauli_sum_matrix(n, terms)
    want = complex(np.trace(H @ rho.reshape(N, N, order="F")))
    assert abs(O.dm_expectation(terms, rho, n) - want) < 1e-13


def _noisy_items(n, th, p=0.1):
    """The reference's noisy_circuit (test/check_noisy_grad.jl:3-9): a
    variational circuit (RY on every qubit, CRX chain, RZ) and a layer of
    Depolarizing channels, as oracle items (0-based positions)."""
    import vqcb200 as V
    items, k = [], 0
    for q in range(n):
        g = V.RyGate(q + 1, th[k], isparas=True)
        items.append(("gate", [q], g.mat, g.derivatives()))
        k += 1
    for q in range(n - 1):
        g = V.CRxGate(q + 1, q + 2, th[k], isparas=True)
        items.append(("gate", [q, q + 1], g.mat, g.derivatives()))
        k += 1
    for q in range(n):
        g = V.RzGate(q + 1, th[k], isparas=True)
        items.append(("gate", [q], g.mat, g.derivatives()))
        k += 1
    for q in range(n):
        items.append(("map", [q], V.Depolarizing(q + 1, p).kraus))
    return items


def _dm_forward(items, rho, n):
    rho = rho.copy()
    for it in items:
        if it[0] == "map":
            rho = O.dm_apply_channel(rho, n, it[1], it[2])
        else:
            O.dm_apply_gate(rho, n, it[1], it[2])
    return rho


@pytest.mark.parametrize("loss", ["sum", "expectation"])
def test_oracle_noisy_dm_gradient_vs_fd(loss):
    """circuitdiff.jl:42-59 restated (gates: uncompute + Re[tr(D^+ D y) +
    tr(y D^+ D^+)], channels: S^+ on the cotangent, S^-1 on the state)
    against 5-point-free central differences, h = 1e-4 (check_noisy_grad.jl)."""
    from oracle import dense_np as D
    n = 3
    rng = np.random.default_rng(71)
    th = rng.uniform(0, 2 * np.pi, 3 * n - 1)
    N = 1 << n
    rho0 = O.zero_state(2 * n)  # DensityMatrix(n) = |0><0|
    terms = [O.make_term({0: "X", 2: "Y"}, 0.36), O.make_term({1: "Z"}, 0.7), O.make_term({0: "Z", 1: "X"}, -0.5)]
    H = D.pauli_sum_matrix(n, terms)

    def L(t):
        r = _dm_forward(_noisy_items(n, t), rho0, n)
        if loss == "sum":
            return np.sum(r).real
        return np.trace(H @ r.reshape(N, N, order="F")).real

    out = _dm_forward(_noisy_items(n, th), rho0, n)
    delta = np.ones(N * N, dtype=complex) if loss == "sum" else H.conj().T.reshape(-1, order="F").copy()
    g, _, rho_in = O.dm_circuit_gradient(_noisy_items(n, th), out, delta, n)
    h = 1e-4
    fd = np.array([(L(th + h * e) - L(th - h * e)) / (2 * h) for e in np.eye(th.size)])
    assert np.abs(g - fd).max() < 1e-6
    assert np.abs(rho_in - rho0).max() < 1e-10
