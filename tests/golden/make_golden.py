"""Generates the golden fixtures under tests/golden/ from the CPU oracle.

The reference (Julia) cannot run on this image and ships no golden vectors,
so these fixtures are produced by the oracle (oracle/), each cross-checked
here before it is written:
  * against the independent dense NumPy checker (oracle/dense_np.py) for the
    state-vector, operator and density-matrix results;
  * against central finite differences (h = 1e-4, FP64) for the gradients.
Inputs are seeded (NumPy PCG64), so the fixtures are reproducible:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "vqc.jl_b200"))

from oracle import dense_np as D  # noqa: E402
from oracle import gates_ref as GR  # noqa: E402
from oracle import oracle as O  # noqa: E402
from vqcb200 import workloads as W  # noqa: E402


def dense_circuit(psi, gates):
    for pos, U, _ in gates:
        psi = D.apply(psi, list(pos), U)
    return psi


def fd_gradient(spec, terms, psi0, h=1e-4):
    """Central differences of real(expectation(H, circuit(theta) * psi0))."""
    grads = []
    for gi, (name, pos, par) in enumerate(spec):
        for j in range(len(par)):
            vals = []
            for s in (+1, -1):
                p2 = list(par)
                p2[j] += s * h
                sp = list(spec)
                sp[gi] = (name, pos, tuple(p2))
                y = O.apply_circuit(psi0.copy(), O.from_spec(sp))
                vals.append(O.expectation(terms, y).real)
            grads.append((vals[0] - vals[1]) / (2 * h))
    return np.array(grads)


def gates_fixture(rng):
    n = 7
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    cases = []
    for k in range(1, 6):
        for _ in range(4):
            pos = [int(q) for q in rng.choice(n, k, replace=False)]
            U = GR.random_unitary(k, rng)
            out = O.apply_gate(psi.copy(), pos, U)
            assert np.abs(out - D.apply(psi, pos, U)).max() < 1e-12
            cases.append((pos, U, out))
    d = {"n": n, "psi": psi, "ncases": len(cases)}
    for i, (pos, U, out) in enumerate(cases):
        d["pos%d" % i] = np.array(pos)
        d["U%d" % i] = U
        d["out%d" % i] = out
    return d


def hea_fixture(rng):
    n, layers = 12, 6
    theta = rng.uniform(0, 2 * np.pi, layers * 2 * n)
    spec = W.hea_spec(n, layers, theta)
    terms = O.terms_from_spec(W.tfim_spec(n, 0.7))
    psi0 = O.zero_state(n)
    gates = O.from_spec(spec)
    e, g = O.energy_and_gradient(gates, terms, psi0, nthreads=8)
    y = O.apply_circuit(psi0.copy(), gates)
    fd = fd_gradient(spec, terms, psi0)
    assert np.abs(g - fd).max() < 1e-6, np.abs(g - fd).max()
    return {"n": n, "layers": layers, "g": 0.7, "theta": theta, "energy": e, "grads": g, "out": y}


def xxz_fixture(rng):
    n, layers = 8, 2
    theta = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    spec = W.rxyz_crx_spec(n, layers, theta)
    terms = O.terms_from_spec(W.xxz_spec(n, 0.5))
    psi0 = O.zero_state(n)
    gates = O.from_spec(spec)
    e, g = O.energy_and_gradient(gates, terms, psi0)
    y = dense_circuit(psi0.copy(), gates)
    H = D.pauli_sum_matrix(n, terms)
    assert abs(np.vdot(y, H @ y) - e) < 1e-12
    fd = fd_gradient(spec, terms, psi0)
    assert np.abs(g - fd).max() < 1e-6, np.abs(g - fd).max()
    return {"n": n, "layers": layers, "theta": theta, "energy": e, "grads": g, "out": y}


def u3cz_fixture(rng):
    n, layers = 10, 4
    seed = int(rng.integers(1 << 31))
    spec = W.u3_cz_toffoli_spec(n, layers, seed)
    gates = O.from_spec(spec)
    psi0 = O.zero_state(n)
    y = O.apply_circuit(psi0.copy(), gates)
    assert np.abs(y - dense_circuit(psi0.copy(), gates)).max() < 1e-12
    return {"n": n, "layers": layers, "seed": seed, "out": y}


def dm_fixture(rng):
    n, layers = 5, 3
    seed = int(rng.integers(1 << 31))
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    spec = W.u3_cnot_spec(n, layers, seed)
    gates = O.from_spec(spec)
    rho = O.density_matrix(psi)
    O.dm_apply_circuit(rho, n, gates)
    # rho must equal |y><y| for the evolved pure state
    y = dense_circuit(psi.copy(), gates)
    assert np.abs(rho - O.density_matrix(y)).max() < 1e-12
    sites = [3, 4]  # the top two qubits (0-based), 1-based 4 and 5
    red = O.dm_ptrace(rho, n, sites)
    assert np.abs(red - O.sv_ptrace(y, sites)).max() < 1e-12
    probs = O.dm_probs(rho, n)
    assert np.abs(probs - np.abs(y) ** 2).max() < 1e-12
    return {"n": n, "layers": layers, "seed": seed, "psi": psi, "rho": rho, "sites": np.array(sites),
            "ptrace": red, "probs": probs}


def pauli_fixture(rng):
    n = 9
    psi = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    psi /= np.linalg.norm(psi)
    nterms = 40
    xs, zs, cs = [], [], []
    spec = []
    for _ in range(nterms):
        k = int(rng.integers(1, 5))
        qs = rng.choice(n, k, replace=False)
        ops = {int(q) + 1: "XYZ"[int(rng.integers(3))] for q in qs}
        c = complex(rng.standard_normal(), 0.3 * rng.standard_normal())
        spec.append((c, ops))
        x = sum(1 << (q - 1) for q, o in ops.items() if o in "XY")
        z = sum(1 << (q - 1) for q, o in ops.items() if o in "ZY")
        xs.append(x)
        zs.append(z)
        cs.append(c)
    terms = O.terms_from_spec(spec)
    e = O.expectation(terms, psi)
    hpsi = O.apply_operator(terms, psi)
    H = D.pauli_sum_matrix(n, terms)
    assert abs(np.vdot(psi, H @ psi) - e) < 1e-12
    assert np.abs(H @ psi - hpsi).max() < 1e-12
    return {"n": n, "psi": psi, "xmask": np.array(xs, dtype=np.uint64), "zmask": np.array(zs, dtype=np.uint64),
            "coeff": np.array(cs), "energy": e, "hpsi": hpsi}


def _kraus2(rng):
    A = [rng.standard_normal((4, 4)) + 1j * rng.standard_normal((4, 4)) for _ in range(3)]
    S = sum(a.conj().T @ a for a in A)
    w, U = np.linalg.eigh(S)
    return [a @ (U @ np.diag(w ** -0.5) @ U.conj().T) for a in A]


def noisy_dm_fixture(rng):
    """A noisy circuit on a density matrix (channels: apply_qmaps.jl; the DM
    pullback: circuitdiff.jl:35-75; tr(H rho): expecs_dm.jl), checked against
    dense NumPy (sum_i K_i rho K_i^dagger, U rho U^dagger, tr(H rho)) and the
    gradient against central differences of real(tr(H rho_out))."""
    import vqcb200 as V
    n = 4
    N = 1 << n
    psi = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    psi /= np.linalg.norm(psi)
    th = rng.uniform(0, 2 * np.pi, 3 * n - 1)

    def items_of(t):
        its, k = [], 0
        for q in range(n):
            g = V.U3Gate(q + 1, t[k], 0.3, -0.2, isparas=[True, False, False])
            its.append(("gate", [q], g.mat, g.derivatives()))
            k += 1
        its.append(("map", [1], V.Depolarizing(2, 0.15).kraus))
        for q in range(n - 1):
            g = V.CRxGate(q + 1, q + 2, t[k], isparas=True)
            its.append(("gate", [q, q + 1], g.mat, g.derivatives()))
            k += 1
        its.append(("map", [3, 0], K2))
        for q in range(n):
            g = V.RyGate(q + 1, t[k], isparas=True)
            its.append(("gate", [q], g.mat, g.derivatives()))
            k += 1
        its.append(("map", [2], V.AmplitudeDamping(3, 0.25).kraus))
        return its

    K2 = _kraus2(rng)
    spec = [(0.36, {1: "X", 4: "Y"}), (0.7, {2: "Z"}), (-0.5, {1: "Z", 3: "X"}), (0.2, {2: "Y", 3: "Y"})]
    terms = O.terms_from_spec(spec)
    H = D.pauli_sum_matrix(n, terms)

    def forward(t):
        rho = O.density_matrix(psi)
        R = rho.reshape(N, N, order="F").copy()
        for kind, pos, *rest in items_of(t):
            if kind == "map":
                rho = O.dm_apply_channel(rho, n, pos, rest[0])
                R = sum(D.full_operator(n, pos, K) @ R @ D.full_operator(n, pos, K).conj().T for K in rest[0])
            else:
                O.dm_apply_gate(rho, n, pos, rest[0])
                Uf = D.full_operator(n, pos, rest[0])
                R = Uf @ R @ Uf.conj().T
            assert np.abs(rho - R.reshape(-1, order="F")).max() < 1e-12
        return rho

    rho = forward(th)
    e = O.dm_expectation(terms, rho, n)
    assert abs(e - np.trace(H @ rho.reshape(N, N, order="F"))) < 1e-12
    its = items_of(th)
    g, d_in, y_in = O.dm_circuit_gradient(its, rho, H.conj().T.reshape(-1, order="F").copy(), n)
    assert np.abs(y_in - O.density_matrix(psi)).max() < 1e-10
    h = 1e-4
    fd = np.array([(O.dm_expectation(terms, forward(th + h * u), n).real -
                    O.dm_expectation(terms, forward(th - h * u), n).real) / (2 * h) for u in np.eye(th.size)])
    assert np.abs(g - fd).max() < 1e-6
    out = {"n": n, "psi": psi, "theta": th, "kraus2": np.array(K2), "rho": rho, "energy": e, "grads": g,
           "delta_in": d_in, "nitems": len(its),
           "xmask": np.array([sum(1 << (q - 1) for q, o in ops.items() if o in "XY") for _, ops in spec], np.uint64),
           "zmask": np.array([sum(1 << (q - 1) for q, o in ops.items() if o in "ZY") for _, ops in spec], np.uint64),
           "coeff": np.array([c for c, _ in spec], dtype=complex)}
    for i, (kind, pos, *rest) in enumerate(its):
        out["kind%d" % i] = np.array(0 if kind == "gate" else 1)
        out["pos%d" % i] = np.array(pos)
        if kind == "gate":
            out["mat%d" % i] = rest[0]
            out["der%d" % i] = np.array(rest[1]) if rest[1] else np.zeros((0, 1 << len(pos), 1 << len(pos)))
        else:
            out["kraus%d" % i] = np.array(rest[0])
    return out


FIXTURES = {
    "gates_n7": gates_fixture,
    "hea_tfim_n12": hea_fixture,
    "rxyz_crx_xxz_n8": xxz_fixture,
    "u3_cz_toffoli_n10": u3cz_fixture,
    "dm_u3_cnot_n5": dm_fixture,
    "pauli_sum_n9": pauli_fixture,
    "noisy_dm_n4": noisy_dm_fixture,
}


def main(names=None):
    """Writes every fixture, or only the named ones (python make_golden.py NAME...)."""
    for i, (name, fn) in enumerate(FIXTURES.items()):
        if names and name not in names:
            continue
        rng = np.random.default_rng(20261203 + i)
        d = fn(rng)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **d)
        print("wrote", name)


if __name__ == "__main__":
    main(sys.argv[1:])
