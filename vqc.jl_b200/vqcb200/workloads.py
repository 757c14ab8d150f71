"""Circuit and Hamiltonian builders for the benchmark workloads.

Each circuit builder returns a neutral description [(name, positions, params)]
with 1-based positions, so the device engine (`to_circuit`) and the CPU oracle
(its own gate library) build their matrices independently from the same input.
The layouts follow the reference's Utilities module (variational_circuit_1d,
utility/variationalcircuit.jl:5-39; spin chains, utility/spin_hamiltonians.jl)
with the structures the benchmark configurations name.
"""
import numpy as np

from . import gates as G
from .circuit import QCircuit
from .operators import QubitsOperator, QubitsTerm

_BUILD = {
    "rx": lambda p, a: G.RxGate(p[0], a[0], isparas=True),
    "ry": lambda p, a: G.RyGate(p[0], a[0], isparas=True),
    "rz": lambda p, a: G.RzGate(p[0], a[0], isparas=True),
    "u3": lambda p, a: G.U3Gate(p[0], a[0], a[1], a[2], isparas=True),
    "h": lambda p, a: G.HGate(p[0]),
    "x": lambda p, a: G.XGate(p[0]),
    "cnot": lambda p, a: G.CNOTGate(p[0], p[1]),
    "cz": lambda p, a: G.CZGate(p[0], p[1]),
    "crx": lambda p, a: G.CRxGate(p[0], p[1], a[0], isparas=True),
    "toffoli": lambda p, a: G.TOFFOLIGate(*p),
}


def to_circuit(spec):
    return QCircuit([_BUILD[name](pos, par) for name, pos, par in spec])


def hea_spec(n, layers, thetas):
    """Hardware-efficient ansatz: per layer RY(t), RZ(t) on every qubit, then
    CNOT(i, i+1) for i = 1..n-1 (layers * 2n parameters)."""
    thetas = np.asarray(thetas, dtype=float)
    assert thetas.size == layers * 2 * n
    spec, k = [], 0
    for _ in range(layers):
        for q in range(1, n + 1):
            spec.append(("ry", (q,), (thetas[k],)))
            spec.append(("rz", (q,), (thetas[k + 1],)))
            k += 2
        for q in range(1, n):
            spec.append(("cnot", (q, q + 1), ()))
    return spec


def rxyz_crx_spec(n, layers, thetas):
    """Per layer RX, RY, RZ on every qubit, then CRX(i, i+1) for i = 1..n-1
    (layers * (3n + n - 1) parameters)."""
    thetas = np.asarray(thetas, dtype=float)
    assert thetas.size == layers * (4 * n - 1)
    spec, k = [], 0
    for _ in range(layers):
        for q in range(1, n + 1):
            for name in ("rx", "ry", "rz"):
                spec.append((name, (q,), (thetas[k],)))
                k += 1
        for q in range(1, n):
            spec.append(("crx", (q, q + 1), (thetas[k],)))
            k += 1
    return spec


def u3_cz_toffoli_spec(n, layers, rng):
    """Per layer U3 (3 angles uniform in [0, 2 pi)) on every qubit, CZ on the
    brickwork pairs (1,2),(3,4).. on odd layers and (2,3),(4,5).. on even
    layers, and one Toffoli on a seeded random triple."""
    rng = np.random.default_rng(rng)
    spec = []
    for layer in range(layers):
        for q in range(1, n + 1):
            spec.append(("u3", (q,), tuple(rng.uniform(0, 2 * np.pi, 3))))
        start = 1 if layer % 2 == 0 else 2
        for q in range(start, n, 2):
            spec.append(("cz", (q, q + 1), ()))
        trip = rng.choice(np.arange(1, n + 1), 3, replace=False)
        spec.append(("toffoli", tuple(int(t) for t in trip), ()))
    return spec


def u3_cnot_spec(n, layers, rng):
    """Per layer U3 on every qubit then the CNOT ladder (i, i+1), i = 1..n-1."""
    rng = np.random.default_rng(rng)
    spec = []
    for _ in range(layers):
        for q in range(1, n + 1):
            spec.append(("u3", (q,), tuple(rng.uniform(0, 2 * np.pi, 3))))
        for q in range(1, n):
            spec.append(("cnot", (q, q + 1), ()))
    return spec


def nparams(spec):
    return sum(len(p) for name, _, p in spec if name in ("rx", "ry", "rz", "u3", "crx"))


# ----------------------------------------------------------------------------- Hamiltonians
def tfim_spec(n, g):
    """Open-chain transverse-field Ising: sum Z_i Z_{i+1} + g sum X_i."""
    terms = [(1.0, {i: "Z", i + 1: "Z"}) for i in range(1, n)]
    terms += [(g, {i: "X"}) for i in range(1, n + 1)]
    return terms


def xxz_spec(n, jz=0.5):
    """Open-chain XXZ: sum (X_i X_{i+1} + Y_i Y_{i+1} + jz Z_i Z_{i+1})."""
    terms = []
    for i in range(1, n):
        terms += [(1.0, {i: "X", i + 1: "X"}), (1.0, {i: "Y", i + 1: "Y"}), (jz, {i: "Z", i + 1: "Z"})]
    return terms


def to_operator(terms):
    return QubitsOperator(*[QubitsTerm(ops, coeff=c) for c, ops in terms])
