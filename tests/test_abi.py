"""CPU tests of the boundary and the host logic (no GPU): the C-ABI library
loads and exports every symbol include/vqc_b200.h declares; the host mirror
packs circuits and operators into the ABI arrays correctly."""
import os
import re

import numpy as np
import pytest

from helpers import max_abs
from oracle import dense_np as D
from oracle import oracle as O

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(REPO, "include", "vqc_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vqc_\w+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    from vqcb200 import _lib
    lib = _lib.load()
    declared = header_functions()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(declared) == sorted(_lib.exported_symbols())


def test_library_reports_no_device_without_gpu():
    from vqcb200 import _lib
    lib = _lib.load()
    n = lib.vqc_device_count()
    # here (no GPU) a negative status; on a GPU box the device count
    assert n != 0


def test_pack_circuit_layout():
    import vqcb200 as V
    from vqcb200.circuit import Packed
    c = V.QCircuit([V.RxGate(2, 0.3, isparas=True), V.CNOTGate(1, 3), V.U3Gate(3, 0.1, 0.2, 0.3, isparas=True)])
    p = Packed(c)
    assert p.ngates == 3 and p.nparams == 4
    assert p.gates[0].nq == 1 and p.gates[0].pos[0] == 1
    assert p.gates[1].nq == 2 and list(p.gates[1].pos)[:2] == [0, 2]
    m = p.mats[p.gates[1].mat:p.gates[1].mat + 32].view(np.complex128).reshape(4, 4)
    assert np.array_equal(m, c[1].mat)
    assert [p.params[j].gate for j in range(4)] == [0, 2, 2, 2]
    d = p.mats[p.params[0].dmat:p.params[0].dmat + 8].view(np.complex128).reshape(2, 2)
    assert np.allclose(d, c[0].derivatives()[0])


def test_operator_pauli_expansion_is_exact():
    """Every QubitsTerm is expanded into Pauli strings; the sum must equal the
    dense key matrices of hamiltonian/util.jl:6-15."""
    import vqcb200 as V
    rng = np.random.default_rng(5)
    n = 5
    sp = np.array([[0, 1], [0, 0]], dtype=complex)
    terms = [V.QubitsTerm({1: "+", 4: "-"}, coeff=0.77), V.QubitsTerm({2: "X", 3: "Y"}, coeff=1.5 - 0.2j),
             V.QubitsTerm({5: rng.standard_normal((2, 2)) + 1j * rng.standard_normal((2, 2))}, coeff=0.3),
             V.QubitsTerm({1: sp, 2: "Z", 5: "X"}, coeff=-1.1)]
    H = V.QubitsOperator(*terms)
    dense = np.zeros((1 << n, 1 << n), dtype=complex)
    for t in terms:
        m = t.matrix()
        dense += D.full_operator(n, [q - 1 for q in t.positions], m)
    from oracle.dense_np import pauli_sum_matrix
    P = {"I": np.eye(2), "X": O.PAULI["X"], "Y": O.PAULI["Y"], "Z": O.PAULI["Z"]}
    acc = np.zeros_like(dense)
    for x, z, c in H.pauli_strings():
        ops = {}
        for q in range(n):
            b = ((x >> q) & 1, (z >> q) & 1)
            letter = {(0, 0): "I", (1, 0): "X", (0, 1): "Z", (1, 1): "Y"}[b]
            if letter != "I":
                ops[q] = P[letter]
        acc += pauli_sum_matrix(n, [O.make_term(ops, c)]) if ops else c * np.eye(1 << n)
    assert max_abs(acc, dense) < 1e-13


def test_workload_parameter_counts():
    from vqcb200 import workloads as W
    assert W.nparams(W.hea_spec(12, 6, np.zeros(144))) == 144
    assert W.nparams(W.rxyz_crx_spec(26, 20, np.zeros(20 * 103))) == 2060
    spec = W.u3_cz_toffoli_spec(30, 10, 7)
    assert sum(1 for s in spec if s[0] == "toffoli") == 10
    assert sum(1 for s in spec if s[0] == "u3") == 300


def test_host_rejects_wide_gate_before_device():
    import vqcb200 as V
    g = V.QuantumGate((1, 2, 3, 4, 5, 6), np.eye(64))
    with pytest.raises(NotImplementedError):
        V.apply(g, object())
