"""Gate library of the host mirror (closed-form matrices, FP64).

VQC.jl takes its gates from QuantumCircuits.jl (not vendored, unpinned), and
calls `ordered_positions`, `ordered_mat`, `nparameters` and `differentiate` on
them (applygates/generic/generic.jl:43,50; circuitdiff.jl:28-29).  This module
states the conventions explicitly:

  * positions are 1-based, as in the reference's API; bit b of a gate
    matrix's row/column index belongs to positions[b] (first position = least
    significant bit, as `QuantumGate((j, k), kron(m1, m2))` in
    test/check_qubits_ham.jl:20-28 shows);
  * controlled gates take their control(s) first (czgate.jl:57-61,
    fredkingate.jl:67-75);
  * RX(t) = exp(-i t X/2), RY(t) = exp(-i t Y/2), RZ(t) = exp(-i t Z/2),
    U3(t, p, l) = [[cos t/2, -e^{il} sin t/2], [e^{ip} sin t/2, e^{i(p+l)} cos t/2]],
    PHASE(p) = diag(1, e^{ip}); CRX/CRY/CRZ = |0><0| (x) I + |1><1| (x) R.

A gate carries its matrix and, for each active parameter, dU/dtheta (the
derivative the adjoint sweep contracts with, circuitdiff.jl:29).
"""
import cmath
import math

import numpy as np

_X = np.array([[0, 1], [1, 0]], dtype=complex)
_Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
_Z = np.array([[1, 0], [0, -1]], dtype=complex)
_I = np.eye(2, dtype=complex)


class Gate:
    """A k-qubit gate (k <= 5 on the device path; generic.jl:35-39)."""

    def __init__(self, positions, mat, params=(), isparas=None, dmats=None, name="QuantumGate"):
        if isinstance(positions, int):
            positions = (positions,)
        self.positions = tuple(int(p) for p in positions)
        self.mat = np.ascontiguousarray(np.asarray(mat, dtype=np.complex128))
        k = len(self.positions)
        if self.mat.shape != (1 << k, 1 << k):
            raise ValueError("wrong input matrix size.")
        if len(set(self.positions)) != k:
            raise ValueError("duplicate gate positions")
        self.params = tuple(float(p) for p in params)
        if isparas is None:
            isparas = [False] * len(self.params)
        elif isinstance(isparas, bool):
            isparas = [isparas] * len(self.params)
        self.isparas = tuple(bool(b) for b in isparas)
        self._dmats = list(dmats) if dmats is not None else []
        self.name = name

    # QuantumCircuits API mirrored by the reference
    @property
    def nqubits(self):
        return len(self.positions)

    def nparameters(self):
        return sum(self.isparas)

    def active_parameters(self):
        return [p for p, a in zip(self.params, self.isparas) if a]

    def derivatives(self):
        """dU/dtheta for each active parameter, in parameter order."""
        return [d for d, a in zip(self._dmats, self.isparas) if a]

    def adjoint(self):
        """gate' (the reference's AdjointQuantumGate)."""
        return Gate(self.positions, self.mat.conj().T, name=self.name + "'")

    def __repr__(self):
        return "%s%s" % (self.name, self.positions)


def QuantumGate(positions, mat):
    return Gate(positions, mat)


def _controlled(V):
    """control on bit 0, V on the higher bits."""
    d = V.shape[0]
    M = np.zeros((2 * d, 2 * d), dtype=complex)
    for a in range(d):
        M[2 * a, 2 * a] = 1
        for b in range(d):
            M[2 * a + 1, 2 * b + 1] = V[a, b]
    return M


def _dcontrolled(dV):
    d = dV.shape[0]
    M = np.zeros((2 * d, 2 * d), dtype=complex)
    for a in range(d):
        for b in range(d):
            M[2 * a + 1, 2 * b + 1] = dV[a, b]
    return M


def _rx(t):
    c, s = math.cos(t / 2), math.sin(t / 2)
    return np.array([[c, -1j * s], [-1j * s, c]]), 0.5 * np.array([[-s, -1j * c], [-1j * c, -s]])


def _ry(t):
    c, s = math.cos(t / 2), math.sin(t / 2)
    return np.array([[c, -s], [s, c]], dtype=complex), 0.5 * np.array([[-s, -c], [c, -s]], dtype=complex)


def _rz(t):
    a, b = cmath.exp(-0.5j * t), cmath.exp(0.5j * t)
    return np.diag([a, b]), np.diag([-0.5j * a, 0.5j * b])


def XGate(q):
    return Gate((q,), _X, name="X")


def YGate(q):
    return Gate((q,), _Y, name="Y")


def ZGate(q):
    return Gate((q,), _Z, name="Z")


def HGate(q):
    return Gate((q,), np.array([[1, 1], [1, -1]], dtype=complex) / math.sqrt(2), name="H")


def SGate(q):
    return Gate((q,), np.diag([1, 1j]), name="S")


def TGate(q):
    return Gate((q,), np.diag([1, cmath.exp(0.25j * math.pi)]), name="T")


def PHASEGate(q, phi, isparas=False):
    e = cmath.exp(1j * phi)
    return Gate((q,), np.diag([1, e]), (phi,), isparas, [np.diag([0, 1j * e])], name="PHASE")


def RxGate(q, theta, isparas=False):
    U, dU = _rx(theta)
    return Gate((q,), U, (theta,), isparas, [dU], name="Rx")


def RyGate(q, theta, isparas=False):
    U, dU = _ry(theta)
    return Gate((q,), U, (theta,), isparas, [dU], name="Ry")


def RzGate(q, theta, isparas=False):
    U, dU = _rz(theta)
    return Gate((q,), U, (theta,), isparas, [dU], name="Rz")


def U3Gate(q, theta, phi, lam, isparas=False):
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    ep, el, epl = cmath.exp(1j * phi), cmath.exp(1j * lam), cmath.exp(1j * (phi + lam))
    U = np.array([[c, -el * s], [ep * s, epl * c]])
    dt = 0.5 * np.array([[-s, -el * c], [ep * c, -epl * s]])
    dp = np.array([[0, 0], [1j * ep * s, 1j * epl * c]])
    dl = np.array([[0, -1j * el * s], [0, 1j * epl * c]])
    return Gate((q,), U, (theta, phi, lam), isparas, [dt, dp, dl], name="U3")


def CONTROLGate(positions, V):
    return Gate(positions, _controlled(np.asarray(V, dtype=complex)), name="CONTROL")


def CNOTGate(c, t=None):
    if t is None:
        c, t = c
    return Gate((c, t), _controlled(_X), name="CNOT")


def CZGate(c, t=None):
    if t is None:
        c, t = c
    return Gate((c, t), _controlled(_Z), name="CZ")


def _crot(f, name):
    def make(c, t, theta=None, isparas=False):
        if theta is None:  # CRxGate((c, t), theta)
            (c, t), theta = c, t
        U, dU = f(theta)
        return Gate((c, t), _controlled(U), (theta,), isparas, [_dcontrolled(dU)], name=name)
    return make


CRxGate = _crot(_rx, "CRx")
CRyGate = _crot(_ry, "CRy")
CRzGate = _crot(_rz, "CRz")


def CPHASEGate(a, b, phi, isparas=False):
    e = cmath.exp(1j * phi)
    return Gate((a, b), np.diag([1, 1, 1, e]), (phi,), isparas, [np.diag([0, 0, 0, 1j * e])], name="CPHASE")


def SWAPGate(a, b):
    return Gate((a, b), np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex), name="SWAP")


def iSWAPGate(a, b):
    return Gate((a, b), np.array([[1, 0, 0, 0], [0, 0, 1j, 0], [0, 1j, 0, 0], [0, 0, 0, 1]], dtype=complex),
                name="iSWAP")


def TOFFOLIGate(a, b, c):
    M = np.eye(8, dtype=complex)
    M[[3, 7]] = M[[7, 3]]
    return Gate((a, b, c), M, name="TOFFOLI")


def FREDKINGate(a, b, c):
    S = SWAPGate(1, 2).mat
    return Gate((a, b, c), _controlled(S), name="FREDKIN")


def CCPHASEGate(a, b, c, phi, isparas=False):
    e = cmath.exp(1j * phi)
    d = np.ones(8, dtype=complex)
    d[7] = e
    dd = np.zeros(8, dtype=complex)
    dd[7] = 1j * e
    return Gate((a, b, c), np.diag(d), (phi,), isparas, [np.diag(dd)], name="CCPHASE")


class QuantumMap:
    """A quantum channel rho -> sum_i K_i rho K_i^dagger on 1 or 2 qubits
    (QuantumCircuits.jl's QuantumMap, applied by applygates/apply_qmaps.jl).
    Kraus matrices follow the gate conventions: bit b of an index belongs to
    positions[b] (1-based positions)."""

    def __init__(self, positions, kraus, name="QuantumMap"):
        if isinstance(positions, int):
            positions = (positions,)
        self.positions = tuple(int(p) for p in positions)
        k = len(self.positions)
        if len(set(self.positions)) != k:
            raise ValueError("duplicate channel positions")
        self.kraus = [np.ascontiguousarray(np.asarray(m, dtype=np.complex128)) for m in kraus]
        if not self.kraus or any(m.shape != (1 << k, 1 << k) for m in self.kraus):
            raise ValueError("wrong Kraus matrix size.")
        self.name = name

    @property
    def nqubits(self):
        return len(self.positions)

    def nparameters(self):
        return 0

    def active_parameters(self):
        return []

    def derivatives(self):
        return []

    def supermat(self):
        """The 4^k x 4^k matrix acting on (positions, positions + n) of the
        vectorised rho: sum_i kron(conj(K_i), K_i) (column bits high)."""
        return sum(np.kron(m.conj(), m) for m in self.kraus)

    def __repr__(self):
        return "%s%s" % (self.name, self.positions)


# Channel conventions (QuantumCircuits.jl is not vendored; these are the
# standard Kraus forms, fixed here):
#   Depolarizing(p):     sqrt(1-p) I, sqrt(p/3) X, sqrt(p/3) Y, sqrt(p/3) Z
#   AmplitudeDamping(g): [[1, 0], [0, sqrt(1-g)]], [[0, sqrt(g)], [0, 0]]
#   PhaseDamping(g):     [[1, 0], [0, sqrt(1-g)]], [[0, 0], [0, sqrt(g)]]
def Depolarizing(q, p):
    a, b = math.sqrt(1 - p), math.sqrt(p / 3)
    return QuantumMap((q,), [a * _I, b * _X, b * _Y, b * _Z], name="Depolarizing")


def AmplitudeDamping(q, gamma):
    return QuantumMap((q,), [np.array([[1, 0], [0, math.sqrt(1 - gamma)]]), np.array([[0, math.sqrt(gamma)], [0, 0]])],
                      name="AmplitudeDamping")


def PhaseDamping(q, gamma):
    return QuantumMap((q,), [np.array([[1, 0], [0, math.sqrt(1 - gamma)]]), np.array([[0, 0], [0, math.sqrt(gamma)]])],
                      name="PhaseDamping")
