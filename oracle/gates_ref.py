"""Gate matrices for the oracle (test infrastructure only).

The reference takes every gate matrix from the un-vendored, unpinned
QuantumCircuits.jl (called at applygates/generic/generic.jl:43,50 through
`ordered_positions` / `ordered_mat`, and at circuitdiff.jl:28-29 through
`nparameters` / `differentiate`).  Its conventions are therefore unpinned; this
module fixes them, and builds each matrix a different way from the product's
host library (matrix exponentials of generators here, closed forms there) so
that the two are an independent check of each other:

  RX(t) = exp(-i t X / 2), RY(t) = exp(-i t Y / 2), RZ(t) = exp(-i t Z / 2)
  U3(t, p, l) = exp(i (p + l) / 2) RZ(p) RY(t) RZ(l)      (OpenQASM U3)
  PHASE(p) = diag(1, e^{ip}),  CPHASE(p) = diag(1, 1, 1, e^{ip}),
  CCPHASE(p) = diag(1, ..., 1, e^{ip})
  controlled gates: the FIRST listed position is the control (czgate.jl:57-61,
  fredkingate.jl:67-75); matrix index bit b <-> listed position b.

Each function returns (positions, U, [dU/dtheta_j, ...]) with 0-based
positions.
"""
import numpy as np
from scipy.linalg import expm

I2 = np.eye(2, dtype=complex)
X = np.array([[0, 1], [1, 0]], dtype=complex)
Y = np.array([[0, -1j], [1j, 0]], dtype=complex)
Z = np.array([[1, 0], [0, -1]], dtype=complex)
P0 = np.array([[1, 0], [0, 0]], dtype=complex)
P1 = np.array([[0, 0], [0, 1]], dtype=complex)


def kron_lsb(*ops):
    """kron of single-qubit operators, first argument on the least significant bit."""
    m = np.array([[1.0 + 0j]])
    for op in ops:
        m = np.kron(op, m)
    return m


def rot(P, t):
    return expm(-0.5j * t * P)


def drot(P, t):
    return -0.5j * P @ rot(P, t)


def rx(q, t):
    return (q,), rot(X, t), [drot(X, t)]


def ry(q, t):
    return (q,), rot(Y, t), [drot(Y, t)]


def rz(q, t):
    return (q,), rot(Z, t), [drot(Z, t)]


def u3(q, t, p, l):
    g = np.exp(0.5j * (p + l))
    A, B, C = rot(Z, p), rot(Y, t), rot(Z, l)
    U = g * A @ B @ C
    dt = g * A @ drot(Y, t) @ C
    dp = 0.5j * U + g * drot(Z, p) @ B @ C
    dl = 0.5j * U + g * A @ B @ drot(Z, l)
    return (q,), U, [dt, dp, dl]


def h(q):
    return (q,), (X + Z) / np.sqrt(2), []


def x(q):
    return (q,), X.copy(), []


def y(q):
    return (q,), Y.copy(), []


def z(q):
    return (q,), Z.copy(), []


def s(q):
    return (q,), np.diag([1, 1j]).astype(complex), []


def t(q):
    return (q,), np.diag([1, np.exp(0.25j * np.pi)]).astype(complex), []


def phase(q, p):
    return (q,), expm(1j * p * P1), [1j * P1 @ expm(1j * p * P1)]


def controlled(c, targets, V):
    """Control on c (bit 0 of the matrix index), V on targets (higher bits)."""
    d = V.shape[0]
    return kron_lsb(P0, np.eye(d)) + np.kron(V, P1)


def cnot(c, tq):
    return (c, tq), controlled(c, (tq,), X), []


def cz(a, b):
    return (a, b), controlled(a, (b,), Z), []


def crx(c, tq, th):
    return (c, tq), controlled(c, (tq,), rot(X, th)), [np.kron(drot(X, th), P1)]


def cry(c, tq, th):
    return (c, tq), controlled(c, (tq,), rot(Y, th)), [np.kron(drot(Y, th), P1)]


def crz(c, tq, th):
    return (c, tq), controlled(c, (tq,), rot(Z, th)), [np.kron(drot(Z, th), P1)]


def cphase(a, b, p):
    G = kron_lsb(P1, P1)
    return (a, b), expm(1j * p * G), [1j * G @ expm(1j * p * G)]


def swap(a, b):
    S = np.zeros((4, 4), dtype=complex)
    for i in range(4):
        S[((i & 1) << 1) | (i >> 1), i] = 1
    return (a, b), S, []


def iswap(a, b):
    S = swap(a, b)[1]
    S[1, 2] = S[2, 1] = 1j
    return (a, b), S, []


def toffoli(c1, c2, tq):
    U = np.eye(8, dtype=complex)
    U[[3, 7], :] = U[[7, 3], :]
    return (c1, c2, tq), U, []


def fredkin(c, a, b):
    return (c, a, b), controlled(c, (a, b), swap(a, b)[1]), []


def ccphase(a, b, c, p):
    G = kron_lsb(P1, P1, P1)
    return (a, b, c), expm(1j * p * G), [1j * G @ expm(1j * p * G)]


def random_unitary(k, rng):
    """exp(i(M + M^dagger)) with M complex normal (test/runtests.jl:23-27), seeded."""
    d = 1 << k
    m = rng.standard_normal((d, d)) + 1j * rng.standard_normal((d, d))
    return expm(1j * (m + m.conj().T))
