"""Independent dense NumPy checker for the oracle (test infrastructure only).

The reference's own tests check kernels against dense matrices
(`matrix(L, h) * psi`, test/check_high_qubit_gate.jl, test/check_qubits_ham.jl:
73-101).  This module does the same by tensor contraction, with none of the
oracle's index arithmetic, for n <= ~12.  Qubit q is bit q of the index, i.e.
axis n-1-q of the C-order reshape to (2,)*n.
"""
import numpy as np


def apply(psi, pos, U):
    """psi <- U on pos, U's index bit b <-> pos[b] (returns a new array)."""
    n = int(round(np.log2(psi.size)))
    k = len(pos)
    t = psi.reshape((2,) * n)
    # U as a tensor: out bits (k-1..0), in bits (k-1..0) in C order
    Ut = U.reshape((2,) * (2 * k))
    # state axes for pos[k-1], ..., pos[0] (matching Ut's C-order bit order)
    axes = [n - 1 - pos[b] for b in reversed(range(k))]
    r = np.tensordot(Ut, t, axes=(list(range(k, 2 * k)), axes))
    # r's axes: out bits (k-1..0) followed by the remaining state axes in order
    rest = [a for a in range(n) if a not in axes]
    order = axes + rest
    inv = np.argsort(order)
    return np.transpose(r, inv).reshape(-1)


def full_operator(n, pos, U):
    """The 2^n x 2^n matrix of U on pos (columns = images of basis states)."""
    d = 1 << n
    M = np.zeros((d, d), dtype=complex)
    for j in range(d):
        e = np.zeros(d, dtype=complex)
        e[j] = 1
        M[:, j] = apply(e, pos, U)
    return M


def pauli_sum_matrix(n, terms):
    """sum_t c_t kron(...) for terms (positions, ops, coeff)."""
    d = 1 << n
    H = np.zeros((d, d), dtype=complex)
    for pos, ops, c in terms:
        if len(pos) == 0:
            H += c * np.eye(d)
            continue
        m = np.array([[1.0 + 0j]])
        for op in ops:
            m = np.kron(op, m)
        H += c * full_operator(n, pos, m)
    return H
