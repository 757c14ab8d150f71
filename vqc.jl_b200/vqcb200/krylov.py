"""ground_state and time_evolution (utility/groundstate.jl:4-25) on the device.

The reference hands the operator's matvec x -> H x to KrylovKit
(eigsolve(..., 1, :SR; ishermitian=true) and exponentiate(..., t, v;
ishermitian=true); KrylovKit is a dependency without a pinned version and is
not vendored).  This module restates the published Krylov methods for a
Hermitian operator:
  * ground_state: Lanczos with full re-orthogonalisation, restarted from the
    lowest Ritz vector until the residual norm |beta_m y_m| < tol;
  * time_evolution: exp(t H) v by the Lanczos approximation
    ||v|| V_m exp(t T_m) e_1, with t cut into sub-steps until the last
    coefficient of the small exponential is below tol.
Every vector operation runs on the device (the Pauli-sum matvec, FP64
inner products, the axpby update); only the m x m tridiagonal problems are
solved on the host in FP64.
"""
import ctypes

import numpy as np
import scipy.linalg

from . import _lib
from .operators import QubitsOperator, QubitsTerm
from .state import StateVector, apply_operator, rand_state


def _axpby(y, a, x, b):
    """y <- a x + b y on the device."""
    av = (ctypes.c_double * 2)(complex(a).real, complex(a).imag)
    bv = (ctypes.c_double * 2)(complex(b).real, complex(b).imag)
    _lib.check(_lib.load().vqc_state_axpby(y.handle, av, x.handle, bv))


def _hermitian(H):
    if isinstance(H, QubitsTerm):
        H = QubitsOperator(H)
    if not H.is_hermitian():
        raise ValueError("input operator is not hermitian.")
    return H


def _lanczos(H, v, m):
    """m-step Lanczos from v (normalised in place), full re-orthogonalisation.
    Returns (basis list, alpha, beta) with beta[m-1] the residual norm."""
    V = [v]
    alpha, beta = [], []
    for j in range(m):
        w = apply_operator(H, V[j])
        a = V[j].dot(w).real
        alpha.append(a)
        for i, u in enumerate(V):  # full re-orthogonalisation (twice is enough)
            _axpby(w, -u.dot(w), u, 1.0)
        for u in V:
            _axpby(w, -u.dot(w), u, 1.0)
        b = w.norm()
        beta.append(b)
        if b < 1e-14 or j == m - 1:
            break
        _axpby(w, 0.0, w, 1.0 / b)
        V.append(w)
    return V, np.array(alpha), np.array(beta)


def _combine(V, coeffs, like):
    out = StateVector(like.nqubits, dtype=like.dtype, device=like.device)
    _axpby(out, 0.0, out, 0.0)
    for c, u in zip(coeffs, V):
        _axpby(out, c, u, 1.0)
    return out


def ground_state(H, nqubits=None, krylov_dim=30, tol=1e-10, maxiter=100, dtype=np.complex128, rng=None):
    """ground_state(h) (groundstate.jl:4-13): (lowest eigenvalue, eigenvector)
    of a Hermitian QubitsOperator; the start vector is rand_state(n)."""
    H = _hermitian(H)
    n = nqubits or H.max_position()
    v = rand_state(n, dtype=dtype, rng=rng)
    for _ in range(maxiter):
        V, alpha, beta = _lanczos(H, v, min(krylov_dim, 1 << n))
        m = len(alpha)
        T = np.diag(alpha) + np.diag(beta[:m - 1], 1) + np.diag(beta[:m - 1], -1)
        w, Y = np.linalg.eigh(T)
        y = Y[:, 0]
        v = _combine(V, y, v)
        _axpby(v, 0.0, v, 1.0 / v.norm())
        if abs(beta[m - 1] * y[-1]) < tol * max(1.0, abs(w[0])) or m < min(krylov_dim, 1 << n):
            return float(w[0]), v
    raise RuntimeError("eigsolve fails to converge.")


def time_evolution(H, t, v, krylov_dim=30, tol=1e-12):
    """time_evolution(h, t, v) (groundstate.jl:16-25): exp(t H) v for a
    Hermitian QubitsOperator H and a (complex) scalar t; returns a new state."""
    H = _hermitian(H)
    if H.max_position() > v.nqubits:
        raise ValueError("number of qubits mismatch.")
    out = v.copy()
    remaining, step = complex(t), complex(t)
    while abs(remaining) > 0:
        step = remaining if abs(step) > abs(remaining) else step
        nrm = out.norm()
        if nrm == 0:
            return out
        start = out.copy()
        _axpby(start, 0.0, start, 1.0 / nrm)
        V, alpha, beta = _lanczos(H, start, min(krylov_dim, 1 << v.nqubits))
        m = len(alpha)
        T = np.diag(alpha) + np.diag(beta[:m - 1], 1) + np.diag(beta[:m - 1], -1)
        while True:
            c = scipy.linalg.expm(step * T)[:, 0]
            # error estimate: the coupling out of the Krylov space
            if m < min(krylov_dim, 1 << v.nqubits) or abs(beta[m - 1] * c[-1]) < tol:
                break
            step *= 0.5
        out = _combine(V, nrm * c, out)
        remaining -= step
        if abs(remaining) < 1e-15 * abs(complex(t)):
            break
    return out
