"""Python front of the CPU oracle (test infrastructure only).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import this module, as the checker or as the timed CPU restatement of the
reference's multithreaded path.  The product library never loads it.

Parity status: UNPINNED against outputs of the reference itself (Julia is not
available, and the reference ships no golden vectors); pinned by line-for-line
restatement and by the reference's relational and known-answer tests restated
under tests/.

The kernels live in vqc_oracle.cpp (liboracle.so, built by the Makefile beside
this file).  This module adds the drivers that the reference writes in Julia:
  * circuit application            applygates/generic/generic.jl:26-33
  * QubitsOperator grouping by key hamiltonian/util.jl:6-15, expecs.jl:22-42
  * H * psi                        hamiltonian/apply_qterms/apply_qterms.jl:13-28
  * expectation pullback           expecdiff.jl:30-33
  * circuit pullback (uncompute)   circuitdiff.jl:2-8, 23-32, 61-75
  * density-matrix circuit, ptrace, probabilities
                                   generic.jl:54-64, ptrace.jl:4-53, measure.jl:69-81
All positions are 0-based (the reference's are 1-based).
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Compile liboracle.so beside this file (g++, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        dp, fp, ip = (ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float),
                      ctypes.POINTER(ctypes.c_int))
        i = ctypes.c_int
        for name, args in [
            ("or_apply_gate_c128", [dp, i, i, ip, dp, i]),
            ("or_apply_gate_c64", [fp, i, i, ip, fp, i]),
            ("or_apply_gate_add_c128", [dp, dp, i, i, ip, dp, i]),
            ("or_apply_gate_add_c64", [fp, fp, i, i, ip, fp, i]),
            ("or_expect_c128", [dp, dp, i, i, ip, dp, dp, i]),
            ("or_expect_c64", [fp, fp, i, i, ip, fp, fp, i]),
            ("or_dm_apply_gate_c128", [dp, i, i, ip, dp, i]),
            ("or_dm_ptrace_c128", [dp, i, i, ip, dp]),
            ("or_sv_ptrace_c128", [dp, i, i, ip, dp]),
            ("or_dm_probs_c128", [dp, i, dp]),
        ]:
            f = getattr(L, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        L.or_dm_prob_zero_c128.argtypes = [dp, i, i]
        L.or_dm_prob_zero_c128.restype = ctypes.c_double
        L.or_max_threads.restype = ctypes.c_int
        _LIB = L
    return _LIB


def default_threads():
    return max(1, lib().or_max_threads())


def _ptr(a):
    if a is None:
        return None
    if a.dtype == np.complex128 or a.dtype == np.float64:
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    if a.dtype == np.complex64 or a.dtype == np.float32:
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    raise TypeError(a.dtype)


def _ipos(pos):
    a = np.ascontiguousarray(pos, dtype=np.int32)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _nq(v):
    n = int(round(np.log2(v.size)))
    assert (1 << n) == v.size
    return n


def _sfx(v):
    if v.dtype == np.complex128:
        return "c128"
    if v.dtype == np.complex64:
        return "c64"
    raise TypeError(v.dtype)


# ----------------------------------------------------------------------------- state vectors
def zero_state(n, dtype=np.complex128):
    """StateVector(n): |0...0> (statevector.jl:15-21)."""
    v = np.zeros(1 << n, dtype=dtype)
    v[0] = 1
    return v


def apply_gate(v, pos, U, nthreads=1):
    """In place: v <- U on pos (generic.jl:6-14; serial_short_range.jl / threaded_*)."""
    assert v.flags.c_contiguous
    U = np.ascontiguousarray(U, dtype=v.dtype)
    p, pp = _ipos(pos)
    err = getattr(lib(), "or_apply_gate_" + _sfx(v))(_ptr(v), _nq(v), len(p), pp, _ptr(U), nthreads)
    if err:
        raise ValueError("oracle apply_gate: bad positions %s for n=%d" % (list(pos), _nq(v)))
    return v


def apply_gate_add(v, vout, pos, U, nthreads=1):
    """vout += U v on pos (apply_qterms/short_range_serial.jl)."""
    U = np.ascontiguousarray(U, dtype=v.dtype)
    p, pp = _ipos(pos)
    err = getattr(lib(), "or_apply_gate_add_" + _sfx(v))(_ptr(v), _ptr(vout), _nq(v), len(p), pp, _ptr(U),
                                                          nthreads)
    if err:
        raise ValueError("oracle apply_gate_add: bad positions")
    return vout


def expect_dense(v, pos, M, vc=None, nthreads=1):
    """sum vc^dagger M v over groups (expec_serial.jl; vc=None: one-state form)."""
    M = np.ascontiguousarray(M, dtype=v.dtype)
    p, pp = _ipos(pos)
    out = np.zeros(2, dtype=np.float64 if v.dtype == np.complex128 else np.float32)
    err = getattr(lib(), "or_expect_" + _sfx(v))(_ptr(v), _ptr(vc), _nq(v), len(p), pp, _ptr(M), _ptr(out),
                                                  nthreads)
    if err:
        raise ValueError("oracle expect: bad positions")
    return complex(out[0], out[1])


def apply_circuit(v, gates, nthreads=1):
    """apply!(circuit, state): gates in order, no fusion (generic.jl:26-31)."""
    for g in gates:
        apply_gate(v, g[0], g[1], nthreads)
    return v


# ----------------------------------------------------------------------------- operators
PAULI = {
    "I": np.eye(2, dtype=complex),
    "X": np.array([[0, 1], [1, 0]], dtype=complex),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=complex),
    "Z": np.array([[1, 0], [0, -1]], dtype=complex),
}


def make_term(ops, coeff=1.0):
    """A QubitsTerm: ops = {position: 2x2 matrix or 'X'/'Y'/'Z'}, coefficient."""
    items = sorted((int(q), PAULI[o] if isinstance(o, str) else np.asarray(o, dtype=complex))
                   for q, o in ops.items())
    return tuple(q for q, _ in items), [m for _, m in items], complex(coeff)


def group_by_key(terms):
    """QubitsOperator.data: terms grouped by their position tuple; each key's
    matrix is sum_t coeff_t kron(reverse(ops_t)) (hamiltonian/util.jl:6-15)."""
    keys = {}
    for pos, ops, c in terms:
        m = np.array([[1.0 + 0j]])
        for op in ops:  # first position on the least significant bit
            m = np.kron(op, m)
        if pos in keys:
            keys[pos] = keys[pos] + c * m
        else:
            keys[pos] = c * m
    return keys


def expectation(terms, v, vc=None, nthreads=1):
    """expectation(H, psi) / expectation(phi, H, psi): one pass per key (expecs.jl:22-74).
    The empty key (identity) contributes coeff * <vc|v>."""
    r = 0j
    for pos, M in group_by_key(terms).items():
        if len(pos) == 0:
            w = v if vc is None else vc
            r += M[0, 0] * complex(np.vdot(w.astype(np.complex128), v.astype(np.complex128)))
        else:
            r += expect_dense(v, pos, M, vc, nthreads)
    return r


def apply_operator(terms, v, nthreads=1):
    """H * psi = sum_key M_key psi (apply_qterms.jl:13-28)."""
    out = np.zeros_like(v)
    for pos, M in group_by_key(terms).items():
        if len(pos) == 0:
            out += M[0, 0] * v
        else:
            apply_gate_add(v, out, pos, M, nthreads)
    return out


def adjoint_terms(terms):
    return [(p, [o.conj().T for o in ops], np.conj(c)) for p, ops, c in terms]


def from_spec(spec):
    """Gate list from a neutral description [(name, 1-based positions, params)],
    matrices from this directory's own gate library (gates_ref.py)."""
    from . import gates_ref as G
    return [getattr(G, name.lower())(*[q - 1 for q in pos], *par) for name, pos, par in spec]


def terms_from_spec(spec):
    """Operator from [(coeff, {1-based position: 'X'|'Y'|'Z'|matrix}), ...]."""
    return [make_term({q - 1: o for q, o in ops.items()}, c) for c, ops in spec]


# ----------------------------------------------------------------------------- gradients
def circuit_gradient(gates, psi0, delta, nthreads=1):
    """Reverse pass of the circuit pullback (circuitdiff.jl:23-32, 61-75).

    gates: list of (positions, U, [dU/dtheta_j ...]) in circuit order;
    delta: cotangent of the output state.  The forward states are uncomputed
    (y <- U^dagger y) instead of stored; each parameter's partial is
    real(expectation(y, G_j, delta)) with G_j = (dU/dtheta_j)^dagger U, the
    form that makes it equal Re <delta_out | dU/dtheta_j | y_in>.
    Returns (gradients in circuit order, cotangent of the input state)."""
    y = apply_circuit(psi0.copy(), gates, nthreads)
    d = delta.copy()
    per_gate = []
    for pos, U, dUs in reversed(gates):
        Ud = U.conj().T
        apply_gate(d, pos, Ud, nthreads)
        apply_gate(y, pos, Ud, nthreads)
        if dUs:
            per_gate.append([expect_dense(d, pos, dU.conj().T @ U, vc=y, nthreads=nthreads).real for dU in dUs])
    grads = []
    for g in reversed(per_gate):
        grads.extend(g)
    return np.array(grads), d


def energy_and_gradient(gates, terms, psi0, nthreads=1):
    """gradient(theta -> real(expectation(H, circuit(theta) * psi0))):
    forward, expectation, expectation pullback with z = 1 ((conj(z) H + z H')psi,
    expecdiff.jl:30-33), then the circuit pullback."""
    y = apply_circuit(psi0.copy(), gates, nthreads)
    e = expectation(terms, y, nthreads=nthreads)
    delta = apply_operator(terms, y, nthreads) + apply_operator(adjoint_terms(terms), y, nthreads)
    g, _ = circuit_gradient(gates, psi0, delta, nthreads)
    return e, g


# ----------------------------------------------------------------------------- density matrices
def density_matrix(psi):
    """DensityMatrix(psi) = kron(conj psi, psi) flattened (densitymatrix.jl:27)."""
    return np.kron(psi.conj(), psi)


def dm_apply_gate(rho, n, pos, U, nthreads=1):
    """generic.jl:54-64: U on pos, conj(U) on pos + n."""
    U = np.ascontiguousarray(U, dtype=np.complex128)
    p, pp = _ipos(pos)
    if lib().or_dm_apply_gate_c128(_ptr(rho), n, len(p), pp, _ptr(U), nthreads):
        raise ValueError("oracle dm_apply_gate: bad positions")
    return rho


def dm_apply_circuit(rho, n, gates, nthreads=1):
    for g in gates:
        dm_apply_gate(rho, n, g[0], g[1], nthreads)
    return rho


def dm_ptrace(rho, n, sites):
    """partial_tr(rho, sites) (ptrace.jl:4-10, 38-53); returns the flattened
    2^(n-m) x 2^(n-m) column-major result."""
    s, sp = _ipos(sites)
    m = n - len(s)
    out = np.zeros(1 << (2 * m), dtype=np.complex128)
    if lib().or_dm_ptrace_c128(_ptr(rho), n, len(s), sp, _ptr(out)):
        raise ValueError("oracle ptrace: bad sites")
    return out


def sv_ptrace(psi, sites):
    """partial_tr(psi, sites) (ptrace.jl:13-27)."""
    n = _nq(psi)
    s, sp = _ipos(sites)
    m = n - len(s)
    out = np.zeros(1 << (2 * m), dtype=np.complex128)
    if lib().or_sv_ptrace_c128(_ptr(psi), n, len(s), sp, _ptr(out)):
        raise ValueError("oracle ptrace: bad sites")
    return out


def dm_probs(rho, n):
    out = np.zeros(1 << n, dtype=np.float64)
    lib().or_dm_probs_c128(_ptr(rho), n, _ptr(out))
    return out


def dm_prob_zero(rho, n, q):
    """compute_probability_zero(rho, q) (measure.jl:69-81)."""
    return lib().or_dm_prob_zero_c128(_ptr(rho), n, q)


def dm_apply_channel(rho, n, pos, kraus, mode=0, nthreads=1):
    """apply!(::QuantumMap, rho) (apply_qmaps.jl:5-14, 67-77): the channel's
    supermatrix sum_i kron(conj K_i, K_i) as a gate on (pos..., pos + n...)
    of the vectorised rho; mode 1 its adjoint (apply_dagger!, :21-30,
    79-86), mode 2 its inverse (apply_inverse!, :36-45)."""
    S = sum(np.kron(np.asarray(K, dtype=np.complex128).conj(), np.asarray(K, dtype=np.complex128)) for K in kraus)
    if mode == 1:
        S = S.conj().T
    elif mode == 2:
        S = np.linalg.inv(S)
    return apply_gate(rho, list(pos) + [p + n for p in pos], S, nthreads)


def dm_expectation(terms, rho, n):
    """expectation(H, rho) (expecs_dm.jl:19-30): sum over position keys of
    tr(M_key rho_key), rho_key the reduced matrix of the key's qubits (the
    blocks expec_dm_serial.jl sums); the empty key gives coeff * tr(rho)."""
    r = 0j
    for pos, M in group_by_key(terms).items():
        if len(pos) == 0:
            r += M[0, 0] * complex(np.sum(dm_probs(rho, n)))
            continue
        rest = [q for q in range(n) if q not in pos]
        red = dm_ptrace(rho, n, rest) if rest else rho
        d = 1 << len(pos)
        r += complex(np.trace(M @ red.reshape(d, d, order="F")))
    return r


def dm_trace_prod(a, b, n, pos, M, dag_a=False, dag_b=False):
    """tr(op(a) M op(b)) with M on the row qubits pos (circuitdiff.jl:35-40)."""
    N = 1 << n
    A = a.reshape(N, N, order="F")
    B = b.reshape(N, N, order="F")
    A = A.conj().T if dag_a else A
    B = B.conj().T if dag_b else B
    MB = apply_gate(np.array(B.reshape(-1, order="F"), dtype=np.complex128), list(pos),
                    np.asarray(M, dtype=np.complex128))
    return complex(np.sum(A * MB.reshape(N, N, order="F").T))


def dm_circuit_gradient(items, rho_out, delta_out, n):
    """back_propagate for density matrices (circuitdiff.jl:42-59, 61-75).
    items: ("gate", pos, U, [dU...]) or ("map", pos, [K...]); returns
    (grads, delta_in, rho_in)."""
    y, d = rho_out.copy(), delta_out.copy()
    per = []
    for it in reversed(items):
        if it[0] == "map":
            _, pos, kraus = it
            d = dm_apply_channel(d, n, pos, kraus, mode=1)
            y = dm_apply_channel(y, n, pos, kraus, mode=2)
            continue
        _, pos, U, ders = it
        Ud = np.asarray(U, dtype=np.complex128).conj().T
        dm_apply_gate(d, n, pos, Ud)
        dm_apply_gate(y, n, pos, Ud)
        g = []
        for dU in ders:
            D = Ud @ np.asarray(dU, dtype=np.complex128)
            g.append((dm_trace_prod(d, y, n, pos, D, dag_a=True) + dm_trace_prod(y, d, n, pos, D.conj().T, dag_b=True)).real)
        if g:
            per.append(g)
    return np.array([x for g in reversed(per) for x in g]), d, y


# ----------------------------------------------------------------------------- measurement
def sv_prob_zero(v, q):
    """compute_probability_zero(v, key) (measure.jl:47-59): sum of |v_i|^2
    over the indices with bit q clear (0-based q)."""
    idx = np.arange(v.size)
    return float(np.sum(np.abs(v[(idx >> q) & 1 == 0]) ** 2))


def collapse(v, q, i, p, reset):
    """The collapse of apply!(::QMeasure, ...) (measure.jl:4-16) on a state
    vector: |i> -> |0> (reset) or |i>, scaled by 1/sqrt(p), other branch 0."""
    m = np.zeros((2, 2), dtype=complex)
    m[0 if reset else i, i] = 1 / np.sqrt(p)
    return apply_gate(np.array(v, dtype=np.complex128), [q], m)


def take_qubit(v, q, value):
    """The slice of qubit q at `value` (measure.jl:38-46, postselect.jl:37-44:
    swap the qubit to position 1, keep one row of the 2 x L/2 reshape)."""
    idx = np.arange(v.size)
    return np.array(v[(idx >> q) & 1 == value], dtype=np.complex128)
