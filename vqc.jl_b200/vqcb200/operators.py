"""QubitsTerm / QubitsOperator of the host mirror.

The reference's operators come from QuantumCircuits.jl: a QubitsTerm is a
coefficient times single-qubit 2x2 operators on positions; a QubitsOperator is
a sum of terms grouped by position key (hamiltonian/util.jl:3-27 builds each
key's matrix as kron(reverse(ops)) * coeff).  On the device every operator is
run as a Pauli sum in one pass: each 2x2 operator is expanded in the Pauli
basis (A = sum_P tr(P A)/2 P), products are expanded, identical strings are
merged.  That is exact and turns sigma+/- (heisenberg_chain,
spin_hamiltonians.jl:7-22) into X/Y strings.
"""
import itertools

import numpy as np

from . import _lib

PAULI = {
    "I": np.eye(2, dtype=complex),
    "X": np.array([[0, 1], [1, 0]], dtype=complex),
    "Y": np.array([[0, -1j], [1j, 0]], dtype=complex),
    "Z": np.array([[1, 0], [0, -1]], dtype=complex),
    "+": np.array([[0, 1], [0, 0]], dtype=complex),
    "-": np.array([[0, 0], [1, 0]], dtype=complex),
    "0": np.array([[1, 0], [0, 0]], dtype=complex),
    "1": np.array([[0, 0], [0, 1]], dtype=complex),
}
# (x, z) bits of each Pauli letter
_XZ = {"I": (0, 0), "X": (1, 0), "Z": (0, 1), "Y": (1, 1)}


def _op(o):
    if isinstance(o, str):
        return PAULI[o]
    a = np.asarray(o, dtype=complex)
    if a.shape != (2, 2):
        raise ValueError("a QubitsTerm takes 2x2 single-qubit operators")
    return a


class QubitsTerm:
    """coeff * prod_i ops[i] on positions[i] (1-based)."""

    def __init__(self, ops=None, coeff=1.0, **kw):
        ops = dict(ops or {})
        items = sorted((int(q), _op(o)) for q, o in ops.items())
        self.positions = tuple(q for q, _ in items)
        self.ops = [m for _, m in items]
        self.coeff = complex(coeff)

    def adjoint(self):
        t = QubitsTerm()
        t.positions = self.positions
        t.ops = [o.conj().T for o in self.ops]
        t.coeff = np.conj(self.coeff)
        return t

    def __mul__(self, a):
        t = QubitsTerm()
        t.positions, t.ops, t.coeff = self.positions, list(self.ops), self.coeff * complex(a)
        return t

    __rmul__ = __mul__

    def matrix(self):
        m = np.array([[1.0 + 0j]])
        for o in self.ops:
            m = np.kron(o, m)
        return self.coeff * m

    def pauli_strings(self):
        """[(xmask, zmask, coeff)] with 0-based masks."""
        per_site = []
        for q, o in zip(self.positions, self.ops):
            comps = []
            for letter in "IXYZ":
                c = np.trace(PAULI[letter] @ o) / 2
                if c != 0:
                    comps.append((q - 1, letter, c))
            per_site.append(comps)
        out = []
        for combo in itertools.product(*per_site):
            x = z = 0
            c = self.coeff
            for q, letter, a in combo:
                bx, bz = _XZ[letter]
                x |= bx << q
                z |= bz << q
                c *= a
            out.append((x, z, c))
        return out


class QubitsOperator:
    def __init__(self, *terms):
        self.terms = []
        for t in terms:
            self.add(t)

    def add(self, t):
        if isinstance(t, QubitsOperator):
            self.terms.extend(t.terms)
        else:
            self.terms.append(t)
        return self

    def __add__(self, other):
        r = QubitsOperator(*self.terms)
        return r.add(other)

    def __mul__(self, a):
        return QubitsOperator(*[t * a for t in self.terms])

    __rmul__ = __mul__

    def adjoint(self):
        return QubitsOperator(*[t.adjoint() for t in self.terms])

    def max_position(self):
        return max((max(t.positions) for t in self.terms if t.positions), default=0)

    def keys(self):
        """QubitsOperator.data: position key -> dense matrix (util.jl:6-15)."""
        d = {}
        for t in self.terms:
            m = t.matrix()
            d[t.positions] = d.get(t.positions, 0) + m
        return d

    def pauli_strings(self):
        acc = {}
        for t in self.terms:
            for x, z, c in t.pauli_strings():
                acc[(x, z)] = acc.get((x, z), 0) + c
        return [(x, z, c) for (x, z), c in acc.items() if c != 0]

    def packed(self):
        """ctypes vqc_pauli array of the merged Pauli strings (cached while
        the operator holds the same terms with the same coefficients)."""
        key = [(t, t.coeff) for t in self.terms]
        cache = getattr(self, "_packed", None)
        if cache is not None and len(cache[0]) == len(key) and all(
                a[0] is b[0] and a[1] == b[1] for a, b in zip(cache[0], key)):
            return cache[1], cache[2]
        ps = self.pauli_strings()
        arr = (_lib.Pauli_t * max(len(ps), 1))()
        for i, (x, z, c) in enumerate(ps):
            arr[i].xmask, arr[i].zmask = x, z
            arr[i].coeff_re, arr[i].coeff_im = c.real, c.imag
        self._packed = (key, arr, len(ps))
        return arr, len(ps)

    def is_hermitian(self):
        return all(abs(np.conj(c) - c) < 1e-14 for _, _, c in self.pauli_strings())


def pauli(spec, coeff=1.0):
    """QubitsTerm from {position: 'X'|'Y'|'Z'} (1-based)."""
    return QubitsTerm(spec, coeff=coeff)
