"""QCircuit of the host mirror and its packing into the C ABI arrays.

QCircuit is a gate list (QuantumCircuits.jl's QCircuit, iterated by
applygates/generic/generic.jl:26-31).  `pack` turns it into the vqc_gate /
vqc_param arrays and the FP64 matrix pool of include/vqc_b200.h.
"""
import ctypes

import numpy as np

from . import _lib
from .gates import Gate, QuantumMap


class QCircuit:
    def __init__(self, gates=()):
        self.gates = []
        for g in gates:
            self.push(g)

    def push(self, g):
        if not isinstance(g, (Gate, QuantumMap)):
            raise TypeError("QCircuit holds Gate and QuantumMap objects")
        self.gates.append(g)
        self._packed = None
        return self

    append = push

    def __iter__(self):
        return iter(self.gates)

    def __len__(self):
        return len(self.gates)

    def __getitem__(self, i):
        return self.gates[i]

    def nparameters(self):
        return sum(g.nparameters() for g in self.gates)

    def active_parameters(self):
        out = []
        for g in self.gates:
            out.extend(g.active_parameters())
        return out

    def adjoint(self):
        return QCircuit([g.adjoint() for g in reversed(self.gates)])

    def max_position(self):
        return max((max(g.positions) for g in self.gates), default=0)

    def __mul__(self, state):
        """circuit * state: apply to a copy (generic.jl:33)."""
        from .state import apply
        return apply(self, state.copy())


_GATE_DT = np.dtype([("nq", "<i4"), ("pos", "<i4", (5,)), ("mat", "<i8")], align=True)
_PARAM_DT = np.dtype([("gate", "<i4"), ("kind", "<i4"), ("dmat", "<i8")], align=True)
assert _GATE_DT.itemsize == ctypes.sizeof(_lib.Gate_t) and _PARAM_DT.itemsize == ctypes.sizeof(_lib.Param_t)


def _gate_pack(g):
    """Per-gate packing (0-based padded positions, FP64 matrix and derivative
    matrices flattened re/im), computed once per Gate object: gates are
    values, not changed after construction."""
    pk = getattr(g, "_pk", None)
    if pk is None:
        pos = tuple(p - 1 for p in g.positions) + (0,) * (5 - g.nqubits)
        mat = np.ascontiguousarray(g.mat, dtype=np.complex128).view(np.float64).ravel()
        ders = tuple(np.ascontiguousarray(d, dtype=np.complex128).view(np.float64).ravel() for d in g.derivatives())
        pk = g._pk = (g.nqubits, pos, mat, ders)
    return pk


class Packed:
    """ctypes arrays for one circuit: gates, matrix pool, parameters.

    Built with numpy (the C structs' layouts as structured dtypes) and cached
    on the QCircuit for as long as it holds the same gate objects, so a
    circuit evaluated repeatedly (an optimisation loop) is packed once."""

    def __new__(cls, circuit, with_params=True):
        cache = getattr(circuit, "_packed", None) if isinstance(circuit, QCircuit) else None
        gates = list(circuit)
        if cache is not None:
            key_gates, wp, packed = cache
            if wp == with_params and len(key_gates) == len(gates) and all(a is b for a, b in zip(key_gates, gates)):
                return packed
        self = super().__new__(cls)
        self._build(gates, with_params)
        if isinstance(circuit, QCircuit):
            circuit._packed = (gates, with_params, self)
        return self

    def __init__(self, circuit, with_params=True):
        pass

    def _build(self, gates, with_params):
        if any(isinstance(g, QuantumMap) for g in gates):
            raise TypeError("a circuit with quantum channels applies to a DensityMatrix, gate run by gate run")
        ng = len(gates)
        pks = [_gate_pack(g) for g in gates]
        chunks, offs, params = [], [], []
        off = 0
        for i, (k, pos, mat, ders) in enumerate(pks):
            offs.append(off)
            chunks.append(mat)
            off += mat.size
            if with_params:
                for d in ders:
                    params.append((i, off))
                    chunks.append(d)
                    off += d.size
        self._garr = np.zeros(max(ng, 1), _GATE_DT)
        if ng:
            self._garr["nq"][:ng] = [pk[0] for pk in pks]
            self._garr["pos"][:ng] = [pk[1] for pk in pks]
            self._garr["mat"][:ng] = offs
        self._parr = np.zeros(max(len(params), 1), _PARAM_DT)
        if params:
            pa = np.asarray(params, dtype=np.int64)
            self._parr["gate"][:len(params)] = pa[:, 0]
            self._parr["dmat"][:len(params)] = pa[:, 1]
        self.gates = (_lib.Gate_t * len(self._garr)).from_buffer(self._garr)
        self.params = (_lib.Param_t * len(self._parr)).from_buffer(self._parr)
        self.mats = np.concatenate(chunks) if chunks else np.zeros(1)
        self.ngates = ng
        self.nparams = len(params)

    def mats_ptr(self):
        return self.mats.ctypes.data_as(_lib._D)
