"""QCircuit of the host mirror and its packing into the C ABI arrays.

QCircuit is a gate list (QuantumCircuits.jl's QCircuit, iterated by
applygates/generic/generic.jl:26-31).  `pack` turns it into the vqc_gate /
vqc_param arrays and the FP64 matrix pool of include/vqc_b200.h.
"""
import numpy as np

from . import _lib
from .gates import Gate


class QCircuit:
    def __init__(self, gates=()):
        self.gates = []
        for g in gates:
            self.push(g)

    def push(self, g):
        if not isinstance(g, Gate):
            raise TypeError("QCircuit holds Gate objects")
        self.gates.append(g)
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


class Packed:
    """ctypes arrays for one circuit: gates, matrix pool, parameters."""

    def __init__(self, circuit, with_params=True):
        gates = list(circuit)
        ng = len(gates)
        self.gates = (_lib.Gate_t * max(ng, 1))()
        chunks, off = [], 0
        params = []
        for i, g in enumerate(gates):
            k = g.nqubits
            t = self.gates[i]
            t.nq = k
            for b in range(k):
                t.pos[b] = g.positions[b] - 1  # 1-based -> 0-based
            t.mat = off
            m = np.ascontiguousarray(g.mat, dtype=np.complex128).view(np.float64).ravel()
            chunks.append(m)
            off += m.size
            if with_params:
                for dU in g.derivatives():
                    d = np.ascontiguousarray(dU, dtype=np.complex128).view(np.float64).ravel()
                    params.append((i, off))
                    chunks.append(d)
                    off += d.size
        self.mats = np.concatenate(chunks) if chunks else np.zeros(1)
        self.ngates = ng
        self.nparams = len(params)
        self.params = (_lib.Param_t * max(len(params), 1))()
        for j, (gi, o) in enumerate(params):
            self.params[j].gate = gi
            self.params[j].dmat = o

    def mats_ptr(self):
        return self.mats.ctypes.data_as(_lib._D)
