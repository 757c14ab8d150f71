"""Adjoint-mode differentiation through the device engine.

Mirrors the reference's Zygote adjoints: `*(circuit, psi)` with the circuit
pullback `back_propagate` (circuitdiff.jl:2-8, 23-32, 61-75) and
`expectation(H, psi)` with its pullback (expecdiff.jl:30-33, 68).  The Julia
wrapper exposes the same through a ChainRules `rrule`; this module is the
executable Python form.
"""
import ctypes

import numpy as np

from . import _lib
from .circuit import Packed
from .operators import QubitsOperator, QubitsTerm


def energy_and_gradient(H, circuit, psi0):
    """(E, dE/dtheta) for E = expectation(H, circuit * psi0).

    The gradient is that of real(E) with respect to the circuit's active
    parameters, in circuit order (active_parameters(circuit)), as
    `gradient(c -> real(expectation(H, c * psi0)), circuit)` returns it."""
    lib = _lib.load()
    if isinstance(H, QubitsTerm):
        H = QubitsOperator(H)
    p = Packed(circuit)
    arr, nt = H.packed()
    energy = (ctypes.c_double * 2)()
    grads = np.zeros(max(p.nparams, 1), dtype=np.float64)
    _lib.check(lib.vqc_adjoint_grad(psi0.handle, p.gates, p.ngates, p.mats_ptr(), p.params, p.nparams, arr, nt, energy,
                                    grads.ctypes.data_as(_lib._D)))
    return complex(energy[0], energy[1]), grads[:p.nparams]


def trace_prod(a, b, positions, M, dag_a=False, dag_b=False):
    """tr(op(a) M op(b)) of two DensityMatrix objects, M on the row qubits
    `positions` (1-based), op = identity or the conjugate transpose
    (expectation(x::DensityMatrix, m::Gate, y::DensityMatrix) is
    tr(x M y), circuitdiff.jl:35-40)."""
    from .state import _mat_ptr, _pos_array
    keep, mp = _mat_ptr(M)
    out = (ctypes.c_double * 2)()
    _lib.check(_lib.load().vqc_dm_trace_prod(a.handle, 1 if dag_a else 0, b.handle, 1 if dag_b else 0,
                                             len(positions), _pos_array(positions), mp, out))
    return complex(out[0], out[1])


def _dm_back_propagate(delta, circuit, y):
    """back_propagate(::AbstractMatrix, circuit, ::DensityMatrix)
    (circuitdiff.jl:42-59, 61-75), on the device, in place.  Per item, last
    to first: a gate uncomputes both, delta <- U^dagger delta U and
    y <- U^dagger y U, then each parameter's partial is
        Re[tr(delta^dagger D y) + tr(y D^dagger delta^dagger)],  D = U^dagger dU/dtheta
    (the derivative of Re <delta_out, U rho U^dagger>); a channel
    propagates delta <- S^dagger delta and y <- S^-1 y (apply_dagger!,
    apply_inverse!)."""
    from .gates import QuantumMap
    from .state import apply, apply_dagger, apply_inverse
    per_item = []
    for item in reversed(list(circuit)):
        if isinstance(item, QuantumMap):
            apply_dagger(item, delta)
            apply_inverse(item, y)
            continue
        ud = item.adjoint()
        apply(ud, delta)
        apply(ud, y)
        g = []
        for dU in item.derivatives():
            D = item.mat.conj().T @ np.asarray(dU, dtype=np.complex128)
            t1 = trace_prod(delta, y, item.positions, D, dag_a=True)
            t2 = trace_prod(y, delta, item.positions, D.conj().T, dag_b=True)
            g.append((t1 + t2).real)
        if g:
            per_item.append(g)
    grads = [x for g in reversed(per_item) for x in g]
    return delta, np.asarray(grads, dtype=np.float64), y


def back_propagate(delta, circuit, y):
    """back_propagate(delta, circuit, y) (circuitdiff.jl:61-75), in place:
    y (the circuit's output state) becomes the input state, delta (the
    cotangent of the output) becomes the cotangent of the input; returns
    (delta, grads, y) with grads[j] = Re <delta_out | dU/dtheta_j | y_in>.
    For density matrices (y a DensityMatrix, delta the cotangent matrix as a
    DensityMatrix) the circuit may hold quantum channels."""
    from .state import DensityMatrix
    if isinstance(y, DensityMatrix):
        return _dm_back_propagate(delta, circuit, y)
    lib = _lib.load()
    p = Packed(circuit)
    grads = np.zeros(max(p.nparams, 1), dtype=np.float64)
    _lib.check(lib.vqc_circuit_backward(y.handle, delta.handle, p.gates, p.ngates, p.mats_ptr(), p.params, p.nparams,
                                        grads.ctypes.data_as(_lib._D)))
    return delta, grads[:p.nparams], y
