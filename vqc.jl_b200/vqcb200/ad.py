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


def back_propagate(delta, circuit, y):
    """back_propagate(delta, circuit, y) (circuitdiff.jl:61-75), in place:
    y (the circuit's output state) becomes the input state, delta (the
    cotangent of the output) becomes the cotangent of the input; returns
    (delta, grads, y) with grads[j] = Re <delta_out | dU/dtheta_j | y_in>."""
    lib = _lib.load()
    p = Packed(circuit)
    grads = np.zeros(max(p.nparams, 1), dtype=np.float64)
    _lib.check(lib.vqc_circuit_backward(y.handle, delta.handle, p.gates, p.ngates, p.mats_ptr(), p.params, p.nparams,
                                        grads.ctypes.data_as(_lib._D)))
    return delta, grads[:p.nparams], y
