"""vqcb200: the Python host mirror of VQC.jl's state-vector API, running on
the B200 engine libvqcb200.so through its C ABI (include/vqc_b200.h).

Julia names map as: apply! -> apply, expectation -> expectation,
partial_tr -> partial_tr, circuit * psi -> circuit * psi, the Zygote
gradient of real(expectation(H, circuit * psi0)) -> energy_and_gradient.
"""
from . import _lib
from .ad import back_propagate, energy_and_gradient
from .circuit import QCircuit
from .gates import *  # noqa: F401,F403
from .krylov import ground_state, time_evolution
from .measure import measure, measure_inplace, post_select, post_select_inplace, prob_zero
from .operators import QubitsOperator, QubitsTerm, pauli
from .state import (DensityMatrix, StateVector, apply, apply_dagger, apply_inverse, apply_operator, expectation,
                    fidelity, partial_tr,
                    probabilities, rand_state)


def load():
    """Load libvqcb200.so (raises if it has not been built)."""
    return _lib.load()
