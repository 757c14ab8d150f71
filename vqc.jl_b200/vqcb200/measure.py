"""Measurement and post-selection (measure.jl, postselect.jl) on the device.

Julia's in-place forms map to *_inplace names:
  measure!(psi, pos; auto_reset)  -> measure_inplace(psi, pos, auto_reset, rng)
  measure(psi, pos)               -> measure(psi, pos, rng)
  post_select!(psi, key, state)   -> post_select_inplace(psi, key, state)
  post_select(psi, key, state; keep) -> post_select(psi, key, state, keep)
Positions are 1-based.  The outcome is drawn from [p0, 1 - p0] with the
numpy Generator `rng` (the reference's discrete_sample on Julia's global
RNG); pass a seeded one for reproducible runs.  All arithmetic on the state
(probabilities, collapse, normalisation) runs on the device.
"""
import numpy as np

from .gates import Gate
from .operators import QubitsOperator, QubitsTerm
from .state import DensityMatrix, StateVector, apply, expectation
from . import _lib


def prob_zero(state, pos):
    """compute_probability_zero(state, pos) (measure.jl:47-59, 69-81): the
    weight of the amplitudes (or diagonal entries) with qubit pos at 0,
    (norm^2 + <Z_pos>) / 2 from the device's FP64 reductions."""
    z = expectation(QubitsOperator(QubitsTerm({pos: "Z"})), state).real
    total = state.tr().real if isinstance(state, DensityMatrix) else state.norm() ** 2
    return 0.5 * (total + z)


def _draw(p0, rng):
    u = (rng if rng is not None else np.random.default_rng()).random()
    return (0, p0) if u < p0 else (1, 1.0 - p0)


def measure_inplace(state, pos, auto_reset=True, rng=None):
    """measure!(state, pos; auto_reset) (measure.jl:4-27): samples the qubit,
    collapses the state in place (the measured qubit reset to 0 if
    auto_reset) and returns (outcome, probability)."""
    i, p = _draw(prob_zero(state, pos), rng)
    m = np.zeros((2, 2), dtype=complex)
    m[0 if auto_reset else i, i] = 1.0 / np.sqrt(p)
    apply(Gate((pos,), m), state)  # m rho m^dagger for a density matrix
    return i, p


def measure(state, pos, rng=None):
    """measure(psi, pos) (measure.jl:30-46): (the collapsed state without the
    measured qubit, outcome, probability)."""
    if isinstance(state, DensityMatrix):
        raise TypeError("measure(psi, pos) takes a StateVector")
    i, p = _draw(prob_zero(state, pos), rng)
    out = StateVector(state.nqubits - 1, dtype=state.dtype, device=state.device)
    _lib.check(_lib.load().vqc_state_take_qubit(state.handle, pos - 1, i, 1.0 / np.sqrt(p), out.handle))
    return out, i, p


def post_select_inplace(state, key, value=0):
    """post_select!(psi, key, state) (postselect.jl:3-15): projects qubit key
    on |value>, normalises in place, returns the norm before normalising."""
    p0 = prob_zero(state, key)
    p = p0 if value == 0 else 1.0 - p0
    m = np.zeros((2, 2), dtype=complex)
    m[value, value] = 1.0 / np.sqrt(p)
    apply(Gate((key,), m), state)
    return float(np.sqrt(p))


def post_select(state, key, value=0, keep=False):
    """post_select(psi, key, state; keep) (postselect.jl:17-44): (the
    normalised projected state, its norm); without keep the qubit is removed."""
    p0 = prob_zero(state, key)
    p = p0 if value == 0 else 1.0 - p0
    if keep:
        out = state.copy()
        m = np.zeros((2, 2), dtype=complex)
        m[value, value] = 1.0 / np.sqrt(p)
        apply(Gate((key,), m), out)
        return out, float(np.sqrt(p))
    out = StateVector(state.nqubits - 1, dtype=state.dtype, device=state.device)
    _lib.check(_lib.load().vqc_state_take_qubit(state.handle, key - 1, value, 1.0 / np.sqrt(p), out.handle))
    return out, float(np.sqrt(p))
