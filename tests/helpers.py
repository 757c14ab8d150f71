"""Shared checks for the parity tests.

Bounds (stated once here and asserted as they stand, with no multipliers):
  * FP64 (complex128) device results against the FP64 oracle: 1e-12 --
    max-abs on normalised states (`max_abs`), relative on scalars (`rel_scalar`)
    and norm-wise relative on vectors that are not normalised: gradients,
    H psi, density matrices after non-unitary maps (`rel`, `max_rel`);
  * FP32 (complex64) states with FP64 accumulation: 1e-5, in the same forms
    (relative on expectations, norm-wise relative on gradients, max-abs on
    normalised states).

Identical inputs: the device computes an FP32 state from the FP32-rounded
input, so FP32 results are compared against the oracle run on exactly that
input (`as_input`), held in FP64.  The bound then measures the device's own
arithmetic, not the rounding of the input.
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = {np.dtype(np.complex128): 1e-12, np.dtype(np.complex64): 1e-5}


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def tol(dtype):
    return TOL[np.dtype(dtype)]


def as_input(a, dtype):
    """The array the device holds when given `a` in `dtype`, as complex128."""
    return np.asarray(a).astype(dtype).astype(np.complex128)


def max_abs(a, b):
    return float(np.abs(np.asarray(a, dtype=np.complex128) - np.asarray(b, dtype=np.complex128)).max())


def max_rel(a, b):
    """max |a - b| relative to max |b| (vectors that are not normalised)."""
    b = np.asarray(b, dtype=np.complex128)
    return max_abs(a, b) / max(float(np.abs(b).max()), 1e-300)


def rel(a, b):
    """Norm-wise relative difference ||a - b|| / ||b||."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    den = max(float(np.linalg.norm(b)), 1e-300)
    return float(np.linalg.norm(a - b)) / den


def rel_scalar(a, b):
    """|a - b| / |b| for scalars (energies, traces, inner products)."""
    return abs(complex(a) - complex(b)) / max(abs(complex(b)), 1e-300)


def rand_psi(rng, n):
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)


def max_abs_chunked(dev, ref, chunk=1 << 26):
    """max |dev - ref| over two long vectors, a chunk at a time (bounded
    temporary memory for states of 2^30 amplitudes)."""
    m = 0.0
    for i in range(0, ref.size, chunk):
        d = dev[i:i + chunk].astype(np.complex128) - ref[i:i + chunk]
        m = max(m, float(np.abs(d).max()))
    return m
