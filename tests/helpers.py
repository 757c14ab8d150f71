"""Shared checks for the parity tests.

Tolerances (stated once, used everywhere):
  * FP64 (complex128) device results vs the FP64 oracle: 1e-12, max-abs on
    normalised states and relative on scalars / gradient vectors;
  * FP32 (complex64) states with FP64 accumulation: 1e-5 relative on
    expectations (relative to max(|E|, 1): these Hamiltonians have norm of
    order n, so an energy that cancels to ~0 is compared against that scale)
    and norm-wise on gradients; 1e-5 max-abs on normalised states
    after short circuits (the error grows with circuit depth: long-circuit
    tests state their own bound).
"""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = {np.dtype(np.complex128): 1e-12, np.dtype(np.complex64): 1e-5}


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False))


def tol(dtype):
    return TOL[np.dtype(dtype)]


def max_abs(a, b):
    return float(np.abs(np.asarray(a, dtype=np.complex128) - np.asarray(b, dtype=np.complex128)).max())


def rel(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    den = max(float(np.linalg.norm(b)), 1e-300)
    return float(np.linalg.norm(a - b)) / den


def rand_psi(rng, n):
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    return v / np.linalg.norm(v)
