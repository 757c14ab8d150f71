"""Pauli sums on states of 2^18 and more amplitudes: the tile passes (a pass
stages 2^13 FP32 / 2^12 FP64 amplitudes over chosen qubits in shared memory;
flip masks inside them read their partners there, the others from global
memory) against the oracle's per-key restatement of expecs.jl:22-74 and
apply_qterms.jl:13-28, and against the single global pass (VQC_PAULI_TILE=0),
on the same inputs.  At n = 18 the passes run on the generic tile kernel, from
n = 20 on the kernels compiled per operator structure (VQC_JIT=off: generic).
Bounds: helpers.py (1e-12 FP64, 1e-5 FP32)."""
import numpy as np
import pytest

import vqcb200 as V
from helpers import as_input, max_rel, rel, rel_scalar, tol
from oracle import oracle as O
from vqcb200 import workloads as W

pytestmark = pytest.mark.gpu
DTYPES = [np.complex128, np.complex64]
NTHREADS = 8


def product_like(rng, n, noise=0.05):
    """A product state plus a little noise: every Pauli string has an O(1)
    expectation, so relative bounds on scalars are meaningful."""
    v = np.ones(1, dtype=np.complex128)
    for _ in range(n):
        a = rng.standard_normal(2) + 1j * rng.standard_normal(2)
        v = np.kron(a / np.linalg.norm(a), v)
    v = v + noise * (rng.standard_normal(v.size) + 1j * rng.standard_normal(v.size)) / np.sqrt(v.size)
    return v / np.linalg.norm(v)


def random_terms(rng, n, nterms, complex_coeff):
    spec = []
    for _ in range(nterms):
        w = int(rng.integers(1, 5))
        qs = rng.choice(n, w, replace=False)
        ops = {int(q) + 1: "XYZ"[int(rng.integers(3))] for q in qs}
        c = float(rng.standard_normal())
        if complex_coeff:
            c = complex(c, float(rng.standard_normal()))
        spec.append((c, ops))
    return spec


OPERATORS = {
    "xxz": lambda rng, n: W.xxz_spec(n),
    "tfim": lambda rng, n: W.tfim_spec(n, 0.7),
    "random_real": lambda rng, n: random_terms(rng, n, 40, False),
    "random_complex": lambda rng, n: random_terms(rng, n, 40, True),
    # flip masks joining a low and a high qubit (no pass covers them) and Z fields
    "far_pairs": lambda rng, n: ([(0.3 + 0.1 * k, {1 + k: "X", n - k: "Y"}) for k in range(n // 2)]
                                 + [(0.5, {q: "Z"}) for q in range(1, n + 1)]),
}


def oterms(spec):
    return [O.make_term({q - 1: o for q, o in ops.items()}, c) for c, ops in spec]


def sv(a, dtype):
    return V.StateVector(np.asarray(a, dtype=dtype), dtype=dtype)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", sorted(OPERATORS))
@pytest.mark.parametrize("n", [18, 21])
def test_tile_passes_match_oracle(dtype, name, n):
    rng = np.random.default_rng(1800 + n)
    spec = OPERATORS[name](rng, n)
    H, T = W.to_operator(spec), oterms(spec)
    psi = product_like(rng, n)
    phi = psi + 0.1 * product_like(rng, n)
    phi /= np.linalg.norm(phi)
    pin, fin = as_input(psi, dtype), as_input(phi, dtype)
    e = V.expectation(H, sv(psi, dtype))
    assert rel_scalar(e, O.expectation(T, pin, nthreads=NTHREADS)) < tol(dtype)
    e2 = V.expectation(sv(phi, dtype), H, sv(psi, dtype))
    assert rel_scalar(e2, O.expectation(T, pin, vc=fin, nthreads=NTHREADS)) < tol(dtype)
    out = V.apply_operator(H, sv(psi, dtype))
    assert max_rel(out.storage(), O.apply_operator(T, pin, nthreads=NTHREADS)) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", ["xxz", "random_complex", "far_pairs"])
def test_tile_passes_agree_with_one_global_pass(dtype, name, monkeypatch):
    n = 20
    rng = np.random.default_rng(2000)
    spec = OPERATORS[name](rng, n)
    H = W.to_operator(spec)
    psi = product_like(rng, n)
    res = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("VQC_PAULI_TILE", mode)
        res[mode] = (V.expectation(H, sv(psi, dtype)), V.apply_operator(H, sv(psi, dtype)).storage())
    assert rel_scalar(res["1"][0], res["0"][0]) < tol(dtype)
    assert max_rel(res["1"][1], res["0"][1]) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
@pytest.mark.parametrize("name", ["xxz", "random_complex", "tfim"])
def test_compiled_passes_agree_with_generic_tile_kernel(dtype, name, monkeypatch):
    n = 21
    rng = np.random.default_rng(2100)
    spec = OPERATORS[name](rng, n)
    H = W.to_operator(spec)
    psi = product_like(rng, n)
    phi = psi + 0.1 * product_like(rng, n)
    phi /= np.linalg.norm(phi)
    res = {}
    for mode in ("auto", "off"):
        monkeypatch.setenv("VQC_JIT", mode)
        res[mode] = (V.expectation(H, sv(psi, dtype)), V.expectation(sv(phi, dtype), H, sv(psi, dtype)),
                     V.apply_operator(H, sv(psi, dtype)).storage())
    for i in range(2):
        assert rel_scalar(res["auto"][i], res["off"][i]) < tol(dtype)
    assert max_rel(res["auto"][2], res["off"][2]) < tol(dtype)


@pytest.mark.parametrize("dtype", DTYPES)
def test_gradient_through_tile_passes(dtype, monkeypatch):
    # the gradient's Pauli pass: E and (H + H^dagger) psi in one sweep
    n = 20
    rng = np.random.default_rng(1818)
    spec = W.rxyz_crx_spec(n, 2, rng.uniform(0, 2 * np.pi, 2 * (4 * n - 1)))
    H = W.to_operator(W.xxz_spec(n))
    res = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("VQC_PAULI_TILE", mode)
        res[mode] = V.energy_and_gradient(H, W.to_circuit(spec), V.StateVector(n, dtype=dtype))
    e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(W.xxz_spec(n)), O.zero_state(n),
                                         nthreads=NTHREADS)
    for mode in ("1", "0"):
        assert rel_scalar(res[mode][0], e_ref) < tol(dtype), mode
        assert rel(res[mode][1], g_ref) < tol(dtype), mode
