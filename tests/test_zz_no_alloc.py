"""The allocation-free expectation entry point (vqc_expect_pauli_noalloc).

It serves callers that cannot allocate device memory: an application that
hands the library a fixed arena at start-up and forbids cudaMalloc/cudaFree
afterwards.  Its scratch lives in a static device array shared by all calls,
so this test calls it twice in a row on caller-owned device buffers and
checks both results against the regular entry point (vqc_expect_pauli), at
the tolerances of helpers.py.  It runs last (file name) so a failure here
leaves every other test already run; it also passes alone in a fresh process
(the first call on the device does the one-time symbol lookup)."""
import ctypes

import numpy as np
import pytest

import vqcb200 as V
from helpers import rand_psi
from vqcb200 import _lib
from vqcb200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype,tol", [(np.complex128, 1e-12), (np.complex64, 1e-5)])
def test_noalloc_expectation_matches_regular_entry_point(dtype, tol):
    import torch
    lib = V.load()
    rng = np.random.default_rng(77)
    code = _lib.VQC_C64 if dtype == np.complex64 else _lib.VQC_C128
    cases = []
    for n, hspec in ((14, W.xxz_spec(14, 0.5)), (20, W.tfim_spec(20, 0.9))):
        H = W.to_operator(hspec)
        arr, nt = H.packed()
        cases.append((n, H, arr, nt))
    # a random operator with many groups, within the 1024-term limit
    n = 12
    terms = []
    for _ in range(300):
        qs = rng.choice(n, int(rng.integers(1, 4)), replace=False)
        terms.append(V.QubitsTerm({int(q) + 1: "XYZ"[int(rng.integers(3))] for q in qs},
                                  coeff=complex(rng.standard_normal(), 0.2 * rng.standard_normal())))
    H = V.QubitsOperator(*terms)
    arr, nt = H.packed()
    cases.append((n, H, arr, nt))
    for n, H, arr, nt in cases:
        psi = V.StateVector(rand_psi(rng, n).astype(dtype), dtype=dtype)
        ref = V.expectation(H, psi)
        # the caller's own device buffer and stream (allocated by the caller, here torch)
        buf = torch.from_numpy(psi.storage().view(np.float32 if dtype == np.complex64 else np.float64).copy()).cuda()
        stream = torch.cuda.current_stream().cuda_stream
        torch.cuda.synchronize()
        for _ in range(2):  # two calls in a row share the static scratch
            out = (ctypes.c_double * 2)()
            _lib.check(lib.vqc_expect_pauli_noalloc(ctypes.c_void_p(buf.data_ptr()), n, code, arr, nt,
                                                    ctypes.c_void_p(stream), out))
            got = complex(out[0], out[1])
            assert abs(got - ref) <= tol * max(abs(ref), 1.0), (n, got, ref)


def test_noalloc_rejects_too_many_terms():
    import torch
    lib = V.load()
    buf = torch.zeros(2 << 10, dtype=torch.float64, device="cuda")
    arr = (_lib.Pauli_t * 1025)()
    for i in range(1025):
        arr[i].zmask = 1 << (i % 10)
        arr[i].coeff_re = 1.0
    out = (ctypes.c_double * 2)()
    rc = lib.vqc_expect_pauli_noalloc(ctypes.c_void_p(buf.data_ptr()), 10, _lib.VQC_C128, arr, 1025, None, out)
    assert rc == -1
    assert b"1024" in lib.vqc_last_error()


def test_noalloc_rejects_a_host_pointer():
    """A host buffer is refused before any launch (a kernel given it would fault)."""
    lib = V.load()
    host = np.zeros(2 << 10, dtype=np.float64)
    arr = (_lib.Pauli_t * 1)()
    arr[0].zmask = 1
    arr[0].coeff_re = 1.0
    out = (ctypes.c_double * 2)()
    rc = lib.vqc_expect_pauli_noalloc(ctypes.c_void_p(host.ctypes.data), 10, _lib.VQC_C128, arr, 1, None, out)
    assert rc == -1
    assert b"device" in lib.vqc_last_error()
