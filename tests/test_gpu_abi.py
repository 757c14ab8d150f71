"""GPU tests of C-ABI behaviour that the host mirror does not exercise on its
own: parameter conventions, error statuses, stream interop, profiling."""
import ctypes

import numpy as np
import pytest

import vqcb200 as V
from helpers import rand_psi, rel
from oracle import oracle as O
from vqcb200 import _lib
from vqcb200 import workloads as W
from vqcb200.circuit import Packed

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [8, 13])
def test_generator_kind_matches_derivative_kind(n):
    """VQC_PARAM_GENERATOR takes the gate G of QuantumCircuits' differentiate
    (grad = real(expectation(y_in, G, delta_in)), circuitdiff.jl:29); with
    G = (dU/dtheta)^dagger U it must give the same gradients as the
    derivative form."""
    rng = np.random.default_rng(40 + n)
    layers = 2
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    c = W.to_circuit(W.rxyz_crx_spec(n, layers, th))
    H = W.to_operator(W.xxz_spec(n, 0.5))
    e1, g1 = V.energy_and_gradient(H, c, V.StateVector(n))
    p = Packed(c)
    # rewrite every parameter as generator kind
    gates = list(c)
    chunks = [p.mats]
    off = p.mats.size
    for j in range(p.nparams):
        gi = p.params[j].gate
        U = gates[gi].mat
        k = gates[gi].nqubits
        dU = p.mats[p.params[j].dmat:p.params[j].dmat + 2 * 4 ** k].view(np.complex128).reshape(1 << k, 1 << k)
        G = dU.conj().T @ U
        chunks.append(np.ascontiguousarray(G).view(np.float64).ravel())
        p.params[j].kind = 1
        p.params[j].dmat = off
        off += 2 * 4 ** k
    mats = np.concatenate(chunks)
    arr, nt = H.packed()
    energy = (ctypes.c_double * 2)()
    g2 = np.zeros(p.nparams)
    psi0 = V.StateVector(n)  # keep a reference: the handle lives as long as the object
    _lib.check(V.load().vqc_adjoint_grad(psi0.handle, p.gates, p.ngates,
                                         mats.ctypes.data_as(_lib._D), p.params, p.nparams, arr, nt, energy,
                                         g2.ctypes.data_as(_lib._D)))
    assert abs(complex(energy[0], energy[1]) - e1) < 1e-12
    assert rel(g2, g1) < 1e-12


def test_bad_parameter_kind_and_gate_index():
    c = V.QCircuit([V.RxGate(1, 0.3, isparas=True)])
    p = Packed(c)
    H = V.QubitsOperator(V.pauli({1: "Z"}))
    arr, nt = H.packed()
    energy = (ctypes.c_double * 2)()
    g = np.zeros(1)
    lib = V.load()
    psi0 = V.StateVector(3)
    p.params[0].kind = 7
    rc = lib.vqc_adjoint_grad(psi0.handle, p.gates, p.ngates, p.mats_ptr(), p.params, 1, arr, nt, energy,
                              g.ctypes.data_as(_lib._D))
    assert rc == -1
    p.params[0].kind = 0
    p.params[0].gate = 5
    rc = lib.vqc_adjoint_grad(psi0.handle, p.gates, p.ngates, p.mats_ptr(), p.params, 1, arr, nt, energy,
                              g.ctypes.data_as(_lib._D))
    assert rc == -1
    assert b"out of range" in lib.vqc_last_error()


def test_upload_size_mismatch_and_null_handles():
    lib = V.load()
    s = V.StateVector(4)
    buf = np.zeros(8, dtype=np.complex128)
    assert lib.vqc_state_upload(s.handle, buf.ctypes.data, buf.nbytes) == -1
    assert lib.vqc_state_norm(None, None) == -1
    h = ctypes.c_void_p()
    assert lib.vqc_state_create(0, 1, 0, ctypes.byref(h)) == -1
    assert lib.vqc_state_create(4, 7, 0, ctypes.byref(h)) == -1


def test_stream_interop_and_profile():
    import torch
    s = V.StateVector(20)
    ptr = V.load().vqc_state_stream(s.handle)
    assert ptr
    st = torch.cuda.ExternalStream(ptr)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    _lib.profile_enable(True)
    a.record(st)
    V.apply(V.HGate(20), s)
    V.apply(V.CZGate(1, 20), s)
    b.record(st)
    b.synchronize()
    prof = _lib.profile_read()
    _lib.profile_enable(False)
    assert prof["gate_dense"][0] == 1 and prof["gate_diag"][0] == 1
    assert a.elapsed_time(b) > 0


def test_energy_matches_oracle_at_22_qubits_fp32():
    """A mid-size FP32 check of the headline path (fused forward, Pauli pass,
    fused reverse sweep) against the FP64 oracle: 1e-5 relative."""
    n, layers = 22, 2
    rng = np.random.default_rng(44)
    th = rng.uniform(0, 2 * np.pi, layers * (4 * n - 1))
    spec = W.rxyz_crx_spec(n, layers, th)
    hspec = W.xxz_spec(n, 0.5)
    e, g = V.energy_and_gradient(W.to_operator(hspec), W.to_circuit(spec), V.StateVector(n, dtype=np.complex64))
    e_ref, g_ref = O.energy_and_gradient(O.from_spec(spec), O.terms_from_spec(hspec), O.zero_state(n), nthreads=16)
    assert abs(e - e_ref) / abs(e_ref) < 1e-5
    assert rel(g, g_ref) < 1e-5
