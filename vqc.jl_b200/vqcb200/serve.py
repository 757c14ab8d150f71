"""Serving: many circuits batched on one GPU (continuous batching).

A `Server` wraps the C-ABI serving loop (vqc_serve_* in include/vqc_b200.h):
requests are queued from any thread; the device worker admits them by
memory, advances every admitted request by one step per loop iteration with
one launch per step kind, and retires them as they finish.
"""
import ctypes
import threading

import numpy as np

from . import _lib
from .circuit import Packed
from .operators import QubitsOperator, QubitsTerm

_DT = {np.dtype(np.complex64): _lib.VQC_C64, np.dtype(np.complex128): _lib.VQC_C128}


class Ticket:
    """A submitted request: keeps its input and output arrays alive."""

    def __init__(self, tid, packed, terms, grads, want_grad):
        self.id = tid
        self._packed = packed
        self._terms = terms
        self.grads = grads
        self.want_grad = want_grad
        self.energy = None
        self.latency = None


class Server:
    def __init__(self, device=0, dtype=np.complex64, memory_bytes=8 << 30, max_active=512, planner_threads=4):
        self._lib = _lib.load()
        self._h = ctypes.c_void_p()
        _lib.check(self._lib.vqc_serve_open(device, _DT[np.dtype(dtype)], memory_bytes, max_active, planner_threads,
                                            ctypes.byref(self._h)))
        self._lock = threading.Lock()

    def submit(self, nqubits, circuit, H, want_grad=True):
        """Queue expectation(H, circuit * |0...0>) [and its gradient]."""
        if isinstance(H, QubitsTerm):
            H = QubitsOperator(H)
        p = Packed(circuit, with_params=want_grad)
        arr, nt = H.packed()
        grads = np.zeros(max(p.nparams, 1))
        tid = ctypes.c_int64()
        _lib.check(self._lib.vqc_serve_submit(self._h, nqubits, p.gates, p.ngates, p.mats_ptr(), p.params,
                                              p.nparams if want_grad else 0, arr, nt, 1 if want_grad else 0,
                                              grads.ctypes.data_as(_lib._D), ctypes.byref(tid)))
        t = Ticket(tid.value, p, arr, grads, want_grad)
        t.nparams = p.nparams
        return t

    def submit_packed(self, nqubits, packed, terms, nterms, want_grad=True):
        """submit() with a circuit already packed (vqcb200.circuit.Packed) and a
        Pauli array (QubitsOperator.packed()); the objects must outlive the ticket."""
        grads = np.zeros(max(packed.nparams, 1))
        tid = ctypes.c_int64()
        _lib.check(self._lib.vqc_serve_submit(self._h, nqubits, packed.gates, packed.ngates, packed.mats_ptr(),
                                              packed.params, packed.nparams if want_grad else 0, terms, nterms,
                                              1 if want_grad else 0, grads.ctypes.data_as(_lib._D),
                                              ctypes.byref(tid)))
        t = Ticket(tid.value, packed, terms, grads, want_grad)
        t.nparams = packed.nparams
        return t

    def _finish(self, t, e, lat):
        t.energy = complex(e[0], e[1])
        t.latency = lat.value
        return t.energy, (t.grads[:t.nparams] if t.want_grad else None), t.latency

    def wait(self, t, timeout=120.0):
        """(energy, gradient or None, latency in seconds)."""
        e = (ctypes.c_double * 2)()
        lat = ctypes.c_double()
        _lib.check(self._lib.vqc_serve_wait(self._h, t.id, int(timeout * 1000), e, ctypes.byref(lat)))
        return self._finish(t, e, lat)

    def poll(self, t):
        e = (ctypes.c_double * 2)()
        lat = ctypes.c_double()
        rc = _lib.check(self._lib.vqc_serve_poll(self._h, t.id, e, ctypes.byref(lat)))
        if rc == 0:
            return None
        return self._finish(t, e, lat)

    def cancel(self, t):
        """Cancel a request; True when it was cancelled, False when it had
        already finished (its result can still be collected)."""
        return _lib.check(self._lib.vqc_serve_cancel(self._h, t.id)) == 1

    def stats(self):
        out = (ctypes.c_longlong * 7)()
        _lib.check(self._lib.vqc_serve_stats(self._h, out))
        keys = ["completed", "iterations", "launches", "request_steps", "bytes_admitted", "running", "waiting"]
        return dict(zip(keys, list(out)))

    def timing(self):
        out = (ctypes.c_double * 6)()
        _lib.check(self._lib.vqc_serve_timing(self._h, out))
        keys = ["plan_mean_s", "plan_max_s", "wait_mean_s", "wait_max_s", "run_mean_s", "run_max_s"]
        return dict(zip(keys, list(out)))

    def loop_timing(self):
        """Per busy loop iteration (one that launched work): mean host time building and
        enqueueing, mean wait for the device, mean host time retiring (seconds)."""
        out = (ctypes.c_double * 4)()
        _lib.check(self._lib.vqc_serve_loop_timing(self._h, out))
        n = max(out[3], 1.0)
        return {"iterations": int(out[3]), "build_s": out[0] / n, "device_wait_s": out[1] / n,
                "retire_s": out[2] / n}

    def close(self):
        if self._h:
            self._lib.vqc_serve_close(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
