"""StateVector / DensityMatrix of the host mirror, and the reference's
operations on them: apply! (here `apply`), expectation, partial_tr,
probabilities, norm, dot, fidelity, distance.

Every operation runs on the device through libvqcb200 (include/vqc_b200.h).
Positions are 1-based, as in VQC.jl.
"""
import ctypes

import numpy as np

from . import _lib
from .circuit import Packed, QCircuit
from .gates import Gate, QuantumMap
from .operators import QubitsOperator, QubitsTerm

_DTYPES = {np.dtype(np.complex64): _lib.VQC_C64, np.dtype(np.complex128): _lib.VQC_C128}


def _dt(dtype):
    dtype = np.dtype(dtype)
    if dtype not in _DTYPES:
        raise TypeError("StateVector holds complex64 or complex128 amplitudes")
    return dtype


class _Handle:
    def __init__(self):
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            if self.h and _lib._lib is not None:
                _lib._lib.vqc_state_destroy(self.h)
        except Exception:
            pass


class StateVector:
    """StateVector{T} (statevector.jl:1-21): 2^n amplitudes on a CUDA device."""

    def __init__(self, data, nqubits=None, dtype=None, device=0):
        lib = _lib.load()
        if isinstance(data, (int, np.integer)):
            n, arr = int(data), None
            self.dtype = _dt(np.complex128 if dtype is None else dtype)
        else:
            arr = np.asarray(data)
            if dtype is None:
                dtype = arr.dtype if arr.dtype == np.complex64 else np.complex128
            self.dtype = _dt(dtype)
            arr = np.ascontiguousarray(arr, dtype=self.dtype).ravel()
            n = int(round(np.log2(arr.size)))
            if (1 << n) != arr.size:
                raise ValueError("state can not be interpretted as a qubit state.")
            if nqubits is not None and nqubits != n:
                raise ValueError("length(data) must be 2^nqubits")
        self._n = n
        self.device = device
        self._h = _Handle()
        _lib.check(self._create(lib, n))
        if arr is not None:
            self.upload(arr)

    def _create(self, lib, n):
        return lib.vqc_state_create(n, _DTYPES[self.dtype], self.device, ctypes.byref(self._h.h))

    @property
    def handle(self):
        return self._h.h

    @property
    def nqubits(self):
        return self._n

    def __len__(self):
        return 1 << self._n

    def upload(self, arr):
        arr = np.ascontiguousarray(arr, dtype=self.dtype).ravel()
        _lib.check(_lib.load().vqc_state_upload(self.handle, arr.ctypes.data, arr.nbytes))
        return self

    def storage(self):
        """storage(x): the amplitudes as a host array (a copy)."""
        out = np.empty(1 << _lib.load().vqc_state_nqubits(self.handle), dtype=self.dtype)
        _lib.check(_lib.load().vqc_state_download(self.handle, out.ctypes.data, out.nbytes))
        return out

    amplitudes = storage

    def copy(self):
        r = self.__class__.__new__(self.__class__)
        r.__dict__.update({k: v for k, v in self.__dict__.items() if k != "_h"})
        r._h = _Handle()
        _lib.check(r._create(_lib.load(), self._n))
        _lib.check(_lib.load().vqc_state_copy(r.handle, self.handle))
        return r

    def astype(self, dtype):
        r = self.__class__.__new__(self.__class__)
        r.__dict__.update({k: v for k, v in self.__dict__.items() if k != "_h"})
        r.dtype = _dt(dtype)
        r._h = _Handle()
        _lib.check(r._create(_lib.load(), self._n))
        _lib.check(_lib.load().vqc_state_copy(r.handle, self.handle))
        return r

    def reset(self):
        """reset!(x) (statevector.jl:110-114)."""
        _lib.check(_lib.load().vqc_state_reset(self.handle))
        return self

    def norm(self):
        out = ctypes.c_double()
        _lib.check(_lib.load().vqc_state_norm(self.handle, ctypes.byref(out)))
        return out.value

    def dot(self, other):
        """<self|other> (statevector.jl:54)."""
        out = (ctypes.c_double * 2)()
        _lib.check(_lib.load().vqc_state_dot(self.handle, other.handle, out))
        return complex(out[0], out[1])

    def sync(self):
        _lib.check(_lib.load().vqc_state_sync(self.handle))


class DensityMatrix(StateVector):
    """DensityMatrix{T} (densitymatrix.jl:1-30): the 4^n entries of rho on the
    device, row qubits on index bits 0..n-1, column qubits on n..2n-1."""

    def __init__(self, data, nqubits=None, dtype=None, device=0):
        lib = _lib.load()
        self.device = device
        if isinstance(data, StateVector):
            self.dtype = data.dtype
            self._n = data.nqubits
            self._h = _Handle()
            _lib.check(self._create(lib, self._n))
            _lib.check(lib.vqc_dm_from_state(self.handle, data.handle))
            return
        if isinstance(data, (int, np.integer)):
            self.dtype = _dt(np.complex128 if dtype is None else dtype)
            self._n = int(data)
            self._h = _Handle()
            _lib.check(self._create(lib, self._n))
            return
        arr = np.asarray(data)
        if dtype is None:
            dtype = arr.dtype if arr.dtype == np.complex64 else np.complex128
        self.dtype = _dt(dtype)
        if arr.ndim == 2:
            arr = arr.reshape(-1, order="F")  # column-major storage, as Julia's reshape
        n = int(round(np.log2(arr.size) / 2))
        if (1 << (2 * n)) != arr.size:
            raise ValueError("DimensionMismatch")
        self._n = n
        self._h = _Handle()
        _lib.check(self._create(lib, n))
        self.upload(arr)

    def _create(self, lib, n):
        return lib.vqc_dm_create(n, _DTYPES[self.dtype], self.device, ctypes.byref(self._h.h))

    def __len__(self):
        return 1 << (2 * self._n)

    def storage(self):
        """storage(rho): the L x L matrix (a copy)."""
        flat = StateVector.storage(self)
        L = 1 << self._n
        return flat.reshape((L, L), order="F")

    def data(self):
        return StateVector.storage(self)

    def tr(self):
        out = (ctypes.c_double * 2)()
        _lib.check(_lib.load().vqc_dm_trace(self.handle, out))
        return complex(out[0], out[1])


# ----------------------------------------------------------------------------- operations
def _pos_array(positions):
    arr = (ctypes.c_int * len(positions))(*[p - 1 for p in positions])
    return arr


def _mat_ptr(m):
    a = np.ascontiguousarray(m, dtype=np.complex128).view(np.float64).ravel()
    return a, a.ctypes.data_as(_lib._D)


def apply(x, state, fuse=True):
    """apply!(x, state) in place (applygates/generic/generic.jl:6-31); returns state."""
    lib = _lib.load()
    dm = isinstance(state, DensityMatrix)
    if isinstance(x, Gate):
        if x.nqubits > 5:
            raise NotImplementedError("only implement 5-qubit gates and less currently.")
        if max(x.positions) > state.nqubits or min(x.positions) < 1:
            raise ValueError("gate position out of range")
        keep, mp = _mat_ptr(x.mat)
        f = lib.vqc_dm_apply_gate if dm else lib.vqc_apply_gate
        _lib.check(f(state.handle, x.nqubits, _pos_array(x.positions), mp))
        return state
    if isinstance(x, QuantumMap):
        return _apply_channel(x, state, 0)
    if isinstance(x, QCircuit):
        if any(isinstance(g, QuantumMap) for g in x):
            # gate runs through the tile engine, channels one by one (on rho)
            if not dm:
                state = DensityMatrix(state)
            run = []
            for g in list(x) + [None]:
                if isinstance(g, Gate):
                    run.append(g)
                    continue
                if run:
                    apply(QCircuit(run), state, fuse=fuse)
                    run = []
                if g is not None:
                    _apply_channel(g, state, 0)
            return state
        for g in x:
            if g.nqubits > 5:
                raise NotImplementedError("only implement 5-qubit gates and less currently.")
        p = Packed(x, with_params=False)
        f = lib.vqc_dm_apply_circuit if dm else lib.vqc_apply_circuit
        _lib.check(f(state.handle, p.gates, p.ngates, p.mats_ptr(), 1 if fuse else 0))
        return state
    raise TypeError("apply takes a Gate or a QCircuit")


def _apply_channel(x, state, mode):
    """apply!(::QuantumMap, rho) (apply_qmaps.jl:5-14); a StateVector becomes
    DensityMatrix(state) first (apply_qmaps.jl:16).  mode 1: apply_dagger!,
    2: apply_inverse!."""
    if not isinstance(state, DensityMatrix):
        state = DensityMatrix(state)
    if max(x.positions) > state.nqubits or min(x.positions) < 1:
        raise ValueError("channel position out of range")
    kr = np.ascontiguousarray(np.stack(x.kraus), dtype=np.complex128).view(np.float64).ravel()
    _lib.check(_lib.load().vqc_dm_apply_channel(state.handle, x.nqubits, _pos_array(x.positions), len(x.kraus),
                                                kr.ctypes.data_as(_lib._D), mode))
    return state


def apply_dagger(x, rho):
    """apply_dagger!(::QuantumMap, rho) (apply_qmaps.jl:21-30): the adjoint of
    the channel's supermatrix, in place."""
    return _apply_channel(x, rho, 1)


def apply_inverse(x, rho):
    """apply_inverse!(::QuantumMap, rho) (apply_qmaps.jl:36-45): the inverse of
    the channel's supermatrix, in place (raises if it is singular)."""
    return _apply_channel(x, rho, 2)


def _as_operator(m):
    if isinstance(m, QubitsTerm):
        return QubitsOperator(m)
    return m


def expectation(*args):
    """expectation(H, psi) or expectation(phi, H, psi) (expecs.jl:12-78).

    H: QubitsOperator / QubitsTerm (Pauli-sum path), or a Gate (one dense key,
    expectation_value(ordered_positions(m), ordered_mat(m), ...))."""
    lib = _lib.load()
    if len(args) == 2:
        m, psi = args
        phi = None
    elif len(args) == 3:
        phi, m, psi = args
    else:
        raise TypeError("expectation(H, psi) or expectation(phi, H, psi)")
    out = (ctypes.c_double * 2)()
    m = _as_operator(m)
    if isinstance(psi, DensityMatrix):
        # tr(H rho) (expecs_dm.jl:19-30)
        if phi is not None or not isinstance(m, QubitsOperator):
            raise TypeError("expectation(H, rho) takes a QubitsOperator / QubitsTerm")
        arr, nt = m.packed()
        _lib.check(lib.vqc_dm_expect_pauli(psi.handle, arr, nt, out))
        return complex(out[0], out[1])
    if isinstance(m, QubitsOperator):
        arr, nt = m.packed()
        if phi is None:
            _lib.check(lib.vqc_expect_pauli(psi.handle, arr, nt, out))
        else:
            _lib.check(lib.vqc_expect_pauli2(phi.handle, psi.handle, arr, nt, out))
    elif isinstance(m, Gate):
        keep, mp = _mat_ptr(m.mat)
        _lib.check(lib.vqc_expect_dense(phi.handle if phi is not None else None, psi.handle, m.nqubits,
                                        _pos_array(m.positions), mp, out))
    else:
        raise TypeError("unsupported observable")
    return complex(out[0], out[1])


def apply_operator(m, psi):
    """H * psi as a new state (apply_qterms.jl:13-28)."""
    lib = _lib.load()
    m = _as_operator(m)
    out = StateVector(psi.nqubits, dtype=psi.dtype, device=psi.device)
    if isinstance(m, QubitsOperator):
        arr, nt = m.packed()
        _lib.check(lib.vqc_apply_pauli(psi.handle, out.handle, arr, nt))
    elif isinstance(m, Gate):
        _lib.check(lib.vqc_apply_pauli(psi.handle, out.handle, None, 0))  # zero
        keep, mp = _mat_ptr(m.mat)
        _lib.check(lib.vqc_apply_dense_add(psi.handle, out.handle, m.nqubits, _pos_array(m.positions), mp))
    else:
        raise TypeError("unsupported operator")
    return out


def partial_tr(rho, sites):
    """partial_tr(rho, sites) (ptrace.jl:4-10): returns the reduced matrix
    (numpy, L' x L'); tracing out every site returns tr(rho)."""
    lib = _lib.load()
    n = rho.nqubits
    sites = list(sites)
    if len(sites) == 0:
        return rho.storage()
    if len(set(sites)) != len(sites):
        raise ValueError("duplicate sites not allowed.")
    for s in sites:
        if not (1 <= s <= n):
            raise ValueError("site out of range.")
    if len(sites) == n:
        return rho.tr()
    m = n - len(sites)
    out = np.zeros(1 << (2 * m), dtype=np.complex128)
    _lib.check(lib.vqc_dm_ptrace(rho.handle, len(sites), _pos_array(sites), out.view(np.float64).ctypes.data_as(_lib._D)))
    L = 1 << m
    return out.reshape((L, L), order="F")


def probabilities(rho):
    """real(diag(storage(rho))): the basis distribution of a density matrix."""
    out = np.zeros(1 << rho.nqubits, dtype=np.float64)
    _lib.check(_lib.load().vqc_dm_probs(rho.handle, out.ctypes.data_as(_lib._D)))
    return out


def fidelity(x, y):
    """abs2(dot(x, y)) for pure states (statevector.jl:63)."""
    return abs(x.dot(y)) ** 2


def rand_state(n, dtype=np.complex128, rng=None, device=0):
    """rand_state (statevector.jl:152-158) with a seeded generator."""
    rng = np.random.default_rng(rng)
    v = rng.standard_normal(1 << n) + 1j * rng.standard_normal(1 << n)
    v /= np.linalg.norm(v)
    return StateVector(v.astype(dtype), dtype=dtype, device=device)
