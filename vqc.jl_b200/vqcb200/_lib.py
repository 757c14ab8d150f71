"""ctypes binding of libvqcb200.so (the C ABI declared in include/vqc_b200.h).

The library is the product: there is no CPU or PyTorch fallback.  If it is
missing or fails to load, every call raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
# VQC_DEBUG_LIB=1 loads the debug build (device-side index checks, see
# vqc_debug_status in include/vqc_b200.h) instead of the release library
LIB_PATH = os.path.join(HERE, "libvqcb200_debug.so" if os.environ.get("VQC_DEBUG_LIB") == "1" else "libvqcb200.so")

VQC_C64 = 0
VQC_C128 = 1

STATUS = {
    -1: ValueError,       # VQC_ERR_ARG
    -2: MemoryError,      # VQC_ERR_OOM
    -3: RuntimeError,     # VQC_ERR_CUDA
    -4: NotImplementedError,  # VQC_ERR_UNSUPPORTED
    -5: TimeoutError,     # VQC_ERR_TIMEOUT
    -6: BlockingIOError,  # VQC_ERR_BUSY
}


class Cancelled(RuntimeError):
    """VQC_ERR_CANCELED: the serving request was cancelled."""


STATUS[-7] = Cancelled


class VqcError(RuntimeError):
    pass


class Gate_t(ctypes.Structure):
    _fields_ = [("nq", ctypes.c_int32), ("pos", ctypes.c_int32 * 5), ("mat", ctypes.c_int64)]


class Param_t(ctypes.Structure):
    _fields_ = [("gate", ctypes.c_int32), ("kind", ctypes.c_int32), ("dmat", ctypes.c_int64)]


class Pauli_t(ctypes.Structure):
    _fields_ = [("xmask", ctypes.c_uint64), ("zmask", ctypes.c_uint64), ("coeff_re", ctypes.c_double),
                ("coeff_im", ctypes.c_double)]


_lib = None

# name -> (argtypes, restype)
_H = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)
_V = ctypes.c_void_p
_S = ctypes.c_size_t
SIGNATURES = {
    "vqc_last_error": ([], ctypes.c_char_p),
    "vqc_version": ([], ctypes.c_char_p),
    "vqc_device_count": ([], _I),
    "vqc_state_create": ([_I, _I, _I, ctypes.POINTER(_H)], _I),
    "vqc_state_destroy": ([_H], _I),
    "vqc_state_nqubits": ([_H], _I),
    "vqc_state_dtype": ([_H], _I),
    "vqc_state_upload": ([_H, _V, _S], _I),
    "vqc_state_download": ([_H, _V, _S], _I),
    "vqc_state_reset": ([_H], _I),
    "vqc_state_copy": ([_H, _H], _I),
    "vqc_state_norm": ([_H, _D], _I),
    "vqc_state_dot": ([_H, _H, _D], _I),
    "vqc_state_sync": ([_H], _I),
    "vqc_state_device_ptr": ([_H], _V),
    "vqc_state_stream": ([_H], _V),
    "vqc_profile_enable": ([_I], _I),
    "vqc_profile_count": ([], _I),
    "vqc_profile_get": ([_I, ctypes.c_char_p, _I, ctypes.POINTER(ctypes.c_longlong), _D, _D], _I),
    "vqc_profile_flops": ([_I, _D], _I),
    "vqc_fma_peak": ([_I, _I, _D], _I),
    "vqc_debug_status": ([_I, ctypes.POINTER(ctypes.c_longlong)], _I),
    "vqc_debug_build": ([], _I),
    "vqc_apply_gate": ([_H, _I, _IP, _D], _I),
    "vqc_apply_circuit": ([_H, ctypes.POINTER(Gate_t), _I, _D, _I], _I),
    "vqc_expect_pauli": ([_H, ctypes.POINTER(Pauli_t), _I, _D], _I),
    "vqc_expect_pauli2": ([_H, _H, ctypes.POINTER(Pauli_t), _I, _D], _I),
    "vqc_expect_dense": ([_H, _H, _I, _IP, _D, _D], _I),
    "vqc_apply_pauli": ([_H, _H, ctypes.POINTER(Pauli_t), _I], _I),
    "vqc_apply_dense_add": ([_H, _H, _I, _IP, _D], _I),
    "vqc_adjoint_grad": ([_H, ctypes.POINTER(Gate_t), _I, _D, ctypes.POINTER(Param_t), _I,
                          ctypes.POINTER(Pauli_t), _I, _D, _D], _I),
    "vqc_circuit_backward": ([_H, _H, ctypes.POINTER(Gate_t), _I, _D, ctypes.POINTER(Param_t), _I, _D], _I),
    "vqc_dm_create": ([_I, _I, _I, ctypes.POINTER(_H)], _I),
    "vqc_dm_nqubits": ([_H], _I),
    "vqc_dm_from_state": ([_H, _H], _I),
    "vqc_dm_apply_gate": ([_H, _I, _IP, _D], _I),
    "vqc_dm_apply_circuit": ([_H, ctypes.POINTER(Gate_t), _I, _D, _I], _I),
    "vqc_dm_ptrace": ([_H, _I, _IP, _D], _I),
    "vqc_dm_probs": ([_H, _D], _I),
    "vqc_dm_trace": ([_H, _D], _I),
    "vqc_dm_apply_channel": ([_H, _I, _IP, _I, _D, _I], _I),
    "vqc_state_take_qubit": ([_H, _I, _I, ctypes.c_double, _H], _I),
    "vqc_state_axpby": ([_H, _D, _H, _D], _I),
    "vqc_dm_trace_prod": ([_H, _I, _H, _I, _I, _IP, _D, _D], _I),
    "vqc_dm_expect_pauli": ([_H, ctypes.POINTER(Pauli_t), _I, _D], _I),
    "vqc_expect_pauli_noalloc": ([_V, _I, _I, ctypes.POINTER(Pauli_t), _I, _V, _D], _I),
    "vqc_serve_open": ([_I, _I, _S, _I, _I, ctypes.POINTER(_H)], _I),
    "vqc_serve_submit": ([_H, _I, ctypes.POINTER(Gate_t), _I, _D, ctypes.POINTER(Param_t), _I,
                          ctypes.POINTER(Pauli_t), _I, _I, _D, ctypes.POINTER(ctypes.c_int64)], _I),
    "vqc_serve_poll": ([_H, ctypes.c_int64, _D, _D], _I),
    "vqc_serve_wait": ([_H, ctypes.c_int64, _I, _D, _D], _I),
    "vqc_serve_cancel": ([_H, ctypes.c_int64], _I),
    "vqc_serve_stats": ([_H, ctypes.POINTER(ctypes.c_longlong)], _I),
    "vqc_serve_timing": ([_H, _D], _I),
    "vqc_serve_loop_timing": ([_H, _D], _I),
    "vqc_serve_close": ([_H], _I),
}


def load(path=LIB_PATH):
    """Load the engine.  Raises if it is absent: there is no fallback path."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise VqcError("libvqcb200.so not found at %s: build it with vqcb200._build.build()" % path)
    lib = ctypes.CDLL(path)
    for name, (args, res) in SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = res
    _lib = lib
    return lib


def check(rc):
    """Raise the Python exception of a negative vqc status."""
    if rc < 0:
        msg = load().vqc_last_error().decode("utf-8", "replace")
        raise STATUS.get(rc, VqcError)(msg)
    return rc


def profile_enable(on):
    check(load().vqc_profile_enable(1 if on else 0))


def profile_read(with_flops=False):
    """{kernel class: (launches, total_ms, total_algorithmic_bytes)}, with a
    fourth entry, the total FMA-pipe flops, when with_flops is set."""
    lib = load()
    out = {}
    for i in range(check(lib.vqc_profile_count())):
        name = ctypes.create_string_buffer(64)
        n = ctypes.c_longlong()
        ms = ctypes.c_double()
        by = ctypes.c_double()
        check(lib.vqc_profile_get(i, name, 64, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by)))
        rec = (n.value, ms.value, by.value)
        if with_flops:
            fl = ctypes.c_double()
            check(lib.vqc_profile_flops(i, ctypes.byref(fl)))
            rec = rec + (fl.value,)
        out[name.value.decode()] = rec
    return out


def debug_status(reset=False):
    """(violations, first source line, first index, its limit) recorded by the
    debug build's device-side index checks; (0, 0, 0, 0) in the release build."""
    out = (ctypes.c_longlong * 4)()
    check(load().vqc_debug_status(1 if reset else 0, out))
    return tuple(out)


def fma_peak(device=0, kind=0):
    """Measured FMA-pipe peak in TFLOP/s: kind 0 packed FP32, 1 scalar FP32, 2 FP64."""
    out = ctypes.c_double()
    check(load().vqc_fma_peak(device, kind, ctypes.byref(out)))
    return out.value


def exported_symbols():
    return sorted(SIGNATURES)
