"""ctypes binding of ``libpaulistrings_b200.so`` (the C ABI in ``include/paulistrings_b200.h``).

The library is built in-tree by ``csrc/Makefile``; there is no other implementation of
the layer path, so every entry point here raises when the library or a CUDA device is
missing.  Set ``PAULISTRINGS_B200_CHECKED=1`` to load the bounds-checked build.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_NAME = "libpaulistrings_b200.so"
CHECKED_LIB_NAME = "libpaulistrings_b200_checked.so"

PS_MAX_W = 16
PS_MAX_ENTRIES = 16
PS_MAX_KEEP_NODES = 15
PS_MAX_PASSES = 4

PS_OK, PS_ERR_OOM, PS_ERR_UNSUPPORTED, PS_ERR_INVALID, PS_ERR_DEVICE, PS_ERR_TIMEOUT, PS_ERR_NO_DEVICE = range(7)
PS_F64, PS_F32 = 0, 1
PS_FORWARD, PS_HEISENBERG = 0, 1
PS_KEEP_TRUE, PS_KEEP_COEFF, PS_KEEP_WEIGHT, PS_KEEP_AND, PS_KEEP_OR = range(5)
PS_PASS_NONE, PS_PASS_TOPN, PS_PASS_SCORED_TOPN, PS_PASS_APPROX_TOPN, PS_PASS_COLLAPSE_SAMPLE = 0, 1, 2, 3, 4
(PS_CH_PAULI_ROTATION, PS_CH_DEPOLARIZING, PS_CH_HADAMARD, PS_CH_PHASE, PS_CH_PHASE_DAGGER, PS_CH_PAULI_X,
 PS_CH_PAULI_Y, PS_CH_PAULI_Z, PS_CH_CNOT, PS_CH_CZ, PS_CH_SWAP, PS_CH_UNITARY, PS_CH_DEPHASING,
 PS_CH_PAULI_CHANNEL, PS_CH_DEPOLARIZING_2Q, PS_CH_AMPLITUDE_DAMPING) = range(1, 17)
PS_TABLE_LOCAL, PS_TABLE_ROTATION = 1, 2
PS_PATH_RESCALE, PS_PATH_ROTATION, PS_PATH_SORT = 1, 2, 3

EXPORTED = (
    "ps_abi_version",
    "ps_device_count",
    "ps_create",
    "ps_destroy",
    "ps_last_error",
    "ps_width",
    "ps_num_qubits",
    "ps_dtype_of",
    "ps_upload",
    "ps_len",
    "ps_download",
    "ps_prepare_channel",
    "ps_apply_layer",
    "ps_finalize_layer",
    "ps_propagate",
    "ps_expectation",
    "ps_set_profiling",
    "ps_read_profile",
    "ps_expectation_device_noalloc",
    "ps_inject_fault",
    "ps_synchronize",
    "ps_set_compensated_sums",
    "ps_scorer_create",
    "ps_scorer_destroy",
    "ps_scorer_last_error",
    "ps_scorer_num_params",
    "ps_scorer_get_params",
    "ps_scorer_set_params",
    "ps_scorer_score",
    "ps_scorer_gradients",
    "ps_scorer_train",
    "ps_scorer_set_site_map",
    "ps_set_scorer",
)

PS_FAULT_NONE, PS_FAULT_OOM, PS_FAULT_STALL, PS_FAULT_FLAG = 0, 1, 2, 3

NOALLOC_MAX_TERMS = 1 << 30


class KeepNode(ctypes.Structure):
    _fields_ = [("op", ctypes.c_int32), ("reserved", ctypes.c_int32), ("iarg", ctypes.c_int64), ("farg", ctypes.c_double)]


class ScorerConfig(ctypes.Structure):
    _fields_ = [
        ("num_qubits", ctypes.c_int32),
        ("residual", ctypes.c_int32),
        ("layers_per_unit", ctypes.c_double),
        ("feature_scale", ctypes.c_float * 3),
        ("init_scale", ctypes.c_float),
        ("seed", ctypes.c_uint64),
    ]


class Pass(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("reserved", ctypes.c_int32), ("n", ctypes.c_uint64),
                ("samples", ctypes.c_uint64), ("seed", ctypes.c_uint64), ("call", ctypes.c_uint64)]


class Policy(ctypes.Structure):
    _fields_ = [
        ("num_nodes", ctypes.c_int32),
        ("num_passes", ctypes.c_int32),
        ("nodes", KeepNode * PS_MAX_KEEP_NODES),
        ("passes", Pass * PS_MAX_PASSES),
    ]


class Channel(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("num_support", ctypes.c_int32),
        ("qubits", ctypes.POINTER(ctypes.c_uint32)),
        ("paulis", ctypes.c_char_p),
        ("param", ctypes.c_double),
        ("matrix", ctypes.POINTER(ctypes.c_double)),
        ("params", ctypes.c_double * 3),
        ("adjoint", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class TableEntry(ctypes.Structure):
    _fields_ = [
        ("local_delta", ctypes.c_uint32),
        ("reserved", ctypes.c_uint32),
        ("mask_x", ctypes.c_uint64 * PS_MAX_W),
        ("mask_z", ctypes.c_uint64 * PS_MAX_W),
        ("amplitude", ctypes.c_double * PS_MAX_ENTRIES),
    ]


class Table(ctypes.Structure):
    _fields_ = [
        ("mode", ctypes.c_int32),
        ("k", ctypes.c_int32),
        ("qubits", ctypes.c_uint32 * 2),
        ("num_entries", ctypes.c_int32),
        ("width", ctypes.c_int32),
        ("entries", TableEntry * PS_MAX_ENTRIES),
        ("gen_x", ctypes.c_uint64 * PS_MAX_W),
        ("gen_z", ctypes.c_uint64 * PS_MAX_W),
        ("cos_theta", ctypes.c_double),
        ("sin_theta", ctypes.c_double),
    ]


class LayerStats(ctypes.Structure):
    _fields_ = [
        ("terms_in", ctypes.c_uint64),
        ("partners", ctypes.c_uint64),
        ("terms_out", ctypes.c_uint64),
        ("terms_after_passes", ctypes.c_uint64),
        ("path", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
    ]


class RunStats(ctypes.Structure):
    _fields_ = [
        ("layers", ctypes.c_uint64),
        ("peak_terms", ctypes.c_uint64),
        ("final_terms", ctypes.c_uint64),
        ("total_terms_in", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64),
        ("device_ms", ctypes.c_double),
        ("collapses", ctypes.c_uint64),
        ("layers_skipped", ctypes.c_uint64),
        ("skipped_terms_in", ctypes.c_uint64),
    ]


class KernelProfile(ctypes.Structure):
    _fields_ = [
        ("name", ctypes.c_char * 32),
        ("launches", ctypes.c_uint64),
        ("timed_launches", ctypes.c_uint64),
        ("total_ms", ctypes.c_double),
        ("algorithmic_bytes", ctypes.c_double),
    ]


class PauliStringsError(RuntimeError):
    """A failed library call; ``status`` is the ``ps_status`` code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def library_path(checked: bool | None = None) -> Path:
    if checked is None:
        checked = os.environ.get("PAULISTRINGS_B200_CHECKED", "") not in ("", "0")
    return HERE / (CHECKED_LIB_NAME if checked else LIB_NAME)


_lib = None


def lib():
    """The loaded library; raises ``ImportError`` when it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = library_path()
    if not path.exists():
        raise ImportError(
            f"{path.name} is not built; run `make -C paulistrings-rs_b200/csrc` "
            "(or __graft_entry__.build()) first"
        )
    L = ctypes.CDLL(str(path))
    vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int32
    P = ctypes.POINTER
    L.ps_abi_version.restype = i32
    L.ps_device_count.restype = i32
    L.ps_create.argtypes = [i32, i32, i32, P(vp)]
    L.ps_destroy.argtypes = [vp]
    L.ps_last_error.restype = ctypes.c_char_p
    L.ps_last_error.argtypes = [vp]
    for name in ("ps_width", "ps_num_qubits", "ps_dtype_of"):
        getattr(L, name).restype = i32
        getattr(L, name).argtypes = [vp]
    L.ps_upload.argtypes = [vp, vp, vp, vp, u64]
    L.ps_len.argtypes = [vp, P(u64)]
    L.ps_download.argtypes = [vp, vp, vp, vp, u64, P(u64)]
    L.ps_prepare_channel.argtypes = [i32, i32, P(Channel), i32, P(Table)]
    L.ps_apply_layer.argtypes = [vp, P(Table), P(Policy), P(LayerStats)]
    L.ps_finalize_layer.argtypes = [vp, P(Policy)]
    L.ps_propagate.argtypes = [vp, P(Channel), u64, P(Policy), i32, vp, P(RunStats)]
    L.ps_expectation.argtypes = [vp, vp, vp, vp, P(ctypes.c_double)]
    L.ps_set_profiling.argtypes = [vp, i32]
    L.ps_read_profile.argtypes = [vp, P(KernelProfile), i32, P(i32)]
    L.ps_expectation_device_noalloc.argtypes = [vp, vp, i32, i32, u64, vp, vp, vp, vp, vp]
    L.ps_inject_fault.argtypes = [vp, i32, u64]
    L.ps_synchronize.argtypes = [vp]
    L.ps_set_compensated_sums.argtypes = [vp, i32]
    L.ps_scorer_create.argtypes = [i32, P(ScorerConfig), P(vp)]
    L.ps_scorer_destroy.argtypes = [vp]
    L.ps_scorer_last_error.restype = ctypes.c_char_p
    L.ps_scorer_last_error.argtypes = [vp]
    L.ps_scorer_num_params.restype = u64
    L.ps_scorer_num_params.argtypes = [vp]
    L.ps_scorer_get_params.argtypes = [vp, vp]
    L.ps_scorer_set_params.argtypes = [vp, vp]
    L.ps_scorer_score.argtypes = [vp, vp, vp, vp, u64, vp]
    L.ps_scorer_gradients.argtypes = [vp, vp, vp, vp, vp, u64, vp, vp]
    L.ps_scorer_train.argtypes = [vp, vp, vp, vp, vp, u64, i32, i32, ctypes.c_float, vp]
    L.ps_set_scorer.argtypes = [vp, vp, ctypes.c_double]
    L.ps_scorer_set_site_map.argtypes = [vp, i32, vp]
    for name in EXPORTED:
        fn = getattr(L, name)
        if name not in ("ps_abi_version", "ps_device_count", "ps_last_error", "ps_width", "ps_num_qubits",
                        "ps_dtype_of", "ps_scorer_last_error", "ps_scorer_num_params"):
            fn.restype = i32
    _lib = L
    return L


def check(status: int, handle=None, what: str = "") -> None:
    if status == PS_OK:
        return
    msg = ""
    if handle is not None:
        raw = lib().ps_last_error(handle)
        msg = raw.decode() if raw else ""
    names = {
        PS_ERR_OOM: "out of device memory",
        PS_ERR_UNSUPPORTED: "unsupported",
        PS_ERR_INVALID: "invalid argument",
        PS_ERR_DEVICE: "CUDA error",
        PS_ERR_TIMEOUT: "device wait timed out",
        PS_ERR_NO_DEVICE: "no CUDA device",
    }
    text = f"{what}: {names.get(status, 'error')}" + (f" ({msg})" if msg else "")
    if status == PS_ERR_INVALID:
        raise ValueError(text)
    if status == PS_ERR_UNSUPPORTED:
        raise NotImplementedError(text)
    if status == PS_ERR_OOM:
        raise MemoryError(text)
    raise PauliStringsError(status, text)


def device_count() -> int:
    return int(lib().ps_device_count())
