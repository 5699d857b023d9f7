"""ctypes binding of the CPU oracle (``ps_oracle.c``).

TEST INFRASTRUCTURE ONLY: imported by ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg, as the checker.  The product package never imports it.

Channels are ``(kind, paulis, qubits, param[, extra])`` tuples: kind ``"rotation"``
(``exp(-i param P / 2)``, ``paulis`` one of ``XYZ`` per qubit), ``"depolarize"`` (single
qubit, ``param = p``), the Cliffords ``"h" "s" "sdg" "x" "y" "z" "cnot" "cz" "swap"``,
``"unitary"`` (``extra["matrix"]``: 2^k x 2^k complex), ``"dephase"``, ``"pauli_channel"``
(``extra["params"] = (px, py, pz)``), ``"depolarize2"`` and ``"amplitude_damping"``;
``extra["adjoint"]`` applies the channel's adjoint.  Policies are ``{"keep": [...postfix nodes...],
"passes": [("topn", n), ...]}`` with nodes ``("coeff", eps)``, ``("weight", k)``,
``("and",)``, ``("or",)``, ``("true",)``.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libps_oracle.so"

F64, F32 = 0, 1
_KEEP = {"true": 0, "coeff": 1, "weight": 2, "and": 3, "or": 4}
_PASS = {"topn": 1, "approx_topn": 3, "collapse_sample": 4}
_KIND = {"rotation": 1, "depolarize": 2, "h": 3, "s": 4, "sdg": 5, "x": 6, "y": 7, "z": 8, "cnot": 9,
         "cz": 10, "swap": 11, "unitary": 12, "dephase": 13, "pauli_channel": 14, "depolarize2": 15,
         "amplitude_damping": 16}


class _Policy(ctypes.Structure):
    _fields_ = [
        ("num_nodes", ctypes.c_int32),
        ("op", ctypes.c_int32 * 16),
        ("iarg", ctypes.c_int64 * 16),
        ("farg", ctypes.c_double * 16),
        ("num_passes", ctypes.c_int32),
        ("pass_kind", ctypes.c_int32 * 4),
        ("pass_n", ctypes.c_uint64 * 4),
        ("pass_samples", ctypes.c_uint64 * 4),
        ("pass_seed", ctypes.c_uint64 * 4),
        ("pass_call", ctypes.c_uint64 * 4),
    ]


class _Channel(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("num_support", ctypes.c_int32),
        ("qubits", ctypes.c_uint32 * 64),
        ("paulis", ctypes.c_char * 64),
        ("param", ctypes.c_double),
        ("params", ctypes.c_double * 3),
        ("matrix", ctypes.c_double * 32),
        ("adjoint", ctypes.c_int32),
    ]


def build() -> Path:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build()
        L = ctypes.CDLL(str(LIB_PATH))
        vp, sz = ctypes.c_void_p, ctypes.c_size_t
        L.pso_new.restype = vp
        L.pso_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.pso_free.argtypes = [vp]
        L.pso_len.restype = sz
        L.pso_len.argtypes = [vp]
        L.pso_set.argtypes = [vp, vp, vp, sz]
        L.pso_get.argtypes = [vp, vp, vp]
        L.pso_apply_channel.argtypes = [vp, ctypes.POINTER(_Channel), ctypes.c_int, ctypes.POINTER(_Policy)]
        L.pso_apply_channel_sorted.argtypes = L.pso_apply_channel.argtypes
        L.pso_finalize_layer.argtypes = [vp, ctypes.POINTER(_Policy)]
        L.pso_propagate.argtypes = [vp, ctypes.POINTER(_Channel), sz, ctypes.POINTER(_Policy), ctypes.c_int, vp]
        L.pso_propagate_sorted.argtypes = L.pso_propagate.argtypes
        L.pso_expectation.restype = ctypes.c_double
        L.pso_expectation.argtypes = [vp, vp, vp, vp]
        L.pso_set_threads.argtypes = [ctypes.c_int]
        L.pso_collapses.restype = ctypes.c_uint64
        L.pso_collapses.argtypes = []
        L.pso_splitmix64_first.restype = ctypes.c_uint64
        L.pso_splitmix64_first.argtypes = [ctypes.c_uint64]
        L.pso_xoshiro_two.argtypes = [vp, vp]
        L.pso_keyed_uniform.restype = ctypes.c_double
        L.pso_keyed_uniform.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.pso_prepare_table.argtypes = [ctypes.POINTER(_Channel), ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp, vp,
                                        vp, vp, vp]
        _lib = L
    return _lib


def policy_struct(policy) -> _Policy | None:
    if policy is None:
        return None
    p = _Policy()
    keep = policy.get("keep", [])
    assert len(keep) <= 15
    p.num_nodes = len(keep)
    for i, node in enumerate(keep):
        p.op[i] = _KEEP[node[0]]
        if node[0] == "coeff":
            p.farg[i] = float(node[1])
        elif node[0] == "weight":
            p.iarg[i] = int(node[1])
    passes = policy.get("passes", [])
    p.num_passes = len(passes)
    for i, ps_ in enumerate(passes):
        p.pass_kind[i] = _PASS[ps_[0]]
        p.pass_n[i] = int(ps_[1])
        if len(ps_) > 2:  # collapse_sample: (kind, cache, samples, seed, call)
            p.pass_samples[i], p.pass_seed[i], p.pass_call[i] = int(ps_[2]), int(ps_[3]), int(ps_[4])
    return p


def collapses() -> int:
    """CollapseSample collapses the oracle performed in this process."""
    return int(lib().pso_collapses())


def channel_array(channels):
    arr = (_Channel * max(1, len(channels)))()
    for i, ch in enumerate(channels):
        kind, paulis, qubits, param = ch[:4]
        extra = ch[4] if len(ch) > 4 else {}
        c = arr[i]
        c.kind = _KIND[kind]
        c.num_support = len(qubits)
        for j, q in enumerate(qubits):
            c.qubits[j] = int(q)
        c.paulis = (paulis or "").encode()
        c.param = float(param)
        for j, v in enumerate(extra.get("params", ())):
            c.params[j] = float(v)
        if "matrix" in extra:
            u = np.asarray(extra["matrix"], dtype=np.complex128).reshape(-1)
            for j, v in enumerate(u):
                c.matrix[2 * j] = float(v.real)
                c.matrix[2 * j + 1] = float(v.imag)
        c.adjoint = 1 if extra.get("adjoint") else 0
    return arr


def prepare_table(channel, num_qubits: int, adjoint: bool = False):
    """The oracle's prepared table of one channel: ``None`` for a wide rotation, else
    ``(qubits, [(local_delta, amplitudes[16]), ...])``; ``ValueError`` when declined."""
    arr = channel_array([channel])
    W = width_for(num_qubits)
    wide, k, ne = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_int(0)
    q = (ctypes.c_uint32 * 2)()
    deltas = (ctypes.c_uint32 * 16)()
    amps = (ctypes.c_double * 256)()
    rc = lib().pso_prepare_table(arr, int(bool(adjoint)), W, num_qubits, ctypes.addressof(wide), ctypes.addressof(k),
                                 ctypes.addressof(q), ctypes.addressof(ne), ctypes.addressof(deltas),
                                 ctypes.addressof(amps))
    if rc:
        raise ValueError(f"oracle declined channel {channel}")
    if wide.value:
        return None
    ents = [(int(deltas[e]), [float(amps[16 * e + s]) for s in range(16)]) for e in range(ne.value)]
    return tuple(int(q[j]) for j in range(k.value)), ents


def width_for(num_qubits: int) -> int:
    for w in (1, 2, 4, 8, 16):
        if num_qubits <= 64 * w:
            return w
    raise ValueError("too many qubits")


class OracleSum:
    """A CPU Pauli sum: sorted unique keys (x words then z words) and coefficients."""

    def __init__(self, num_qubits: int, dtype: str = "f64", width: int | None = None):
        self.num_qubits = num_qubits
        self.W = width or width_for(num_qubits)
        self.dtype = dtype
        self._h = lib().pso_new(self.W, num_qubits, F64 if dtype == "f64" else F32)
        if not self._h:
            raise ValueError("bad oracle sum parameters")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            lib().pso_free(h)
            self._h = None

    def __len__(self):
        return int(lib().pso_len(self._h))

    def set(self, keys: np.ndarray, coeffs: np.ndarray) -> "OracleSum":
        keys = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1, 2 * self.W)
        coeffs = np.ascontiguousarray(coeffs, dtype=np.float64).reshape(-1)
        assert keys.shape[0] == coeffs.shape[0]
        lib().pso_set(self._h, keys.ctypes.data, coeffs.ctypes.data, keys.shape[0])
        return self

    def get(self):
        n = len(self)
        keys = np.zeros((n, 2 * self.W), dtype=np.uint64)
        coeffs = np.zeros(n, dtype=np.float64)
        if n:
            lib().pso_get(self._h, keys.ctypes.data, coeffs.ctypes.data)
        return keys, coeffs

    def apply(self, channel, adjoint=False, policy=None, sorted_engine=False, threads=None):
        arr = channel_array([channel])
        if threads is not None:
            lib().pso_set_threads(int(threads))
        pol = policy_struct(policy)
        fn = lib().pso_apply_channel_sorted if sorted_engine else lib().pso_apply_channel
        rc = fn(self._h, arr, int(bool(adjoint)), ctypes.byref(pol) if pol else None)
        if rc:
            raise ValueError(f"oracle rejected channel {channel}")

    def propagate(self, channels, policy=None, direction="forward", sorted_engine=False, threads=None):
        arr = channel_array(channels)
        pol = policy_struct(policy)
        after = np.zeros(max(1, len(channels)), dtype=np.uint64)
        if threads is not None:
            lib().pso_set_threads(int(threads))
        fn = lib().pso_propagate_sorted if sorted_engine else lib().pso_propagate
        rc = fn(self._h, arr, len(channels), ctypes.byref(pol) if pol else None,
                1 if direction == "heisenberg" else 0, after.ctypes.data)
        if rc:
            raise ValueError("oracle rejected the circuit")
        return after[: len(channels)]

    def expectation(self, state: str) -> float:
        ax, az, neg = product_basis(state, self.num_qubits, self.W)
        return float(lib().pso_expectation(self._h, ax.ctypes.data, az.ctypes.data, neg.ctypes.data))


def product_basis(state: str, num_qubits: int, W: int):
    """Axis/sign masks of a product state: ``x+``/``y+``/``z+`` or one label per qubit from
    ``01+-rl`` (crates/paulistrings-py/src/sum.rs:42-91)."""
    ax = np.zeros(W, dtype=np.uint64)
    az = np.zeros(W, dtype=np.uint64)
    neg = np.zeros(W, dtype=np.uint64)
    uni = state.lower()
    if uni in ("x+", "y+", "z+"):
        full = np.uint64(0xFFFFFFFFFFFFFFFF)
        if uni in ("x+", "y+"):
            ax[:] = full
        if uni in ("z+", "y+"):
            az[:] = full
        return ax, az, neg
    if len(state) != num_qubits:
        raise ValueError("a per-qubit label needs one character per qubit")
    table = {"0": (0, 1, 0), "1": (0, 1, 1), "+": (1, 0, 0), "-": (1, 0, 1), "r": (1, 1, 0), "l": (1, 1, 1)}
    for q, ch in enumerate(state):
        bx, bz, bn = table[ch]
        bit = np.uint64(1) << np.uint64(q % 64)
        if bx:
            ax[q // 64] |= bit
        if bz:
            az[q // 64] |= bit
        if bn:
            neg[q // 64] |= bit
    return ax, az, neg


def pauli_key(label: str, W: int) -> np.ndarray:
    """Key words of an ``IXYZ`` label (character i = qubit i)."""
    k = np.zeros(2 * W, dtype=np.uint64)
    for q, ch in enumerate(label):
        bit = np.uint64(1) << np.uint64(q % 64)
        if ch in "XY":
            k[q // 64] |= bit
        if ch in "ZY":
            k[W + q // 64] |= bit
    return k
