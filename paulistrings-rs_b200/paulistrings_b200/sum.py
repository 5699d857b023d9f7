"""``PauliSum`` (host arrays) and ``GpuPauliSum`` (resident on one CUDA device).

Mirrors the reference's ``PauliSum`` Python surface (crates/paulistrings-py/src/sum.rs):
``from_strings`` / ``from_arrays``, ``x_array`` / ``z_array`` / ``coefficients_array``,
``propagate(circuit, policy=None, direction=None, ..., device=)`` (sum.rs:2132-2183),
``expectation(state)`` (sum.rs:1826-1837) and ``to_device`` (sum.rs:2276-2283).

Every propagation and readout runs on the device through the C ABI; there is no host
engine.  A ``PauliSum`` keeps its terms in numpy arrays sorted by key and uploads them for
each call; a ``GpuPauliSum`` keeps them resident across calls.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .circuit import Circuit
from .truncation import policy_to_c

_DTYPES = {"f64": _lib.PS_F64, "float64": _lib.PS_F64, "f32": _lib.PS_F32, "float32": _lib.PS_F32}


def width_for(num_qubits: int) -> int:
    for w in (1, 2, 4, 8, 16):
        if num_qubits <= 64 * w:
            return w
    raise ValueError(f"num_qubits={num_qubits} exceeds 1024")


def _dtype_code(dtype: str) -> int:
    if dtype in ("c128", "c64", "complex128", "complex64"):
        raise NotImplementedError("complex coefficients are not on the device path; use dtype='f64' or 'f32'")
    try:
        return _DTYPES[dtype]
    except KeyError:
        raise ValueError(f"unknown dtype {dtype!r}; expected 'f64' or 'f32'") from None


def _dtype_name(code: int) -> str:
    return "f64" if code == _lib.PS_F64 else "f32"


def parse_label(label: str, W: int):
    """x and z words of an ``IXYZ`` label; character i is qubit i (crates/paulistrings-py/src/pauli_string.rs:196)."""
    x = np.zeros(W, dtype=np.uint64)
    z = np.zeros(W, dtype=np.uint64)
    for q, ch in enumerate(label):
        bit = np.uint64(1) << np.uint64(q % 64)
        if ch in "XY":
            x[q // 64] |= bit
        if ch in "ZY":
            z[q // 64] |= bit
        if ch not in "IXYZ":
            raise ValueError(f"bad Pauli character {ch!r} in {label!r}")
    return x, z


def product_basis(state: str, num_qubits: int, W: int):
    """Axis and sign masks of a product state (crates/paulistrings-py/src/sum.rs:42-91):
    ``"x+"``, ``"y+"``, ``"z+"`` or one character per qubit from ``01+-rl``."""
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
    table = {"0": (0, 1, 0), "1": (0, 1, 1), "+": (1, 0, 0), "-": (1, 0, 1), "r": (1, 1, 0), "l": (1, 1, 1)}
    if len(state) != num_qubits:
        raise ValueError(
            f"unknown product state {state!r}: a per-qubit label string over \"01+-rl\" needs one character "
            f"per qubit (got {len(state)}, num_qubits is {num_qubits}); the uniform names are \"x+\", \"y+\", \"z+\""
        )
    for q, ch in enumerate(state):
        if ch not in table:
            raise ValueError(f"unknown product state {state!r}: {ch!r} at qubit {q} is not a per-qubit label")
        bx, bz, bn = table[ch]
        bit = np.uint64(1) << np.uint64(q % 64)
        if bx:
            ax[q // 64] |= bit
        if bz:
            az[q // 64] |= bit
        if bn:
            neg[q // 64] |= bit
    return ax, az, neg


def _parse_direction(direction) -> int:
    d = "forward" if direction is None else direction
    if d == "forward":
        return _lib.PS_FORWARD
    if d == "heisenberg":
        return _lib.PS_HEISENBERG
    raise ValueError(f"direction must be 'forward' or 'heisenberg', got {direction!r}")


def _parse_device(device) -> int:
    if device is None or device == "auto":
        return 0
    if isinstance(device, (list, tuple)):
        if len(device) != 1:
            raise NotImplementedError("one device per sum: the layer path does not shard")
        device = device[0]
    return int(device)


@dataclass
class PropagationStats:
    """Per-layer term counts of a propagation (PropagationStats, crates/paulistrings-py)."""

    terms_after: list = field(default_factory=list)
    peak_terms: int = 0
    final_terms: int = 0
    layers: int = 0
    device_ms: float = 0.0
    total_terms_in: int = 0
    kernel_launches: int = 0
    collapses: int = 0
    layers_skipped: int = 0     # layers that acted only on qubits no term touched (nothing ran)
    skipped_terms_in: int = 0   # terms entering those layers


class GpuPauliSum:
    """A Pauli sum resident on one CUDA device (the handle of the C ABI)."""

    def __init__(self, num_qubits: int, dtype: str = "f64", device: int = 0):
        self.num_qubits = int(num_qubits)
        self.W = width_for(self.num_qubits)
        self.device = int(device)
        h = ctypes.c_void_p()
        st = _lib.lib().ps_create(self.device, self.num_qubits, _dtype_code(dtype), ctypes.byref(h))
        if st == _lib.PS_ERR_NO_DEVICE:
            raise RuntimeError(f"no CUDA device {device}: the layer path runs only on a GPU")
        _lib.check(st, None, "ps_create")
        self._h = h

    @property
    def dtype(self) -> str:
        return _dtype_name(_lib.lib().ps_dtype_of(self._h))

    def close(self) -> None:
        h = getattr(self, "_h", None)
        if h:
            _lib.lib().ps_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        n = ctypes.c_uint64()
        _lib.check(_lib.lib().ps_len(self._h, ctypes.byref(n)), self._h, "ps_len")
        return int(n.value)

    def upload(self, x: np.ndarray, z: np.ndarray, coeffs: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, self.W)
        z = np.ascontiguousarray(z, dtype=np.uint64).reshape(-1, self.W)
        c = np.ascontiguousarray(coeffs, dtype=np.float64).reshape(-1)
        if not (x.shape[0] == z.shape[0] == c.shape[0]):
            raise ValueError("x, z and coefficients must have the same length")
        st = _lib.lib().ps_upload(self._h, x.ctypes.data, z.ctypes.data, c.ctypes.data, c.shape[0])
        _lib.check(st, self._h, "upload")

    def download(self, out=None):
        """(x, z, coefficients) as new arrays, or written into ``out = (x, z, c)`` (e.g. pinned
        host buffers with at least ``len(self)`` rows), returning views of the filled rows."""
        n = len(self)
        if out is None:
            x = np.zeros((n, self.W), dtype=np.uint64)
            z = np.zeros((n, self.W), dtype=np.uint64)
            c = np.zeros(n, dtype=np.float64)
        else:
            x, z, c = out
            if x.shape[0] < n or z.shape[0] < n or c.shape[0] < n or x.dtype != np.uint64 or c.dtype != np.float64:
                raise ValueError("download: output buffers too small or of the wrong dtype")
            if not (x.flags.c_contiguous and z.flags.c_contiguous and c.flags.c_contiguous):
                raise ValueError("download: output buffers must be C-contiguous")
        got = ctypes.c_uint64()
        st = _lib.lib().ps_download(self._h, x.ctypes.data, z.ctypes.data, c.ctypes.data, x.shape[0], ctypes.byref(got))
        _lib.check(st, self._h, "download")
        return x[:n], z[:n], c[:n]

    def set_profiling(self, enabled: bool) -> None:
        _lib.check(_lib.lib().ps_set_profiling(self._h, int(bool(enabled))), self._h, "set_profiling")

    def read_profile(self) -> dict:
        """{kernel: {launches, timed_launches, total_ms, algorithmic_bytes}}."""
        arr = (_lib.KernelProfile * 32)()
        count = ctypes.c_int32()
        _lib.check(_lib.lib().ps_read_profile(self._h, arr, 32, ctypes.byref(count)), self._h, "read_profile")
        out = {}
        for i in range(min(count.value, 32)):
            r = arr[i]
            out[r.name.decode()] = {
                "launches": int(r.launches),
                "timed_launches": int(r.timed_launches),
                "total_ms": float(r.total_ms),
                "algorithmic_bytes": float(r.algorithmic_bytes),
            }
        return out

    def to_host(self) -> "PauliSum":
        x, z, c = self.download()
        out = PauliSum(self.num_qubits, self.dtype)
        out._set_sorted(x, z, c)
        return out

    def propagate(self, circuit: Circuit, policy=None, direction=None, with_stats: bool = False,
                  remaining_layers=None):
        """``remaining_layers``: layers still to apply when this call starts, for a scored_topn
        policy's remaining-depth feature (default: this circuit's length)."""
        if circuit.num_qubits != self.num_qubits:
            raise ValueError(
                f"circuit acts on {circuit.num_qubits} qubits but the sum has {self.num_qubits}"
            )
        arr, count, keep = circuit.to_c()
        pol = policy_to_c(policy)
        self._attach_scorer(policy, count if remaining_layers is None else remaining_layers)
        after = np.zeros(max(1, count), dtype=np.uint64)
        rs = _lib.RunStats()
        st = _lib.lib().ps_propagate(
            self._h, arr, count, ctypes.byref(pol) if pol is not None else None, _parse_direction(direction),
            after.ctypes.data, ctypes.byref(rs),
        )
        del keep
        if policy is not None:  # the CollapseSample pass counters live in the policy
            for state in policy.collapse_states():
                state["calls"] += int(rs.layers)
                state["collapses"] += int(rs.collapses)
        _lib.check(st, self._h, "propagate")
        if with_stats:
            return PropagationStats(
                terms_after=[int(v) for v in after[:count]],
                peak_terms=int(rs.peak_terms),
                final_terms=int(rs.final_terms),
                layers=int(rs.layers),
                device_ms=float(rs.device_ms),
                total_terms_in=int(rs.total_terms_in),
                kernel_launches=int(rs.kernel_launches),
                collapses=int(rs.collapses),
                layers_skipped=int(rs.layers_skipped),
                skipped_terms_in=int(rs.skipped_terms_in),
            )
        return None

    def _attach_scorer(self, policy, remaining_layers) -> None:
        sc = policy.scorer() if policy is not None else None
        if sc is None:
            _lib.lib().ps_set_scorer(self._h, None, 0.0)
            return
        _lib.check(_lib.lib().ps_set_scorer(self._h, sc._h, float(remaining_layers)), self._h, "set_scorer")
        self._scorer = sc  # keep it alive while attached

    def apply_layer(self, channel, policy=None, adjoint: bool = False) -> _lib.LayerStats:
        """One layer through ``ps_prepare_channel`` + ``ps_apply_layer`` + ``ps_finalize_layer``."""
        c = Circuit(self.num_qubits)
        c.append(channel)
        arr, _, keep = c.to_c()
        table = _lib.Table()
        L = _lib.lib()
        dt = L.ps_dtype_of(self._h)
        _lib.check(L.ps_prepare_channel(self.num_qubits, dt, arr, int(bool(adjoint)), ctypes.byref(table)), None,
                   "prepare_channel")
        del keep
        pol = policy_to_c(policy)
        stats = _lib.LayerStats()
        polp = ctypes.byref(pol) if pol is not None else None
        _lib.check(L.ps_apply_layer(self._h, ctypes.byref(table), polp, ctypes.byref(stats)), self._h, "apply_layer")
        _lib.check(L.ps_finalize_layer(self._h, polp), self._h, "finalize_layer")
        if policy is not None:
            for state in policy.collapse_states():
                state["calls"] += 1
        return stats

    def expectation(self, state: str = "z+") -> float:
        ax, az, neg = product_basis(state, self.num_qubits, self.W)
        out = ctypes.c_double()
        st = _lib.lib().ps_expectation(self._h, ax.ctypes.data, az.ctypes.data, neg.ctypes.data, ctypes.byref(out))
        _lib.check(st, self._h, "expectation")
        return float(out.value)


class PauliSum:
    """Host-side Pauli sum: unique keys sorted lexicographically by (x words, z words), with
    float64 or float32 coefficients."""

    def __init__(self, num_qubits: int, dtype: str = "f64"):
        _dtype_code(dtype)
        self.num_qubits = int(num_qubits)
        self.W = width_for(self.num_qubits)
        self.dtype = "f64" if dtype in ("f64", "float64") else "f32"
        self._x = np.zeros((0, self.W), dtype=np.uint64)
        self._z = np.zeros((0, self.W), dtype=np.uint64)
        self._c = np.zeros(0, dtype=np.float64)

    # -- construction -------------------------------------------------------
    @classmethod
    def from_strings(cls, terms: dict, num_qubits: int | None = None, dtype: str = "f64", device=None) -> "PauliSum":
        labels = list(terms.keys())
        if num_qubits is None:
            if not labels:
                raise ValueError("num_qubits is required for an empty sum")
            num_qubits = len(labels[0])
        W = width_for(num_qubits)
        x = np.zeros((len(labels), W), dtype=np.uint64)
        z = np.zeros((len(labels), W), dtype=np.uint64)
        c = np.zeros(len(labels), dtype=np.float64)
        for i, lab in enumerate(labels):
            if len(lab) != num_qubits:
                raise ValueError(f"label {lab!r} has {len(lab)} characters, num_qubits is {num_qubits}")
            x[i], z[i] = parse_label(lab, W)
            v = terms[lab]
            if isinstance(v, complex):
                if v.imag != 0.0:
                    raise ValueError("a real dtype cannot hold an imaginary coefficient")
                v = v.real
            c[i] = float(v)
        return cls.from_arrays(x, z, c, num_qubits=num_qubits, dtype=dtype, device=device)

    @classmethod
    def from_arrays(cls, x, z, coeffs, num_qubits: int, dtype: str = "f64", device=None) -> "PauliSum":
        """Duplicates summed in input order, exact zeros dropped (pauli_sum/accumulator.rs:35-56),
        normalized on the device."""
        out = cls(num_qubits, dtype)
        g = GpuPauliSum(num_qubits, dtype, _parse_device(device))
        try:
            g.upload(np.asarray(x).reshape(-1, out.W), np.asarray(z).reshape(-1, out.W), np.asarray(coeffs))
            out._set_sorted(*g.download())
        finally:
            g.close()
        return out

    def _set_sorted(self, x, z, c):
        self._x = np.ascontiguousarray(x, dtype=np.uint64).reshape(-1, self.W)
        self._z = np.ascontiguousarray(z, dtype=np.uint64).reshape(-1, self.W)
        self._c = np.ascontiguousarray(c, dtype=np.float64).reshape(-1)

    # -- accessors ----------------------------------------------------------
    def __len__(self) -> int:
        return int(self._c.shape[0])

    def x_array(self) -> np.ndarray:
        return self._x.copy()

    def z_array(self) -> np.ndarray:
        return self._z.copy()

    def coefficients_array(self) -> np.ndarray:
        return self._c.astype(np.float32) if self.dtype == "f32" else self._c.copy()

    def copy(self) -> "PauliSum":
        out = PauliSum(self.num_qubits, self.dtype)
        out._set_sorted(self._x.copy(), self._z.copy(), self._c.copy())
        return out

    def to_dict(self) -> dict:
        out = {}
        for i in range(len(self)):
            lab = []
            for q in range(self.num_qubits):
                w, b = q // 64, np.uint64(q % 64)
                xb = (int(self._x[i, w]) >> int(b)) & 1
                zb = (int(self._z[i, w]) >> int(b)) & 1
                lab.append("IXZY"[xb | (zb << 1)])
            out["".join(lab)] = float(self._c[i])
        return out

    def to_device(self, device=None) -> GpuPauliSum:
        g = GpuPauliSum(self.num_qubits, self.dtype, _parse_device(device))
        g.upload(self._x, self._z, self._c)
        return g

    # -- propagation --------------------------------------------------------
    def propagate(self, circuit: Circuit, policy=None, direction=None, target_bucket_len: int = 1024,
                  min_buckets: int = 128, device=None, **unsupported) -> None:
        """Propagate in place on ``device`` (default 0).  On error the sum is left empty, as the
        reference's moved-out sum is (crates/paulistrings-py/src/sum.rs:2104-2106)."""
        self._run(circuit, policy, direction, target_bucket_len, min_buckets, device, unsupported, False)

    def propagate_with_stats(self, circuit: Circuit, policy=None, direction=None, target_bucket_len: int = 1024,
                             min_buckets: int = 128, device=None, **unsupported) -> PropagationStats:
        return self._run(circuit, policy, direction, target_bucket_len, min_buckets, device, unsupported, True)

    def _run(self, circuit, policy, direction, target_bucket_len, min_buckets, device, unsupported, stats):
        if unsupported:
            raise NotImplementedError(
                f"{sorted(unsupported)}: partitioned / distributed runs are not on this path (one device per sum)"
            )
        if target_bucket_len < 1:
            raise ValueError("target_bucket_len must be at least 1")
        if min_buckets < 16:
            raise ValueError("min_buckets must be at least 16")
        d = _parse_direction(direction)
        if circuit.num_qubits != self.num_qubits:
            raise ValueError(f"circuit acts on {circuit.num_qubits} qubits but the sum has {self.num_qubits}")
        g = GpuPauliSum(self.num_qubits, self.dtype, _parse_device(device))
        try:
            g.upload(self._x, self._z, self._c)
            self._set_sorted(np.zeros((0, self.W), np.uint64), np.zeros((0, self.W), np.uint64), np.zeros(0))
            st = g.propagate(circuit, policy, "heisenberg" if d == _lib.PS_HEISENBERG else "forward", with_stats=stats)
            self._set_sorted(*g.download())
        finally:
            g.close()
        return st

    def expectation(self, state: str = "z+", device=None) -> float:
        g = self.to_device(device)
        try:
            return g.expectation(state)
        finally:
            g.close()


def propagated(pauli_sum: PauliSum, circuit: Circuit, policy=None, direction=None, device=None, **kw) -> PauliSum:
    """Copying form of ``PauliSum.propagate`` (python/paulistrings/_propagated.py)."""
    out = pauli_sum.copy()
    out.propagate(circuit, policy=policy, direction=direction, device=device, **kw)
    return out


def propagated_with_stats(pauli_sum: PauliSum, circuit: Circuit, policy=None, direction=None, device=None, **kw):
    out = pauli_sum.copy()
    st = out.propagate_with_stats(circuit, policy=policy, direction=direction, device=device, **kw)
    return out, st


def cuda_available() -> bool:
    try:
        return _lib.device_count() > 0
    except (ImportError, OSError):
        return False
