"""``Circuit`` and the channel factories (``gates``, ``noise``).

Mirrors the reference's Python surface (crates/paulistrings-py/src/circuit.rs:102-345,
crates/paulistrings-py/src/gates.rs:52-255, crates/paulistrings-py/src/noise.rs:19-115): a
circuit is an ordered list of channels, each applied as one layer.  The built-ins are Pauli
rotations ``exp(-i theta P / 2)`` of any weight, the Clifford gates H, S, S^dagger, X, Y, Z,
CNOT, CZ and SWAP, general one- and two-qubit unitaries, and the noise channels depolarize,
dephase, pauli_channel, depolarize2 and amplitude_damping (``PtmChannel``,
crates/paulistrings/src/channel/ptm.rs:15-36).
"""

from __future__ import annotations

import ctypes
import dataclasses
from dataclasses import dataclass

import numpy as np

from . import _lib

UNITARITY_TOLERANCE = 1e-10


@dataclass(frozen=True)
class PauliRotation:
    """``exp(-i theta P / 2)`` with ``P = paulis[j]`` on ``qubits[j]`` (crates/paulistrings/src/channel/rotation.rs:11-41)."""

    paulis: str
    qubits: tuple
    theta: float

    kind = _lib.PS_CH_PAULI_ROTATION

    def __post_init__(self):
        if len(self.paulis) != len(self.qubits):
            raise ValueError(
                f"pauli_rotation: {len(self.paulis)} Pauli labels for {len(self.qubits)} qubits"
            )
        for ch in self.paulis:
            if ch not in "XYZ":
                raise ValueError(f"pauli_rotation: bad Pauli label {ch!r}; expected X, Y or Z")
        if len(set(self.qubits)) != len(self.qubits):
            raise ValueError("pauli_rotation: repeated qubit")

    @property
    def param(self) -> float:
        return self.theta

    def support(self):
        return tuple(self.qubits)

    def adjoint(self) -> "PauliRotation":
        return PauliRotation(self.paulis, self.qubits, -self.theta)


@dataclass(frozen=True)
class Depolarizing:
    """Single-qubit depolarizing noise: X, Y, Z scaled by ``1 - 4p/3`` (ptm/noise.rs:7-16)."""

    qubit: int
    p: float

    kind = _lib.PS_CH_DEPOLARIZING

    def __post_init__(self):
        if not 0.0 <= self.p <= 1.0:
            raise ValueError(f"depolarizing: p must lie in [0, 1], got {self.p}")

    @property
    def paulis(self) -> str:
        return ""

    @property
    def qubits(self):
        return (self.qubit,)

    @property
    def param(self) -> float:
        return self.p

    def support(self):
        return (self.qubit,)

    def adjoint(self) -> "Depolarizing":
        return self


@dataclass(frozen=True)
class PtmChannel:
    """A one- or two-qubit gate or noise channel stored as its Pauli-transfer matrix
    (crates/paulistrings/src/channel/ptm.rs:15-36).  ``name`` is the constructor
    (``"hadamard"``, ``"cnot"``, ...); ``adjoint()`` flips ``is_adjoint``, and ``debug_name``
    then carries ``_adjoint`` as the reference's does (ptm.rs:56-80)."""

    name: str
    kind: int
    qubits: tuple
    param: float = 0.0
    params: tuple = (0.0, 0.0, 0.0)
    matrix: tuple | None = None   # UNITARY: row-major, re/im interleaved
    is_adjoint: bool = False

    paulis = ""

    def support(self):
        return tuple(self.qubits)

    @property
    def debug_name(self) -> str:
        return self.name + ("_adjoint" if self.is_adjoint else "")

    def adjoint(self) -> "PtmChannel":
        return dataclasses.replace(self, is_adjoint=not self.is_adjoint)


def _check_probability(channel: str, name: str, value: float) -> float:
    value = float(value)
    if not 0.0 <= value <= 1.0:
        raise ValueError(f"{channel}: {name} must be between 0 and 1 (got {value})")
    return value


def _distinct(name: str, q0: int, q1: int):
    if int(q0) == int(q1):
        raise ValueError(f"{name}: the two qubit indices must differ (both are {q0})")
    return int(q0), int(q1)


def _read_unitary(matrix, n: int, what: str) -> tuple:
    """A unitary given as an n x n complex array, checked as crates/paulistrings-py/src/gates.rs:13-49
    checks it (every entry of U^dagger U - I at most 1e-10), flattened re/im interleaved."""
    u = np.asarray(matrix, dtype=np.complex128)
    if u.shape != (n, n):
        raise ValueError(f"{what} expects a {n}x{n} complex matrix, got shape {u.shape}")
    dev = np.abs(u.conj().T @ u - np.eye(n))
    worst = float(np.max(dev)) if not np.isnan(dev).any() else float("nan")
    if not worst <= UNITARITY_TOLERANCE:
        raise ValueError(f"{what}: matrix is not unitary (largest entry of U^dagger U - I is {worst:.3e}, "
                         f"tolerance {UNITARITY_TOLERANCE:g})")
    flat = np.empty(2 * n * n, dtype=np.float64)
    flat[0::2] = u.real.reshape(-1)
    flat[1::2] = u.imag.reshape(-1)
    return tuple(float(v) for v in flat)


class gates:  # noqa: N801  (module-like namespace, as the reference's ``gates`` submodule)
    @staticmethod
    def h(qubit: int) -> PtmChannel:
        return PtmChannel("hadamard", _lib.PS_CH_HADAMARD, (int(qubit),))

    @staticmethod
    def s(qubit: int) -> PtmChannel:
        return PtmChannel("phase_gate", _lib.PS_CH_PHASE, (int(qubit),))

    @staticmethod
    def sdg(qubit: int) -> PtmChannel:
        """``S^dagger``: ``phase_gate(qubit).adjoint()`` (crates/paulistrings-py/src/channel_spec.rs:293)."""
        return gates.s(qubit).adjoint()

    @staticmethod
    def x(qubit: int) -> PtmChannel:
        return PtmChannel("pauli_x", _lib.PS_CH_PAULI_X, (int(qubit),))

    @staticmethod
    def y(qubit: int) -> PtmChannel:
        return PtmChannel("pauli_y", _lib.PS_CH_PAULI_Y, (int(qubit),))

    @staticmethod
    def z(qubit: int) -> PtmChannel:
        return PtmChannel("pauli_z", _lib.PS_CH_PAULI_Z, (int(qubit),))

    @staticmethod
    def cnot(control: int, target: int) -> PtmChannel:
        return PtmChannel("cnot", _lib.PS_CH_CNOT, _distinct("cnot", control, target))

    @staticmethod
    def cz(q0: int, q1: int) -> PtmChannel:
        return PtmChannel("cz", _lib.PS_CH_CZ, _distinct("cz", q0, q1))

    @staticmethod
    def swap(q0: int, q1: int) -> PtmChannel:
        return PtmChannel("swap", _lib.PS_CH_SWAP, _distinct("swap", q0, q1))

    @staticmethod
    def unitary_1q(qubit: int, matrix) -> PtmChannel:
        return PtmChannel("unitary_1q", _lib.PS_CH_UNITARY, (int(qubit),),
                          matrix=_read_unitary(matrix, 2, "unitary_1q"))

    @staticmethod
    def unitary_2q(q0: int, q1: int, matrix) -> PtmChannel:
        """``q0`` is the more significant tensor factor: the matrix acts on ``|q0 q1>``."""
        qs = _distinct("unitary_2q", q0, q1)
        return PtmChannel("unitary_2q", _lib.PS_CH_UNITARY, qs, matrix=_read_unitary(matrix, 4, "unitary_2q"))

    @staticmethod
    def pauli_rotation(pauli: str, qubits, theta: float) -> PauliRotation:
        return PauliRotation(str(pauli), tuple(int(q) for q in qubits), float(theta))

    @staticmethod
    def rx(theta: float, qubit: int) -> PauliRotation:
        return PauliRotation("X", (int(qubit),), float(theta))

    @staticmethod
    def ry(theta: float, qubit: int) -> PauliRotation:
        return PauliRotation("Y", (int(qubit),), float(theta))

    @staticmethod
    def rz(theta: float, qubit: int) -> PauliRotation:
        return PauliRotation("Z", (int(qubit),), float(theta))


class noise:  # noqa: N801
    @staticmethod
    def depolarize(p: float, qubit: int) -> Depolarizing:
        return Depolarizing(int(qubit), _check_probability("depolarize", "p", p))

    @staticmethod
    def dephase(p: float, qubit: int) -> PtmChannel:
        return PtmChannel("dephasing", _lib.PS_CH_DEPHASING, (int(qubit),),
                          param=_check_probability("dephase", "p", p))

    @staticmethod
    def amplitude_damping(gamma: float, qubit: int) -> PtmChannel:
        return PtmChannel("amplitude_damping", _lib.PS_CH_AMPLITUDE_DAMPING, (int(qubit),),
                          param=_check_probability("amplitude_damping", "gamma", gamma))

    @staticmethod
    def pauli_channel(px: float, py: float, pz: float, qubit: int) -> PtmChannel:
        """``E(rho) = (1-px-py-pz) rho + px X rho X + py Y rho Y + pz Z rho Z``
        (crates/paulistrings-py/src/noise.rs:52-68, 95-104)."""
        ps = tuple(float(v) for v in (px, py, pz))
        for name, v in zip(("px", "py", "pz"), ps):
            if not v >= 0.0:
                raise ValueError(f"pauli_channel: {name} must be non-negative (got {v})")
        if not sum(ps) <= 1.0:
            raise ValueError(f"pauli_channel: px + py + pz must be at most 1 (got {sum(ps)})")
        return PtmChannel("pauli_channel", _lib.PS_CH_PAULI_CHANNEL, (int(qubit),), params=ps)

    @staticmethod
    def depolarize2(p: float, q0: int, q1: int) -> PtmChannel:
        p = _check_probability("depolarize2", "p", p)
        return PtmChannel("depolarizing_2q", _lib.PS_CH_DEPOLARIZING_2Q, _distinct("depolarize2", q0, q1), param=p)


class Circuit:
    """An ordered list of channels on ``num_qubits`` qubits."""

    def __init__(self, num_qubits: int):
        if num_qubits < 1:
            raise ValueError("a circuit needs at least one qubit")
        self.num_qubits = int(num_qubits)
        self._channels: list = []

    def __len__(self) -> int:
        return len(self._channels)

    def __iter__(self):
        return iter(self._channels)

    def __getitem__(self, i):
        return self._channels[i]

    def _check(self, ch):
        for q in ch.support():
            if not 0 <= q < self.num_qubits:
                raise ValueError(f"qubit {q} is outside the {self.num_qubits}-qubit register")
        return ch

    def append(self, channel) -> None:
        self._channels.append(self._check(channel))

    def extend(self, other: "Circuit") -> None:
        if other.num_qubits != self.num_qubits:
            raise ValueError("circuits on different qubit counts")
        self._channels.extend(other._channels)

    def __add__(self, other: "Circuit") -> "Circuit":
        out = Circuit(self.num_qubits)
        out.extend(self)
        out.extend(other)
        return out

    def adjoint(self) -> "Circuit":
        out = Circuit(self.num_qubits)
        out._channels = [c.adjoint() for c in reversed(self._channels)]
        return out

    def rx(self, theta: float, qubit: int) -> None:
        self.append(gates.rx(theta, qubit))

    def ry(self, theta: float, qubit: int) -> None:
        self.append(gates.ry(theta, qubit))

    def rz(self, theta: float, qubit: int) -> None:
        self.append(gates.rz(theta, qubit))

    def pauli_rotation(self, pauli: str, qubits, theta: float) -> None:
        self.append(gates.pauli_rotation(pauli, qubits, theta))

    def depolarize(self, p: float, qubits) -> None:
        for q in qubits:
            self.append(noise.depolarize(p, q))

    def dephase(self, p: float, qubits) -> None:
        for q in qubits:
            self.append(noise.dephase(p, q))

    def amplitude_damping(self, gamma: float, qubits) -> None:
        for q in qubits:
            self.append(noise.amplitude_damping(gamma, q))

    def pauli_channel(self, px: float, py: float, pz: float, qubits) -> None:
        for q in qubits:
            self.append(noise.pauli_channel(px, py, pz, q))

    def depolarize2(self, p: float, pairs) -> None:
        for q0, q1 in pairs:
            self.append(noise.depolarize2(p, q0, q1))

    def h(self, qubit: int) -> None:
        self.append(gates.h(qubit))

    def s(self, qubit: int) -> None:
        self.append(gates.s(qubit))

    def sdg(self, qubit: int) -> None:
        self.append(gates.sdg(qubit))

    def x(self, qubit: int) -> None:
        self.append(gates.x(qubit))

    def y(self, qubit: int) -> None:
        self.append(gates.y(qubit))

    def z(self, qubit: int) -> None:
        self.append(gates.z(qubit))

    def cnot(self, control: int, target: int) -> None:
        self.append(gates.cnot(control, target))

    def cz(self, q0: int, q1: int) -> None:
        self.append(gates.cz(q0, q1))

    def swap(self, q0: int, q1: int) -> None:
        self.append(gates.swap(q0, q1))

    def unitary_1q(self, qubit: int, matrix) -> None:
        self.append(gates.unitary_1q(qubit, matrix))

    def unitary_2q(self, q0: int, q1: int, matrix) -> None:
        self.append(gates.unitary_2q(q0, q1, matrix))

    def preserves_hermiticity(self) -> bool:
        return True

    def to_c(self):
        """The channels as a ``ps_channel`` array; the returned tuple keeps the buffers alive."""
        n = len(self._channels)
        arr = (_lib.Channel * max(1, n))()
        keep = []
        for i, ch in enumerate(self._channels):
            qs = (ctypes.c_uint32 * max(1, len(ch.qubits)))(*ch.qubits)
            labels = ch.paulis.encode() if ch.paulis else b""
            keep.append((qs, labels))
            arr[i].kind = ch.kind
            arr[i].num_support = len(ch.qubits)
            arr[i].qubits = ctypes.cast(qs, ctypes.POINTER(ctypes.c_uint32))
            arr[i].paulis = labels
            arr[i].param = float(ch.param)
            matrix = getattr(ch, "matrix", None)
            if matrix is not None:
                mbuf = (ctypes.c_double * len(matrix))(*matrix)
                keep.append(mbuf)
                arr[i].matrix = ctypes.cast(mbuf, ctypes.POINTER(ctypes.c_double))
            for j, v in enumerate(getattr(ch, "params", (0.0, 0.0, 0.0))):
                arr[i].params[j] = float(v)
            arr[i].adjoint = 1 if getattr(ch, "is_adjoint", False) else 0
        return arr, n, keep
