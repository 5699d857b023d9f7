"""``Circuit`` and the channel factories (``gates``, ``noise``).

Mirrors the reference's Python surface (crates/paulistrings-py/src/circuit.rs:102-321,
crates/paulistrings-py/src/gates.rs:193): a circuit is an ordered list of channels, each
applied as one layer.  The built-ins on the device path are Pauli rotations
``exp(-i theta P / 2)`` of any weight and single-qubit depolarizing noise.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

from . import _lib


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


class gates:  # noqa: N801  (module-like namespace, as the reference's ``gates`` submodule)
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
    def depolarizing(qubit: int, p: float) -> Depolarizing:
        return Depolarizing(int(qubit), float(p))


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
            self.append(noise.depolarizing(q, p))

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
        return arr, n, keep
