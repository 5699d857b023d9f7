"""paulistrings_b200 -- the per-layer Pauli-propagation path on one NVIDIA B200.

A drop-in for ``PauliSum.propagate(circuit, policy, direction, device=)`` of
lkdvos/paulistrings-rs: the Pauli sum lives on the device as packed symplectic keys plus
float64 or float32 coefficients, and every layer runs as hand-written sm_100a kernels
behind the C ABI in ``include/paulistrings_b200.h``.
"""

from . import truncation
from ._lib import PauliStringsError, device_count
from .circuit import Circuit, Depolarizing, PauliRotation, PtmChannel, gates, noise
from .sum import (
    GpuPauliSum,
    PauliSum,
    PropagationStats,
    cuda_available,
    parse_label,
    product_basis,
    propagated,
    propagated_with_stats,
    width_for,
)


def p(label: str) -> str:
    """A Pauli string label (``IXYZ`` per qubit), validated."""
    for ch in label:
        if ch not in "IXYZ":
            raise ValueError(f"bad Pauli character {ch!r}")
    return label


__all__ = [
    "Circuit",
    "Depolarizing",
    "GpuPauliSum",
    "PauliRotation",
    "PtmChannel",
    "PauliStringsError",
    "PauliSum",
    "PropagationStats",
    "cuda_available",
    "device_count",
    "gates",
    "noise",
    "p",
    "parse_label",
    "product_basis",
    "propagated",
    "propagated_with_stats",
    "truncation",
    "width_for",
]
