"""Pauli-sum file I/O in the ``paulistrings-npz-v1`` format (python/paulistrings/io.py:1-68).

An ``np.savez_compressed`` archive with keys ``format`` (the version string), ``num_qubits``,
``x`` and ``z`` (the ``uint64`` symplectic words, one row per term) and ``coefficients`` (in the
sum's dtype, which ``load`` restores).  ``load`` refuses a missing or unknown ``format``.
Device-resident sums save by downloading and load straight onto a device with
``load_device``.
"""

from __future__ import annotations

import os

import numpy as np

FORMAT = "paulistrings-npz-v1"

__all__ = ["FORMAT", "save", "load", "load_device"]


def _arrays(pauli_sum):
    from .sum import GpuPauliSum

    if isinstance(pauli_sum, GpuPauliSum):
        x, z, c = pauli_sum.download()
        if pauli_sum.dtype == "f32":
            c = c.astype(np.float32)
        return pauli_sum.num_qubits, x, z, c
    return pauli_sum.num_qubits, pauli_sum.x_array(), pauli_sum.z_array(), pauli_sum.coefficients_array()


def save(path: str | os.PathLike, pauli_sum) -> None:
    """Write ``pauli_sum`` (a ``PauliSum`` or a device-resident ``GpuPauliSum``) to ``path``;
    ``numpy.savez_compressed`` appends ``.npz`` when the path lacks it."""
    nq, x, z, c = _arrays(pauli_sum)
    np.savez_compressed(path, format=FORMAT, num_qubits=np.asarray(nq, dtype=np.int64), x=x, z=z, coefficients=c)


def _read(path):
    with np.load(path, allow_pickle=False) as data:
        if "format" not in data:
            raise ValueError(f"{os.fspath(path)!r}: missing 'format' field; not a paulistrings npz file")
        fmt = str(data["format"])
        if fmt != FORMAT:
            raise ValueError(f"{os.fspath(path)!r}: unknown format {fmt!r}, expected {FORMAT!r}")
        return int(data["num_qubits"]), data["x"], data["z"], data["coefficients"]


def _dtype_name(c):
    return "f32" if c.dtype == np.float32 else "f64"


def load(path: str | os.PathLike):
    """Read a ``PauliSum`` written by ``save`` (duplicates summed, zeros dropped, sorted)."""
    from .sum import PauliSum

    nq, x, z, c = _read(path)
    return PauliSum.from_arrays(x, z, c, nq, dtype=_dtype_name(c))


def load_device(path: str | os.PathLike, device: int = 0):
    """Read a saved sum straight into a device-resident ``GpuPauliSum`` on ``device``."""
    from .sum import GpuPauliSum

    nq, x, z, c = _read(path)
    g = GpuPauliSum(nq, _dtype_name(c), device)
    W = g.W
    g.upload(np.asarray(x, np.uint64).reshape(-1, W), np.asarray(z, np.uint64).reshape(-1, W),
             np.asarray(c, np.float64))
    return g
