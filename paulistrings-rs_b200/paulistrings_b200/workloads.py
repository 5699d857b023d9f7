"""Seeded synthetic workloads of the measured configurations.

* ``tfim_2d``: transverse-field Ising Trotter circuit on an L x L periodic lattice, site
  ``i = y * L + x``; per step ``pauli_rotation("ZZ", bond, -2 J dt)`` on every horizontal bond
  (x, y)-(x+1, y) in row-major order, then every vertical bond (x, y)-(x, y+1), then
  ``rx(2 h dt)`` on every qubit; optional depolarizing noise on every qubit after each step.
* ``random_pair_layers``: per layer a seeded Fisher-Yates matching of the qubits into pairs,
  each pair ``exp(-i theta P(x)Q / 2)`` with P, Q uniform in {X, Y, Z} and theta uniform in
  [0, 2 pi), then ``rz(phi)`` on every qubit with phi uniform in [0, 2 pi).
* ``random_observable``: distinct random Pauli strings of weight 1-4 on uniformly chosen
  qubits, coefficients standard normal (Box-Muller) scaled to unit 2-norm.
* ``xxz_chain``: the open XXZ chain of the reference's ``examples/common/circuits.py:292-339``
  (per bond XX, YY, ZZ rotations with theta = 2 dt, 2 dt, 2 dt Jz; even bonds then odd).

All randomness comes from one splitmix64 stream, so every run of a workload is identical.
"""

from __future__ import annotations

import math

import numpy as np

from .circuit import Circuit

MASK64 = (1 << 64) - 1


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014)."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / (1 << 53))

    def below(self, n: int) -> int:
        return int(self.uniform() * n)

    def normal(self) -> float:
        u1 = self.uniform()
        u2 = self.uniform()
        u1 = u1 if u1 > 0.0 else 1.0 / (1 << 53)
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


DEFAULT_SEED = 0xC0FFEE


def tfim_2d(L: int, steps: int, J: float = 1.0, h: float = 1.0, dt: float = 0.1, noise_p: float | None = None) -> Circuit:
    n = L * L
    c = Circuit(n)
    theta_j = -2.0 * J * dt
    theta_h = 2.0 * h * dt
    for _ in range(steps):
        for y in range(L):
            for x in range(L):
                c.pauli_rotation("ZZ", [y * L + x, y * L + (x + 1) % L], theta_j)
        for y in range(L):
            for x in range(L):
                c.pauli_rotation("ZZ", [y * L + x, ((y + 1) % L) * L + x], theta_j)
        for q in range(n):
            c.rx(theta_h, q)
        if noise_p is not None:
            c.depolarize(noise_p, list(range(n)))
    return c


def tfim_magnetization(L: int, axis: str = "X"):
    """``(1 / L^2) * sum_i axis_i`` as {label: coefficient}."""
    n = L * L
    out = {}
    for q in range(n):
        lab = ["I"] * n
        lab[q] = axis
        out["".join(lab)] = 1.0 / n
    return out


def random_pair_layers(num_qubits: int, layers: int, seed: int = DEFAULT_SEED) -> Circuit:
    rng = SplitMix64(seed)
    c = Circuit(num_qubits)
    for _ in range(layers):
        perm = list(range(num_qubits))
        for i in range(num_qubits - 1, 0, -1):
            j = rng.below(i + 1)
            perm[i], perm[j] = perm[j], perm[i]
        for k in range(num_qubits // 2):
            a, b = perm[2 * k], perm[2 * k + 1]
            p = "XYZ"[rng.below(3)]
            q = "XYZ"[rng.below(3)]
            theta = 2.0 * math.pi * rng.uniform()
            c.pauli_rotation(p + q, [a, b], theta)
        for q in range(num_qubits):
            c.rz(2.0 * math.pi * rng.uniform(), q)
    return c


def random_observable(num_qubits: int, count: int, seed: int = DEFAULT_SEED + 1):
    """(x, z, coefficients) of ``count`` distinct random strings, W words per row."""
    W = (num_qubits + 63) // 64
    rng = SplitMix64(seed)
    seen = set()
    xs, zs, cs = [], [], []
    while len(xs) < count:
        w = 1 + rng.below(4)
        qubits = set()
        while len(qubits) < w:
            qubits.add(rng.below(num_qubits))
        x = [0] * W
        z = [0] * W
        for q in sorted(qubits):
            p = rng.below(3)
            if p in (0, 1):
                x[q // 64] |= 1 << (q % 64)
            if p in (1, 2):
                z[q // 64] |= 1 << (q % 64)
        key = (tuple(x), tuple(z))
        if key in seen:
            continue
        seen.add(key)
        xs.append(x)
        zs.append(z)
        cs.append(rng.normal())
    c = np.array(cs, dtype=np.float64)
    c /= np.sqrt(np.sum(c * c))
    return np.array(xs, dtype=np.uint64), np.array(zs, dtype=np.uint64), c


def xxz_chain(n: int, steps: int, Jz: float = 0.5, dt: float = 0.1) -> Circuit:
    bonds = [i for i in range(n - 1) if i % 2 == 0] + [i for i in range(n - 1) if i % 2 == 1]
    c = Circuit(n)
    for _ in range(steps):
        for i in bonds:
            c.pauli_rotation("XX", [i, i + 1], 2.0 * dt)
            c.pauli_rotation("YY", [i, i + 1], 2.0 * dt)
            c.pauli_rotation("ZZ", [i, i + 1], 2.0 * dt * Jz)
    return c


def neel_state(n: int) -> str:
    return "".join("0" if q % 2 == 0 else "1" for q in range(n))
