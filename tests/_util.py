"""Shared test helpers: bridge product objects to the oracle and compare results."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np

from oracle.oracle import OracleSum
from paulistrings_b200 import _lib
from paulistrings_b200.circuit import Circuit, Depolarizing, PauliRotation, PtmChannel

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_golden(name: str):
    return json.loads((GOLDEN / name).read_text())


def circuit_from_gates(num_qubits: int, gates) -> Circuit:
    c = Circuit(num_qubits)
    for kind, paulis, qubits, param in gates:
        assert kind == "rotation"
        c.pauli_rotation(paulis, qubits, param)
    return c


def oracle_channels(circuit: Circuit):
    out = []
    for ch in circuit:
        if isinstance(ch, PauliRotation):
            out.append(("rotation", ch.paulis, list(ch.qubits), ch.theta))
        elif isinstance(ch, Depolarizing):
            out.append(("depolarize", "", [ch.qubit], ch.p))
        elif isinstance(ch, PtmChannel):
            extra = {"adjoint": ch.is_adjoint, "params": ch.params}
            if ch.matrix is not None:
                flat = np.asarray(ch.matrix)
                extra["matrix"] = flat[0::2] + 1j * flat[1::2]
            out.append((_PTM_NAMES[ch.kind], "", list(ch.qubits), ch.param, extra))
        else:
            raise TypeError(ch)
    return out


_PTM_NAMES = {_lib.PS_CH_HADAMARD: "h", _lib.PS_CH_PHASE: "s", _lib.PS_CH_PHASE_DAGGER: "sdg",
              _lib.PS_CH_PAULI_X: "x", _lib.PS_CH_PAULI_Y: "y", _lib.PS_CH_PAULI_Z: "z",
              _lib.PS_CH_CNOT: "cnot", _lib.PS_CH_CZ: "cz", _lib.PS_CH_SWAP: "swap",
              _lib.PS_CH_UNITARY: "unitary", _lib.PS_CH_DEPHASING: "dephase",
              _lib.PS_CH_PAULI_CHANNEL: "pauli_channel", _lib.PS_CH_DEPOLARIZING_2Q: "depolarize2",
              _lib.PS_CH_AMPLITUDE_DAMPING: "amplitude_damping"}


def oracle_policy(policy):
    if policy is None:
        return None
    nodes, passes = policy.lowered()
    names = {_lib.PS_KEEP_TRUE: "true", _lib.PS_KEEP_COEFF: "coeff", _lib.PS_KEEP_WEIGHT: "weight",
             _lib.PS_KEEP_AND: "and", _lib.PS_KEEP_OR: "or"}
    keep = []
    for op, iarg, farg in nodes:
        nm = names[op]
        if nm == "coeff":
            keep.append((nm, farg))
        elif nm == "weight":
            keep.append((nm, iarg))
        else:
            keep.append((nm,))
    names = {_lib.PS_PASS_TOPN: "topn", _lib.PS_PASS_APPROX_TOPN: "approx_topn",
             _lib.PS_PASS_COLLAPSE_SAMPLE: "collapse_sample"}
    return {"keep": keep, "passes": [(names[p[0]],) + tuple(p[1:]) for p in passes if p[0] in names]}


def oracle_sum(num_qubits, x, z, c, dtype="f64") -> OracleSum:
    s = OracleSum(num_qubits, dtype)
    W = s.W
    keys = np.concatenate([np.asarray(x, np.uint64).reshape(-1, W), np.asarray(z, np.uint64).reshape(-1, W)], axis=1)
    s.set(keys, np.asarray(c, np.float64))
    return s


def oracle_arrays(s: OracleSum):
    keys, c = s.get()
    W = s.W
    return keys[:, :W], keys[:, W:], c


def assert_same_terms(got, want, rtol=0.0, what=""):
    """Keys bit-exact; coefficients bit-exact (rtol=0) or within rtol of the larger magnitude."""
    gx, gz, gc = got
    wx, wz, wc = want
    assert gx.shape == wx.shape, f"{what}: {gx.shape[0]} terms vs {wx.shape[0]} expected"
    assert np.array_equal(gx, wx) and np.array_equal(gz, wz), f"{what}: key sets differ"
    if rtol == 0.0:
        # bit-exact; a NaN matches any NaN (payloads differ between host and device arithmetic)
        both_nan = np.isnan(gc) & np.isnan(wc)
        bad = np.nonzero((gc.view(np.uint64) != wc.view(np.uint64)) & ~both_nan)[0]
        assert bad.size == 0, f"{what}: {bad.size} coefficients differ, first {gc[bad[0]]!r} vs {wc[bad[0]]!r}"
    else:
        scale = np.maximum(np.abs(gc), np.abs(wc))
        err = np.abs(gc - wc)
        assert np.all(err <= rtol * scale), f"{what}: max rel err {np.max(err / np.where(scale > 0, scale, 1))}"
