"""The oracle against the reference's own results (CPU only).

Pins the CPU oracle before it is trusted as the parity checker:
* XXZ chain statevector fixtures (examples/xxz_chain/results/statevector.json): final
  term counts exactly, expectation values to the reference's printed digits;
* jl-parity fixtures (benchmarks/python/jl_performance/post-optimization/summary.json):
  XXZ n = 100 and the 127-qubit kicked-Ising circuit (Clifford-point ZZ), final term counts
  exactly and expectations;
* hand-computed rotation identities (python/paulistrings/tests/test_pauli_rotation.py:62-137).
"""

import math

import numpy as np
import pytest

from oracle.oracle import OracleSum, pauli_key
from tests._util import load_golden


def _run(n, gates, eps, obs_z, state, max_weight=None):
    s = OracleSum(n, "f64")
    lab = ["I"] * n
    for q in obs_z:
        lab[q] = "Z"
    s.set(pauli_key("".join(lab), s.W)[None, :], np.array([1.0]))
    keep = [("coeff", eps)]
    if max_weight is not None:
        keep = [("weight", max_weight)] + keep + [("and",)]
    s.propagate([tuple(g) for g in gates], policy={"keep": keep}, direction="heisenberg")
    return len(s), s.expectation(state)


XXZ = load_golden("xxz_statevector.json")["cases"]


@pytest.mark.parametrize("case", [c for c in XXZ if c["final_terms"] <= 200_000],
                         ids=lambda c: f"n{c['n']}-Jz{c['Jz']}-s{c['steps']}-o{len(c['observable_z'])}")
def test_oracle_matches_xxz_statevector_fixture(case):
    terms, value = _run(case["n"], case["gates"], case["epsilon"], case["observable_z"], case["state"])
    assert terms == case["final_terms"]
    # the reference's value and ours differ only by summation order
    assert abs(value - case["expectation"]) <= 1e-14
    assert abs(value - case["statevector"]) <= 1e-9


JL = load_golden("jl_parity.json")["workloads"]


@pytest.mark.parametrize(
    "key,point",
    [(k, p) for k, w in JL.items() for p in w["points"] if p["final_terms"] <= 80_000],
    ids=lambda v: v if isinstance(v, str) else f"eps{v['epsilon']:.3g}-w{v['max_weight']}",
)
def test_oracle_matches_jl_parity_fixture(key, point):
    w = JL[key]
    terms, value = _run(w["n_qubits"], w["gates"], point["epsilon"], w["observable_z"], w["state"], point["max_weight"])
    assert terms == point["final_terms"]
    if point["expectation"] is not None:
        assert abs(value - point["expectation"]) <= 1e-13


def _one(n, label, coeff=1.0):
    s = OracleSum(n, "f64")
    s.set(pauli_key(label, s.W)[None, :], np.array([coeff]))
    return s


def _as_dict(s):
    keys, c = s.get()
    W = s.W
    out = {}
    for k, v in zip(keys, c):
        lab = []
        for q in range(s.num_qubits):
            xb = (int(k[q // 64]) >> (q % 64)) & 1
            zb = (int(k[W + q // 64]) >> (q % 64)) & 1
            lab.append("IXZY"[xb | zb << 1])
        out["".join(lab)] = v
    return out


def test_rz_on_x_is_cos_x_plus_sin_y():
    theta = 0.6
    s = _one(1, "X")
    s.apply(("rotation", "Z", [0], theta))
    assert _as_dict(s) == pytest.approx({"X": math.cos(theta), "Y": math.sin(theta)}, abs=1e-15)


def test_zz_on_xi_is_cos_xi_plus_sin_yz():
    theta = 0.6
    s = _one(2, "XI")
    s.apply(("rotation", "ZZ", [0, 1], theta))
    assert _as_dict(s) == pytest.approx({"XI": math.cos(theta), "YZ": math.sin(theta)}, abs=1e-15)


def test_kicked_ising_bond_maps_xi_to_minus_yz_exactly():
    s = _one(2, "XI")
    s.apply(("rotation", "ZZ", [0, 1], -math.pi / 2))
    assert _as_dict(s) == {"YZ": -1.0}


def test_weight_three_rotation_identity():
    # exp(-i t XYZ / 2) on ZII: Z anticommutes with X; ZII * XYZ = (ZX) Y Z = (iY) Y Z = i IIZ... product via key algebra
    theta = 0.37
    s = _one(3, "ZII")
    s.apply(("rotation", "XYZ", [0, 1, 2], theta))
    d = _as_dict(s)
    assert set(d) == {"ZII", "YYZ"}
    assert d["ZII"] == pytest.approx(math.cos(theta), abs=1e-15)
    assert abs(d["YYZ"]) == pytest.approx(math.sin(theta), abs=1e-15)


def test_heisenberg_round_trip_is_identity():
    gates = [("rotation", "XY", [0, 2], 0.3), ("rotation", "Z", [1], 1.1), ("rotation", "YYZ", [0, 1, 2], -0.7)]
    s = _one(3, "XZY", 0.5)
    s.propagate(gates, direction="forward")
    s.propagate(gates, direction="heisenberg")
    d = _as_dict(s)
    assert d["XZY"] == pytest.approx(0.5, abs=1e-15)
    assert all(abs(v) < 1e-15 for k, v in d.items() if k != "XZY")


def test_depolarizing_scales_non_identity_factors():
    s = OracleSum(2, "f64")
    keys = np.stack([pauli_key(l, 1) for l in ("XI", "IZ", "YZ", "II")])
    s.set(keys, np.array([1.0, 2.0, 3.0, 4.0]))
    s.apply(("depolarize", "", [0], 0.1))
    sc = 1.0 - 4.0 * 0.1 / 3.0
    assert _as_dict(s) == {"XI": 1.0 * sc, "IZ": 2.0, "YZ": 3.0 * sc, "II": 4.0}


def test_topn_keeps_largest_and_ties_in_key_order():
    s = OracleSum(2, "f64")
    labels = ["XI", "YI", "ZI", "IX", "IY", "IZ"]
    keys = np.stack([pauli_key(l, 1) for l in labels])
    s.set(keys, np.array([0.5, -0.5, 0.1, 0.5, 0.9, float("nan")]))
    s.apply(("rotation", "Z", [0], 0.0), policy={"keep": [], "passes": [("topn", 3)]})
    # the three |c| = 0.5 terms tie at the boundary: the first two in key order (x words, then
    # z words) survive, XI = (1, 0) and YI = (1, 1) before IX = (2, 0); NaN is never kept
    assert _as_dict(s) == {"XI": 0.5, "YI": -0.5, "IY": 0.9}


def test_threshold_is_strict():
    s = OracleSum(1, "f64")
    s.set(np.stack([pauli_key("X", 1), pauli_key("Z", 1)]), np.array([0.25, 0.5]))
    s.apply(("rotation", "Z", [0], 0.0), policy={"keep": [("coeff", 0.25)]})
    assert _as_dict(s) == {"Z": 0.5}
