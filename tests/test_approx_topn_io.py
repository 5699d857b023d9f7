"""ApproxTopN (crates/paulistrings/src/truncation/builtin.rs:240-468) and npz I/O
(python/paulistrings/io.py).

ApproxTopN keeps every octave of |c|^2 (its exponent field) above the boundary octave and the
first terms of the boundary octave in key order, n in all; NaN is counted in the top octave
and never kept.  The oracle restates it; GPU tests compare the device pass bit for bit, with
the octave histogram built by the layer's merge (first pass) or by its own kernel (a later
pass).  The npz tests mirror the reference's format checks.
"""

from __future__ import annotations

import numpy as np
import pytest

import paulistrings_b200 as ps
from oracle.oracle import OracleSum, pauli_key
from paulistrings_b200 import io, truncation, workloads

from _util import assert_same_terms, oracle_arrays, oracle_channels, oracle_policy, oracle_sum


def test_oracle_approx_topn_known_answer():
    s = OracleSum(2)
    labels = ["XI", "YI", "ZI", "IX", "IY", "IZ"]
    # octaves of c^2: 0.81 -> -1, 0.25 -> -2 (three terms), 0.01 -> -7
    coeffs = [0.5, -0.5, 0.1, 0.5, 0.9, float("nan")]
    s.set(np.stack([pauli_key(l, 1) for l in labels]), np.array(coeffs))
    s.apply(("rotation", "Z", [0], 0.0), policy={"keep": [], "passes": [("approx_topn", 3)]})
    keys, c = s.get()
    # NaN counted in the top octave (kept_above = 1), then 0.81 (kept_above = 2), then the
    # 0.25 octave overflows: quota 1, its first term in key order
    got = {tuple(k): v for k, v in zip(map(tuple, keys), c)}
    assert len(got) == 2
    assert 0.9 in got.values()
    assert sorted(abs(v) for v in got.values()) == [0.5, 0.9]


def test_npz_rejects_missing_and_unknown_formats(tmp_path):
    p = tmp_path / "bad.npz"
    np.savez_compressed(p, num_qubits=2, x=np.zeros((1, 1), np.uint64), z=np.zeros((1, 1), np.uint64),
                        coefficients=np.ones(1))
    with pytest.raises(ValueError, match="missing 'format'"):
        io.load(p)
    np.savez_compressed(p, format="paulistrings-npz-v0", num_qubits=2, x=np.zeros((1, 1), np.uint64),
                        z=np.zeros((1, 1), np.uint64), coefficients=np.ones(1))
    with pytest.raises(ValueError, match="unknown format"):
        io.load(p)


def test_npz_writes_the_reference_layout(tmp_path):
    s = ps.PauliSum(70, "f32")
    s._set_sorted(np.array([[1, 0], [2, 5]], np.uint64), np.array([[0, 0], [1, 0]], np.uint64),
                  np.array([0.5, -0.25]))
    io.save(tmp_path / "s", s)
    with np.load(tmp_path / "s.npz") as d:
        assert str(d["format"]) == io.FORMAT
        assert int(d["num_qubits"]) == 70
        assert d["x"].dtype == np.uint64 and d["x"].shape == (2, 2)
        assert d["coefficients"].dtype == np.float32


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("first", [True, False])
def test_approx_topn_matches_the_oracle(dtype, first):
    x, z, c = workloads.random_observable(40, 6000, seed=9)
    rng = np.random.default_rng(3)
    c = c * np.exp2(rng.integers(-6, 6, size=len(c)))  # spread the octaves
    circ = workloads.random_pair_layers(40, 2)
    pol = truncation.approx_topn(5000) & truncation.coeff(1e-12) if first else \
        truncation.coeff(1e-12) & truncation.topn(1 << 30) & truncation.approx_topn(5000)
    g = ps.GpuPauliSum(40, dtype)
    g.upload(x, z, c)
    st = g.propagate(circ, pol, "heisenberg", with_stats=True)
    got = g.download()
    o = oracle_sum(40, x, z, c, dtype)
    after = o.propagate(oracle_channels(circ), oracle_policy(pol), "heisenberg")
    assert list(after) == st.terms_after
    assert_same_terms(got, oracle_arrays(o), what=f"approx {dtype} first={first}")
    assert max(st.terms_after) <= 5000


@pytest.mark.gpu
def test_approx_topn_nan_and_ties():
    labels = ["XI", "YI", "ZI", "IX", "IY", "IZ"]
    x = np.stack([pauli_key(l, 1)[:1] for l in labels])
    z = np.stack([pauli_key(l, 1)[1:] for l in labels])
    c = np.array([0.5, -0.5, 0.1, 0.5, 0.9, float("nan")])
    circ = ps.Circuit(2)
    circ.rz(0.0, 0)
    for keep in range(0, 8):
        g = ps.GpuPauliSum(2)
        g.upload(x, z, c)
        g.propagate(circ, truncation.approx_topn(keep), "forward")
        o = oracle_sum(2, x, z, c)
        o.propagate(oracle_channels(circ), {"keep": [], "passes": [("approx_topn", keep)]}, "forward")
        assert_same_terms(g.download(), oracle_arrays(o), what=f"approx nan keep={keep}")


@pytest.mark.gpu
def test_npz_round_trip_host_and_device(tmp_path):
    x, z, c = workloads.random_observable(100, 3000, seed=4)
    s = ps.PauliSum.from_arrays(x, z, c, 100)
    io.save(tmp_path / "a.npz", s)
    back = io.load(tmp_path / "a.npz")
    assert back.num_qubits == 100 and back.dtype == "f64"
    assert np.array_equal(back.x_array(), s.x_array()) and np.array_equal(back.coefficients_array(),
                                                                         s.coefficients_array())
    g = io.load_device(tmp_path / "a.npz")
    circ = workloads.random_pair_layers(100, 1)
    g.propagate(circ, truncation.coeff(1e-9), "heisenberg")
    io.save(tmp_path / "b.npz", g)  # a resident sum saves without a host PauliSum
    s.propagate(circ, truncation.coeff(1e-9), direction="heisenberg", device=0)
    b = io.load(tmp_path / "b.npz")
    assert np.array_equal(b.x_array(), s.x_array()) and np.array_equal(b.coefficients_array(),
                                                                      s.coefficients_array())
    f32 = ps.PauliSum.from_arrays(x, z, c, 100, dtype="f32")
    io.save(tmp_path / "c.npz", f32)
    assert io.load(tmp_path / "c.npz").dtype == "f32"
