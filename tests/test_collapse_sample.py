"""CollapseSample (crates/paulistrings/src/truncation/collapse_sample.rs): whenever a layer leaves
more than `cache` terms, `samples` systematic draws in proportion to |c| replace the sum.

CPU tests pin the oracle's key-addressed stream to the reference's own known values
(crates/paulistrings/src/rng/tests.rs) and check, as the reference's tests do
(crates/paulistrings/tests/propagate.rs:409-470), that trajectories are reproducible per seed,
stay within the cache, differ between seeds and are unbiased over many seeds.  GPU tests
compare the device pass with the oracle bit for bit (the same stretch accumulation per
1024-term block, the same points) and check the pass counter the policy carries.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import paulistrings_b200 as ps
from oracle import oracle as orc
from oracle.oracle import OracleSum, pauli_key
from paulistrings_b200 import truncation, workloads

from _util import assert_same_terms, oracle_arrays, oracle_channels, oracle_policy, oracle_sum


def test_stream_matches_the_reference_known_values():
    L = orc.lib()
    assert L.pso_splitmix64_first(0) == 0xE220A8397B1DCDAF
    st = (ctypes.c_uint64 * 4)(1, 2, 3, 4)
    out = (ctypes.c_uint64 * 2)()
    L.pso_xoshiro_two(ctypes.addressof(st), ctypes.addressof(out))
    assert list(out) == [41943041, 58720359]
    u = np.array([L.pso_keyed_uniform(0xABCD, k) for k in range(20000)])
    assert np.all((u >= 0) & (u < 1))
    assert abs(u.mean() - 0.5) < 5 * np.sqrt(1 / 12 / len(u))
    assert L.pso_keyed_uniform(7, 1) == L.pso_keyed_uniform(7, 1) != L.pso_keyed_uniform(7, 2)


def tfim_chain(n=4, steps=3, theta_j=-0.4, theta_h=0.5):
    c = ps.Circuit(n)
    for _ in range(steps):
        for q in range(n - 1):
            c.pauli_rotation("ZZ", [q, q + 1], theta_j)
        for q in range(n):
            c.rx(theta_h, q)
    return c


def oracle_run(circ, n, seed, cache=6, samples=4, policy=None):
    s = OracleSum(n)
    s.set(pauli_key("Z" + "I" * (n - 1), 1)[None, :], np.array([1.0]))
    pol = policy or {"keep": [], "passes": [("collapse_sample", cache, samples, seed, 0)]}
    s.propagate(oracle_channels(circ), pol, "heisenberg")
    return s


def test_oracle_trajectories_are_reproducible_bounded_and_seeded():
    circ = tfim_chain()
    finals = set()
    for seed in range(10):
        c0 = orc.collapses()
        a = oracle_run(circ, 4, seed)
        assert orc.collapses() - c0 >= 1, "the cache must be hit"
        assert len(a) <= 6
        b = oracle_run(circ, 4, seed)
        ka, ca = a.get()
        kb, cb = b.get()
        assert np.array_equal(ka, kb) and np.array_equal(ca, cb)
        finals.add(ka.tobytes())
    assert len(finals) > 1


def test_oracle_readout_is_unbiased():
    circ = tfim_chain()
    exact = OracleSum(4)
    exact.set(pauli_key("ZIII", 1)[None, :], np.array([1.0]))
    exact.propagate(oracle_channels(circ), None, "heisenberg")
    want = exact.expectation("z+")
    vals = np.array([oracle_run(circ, 4, seed).expectation("z+") for seed in range(2000)])
    err = vals.std(ddof=1) / np.sqrt(len(vals))
    assert err > 0
    assert abs(vals.mean() - want) < 4 * err, (vals.mean(), want, err)


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_small_trajectories_match_the_oracle_bit_for_bit(dtype):
    circ = tfim_chain()
    x = np.array([[0]], np.uint64)
    z = np.array([[1]], np.uint64)
    for seed in range(8):
        pol = truncation.collapse_sample(6, 4, seed)
        g = ps.GpuPauliSum(4, dtype)
        g.upload(x, z, np.array([1.0]))
        st = g.propagate(circ, pol, "heisenberg", with_stats=True)
        o = oracle_sum(4, x, z, [1.0], dtype)
        c0 = orc.collapses()
        after = o.propagate(oracle_channels(circ), {"keep": [], "passes": [("collapse_sample", 6, 4, seed, 0)]},
                            "heisenberg")
        assert st.collapses == orc.collapses() - c0 >= 1
        assert list(after) == st.terms_after and max(after) <= 6
        assert pol.calls == len(circ) and pol.collapses() == st.collapses
        assert_same_terms(g.download(), oracle_arrays(o), what=f"seed {seed} {dtype}")


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_large_collapse_matches_the_oracle(dtype):
    nq = 40
    x, z, c = workloads.random_observable(nq, 20000, seed=31)
    circ = workloads.random_pair_layers(nq, 1, seed=8)
    pol = truncation.coeff(1e-12) & truncation.collapse_sample(15000, 9000, 77)
    g = ps.GpuPauliSum(nq, dtype)
    g.upload(x, z, c)
    st = g.propagate(circ, pol, "heisenberg", with_stats=True)
    assert st.collapses >= 1
    o = oracle_sum(nq, x, z, c, dtype)
    after = o.propagate(oracle_channels(circ), {"keep": [("coeff", 1e-12)],
                                                "passes": [("collapse_sample", 15000, 9000, 77, 0)]},
                        "heisenberg")
    assert list(after) == st.terms_after
    assert_same_terms(g.download(), oracle_arrays(o), what=f"large {dtype}")


@pytest.mark.gpu
def test_a_reused_policy_continues_its_trajectory():
    circ = tfim_chain(steps=2)
    x = np.array([[0]], np.uint64)
    z = np.array([[1]], np.uint64)
    one = truncation.collapse_sample(5, 3, 11)
    g1 = ps.GpuPauliSum(4)
    g1.upload(x, z, np.array([1.0]))
    g1.propagate(circ + circ, one, "heisenberg")
    two = truncation.collapse_sample(5, 3, 11)
    g2 = ps.GpuPauliSum(4)
    g2.upload(x, z, np.array([1.0]))
    g2.propagate(circ, two, "heisenberg")   # Heisenberg: the second half of circ + circ first
    g2.propagate(circ, two, "heisenberg")
    assert two.calls == one.calls == 2 * len(circ)
    assert_same_terms(g2.download(), g1.download(), what="continued")
