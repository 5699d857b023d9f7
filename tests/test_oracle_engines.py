"""The oracle's two CPU engines agree bit for bit: the naive hash-accumulate layer (the
checker) and the sorted-store OpenMP engine in the reference host engine's shape (the timed
CPU baseline)."""

import numpy as np
import pytest

from oracle.oracle import OracleSum
from paulistrings_b200 import truncation, workloads
from tests._util import oracle_channels, oracle_policy


def _both(num_qubits, x, z, c, circ, policy, direction, dtype="f64", threads=4):
    out = []
    for sorted_engine in (False, True):
        s = OracleSum(num_qubits, dtype)
        s.set(np.concatenate([x, z], axis=1), c)
        after = s.propagate(oracle_channels(circ), oracle_policy(policy), direction,
                            sorted_engine=sorted_engine, threads=threads)
        out.append((s.get(), list(after)))
    return out


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_sorted_engine_matches_naive_on_random_pairs_with_topn(dtype):
    circ = workloads.random_pair_layers(24, 2)
    x, z, c = workloads.random_observable(24, 3000)
    pol = truncation.topn(20000) & truncation.coeff(1e-9)
    (ka, la), (kb, lb) = _both(24, x, z, c, circ, pol, "heisenberg", dtype)
    assert la == lb
    assert np.array_equal(ka[0], kb[0])
    assert np.array_equal(ka[1].view(np.uint64), kb[1].view(np.uint64))


def test_sorted_engine_matches_naive_on_noisy_tfim_and_wide_rotations():
    circ = workloads.tfim_2d(3, 2, noise_p=1e-3)
    circ.pauli_rotation("XYZX", [0, 4, 7, 8], 0.3)
    x, z, c = workloads.random_observable(9, 200)
    (ka, la), (kb, lb) = _both(9, x, z, c, circ, truncation.coeff(1e-5), "heisenberg")
    assert la == lb
    assert np.array_equal(ka[0], kb[0])
    assert np.array_equal(ka[1].view(np.uint64), kb[1].view(np.uint64))
