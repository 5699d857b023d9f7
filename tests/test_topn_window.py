"""TopN across layers: after a TopN pass the next layer's merge bins its first select digit in a
window of 1/16 octaves around the last boundary; a boundary that left the window is detected
on the device and the pass reruns in full range.  Both must give the oracle's bits.
"""

from __future__ import annotations

import numpy as np
import pytest

import paulistrings_b200 as ps
from paulistrings_b200 import truncation, workloads

from _util import assert_same_terms, oracle_arrays, oracle_channels, oracle_policy, oracle_sum

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_topn_over_many_layers_matches_the_oracle(dtype):
    nq = 24
    x, z, c = workloads.random_observable(nq, 3000, seed=21)
    circ = workloads.random_pair_layers(nq, 4, seed=5)
    pol = truncation.topn(20000) & truncation.coeff(1e-12)
    g = ps.GpuPauliSum(nq, dtype)
    g.upload(x, z, c)
    st = g.propagate(circ, pol, "heisenberg", with_stats=True)
    o = oracle_sum(nq, x, z, c, dtype)
    after = o.propagate(oracle_channels(circ), oracle_policy(pol), "heisenberg")
    assert list(after) == st.terms_after
    assert max(st.terms_after) == 20000
    assert_same_terms(g.download(), oracle_arrays(o), what=f"topn layers {dtype}")


@pytest.mark.parametrize("scale", [2.0 ** 300, 2.0 ** -300, 1.5])
def test_boundary_far_from_the_window_reruns_in_full_range(scale):
    nq = 24
    x, z, c = workloads.random_observable(nq, 3000, seed=22)
    circ = workloads.random_pair_layers(nq, 1, seed=6)
    pol = truncation.topn(5000)
    g = ps.GpuPauliSum(nq)
    g.upload(x, z, c)
    g.propagate(circ, pol, "heisenberg")  # leaves a window around this layer's boundary
    gx, gz, gc = g.download()
    g.upload(gx, gz, gc * scale)  # the next boundary is octaves away (or not, for 1.5)
    g.propagate(circ, pol, "heisenberg")
    o = oracle_sum(nq, gx, gz, gc * scale)
    o.propagate(oracle_channels(circ), oracle_policy(pol), "heisenberg")
    assert_same_terms(g.download(), oracle_arrays(o), what=f"scale {scale}")
