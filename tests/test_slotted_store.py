"""The slotted merge store, seen from every entry point.

Before a TopN pass the rotation merge writes each tile's rows at the start of a fixed slot
and the TopN pass compacts them; every other reader of the handle compacts the slots first.
These tests drive ``ps_apply_layer`` and ``ps_finalize_layer`` separately (the reference's
apply_layer_body / finalize split) and read the store in between, so each path that meets a
slotted store is compared with the oracle: the length, a download, an expectation, a second
layer without a finalize, a finalize with another policy, and a TopN that does not trigger.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

import paulistrings_b200 as ps
from paulistrings_b200 import _lib, truncation, workloads
from paulistrings_b200.circuit import Circuit, gates
from paulistrings_b200.truncation import policy_to_c

from _util import assert_same_terms, oracle_arrays, oracle_channels, oracle_policy, oracle_sum

pytestmark = pytest.mark.gpu

NQ = 24
KEEP = truncation.coeff(1e-12)


def _channel(theta=0.4):
    return gates.pauli_rotation("XY", [0, 1], theta)


def _apply(g, channel, policy):
    c = Circuit(NQ)
    c.append(channel)
    arr, _, keep = c.to_c()
    table = _lib.Table()
    L = _lib.lib()
    _lib.check(L.ps_prepare_channel(NQ, L.ps_dtype_of(g._h), arr, 0, ctypes.byref(table)), None, "prepare")
    del keep
    pol = policy_to_c(policy)
    stats = _lib.LayerStats()
    _lib.check(L.ps_apply_layer(g._h, ctypes.byref(table), ctypes.byref(pol), ctypes.byref(stats)), g._h, "apply")
    return stats


def _finalize(g, policy):
    pol = policy_to_c(policy)
    _lib.check(_lib.lib().ps_finalize_layer(g._h, ctypes.byref(pol)), g._h, "finalize")


def _length(g):
    n = ctypes.c_uint64()
    _lib.check(_lib.lib().ps_len(g._h, ctypes.byref(n)), g._h, "len")
    return n.value


def _oracle(x, z, c, channels, policy, dtype="f64"):
    o = oracle_sum(NQ, x, z, c, dtype)
    o.propagate(oracle_channels(channels), oracle_policy(policy), "forward")
    return o


def _setup(dtype="f64", count=20000, seed=31):
    x, z, c = workloads.random_observable(NQ, count, seed=seed)
    g = ps.GpuPauliSum(NQ, dtype)
    g.upload(x, z, c)
    circ = Circuit(NQ)
    circ.append(_channel())
    applied = _oracle(x, z, c, circ, KEEP, dtype)  # the layer with the keep program, no pass
    return g, (x, z, c), circ, applied


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_reads_between_apply_and_finalize_see_the_compacted_layer(dtype):
    g, (x, z, c), circ, applied = _setup(dtype)
    live = len(oracle_arrays(applied)[2])
    pol = truncation.topn(live - 3000) & KEEP
    st = _apply(g, _channel(), pol)
    assert st.terms_out == live
    assert _length(g) == live
    assert_same_terms(g.download(), oracle_arrays(applied), what="download after apply")
    _finalize(g, pol)
    want = _oracle(x, z, c, circ, pol, dtype)
    assert_same_terms(g.download(), oracle_arrays(want), what="finalize after download")


def test_expectation_on_a_slotted_store():
    g, (x, z, c), circ, applied = _setup()
    live = len(oracle_arrays(applied)[2])
    pol = truncation.topn(live - 3000) & KEEP
    _apply(g, _channel(), pol)
    got = g.expectation("0" * NQ)
    ref = ps.GpuPauliSum(NQ)
    ref.upload(*oracle_arrays(applied))
    assert got == pytest.approx(ref.expectation("0" * NQ), rel=1e-12, abs=1e-15)
    _finalize(g, pol)
    want = _oracle(x, z, c, circ, pol)
    assert_same_terms(g.download(), oracle_arrays(want), what="finalize after expectation")


def test_topn_that_does_not_trigger_compacts_the_slots():
    g, (x, z, c), circ, applied = _setup()
    live = len(oracle_arrays(applied)[2])
    pol = truncation.topn(live + 100) & KEEP  # below the merge's 2n rows, above the live rows
    assert live + 100 < 2 * 20000
    _apply(g, _channel(), pol)
    _finalize(g, pol)
    assert_same_terms(g.download(), oracle_arrays(applied), what="untriggered topn")


def test_finalize_with_another_policy_compacts_first():
    g, (x, z, c), circ, applied = _setup()
    live = len(oracle_arrays(applied)[2])
    _apply(g, _channel(), truncation.topn(live - 3000) & KEEP)
    _finalize(g, KEEP)
    assert_same_terms(g.download(), oracle_arrays(applied), what="finalize without topn")


def test_second_layer_without_finalize_compacts_first():
    g, (x, z, c), circ, applied = _setup()
    live = len(oracle_arrays(applied)[2])
    pol = truncation.topn(live - 3000) & KEEP
    _apply(g, _channel(), pol)
    second = gates.pauli_rotation("ZX", [2, 5], 0.3)
    _apply(g, second, pol)
    _finalize(g, pol)
    want = oracle_sum(NQ, x, z, c)
    want.propagate(oracle_channels(circ), oracle_policy(KEEP), "forward")
    want.propagate(oracle_channels(_one(second)), oracle_policy(pol), "forward")
    assert_same_terms(g.download(), oracle_arrays(want), what="apply, apply, finalize")


def _one(channel):
    c = Circuit(NQ)
    c.append(channel)
    return c


def test_upload_replaces_a_slotted_store():
    g, (x, z, c), circ, applied = _setup()
    live = len(oracle_arrays(applied)[2])
    _apply(g, _channel(), truncation.topn(live - 3000) & KEEP)
    x2, z2, c2 = workloads.random_observable(NQ, 500, seed=77)
    g.upload(x2, z2, c2)
    assert _length(g) == 500
    assert_same_terms(g.download(), oracle_arrays(oracle_sum(NQ, x2, z2, c2)), what="upload over slots")
