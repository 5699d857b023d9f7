"""Failure handling without a GPU fault (needs a CUDA device).

Failures are injected on the host through ``ps_inject_fault`` (the reference's FaultPlan):
an allocation that reports out-of-memory, a merge launch that skips its first tile so the
next tile's output-offset wait polls a flag nothing sets until its (shortened) bounded limit,
and a device error word written from the host behind a layer's kernels.
In both cases the call must fail with its status, the store must keep the last completed
layer, and the handle must keep working.
"""

import numpy as np
import pytest

import paulistrings_b200 as ps
from paulistrings_b200 import _lib, truncation, workloads
from tests._util import assert_same_terms, oracle_arrays, oracle_channels, oracle_policy, oracle_sum

pytestmark = pytest.mark.gpu


def _sum(num_qubits=32, count=20000, seed=9):
    x, z, c = workloads.random_observable(num_qubits, count, seed=seed)
    g = ps.GpuPauliSum(num_qubits)
    g.upload(x, z, c)
    return g, (x, z, c)


def test_injected_oom_fails_the_layer_and_keeps_the_store():
    g, _ = _sum()
    before = g.download()
    circ = workloads.random_pair_layers(32, 1, seed=4)
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_OOM, 0), g._h, "inject")
    with pytest.raises(MemoryError):
        g.propagate(circ, truncation.coeff(1e-12))
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_NONE, 0), g._h, "disarm")
    assert_same_terms(g.download(), before, what="after-oom")
    # the handle still works, and matches the oracle from the same state
    g.propagate(circ, truncation.coeff(1e-12))
    o = oracle_sum(32, *before)
    o.propagate(oracle_channels(circ), {"keep": [("coeff", 1e-12)]})
    assert_same_terms(g.download(), oracle_arrays(o), what="after-recovery")


def test_injected_stall_times_out_boundedly_and_keeps_the_store():
    g, _ = _sum()
    before = g.download()
    circ = ps.Circuit(32)
    circ.pauli_rotation("XY", [0, 1], 0.4)
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_STALL, 1 << 14), g._h, "inject")
    with pytest.raises(_lib.PauliStringsError) as info:
        g.propagate(circ, truncation.coeff(1e-12))
    assert info.value.status == _lib.PS_ERR_TIMEOUT
    assert_same_terms(g.download(), before, what="after-stall")
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_NONE, 0), g._h, "disarm")
    g.propagate(circ, truncation.coeff(1e-12))
    o = oracle_sum(32, *before)
    o.propagate(oracle_channels(circ), {"keep": [("coeff", 1e-12)]})
    assert_same_terms(g.download(), oracle_arrays(o), what="after-stall-recovery")


def test_injection_can_be_disarmed():
    g, _ = _sum(count=2000)
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_OOM, 0), g._h, "inject")
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_NONE, 0), g._h, "disarm")
    circ = workloads.random_pair_layers(32, 1, seed=2)
    g.propagate(circ, truncation.coeff(1e-12))
    assert len(g) > 2000


def test_disarming_a_stall_restores_the_full_wait_limit():
    """A stall injected with a limit of 64 polls fails its layer; after PS_FAULT_NONE a layer
    over a few million terms (thousands of look-back tiles in flight, whose waits routinely
    take more than 64 polls) runs with the default limit and matches the oracle."""
    g, _ = _sum(num_qubits=48, count=200000, seed=11)
    circ = ps.Circuit(48)
    circ.pauli_rotation("XY", [0, 1], 0.4)
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_STALL, 64), g._h, "inject")
    with pytest.raises(_lib.PauliStringsError) as info:
        g.propagate(circ, truncation.coeff(1e-12))
    assert info.value.status == _lib.PS_ERR_TIMEOUT
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_NONE, 0), g._h, "disarm")
    before = g.download()
    big = workloads.random_pair_layers(48, 1, seed=5)
    g.propagate(big, truncation.coeff(1e-12))
    assert len(g) > 1_000_000
    o = oracle_sum(48, *before)
    o.propagate(oracle_channels(big), {"keep": [("coeff", 1e-12)]})
    assert_same_terms(g.download(), oracle_arrays(o), what="after-disarm")


@pytest.mark.parametrize("policy", ["topn", "threshold"])
def test_injected_device_flag_fails_the_layer_and_keeps_the_store(policy):
    """A device error word set behind a rotation layer fails that layer, also when the layer did
    not wait for its counts and its TopN pass was already queued behind it (the pass must then
    leave the store alone): the store keeps the last completed layer, and the next call works."""
    g, _ = _sum(count=20000)
    pol = truncation.topn(15000) if policy == "topn" else truncation.coeff(1e-12)
    warm = workloads.random_pair_layers(32, 1, seed=6)
    g.propagate(warm, pol)  # at the TopN cap: the layers after this one defer their counts
    before = g.download()
    circ = ps.Circuit(32)
    circ.pauli_rotation("XY", [0, 1], 0.4)
    circ.pauli_rotation("ZZ", [2, 3], 0.3)
    _lib.check(_lib.lib().ps_inject_fault(g._h, _lib.PS_FAULT_FLAG, 0), g._h, "inject")
    with pytest.raises(_lib.PauliStringsError) as info:
        g.propagate(circ, pol)
    assert info.value.status == _lib.PS_ERR_DEVICE
    assert_same_terms(g.download(), before, what=f"after-flag-{policy}")
    g.propagate(circ, pol)  # the injection is spent
    o = oracle_sum(32, *before)
    o.propagate(oracle_channels(circ), oracle_policy(pol))
    assert_same_terms(g.download(), oracle_arrays(o), what=f"after-flag-recovery-{policy}")
