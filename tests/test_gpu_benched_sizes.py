"""Parity at the sizes the benchmark measures, and the precision form's error report.

* The headline workload (64 qubits, random two-qubit rotation layers + RZ sweeps, the
  65,536-term random observable, Heisenberg, ``TopN(2^26) & coeff(1e-10)``, f64) propagated
  through its first 200 channels: the 2^26-term cap binds at channel 184, so the last 16
  channels run the capped path the benchmark times (the slotted merge output, the windowed
  first TopN digit and its compaction).  Every surviving string and coefficient must equal the
  oracle's sorted-store engine bit for bit.
* The precision form (the noisy 6 x 6 transverse-field Ising circuit: 5 Trotter steps,
  depolarizing p = 1e-3 on every qubit after each step, ``coeff(1e-5)``, Heisenberg, readout
  in |0...0>): the f64 run must equal the f64 oracle bit for bit; the f32 run with compensated
  sums is compared with it, and its <O> error and its largest coefficient error over the
  strings both runs keep must stay within the bounds below (f32 carries 24 significant bits;
  540 channels compound at most a few hundred roundings per coefficient).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import paulistrings_b200 as ps
from paulistrings_b200 import _lib, truncation, workloads
from tests._util import assert_same_terms, oracle_arrays, oracle_channels, oracle_policy, oracle_sum

pytestmark = pytest.mark.gpu

HEADLINE_SEED = 0xC0FFEE
HEADLINE_CAP = 1 << 26

# The f32 form against the f64 run on the noisy 6 x 6 circuit.
PRECISION_EXPECTATION_REL = 1e-5      # |<O>_f32 - <O>_f64| / |<O>_f64|
PRECISION_COEFF_REL_TO_MAX = 1e-5     # max |c_f32 - c_f64| over common strings / max |c_f64|


def headline_prefix(num_channels):
    """The first ``num_channels`` channels the headline run applies (Heisenberg order: the last
    layer's channels first), as a forward circuit to propagate with direction="heisenberg"."""
    full = list(workloads.random_pair_layers(64, 30, HEADLINE_SEED))
    circ = ps.Circuit(64)
    for ch in full[len(full) - num_channels:]:
        circ.append(ch)
    return circ


def test_headline_workload_at_the_full_cap_bit_exact():
    circ = headline_prefix(200)
    x, z, c = workloads.random_observable(64, 65536, HEADLINE_SEED + 1)
    policy = truncation.topn(HEADLINE_CAP) & truncation.coeff(1e-10)
    g = ps.GpuPauliSum(64, "f64")
    g.upload(x, z, c)
    after = g.propagate(circ, policy, "heisenberg", with_stats=True).terms_after
    assert int(after[-1]) == HEADLINE_CAP
    capped = int(np.sum(np.asarray(after) == HEADLINE_CAP))
    assert capped >= 12, f"the cap bound on only {capped} channels"
    got = g.download()
    value = g.expectation("z+")
    g.close()
    o = oracle_sum(64, x, z, c)
    o_after = o.propagate(oracle_channels(circ), oracle_policy(policy), "heisenberg", sorted_engine=True,
                          threads=os.cpu_count())
    assert [int(v) for v in after] == [int(v) for v in o_after]
    assert_same_terms(got, oracle_arrays(o), what="headline-at-cap")
    assert value == pytest.approx(o.expectation("z+"), rel=1e-12, abs=1e-15)


def _common_coefficients(a, b):
    """Coefficients of the strings present in both runs (keys sorted in both)."""
    ka = np.concatenate([a[0], a[1]], axis=1)
    kb = np.concatenate([b[0], b[1]], axis=1)
    va = ka.view([("", ka.dtype)] * ka.shape[1]).ravel()
    vb = kb.view([("", kb.dtype)] * kb.shape[1]).ravel()
    _, ia, ib = np.intersect1d(va, vb, assume_unique=True, return_indices=True)
    return a[2][ia], b[2][ib]


def precision_report(steps=5, p=1e-3, threshold=1e-5):
    """The f32-with-compensated-sums run against the f64 run of the noisy 6 x 6 circuit."""
    circ = workloads.tfim_2d(6, steps, J=1.0, h=1.0, dt=0.1, noise_p=p)
    obs = workloads.tfim_magnetization(6, "X")
    out = {}
    for dtype in ("f64", "f32"):
        g = ps.PauliSum.from_strings(obs, num_qubits=36, dtype=dtype).to_device(0)
        if dtype == "f32":
            _lib.check(_lib.lib().ps_set_compensated_sums(g._h, 1), g._h, "compensated")
        g.propagate(circ, truncation.coeff(threshold), "heisenberg")
        out[dtype] = (g.expectation("0" * 36), g.download())
        g.close()
    e64, s64 = out["f64"]
    e32, s32 = out["f32"]
    c64, c32 = _common_coefficients(s64, s32)
    return {
        "expectation_f64": e64, "expectation_f32": e32,
        "abs_error": abs(e32 - e64), "rel_error": abs(e32 - e64) / abs(e64),
        "terms_f64": len(s64[2]), "terms_f32": len(s32[2]), "common_terms": len(c64),
        "max_coeff_abs_error": float(np.max(np.abs(c32 - c64))) if len(c64) else 0.0,
        "max_abs_coeff_f64": float(np.max(np.abs(s64[2]))),
    }, circ, obs, s64


def test_precision_form_f32_against_f64_on_the_noisy_tfim():
    rep, circ, obs, s64 = precision_report()
    print("precision report:", rep)
    # the f64 run is the oracle's, bit for bit
    W = ps.width_for(36)
    x = np.array([ps.parse_label(k, W)[0] for k in obs], np.uint64).reshape(-1, W)
    z = np.array([ps.parse_label(k, W)[1] for k in obs], np.uint64).reshape(-1, W)
    c = np.array(list(obs.values()), np.float64)
    o = oracle_sum(36, x, z, c)
    o.propagate(oracle_channels(circ), {"keep": [("coeff", 1e-5)]}, "heisenberg")
    assert_same_terms(s64, oracle_arrays(o), what="noisy-f64")
    assert rep["rel_error"] <= PRECISION_EXPECTATION_REL
    assert rep["max_coeff_abs_error"] <= PRECISION_COEFF_REL_TO_MAX * rep["max_abs_coeff_f64"]
    # the two runs keep nearly the same strings: only terms whose |c| sits at the cut can differ
    assert rep["common_terms"] >= 0.999 * max(rep["terms_f64"], rep["terms_f32"])
