"""What the trained scorer gains over plain TopN at the same term budget.

A 4 x 4 periodic transverse-field Ising quench (J = 1, dt = 0.05, 10 Trotter steps, observable
(1/16) sum X_i, readout in |0...0>, Heisenberg picture, f32 coefficients for the truncated
runs) — the 8 x 8 learned-truncation configuration shrunk to what a test can afford.  The scorer
is trained on attribution data the engine generates from tight-threshold (1e-6) runs at
h in {0.75, 1.5, 2.5} and compared with plain coefficient-magnitude TopN at budgets of 2^7,
2^9 and 2^11 terms, by |<O> - <O>_ref| at h in {0.5, 1, 2, 3}, the reference being the
threshold-1e-6 run in f64.  Plain TopN is the yardstick: the test asserts the scored policy's
summed error is below plain TopN's.
"""

from __future__ import annotations

import numpy as np
import pytest

import paulistrings_b200 as ps
from paulistrings_b200 import learned, truncation, workloads

pytestmark = pytest.mark.gpu

L_SIDE, STEPS, DT, THRESHOLD = 4, 10, 0.05, 1e-6


def step(h):
    return workloads.tfim_2d(L_SIDE, 1, J=1.0, h=h, dt=DT)


def readout(h, policy, dtype):
    nq = L_SIDE * L_SIDE
    g = ps.PauliSum.from_strings(workloads.tfim_magnetization(L_SIDE, "X"), num_qubits=nq, dtype=dtype).to_device(0)
    circ = ps.Circuit(nq)
    for _ in range(STEPS):
        circ.extend(step(h))
    g.propagate(circ, policy, "heisenberg")
    v = g.expectation("0" * nq)
    g.close()
    return v


def test_trained_scorer_beats_plain_topn_at_equal_budgets():
    nq = L_SIDE * L_SIDE
    obs = ps.PauliSum.from_strings(workloads.tfim_magnetization(L_SIDE, "X"), num_qubits=nq)
    rows = [[], [], [], []]
    for h in (0.75, 1.5, 2.5):
        data = learned.attribution_data(obs, step(h), STEPS, "0" * nq, THRESHOLD, samples_per_step=1024,
                                        seed=int(h * 100), chunk=128, floor=1e-8, top_fraction=0.75, top_pool=8192)
        for r, a in zip(rows, data):
            r.append(a)
    keys, logc, rem, target = (np.concatenate(r) for r in rows)
    sc = learned.Scorer(nq, layers_per_unit=len(step(1.0)), feature_scale=(0.1, 0.1, 0.1), seed=5, residual=True)
    losses = sc.train(keys, logc, rem, target - logc, epochs=40, batch=1024, lr=1e-3)
    assert losses[-1] < 0.5 * losses[1]
    plain = scored = 0.0
    report = []
    for h in (0.5, 1.0, 2.0, 3.0):
        ref = readout(h, truncation.coeff(THRESHOLD), "f64")
        for budget in (1 << 7, 1 << 9, 1 << 11):
            ep = abs(readout(h, truncation.topn(budget), "f32") - ref)
            es = abs(readout(h, truncation.scored_topn(budget, sc), "f32") - ref)
            plain += ep
            scored += es
            report.append((h, budget, round(ep, 4), round(es, 4)))
    print("h, budget, |err| plain TopN, |err| scored TopN:", report)
    print(f"summed error: plain {plain:.4f}, scored {scored:.4f}")
    assert scored < plain
