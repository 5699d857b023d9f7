"""Learned truncation: the scorer network, its training kernels and the scored TopN pass.

CPU tests pin the numpy restatement of the network (``oracle/scorer_ref.py``) against finite
differences of its own forward pass and against torch's bfloat16 rounding, and check the
policy lowering.  GPU tests compare the device scores and the device gradients (tensor-core
forward and backward) with the restatement, check that the scored pass keeps exactly the
terms the scorer ranks highest, and that training lowers the loss.
"""

from __future__ import annotations

import numpy as np
import pytest

import paulistrings_b200 as ps
from oracle import scorer_ref
from paulistrings_b200 import _lib, learned, truncation, workloads
from paulistrings_b200.circuit import Circuit
from tests._util import oracle_sum


def random_params(nq, seed, scale=0.3):
    rng = np.random.default_rng(seed)
    L = learned.layout(nq)
    p = np.zeros(L["total"], np.float32)
    p[L["embed"]] = rng.normal(scale=scale, size=L["embed"].stop - L["embed"].start)
    p[L["u"]] = rng.normal(scale=scale, size=3 * 128)
    p[L["b1"]] = rng.normal(scale=0.1, size=128)
    p[L["w2"]] = rng.normal(scale=1 / np.sqrt(128), size=128 * 128)
    p[L["b2"]] = rng.normal(scale=0.1, size=128)
    p[L["w3"]] = rng.normal(scale=1 / np.sqrt(128), size=128)
    p[L["b3"]] = 0.3
    return p


def random_rows(nq, n, seed):
    x, z, c = workloads.random_observable(nq, n, seed=seed)
    keys = learned.pack_keys(x, z)
    rng = np.random.default_rng(seed + 1)
    logc = np.log(np.abs(c)).astype(np.float32)
    rem = rng.integers(0, 20, size=n).astype(np.float32)
    target = (rng.normal(size=n) - 3.0).astype(np.float32)
    return keys, logc, rem, target


FSCALE = (0.1, 0.1, 0.1)


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------

def test_bf16_rounding_matches_torch():
    import torch

    a = np.random.default_rng(0).normal(size=4096).astype(np.float32) * 10
    want = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(scorer_ref.bf16(a), want)


def test_reference_gradients_match_finite_differences():
    nq, W = 8, 1
    keys, logc, rem, target = random_rows(nq, 64, seed=3)
    p = random_params(nq, 5)
    # exact-arithmetic variant: no bf16 rounding, float64, so differences are clean
    scorer_ref.EXACT = True
    try:
        p64 = p.astype(np.float64)
        g, _ = scorer_ref.gradients(p64, keys, logc, rem, target, nq, W, FSCALE)

        def loss(q):
            y, _ = scorer_ref.forward(q, keys, logc, rem, nq, W, FSCALE)
            return float(np.mean((y - target) ** 2))

        rng = np.random.default_rng(1)
        L = learned.layout(nq)
        for name in ("embed", "u", "b1", "w2", "b2", "w3", "b3"):
            sl = L[name]
            for i in rng.choice(np.arange(sl.start, sl.stop), size=min(6, sl.stop - sl.start), replace=False):
                h = 1e-6
                q1, q2 = p64.copy(), p64.copy()
                q1[i] += h
                q2[i] -= h
                fd = (loss(q1) - loss(q2)) / (2 * h)
                assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (name, i, fd, g[i])
    finally:
        scorer_ref.EXACT = False


def test_scored_topn_lowering():
    sc = object()
    pol = truncation.coeff(1e-8) & truncation.scored_topn(1000, sc)
    nodes, passes = pol.lowered()
    assert passes == [(_lib.PS_PASS_SCORED_TOPN, 1000, 1, 0, 0)]  # samples = the rescore interval
    assert truncation.scored_topn(64, sc, rescore_every=192).lowered()[1] == [(_lib.PS_PASS_SCORED_TOPN, 64, 192, 0, 0)]
    with pytest.raises(ValueError):
        truncation.scored_topn(64, sc, rescore_every=0)
    assert pol.scorer() is sc
    assert truncation.topn(5).scorer() is None
    with pytest.raises(ValueError):
        truncation.coeff(1e-3) | truncation.scored_topn(10, sc)
    with pytest.raises(ValueError):
        (truncation.scored_topn(10, sc) & truncation.scored_topn(20, object())).scorer()


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------

@pytest.mark.gpu
@pytest.mark.parametrize("nq", [16, 64, 100, 200, 256])
def test_device_scores_match_the_reference(nq):
    W = ps.width_for(nq)
    sc = learned.Scorer(nq, layers_per_unit=10.0, feature_scale=FSCALE, seed=2)
    p = random_params(nq, 7)
    sc.set_params(p)
    assert sc.num_params == learned.layout(nq)["total"]
    assert np.array_equal(sc.get_params(), p)
    keys, logc, rem, _ = random_rows(nq, 1000, seed=11)
    got = sc.score(keys, logc, rem)
    want, _ = scorer_ref.forward(p, keys, logc, rem, nq, W, FSCALE)
    assert np.all(np.isfinite(got))
    np.testing.assert_allclose(got, want, rtol=2e-3, atol=2e-3)


def dense_rows(nq, n, seed):
    """Keys with every qubit drawn uniformly from I/X/Y/Z (weight ~ 3/4 of the register)."""
    rng = np.random.default_rng(seed)
    W = ps.width_for(nq)
    x = rng.integers(0, 1 << 63, size=(n, W), dtype=np.int64).astype(np.uint64) << np.uint64(1)
    z = rng.integers(0, 1 << 63, size=(n, W), dtype=np.int64).astype(np.uint64) << np.uint64(1)
    x |= rng.integers(0, 2, size=(n, W)).astype(np.uint64)
    z |= rng.integers(0, 2, size=(n, W)).astype(np.uint64)
    if nq % 64:
        mask = np.uint64((1 << (nq % 64)) - 1)
        x[:, -1] &= mask
        z[:, -1] &= mask
    keys = learned.pack_keys(x, z)
    logc = rng.normal(-8.0, 3.0, size=n).astype(np.float32)
    rem = rng.integers(0, 50, size=n).astype(np.float32)
    return keys, logc, rem


@pytest.mark.gpu
@pytest.mark.parametrize("nq", [64, 200])
def test_device_scores_of_dense_strings_match_the_reference(nq):
    """Strings with about 3/4 of the qubits non-identity: the one-hot operand's sums (the tensor-core
    path at 64 rows, the embedding bag at 200) add dozens of rows per term."""
    W = ps.width_for(nq)
    sc = learned.Scorer(nq, layers_per_unit=10.0, feature_scale=FSCALE, seed=2)
    p = random_params(nq, 19, scale=0.05)
    sc.set_params(p)
    keys, logc, rem = dense_rows(nq, 2000, seed=31)
    got = sc.score(keys, logc, rem)
    want, _ = scorer_ref.forward(p, keys, logc, rem, nq, W, FSCALE)
    np.testing.assert_allclose(got, want, rtol=2e-3, atol=2e-3)


@pytest.mark.gpu
def test_site_mapped_scorer_scores_a_wider_register_like_the_reference():
    """A 64-row scorer on 256-qubit strings through a window map (sites 96..159 onto rows 0..63,
    the sites beyond clamped to the edge rows, every seventh site ignored): the tensor-core
    one-hot operand carries counts up to dozens per row, and the scores must match the
    restatement with the same map.  Training refuses a mapped scorer."""
    rows, sites = 64, 256
    sc = learned.Scorer(rows, layers_per_unit=10.0, feature_scale=FSCALE, seed=2)
    p = random_params(rows, 23, scale=0.05)
    sc.set_params(p)
    site_row = np.clip(np.arange(sites) - 128 + 32, 0, rows - 1).astype(np.int32)
    site_row[::7] = -1
    sc.set_site_map(site_row)
    for keys, logc, rem in (random_rows(sites, 1000, seed=29)[:3], dense_rows(sites, 1000, seed=37)):
        got = sc.score(keys, logc, rem)
        want, _ = scorer_ref.forward(p, keys, logc, rem, rows, 4, FSCALE, site_row=site_row)
        np.testing.assert_allclose(got, want, rtol=2e-3, atol=2e-3)
    k64, l64, r64, t64 = random_rows(rows, 256, seed=41)
    with pytest.raises(Exception):
        sc.train(k64, l64, r64, t64, epochs=1, batch=128)
    sc.set_site_map(None)
    sc.train(k64, l64, r64, t64, epochs=1, batch=128)


@pytest.mark.gpu
@pytest.mark.parametrize("nq,n", [(16, 128), (64, 1000), (100, 777)])
def test_device_gradients_match_the_reference(nq, n):
    W = ps.width_for(nq)
    sc = learned.Scorer(nq, layers_per_unit=10.0, feature_scale=FSCALE, seed=2)
    p = random_params(nq, 9)
    sc.set_params(p)
    keys, logc, rem, target = random_rows(nq, n, seed=13)
    g, loss = sc.gradients(keys, logc, rem, target)
    gw, lw = scorer_ref.gradients(p, keys, logc, rem, target, nq, W, FSCALE)
    assert abs(loss - lw) <= 1e-3 * abs(lw) + 1e-5
    L = learned.layout(nq)
    for name in ("embed", "u", "b1", "w2", "b2", "w3", "b3"):
        a, b = g[L[name]], gw[L[name]]
        err = np.linalg.norm(a - b)
        assert err <= 2e-2 * np.linalg.norm(b) + 1e-6, (name, err, np.linalg.norm(b))


@pytest.mark.gpu
def test_training_lowers_the_loss():
    nq = 16
    keys, logc, rem, _ = random_rows(nq, 8192, seed=21)
    # a learnable target: depends on the weight, the coefficient and the remaining depth
    p = scorer_ref.support(keys, nq, 1)
    weight = (p != 0).sum(axis=1)
    target = (0.8 * logc - 0.3 * weight - 0.05 * rem).astype(np.float32)
    sc = learned.Scorer(nq, layers_per_unit=1.0, feature_scale=FSCALE, seed=4)
    losses = sc.train(keys, logc, rem, target, epochs=15, batch=1024, lr=2e-3)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < 0.1 * losses[0], losses


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_scored_pass_keeps_the_highest_scored_terms(dtype):
    nq = 64
    sc = learned.Scorer(nq, layers_per_unit=1.0, feature_scale=FSCALE, seed=6)
    sc.set_params(random_params(nq, 17))
    x, z, c = workloads.random_observable(nq, 20000, seed=3)
    circ = Circuit(nq)
    circ.pauli_rotation("XY", [3, 17], 0.7)
    full = ps.GpuPauliSum(nq, dtype)
    full.upload(x, z, c)
    full.propagate(circ, None, "forward")
    fx, fz, fc = full.download()
    keep = 9000
    g = ps.GpuPauliSum(nq, dtype)
    g.upload(x, z, c)
    st = g.propagate(circ, truncation.scored_topn(keep, sc), "forward", with_stats=True)
    kx, kz, kc = g.download()
    assert len(kc) == keep and st.final_terms == keep
    scores = sc.score(learned.pack_keys(fx, fz), np.log(np.abs(fc)).astype(np.float32), 0.0)
    order = np.argsort(-scores, kind="stable")
    chosen = np.sort(order[:keep])
    kept = {(a.tobytes(), b.tobytes()) for a, b in zip(kx, kz)}
    want = {(fx[i].tobytes(), fz[i].tobytes()) for i in chosen}
    # the device scores f64 coefficients' log in float64 before rounding; allow a sliver of
    # boundary disagreement from that
    assert len(kept ^ want) <= 4
    assert np.array_equal(kc, fc[np.isin(np.arange(len(fc)), chosen)]) or len(kept ^ want) > 0


# ---------------------------------------------------------------------------
# inherited scores (scored_topn with rescore_every > 1)
# ---------------------------------------------------------------------------

def _rotation_circuit(nq, gates, seed):
    rng = np.random.default_rng(seed)
    circ = Circuit(nq)
    for _ in range(gates):
        a, b = (int(q) for q in rng.choice(nq, size=2, replace=False))
        circ.pauli_rotation("".join(rng.choice(list("XYZ"), size=2)), [a, b], float(rng.uniform(0.3, 1.2)))
    return circ


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_inherited_scores_of_a_constant_network_rank_by_magnitude(dtype):
    """A network whose output is a constant makes log|c| + f a monotone function of |c|: the
    inherited pass (predictions carried by the merge, partners inheriting, the select on
    log|c| + f) must keep what plain TopN keeps, up to |c| values that tie in f32's log."""
    nq, keep = 64, 6000
    sc = learned.Scorer(nq, layers_per_unit=4.0, feature_scale=FSCALE, seed=6, residual=True)
    p = np.zeros(learned.layout(nq)["total"], np.float32)
    p[learned.layout(nq)["b3"]] = 0.5
    sc.set_params(p)
    x, z, c = workloads.random_observable(nq, 4000, seed=8)
    circ = _rotation_circuit(nq, 6, seed=3)
    a = ps.GpuPauliSum(nq, dtype)
    a.upload(x, z, c)
    sa = a.propagate(circ, truncation.scored_topn(keep, sc, rescore_every=4), "forward", with_stats=True)
    b = ps.GpuPauliSum(nq, dtype)
    b.upload(x, z, c)
    sb = b.propagate(circ, truncation.topn(keep), "forward", with_stats=True)
    assert sa.terms_after == sb.terms_after
    ka, kb = a.download(), b.download()
    got = {(u.tobytes(), v.tobytes()) for u, v in zip(ka[0], ka[1])}
    want = {(u.tobytes(), v.tobytes()) for u, v in zip(kb[0], kb[1])}
    assert len(got ^ want) <= 8, len(got ^ want)


def _host_layer(nq, dtype, keys, coefs, channel):
    """One layer through the oracle, no truncation: (keys, coefficients)."""
    W = ps.width_for(nq)
    o = oracle_sum(nq, keys[:, :W], keys[:, W:], coefs, dtype)
    o.apply(("rotation", channel.paulis, list(channel.qubits), channel.theta), adjoint=False, policy=None)
    return o.get()


@pytest.mark.gpu
def test_inherited_scores_follow_their_rows():
    """Three layers, rescored every third: layer 1 scores every row afresh, layers 2 and 3 rank by
    log|c| + the carried prediction (an own row keeps its string's, a new partner takes its
    parent's).  A host restatement (oracle layers, the device scorer's predictions at the
    rescoring, the inheritance rule) must keep nearly the same rows (predictions recovered from
    the device's scores can differ from the carried ones in the last bit)."""
    nq, keep = 40, 1500
    W = ps.width_for(nq)
    sc = learned.Scorer(nq, layers_per_unit=3.0, feature_scale=FSCALE, seed=6, residual=True)
    sc.set_params(random_params(nq, 29, scale=0.3))
    x, z, c = workloads.random_observable(nq, 1200, seed=12)
    circ = _rotation_circuit(nq, 3, seed=5)
    chans = list(circ)
    g = ps.GpuPauliSum(nq, "f64")
    g.upload(x, z, c)
    g.propagate(circ, truncation.scored_topn(keep, sc, rescore_every=3), "forward", remaining_layers=3)
    gx, gz, gc = g.download()

    keys = np.concatenate([x, z], axis=1).astype(np.uint64)
    coefs = c.astype(np.float64)
    order = np.lexsort(keys.T[::-1])
    keys, coefs = keys[order], coefs[order]
    f = None
    for li, ch in enumerate(chans):
        out_k, out_c = _host_layer(nq, "f64", keys, coefs, ch)
        logc = np.maximum(np.log(np.abs(out_c)).astype(np.float32), np.float32(-200.0))
        rem = np.float32((3 - (li + 1)) / 3.0)
        if li == 0:
            y = sc.score(out_k, logc, rem)
            new_f = (y - logc).astype(np.float32)
        else:
            gx_, gz_ = (np.zeros(W, np.uint64) for _ in range(2))
            for q, pch in zip(ch.qubits, ch.paulis):
                if pch in "XY":
                    gx_[q // 64] |= np.uint64(1 << (q % 64))
                if pch in "ZY":
                    gz_[q // 64] |= np.uint64(1 << (q % 64))
            prev = {kk.tobytes(): ff for kk, ff in zip(keys, f)}
            gen = np.concatenate([gx_, gz_])
            new_f = np.array([prev.get(kk.tobytes(), prev.get((kk ^ gen).tobytes())) for kk in out_k], np.float32)
            y = (logc + new_f).astype(np.float32)
        top = np.sort(np.argsort(-y, kind="stable")[:keep])
        keys, coefs, f = out_k[top], out_c[top], new_f[top]
    got = {(u.tobytes(), v.tobytes()) for u, v in zip(gx, gz)}
    want = {(kk[:W].tobytes(), kk[W:].tobytes()) for kk in keys}
    assert len(got) == keep
    assert len(got ^ want) <= 0.01 * keep, len(got ^ want)
