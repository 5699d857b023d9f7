"""Learned truncation: a scorer network ranks terms for ``truncation.scored_topn``.

The scorer is a small MLP (``ps_scorer`` in the C ABI) that predicts, from a term's
per-qubit I/X/Y/Z code, its Pauli weight, ``log|c|`` and the remaining circuit depth, the log
magnitude its descendants contribute to the final expectation.  It plugs in where the
reference's ``TruncationPolicy`` trait takes a layer pass (crates/paulistrings/src/truncation/
mod.rs:30-107); the reference has no built-in learned policy.  Inference runs on the device
inside the truncation pass (tensor cores for the 128 x 128 layer); training runs on the device
with the library's own forward, backward and Adam kernels.

Training data comes from the engine itself (``attribution_data``): at each Trotter-step
boundary of a tight-threshold run, a sample of the terms is tagged with distinct Z strings on
extra qubits that no gate touches, propagated together through the remaining steps under the
same threshold, and read out per tag, which gives each sampled term's own contribution
``c * <psi| U_rest^dagger P U_rest |psi>`` (descendants of different terms never merge, since
their tags differ).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np

from . import _lib
from .circuit import Circuit
from .sum import GpuPauliSum, PauliSum, product_basis, width_for

HIDDEN = 128


def layout(num_qubits: int) -> dict:
    """Slices of the flat parameter vector (the order ``ps_scorer_get_params`` uses)."""
    sizes = [("embed", num_qubits * 3 * HIDDEN), ("u", 3 * HIDDEN), ("b1", HIDDEN), ("w2", HIDDEN * HIDDEN),
             ("b2", HIDDEN), ("w3", HIDDEN), ("b3", 1)]
    out, off = {}, 0
    for name, n in sizes:
        out[name] = slice(off, off + n)
        off += n
    out["total"] = off
    return out


def pack_keys(x: np.ndarray, z: np.ndarray) -> np.ndarray:
    """Rows (x words, z words) as the store and the scorer read them."""
    x = np.asarray(x, np.uint64)
    z = np.asarray(z, np.uint64)
    return np.ascontiguousarray(np.concatenate([x.reshape(len(x), -1), z.reshape(len(z), -1)], axis=1))


class Scorer:
    """A scorer network on one device."""

    def __init__(self, num_qubits: int, layers_per_unit: float, feature_scale=(0.1, 0.1, 0.1),
                 init_scale: float = 0.05, seed: int = 1, device: int = 0, residual: bool = False):
        """``residual``: scores are ``log|c|`` + the network's output, the network predicting the
        log of the descendants' factor (train it with ``target - logc``)."""
        cfg = _lib.ScorerConfig()
        cfg.num_qubits = int(num_qubits)
        cfg.residual = 1 if residual else 0
        cfg.layers_per_unit = float(layers_per_unit)
        for i, v in enumerate(feature_scale):
            cfg.feature_scale[i] = float(v)
        cfg.init_scale = float(init_scale)
        cfg.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        h = ctypes.c_void_p()
        st = _lib.lib().ps_scorer_create(int(device), ctypes.byref(cfg), ctypes.byref(h))
        _lib.check(st, None, "scorer_create")
        self._h = h
        self.num_qubits = int(num_qubits)
        self.W = width_for(self.num_qubits)
        self.layers_per_unit = float(layers_per_unit)
        self.feature_scale = tuple(float(v) for v in feature_scale)
        self.layout = layout(self.num_qubits)
        self.residual = bool(residual)
        self.num_sites, self.key_W = self.num_qubits, self.W

    def close(self) -> None:
        if getattr(self, "_h", None):
            _lib.lib().ps_scorer_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st, what):
        if st != _lib.PS_OK:
            msg = _lib.lib().ps_scorer_last_error(self._h)
            _lib.check(st, None, f"{what}: {msg.decode() if msg else ''}")

    @property
    def num_params(self) -> int:
        return int(_lib.lib().ps_scorer_num_params(self._h))

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        self._check(_lib.lib().ps_scorer_get_params(self._h, out.ctypes.data), "get_params")
        return out

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, np.float32)
        if p.shape != (self.num_params,):
            raise ValueError(f"expected {self.num_params} parameters")
        self._check(_lib.lib().ps_scorer_set_params(self._h, p.ctypes.data), "set_params")

    def _arrays(self, keys, logc, rem, target=None, key_W=None):
        keys = np.ascontiguousarray(keys, np.uint64).reshape(-1, 2 * (key_W or self.W))
        n = keys.shape[0]
        logc = np.ascontiguousarray(np.broadcast_to(np.asarray(logc, np.float32), (n,)))
        rem = np.ascontiguousarray(np.broadcast_to(np.asarray(rem, np.float32), (n,)))
        t = None if target is None else np.ascontiguousarray(target, np.float32).reshape(n)
        return keys, logc, rem, t, n

    def score(self, keys, logc, rem) -> np.ndarray:
        """Scores of terms of ``self.num_sites`` qubits (the site map's, if one is set)."""
        keys, logc, rem, _, n = self._arrays(keys, logc, rem, key_W=self.key_W)
        out = np.zeros(n, np.float32)
        self._check(_lib.lib().ps_scorer_score(self._h, keys.ctypes.data, logc.ctypes.data, rem.ctypes.data, n,
                                               out.ctypes.data), "score")
        return out

    def set_site_map(self, row_of_site=None) -> None:
        """Score sums of ``len(row_of_site)`` qubits: site q adds embedding row ``row_of_site[q]``
        (-1: not an input).  ``None`` restores the identity.  Train before mapping."""
        if row_of_site is None:
            self._check(_lib.lib().ps_scorer_set_site_map(self._h, 0, None), "set_site_map")
            self.num_sites, self.key_W = self.num_qubits, self.W
            return
        rows = np.ascontiguousarray(row_of_site, np.int32)
        self._check(_lib.lib().ps_scorer_set_site_map(self._h, len(rows), rows.ctypes.data), "set_site_map")
        self.num_sites, self.key_W = len(rows), width_for(len(rows))

    def gradients(self, keys, logc, rem, target):
        """Gradients of mean((y - target)^2) over one batch (no update), and that loss."""
        keys, logc, rem, t, n = self._arrays(keys, logc, rem, target)
        grads = np.zeros(self.num_params, np.float32)
        loss = ctypes.c_float()
        self._check(_lib.lib().ps_scorer_gradients(self._h, keys.ctypes.data, logc.ctypes.data, rem.ctypes.data,
                                                   t.ctypes.data, n, grads.ctypes.data, ctypes.byref(loss)),
                    "gradients")
        return grads, float(loss.value)

    def train(self, keys, logc, rem, target, epochs: int = 10, batch: int = 4096, lr: float = 1e-3) -> np.ndarray:
        keys, logc, rem, t, n = self._arrays(keys, logc, rem, target)
        losses = np.zeros(int(epochs), np.float32)
        self._check(_lib.lib().ps_scorer_train(self._h, keys.ctypes.data, logc.ctypes.data, rem.ctypes.data,
                                               t.ctypes.data, n, int(epochs), int(batch), float(lr),
                                               losses.ctypes.data), "train")
        return losses


# ---------------------------------------------------------------------------
# attribution data from the engine
# ---------------------------------------------------------------------------

def widened(circuit: Circuit, num_qubits: int) -> Circuit:
    """The same channels on a register of ``num_qubits`` (extra qubits untouched)."""
    out = Circuit(num_qubits)
    for ch in circuit:
        out.append(ch)
    return out


def tagged_contributions(terms_x, terms_z, terms_c, num_qubits: int, rest: Circuit, policy, state: str,
                         direction: str = "heisenberg", device: int = 0) -> np.ndarray:
    """Each term's own contribution to ``<state| (rest applied) |state>``: the terms carry
    distinct Z tags on ``ceil(log2 n)`` extra qubits, run through ``rest`` together, and the
    final sum is read out per tag."""
    n = len(terms_c)
    tag_bits = max(1, int(math.ceil(math.log2(max(n, 2)))))
    nq2 = num_qubits + tag_bits
    W, W2 = width_for(num_qubits), width_for(nq2)
    x = np.zeros((n, W2), np.uint64)
    z = np.zeros((n, W2), np.uint64)
    x[:, :W] = np.asarray(terms_x, np.uint64).reshape(n, W)
    z[:, :W] = np.asarray(terms_z, np.uint64).reshape(n, W)
    idx = np.arange(n, dtype=np.uint64)
    for b in range(tag_bits):
        q = num_qubits + b
        bit = ((idx >> np.uint64(b)) & np.uint64(1)) << np.uint64(q % 64)
        z[:, q // 64] |= bit
    g = GpuPauliSum(nq2, "f64", device)
    try:
        g.upload(x, z, np.asarray(terms_c, np.float64))
        g.propagate(widened(rest, nq2), policy, direction)
        fx, fz, fc = g.download()
    finally:
        g.close()
    if len(state) != num_qubits:  # a uniform label: x+, y+ or z+ on every system qubit
        state = {"x+": "+", "y+": "r", "z+": "0"}[state.lower()] * num_qubits
    ax, az, neg = product_basis(state + "0" * tag_bits, nq2, W2)  # tags are Z: +1 in |0>
    sup = fx | fz
    mismatch = ((fx ^ (sup & ax)) | (fz ^ (sup & az))).any(axis=1)
    parity = np.bitwise_count(sup & neg[None, :]).sum(axis=1) & 1
    val = np.where(parity.astype(bool), -fc, fc)
    val[mismatch] = 0.0
    tag = np.zeros(len(fc), np.int64)
    for b in range(tag_bits):
        q = num_qubits + b
        tag |= (((fz[:, q // 64] >> np.uint64(q % 64)) & np.uint64(1)).astype(np.int64)) << b
    out = np.zeros(n, np.float64)
    np.add.at(out, tag, val)
    return out


def attribution_data(observable: PauliSum, step: Circuit, steps: int, state: str, threshold: float,
                     samples_per_step: int = 4096, seed: int = 0, floor: float = 1e-12, device: int = 0,
                     truncation_policy=None, chunk: int = 256, every: int = 1, top_fraction: float = 0.0,
                     top_pool: int = 0):
    """Training rows from a tight-threshold Heisenberg run of ``steps`` repetitions of ``step``.

    At every step boundary d (0 <= d < steps) up to ``samples_per_step`` terms of the sum are
    drawn (uniformly, without replacement), each one's contribution to the final expectation
    is measured by ``tagged_contributions`` through the remaining ``steps - d`` steps under the
    same threshold, and a row (key, log|c|, remaining steps, log(|contribution| + floor)) is
    recorded.  The tagged runs take ``chunk`` terms at a time (their light cones never merge,
    so a chunk's sum is about ``chunk`` times one cone); ``every`` > 1 samples only every
    ``every``-th boundary.  With ``top_fraction`` > 0 that share of each sample is drawn from
    the ``top_pool`` largest |c| (the region a TopN budget decides on) and the rest uniformly.
    Returns (keys, logc, rem, target) as numpy arrays."""
    from . import truncation

    rng = np.random.default_rng(seed)
    policy = truncation_policy if truncation_policy is not None else truncation.coeff(threshold)
    nq = observable.num_qubits
    g = observable.to_device(device)
    rows = ([], [], [], [])
    try:
        for d in range(steps):
            x, z, c = g.download()
            take = min(samples_per_step, len(c)) if d % every == 0 else 0
            if take:
                n_top = int(round(take * top_fraction))
                if n_top and top_pool:
                    pool = np.argsort(-np.abs(c), kind="stable")[:max(top_pool, n_top)]
                    top = rng.choice(pool, size=min(n_top, len(pool)), replace=False)
                    others = np.setdiff1d(np.arange(len(c)), top)
                    rest_pick = rng.choice(others, size=min(take - len(top), len(others)), replace=False)
                    pick = np.sort(np.concatenate([top, rest_pick]))
                else:
                    pick = np.sort(rng.choice(len(c), size=take, replace=False))
                rest = Circuit(nq)
                for _ in range(steps - d):
                    rest.extend(step)
                contrib = np.concatenate([
                    tagged_contributions(x[pick[i:i + chunk]], z[pick[i:i + chunk]], c[pick[i:i + chunk]], nq, rest,
                                         policy, state, device=device)
                    for i in range(0, take, chunk)])
                rows[0].append(pack_keys(x[pick], z[pick]))
                rows[1].append(np.log(np.abs(c[pick])).astype(np.float32))
                rows[2].append(np.full(take, steps - d, np.float32))
                rows[3].append(np.log(np.abs(contrib) + floor).astype(np.float32))
            g.propagate(step, policy, "heisenberg")
    finally:
        g.close()
    return tuple(np.concatenate(r) for r in rows)


# ---------------------------------------------------------------------------
# Trotter series with a readout after every step, and a scorer trained for a circuit family
# ---------------------------------------------------------------------------

def trotter_series(observable: dict, num_qubits: int, step: Circuit, steps: int, policy, dtype: str, state: str,
                   device: int = 0) -> dict:
    """Heisenberg propagation of ``steps`` repetitions of ``step`` from ``observable``
    ({label: coefficient}), reading <state| O(t) |state> after every step (the reference's quench
    protocol, docs/figures/ising-quench-convergence/quench_convergence.py:85-94).  Returns the
    readouts (t = 0 .. steps), the wall time of the loop (propagation and readouts, the device
    synchronised at both ends), the device time of the propagations, and term counts."""
    import time

    g = PauliSum.from_strings(observable, num_qubits=num_qubits, dtype=dtype).to_device(device)
    layers = len(step)
    values = [g.expectation(state)]
    dev_ms = 0.0
    terms_in = skipped = launches = 0
    peak = len(g)
    _lib.check(_lib.lib().ps_synchronize(g._h), g._h, "synchronize")
    t0 = time.perf_counter()
    for k in range(steps):
        st = g.propagate(step, policy, "heisenberg", with_stats=True, remaining_layers=layers * (steps - k))
        dev_ms += st.device_ms
        terms_in += st.total_terms_in - st.skipped_terms_in
        skipped += st.layers_skipped
        launches += st.kernel_launches
        peak = max(peak, st.peak_terms)
        values.append(g.expectation(state))
    wall = time.perf_counter() - t0
    final = len(g)
    g.close()
    return {"values": values, "wall_s": wall, "device_ms": dev_ms, "terms_in": terms_in, "layers": layers * steps,
            "layers_skipped": skipped, "peak_terms": peak, "final_terms": final, "gpu_launches": launches}


def train_scorer(observable: dict, num_qubits: int, steps_for, h_values, steps: int, state: str, threshold: float,
                 samples_per_step: int = 1024, every: int = 4, chunk: int = 256, epochs: int = 40,
                 batch: int = 1024, lr: float = 1e-3, seed: int = 5, device: int = 0) -> tuple:
    """A residual scorer trained on attribution rows from tight-threshold runs of the circuit
    family ``steps_for(h)`` (one Trotter step) at each training field in ``h_values``.  Returns
    (scorer, per-epoch losses, rows used, seconds spent on data and on training)."""
    import time

    t0 = time.perf_counter()
    obs = PauliSum.from_strings(observable, num_qubits=num_qubits)
    rows = [[], [], [], []]
    for h in h_values:
        data = attribution_data(obs, steps_for(h), steps, state, threshold, samples_per_step=samples_per_step,
                                seed=int(round(h * 1000)), chunk=chunk, floor=1e-10, every=every,
                                top_fraction=0.75, top_pool=1 << 16, device=device)
        for r, a in zip(rows, data):
            r.append(a)
    keys, logc, rem, target = (np.concatenate(r) for r in rows)
    t_data = time.perf_counter() - t0
    sc = Scorer(num_qubits, layers_per_unit=len(steps_for(h_values[0])), feature_scale=(0.1, 0.1, 0.1), seed=seed,
                residual=True, device=device)
    t1 = time.perf_counter()
    losses = sc.train(keys, logc, rem, target - logc, epochs=epochs, batch=batch, lr=lr)
    t_train = time.perf_counter() - t1
    return sc, losses, len(target), t_data, t_train


def _score_benchmark(log2_terms: int = 22, num_qubits: int = 64) -> None:
    """Score 2^log2_terms terms (the 65,536-term random observable of the bench, tiled) with a
    fresh residual scorer through ``ps_scorer_score``: three warm-up calls, then one timed."""
    import time

    from . import workloads

    x, z, c = workloads.random_observable(num_qubits, 1 << 16, seed=3)
    reps = max(1, (1 << log2_terms) // len(c))
    keys = np.tile(pack_keys(x, z), (reps, 1))
    logc = np.tile(np.log(np.abs(c)).astype(np.float32), reps)
    rem = np.full(len(logc), 5.0, np.float32)
    sc = Scorer(num_qubits, layers_per_unit=96, seed=1, residual=True)
    for _ in range(3):
        sc.score(keys, logc, rem)
    t0 = time.perf_counter()
    s = sc.score(keys, logc, rem)
    dt = time.perf_counter() - t0
    print(f"scored {len(s)} terms, finite {bool(np.all(np.isfinite(s)))}, {dt * 1e3:.2f} ms with host copies")


if __name__ == "__main__":
    import sys

    _score_benchmark(int(sys.argv[1]) if len(sys.argv) > 1 else 22)
