"""Parity of the device layer path against the CPU oracle (needs a CUDA device).

Rotation and depolarizing layers sum at most two contributions per key, so with products
and sums rounded once on both sides the surviving strings AND their coefficients are
bit-exact; the tests assert exactly that.  Expectation values are float64 sums in a
different order, compared at 1e-12 relative.  TopN boundary ties are kept first in key
order on both sides, so truncated runs are bit-exact too.
"""

import math

import numpy as np
import pytest

import paulistrings_b200 as ps
from paulistrings_b200 import truncation, workloads
from tests._util import (
    assert_same_terms,
    circuit_from_gates,
    load_golden,
    oracle_arrays,
    oracle_channels,
    oracle_policy,
    oracle_sum,
)

pytestmark = pytest.mark.gpu


def run_both(num_qubits, x, z, c, circuit, policy=None, direction="forward", dtype="f64"):
    """(device arrays, oracle arrays, device per-layer lengths, oracle per-layer lengths)."""
    g = ps.GpuPauliSum(num_qubits, dtype)
    g.upload(x, z, c)
    st = g.propagate(circuit, policy, direction, with_stats=True)
    got = g.download()
    o = oracle_sum(num_qubits, x, z, c, dtype)
    after = o.propagate(oracle_channels(circuit), oracle_policy(policy), direction)
    return got, oracle_arrays(o), st.terms_after, [int(v) for v in after], g, o


def labels_to_arrays(terms, n):
    W = ps.width_for(n)
    xs, zs, cs = [], [], []
    for lab, v in terms.items():
        x, z = ps.parse_label(lab, W)
        xs.append(x)
        zs.append(z)
        cs.append(v)
    return np.array(xs, np.uint64).reshape(-1, W), np.array(zs, np.uint64).reshape(-1, W), np.array(cs, np.float64)


def test_device_is_visible_and_library_loaded():
    assert ps.cuda_available()
    assert ps.device_count() >= 1


# --- hand-computed identities (python/paulistrings/tests/test_pauli_rotation.py:62-137) -------------


def test_rz_on_x_is_cos_x_plus_sin_y():
    theta = 0.6
    s = ps.PauliSum.from_strings({"X": 1.0}, num_qubits=1)
    c = ps.Circuit(1)
    c.append(ps.gates.pauli_rotation("Z", [0], theta))
    out = ps.propagated(s, circuit=c, direction="forward").to_dict()
    assert out == {"X": math.cos(theta), "Y": math.sin(theta)}


def test_zz_on_xi_is_cos_xi_plus_sin_yz():
    theta = 0.6
    s = ps.PauliSum.from_strings({"XI": 1.0}, num_qubits=2)
    c = ps.Circuit(2)
    c.pauli_rotation("ZZ", [0, 1], theta)
    assert ps.propagated(s, c).to_dict() == {"XI": math.cos(theta), "YZ": math.sin(theta)}


def test_clifford_point_moves_instead_of_splitting():
    s = ps.PauliSum.from_strings({"XI": 1.0}, num_qubits=2)
    c = ps.Circuit(2)
    c.pauli_rotation("ZZ", [0, 1], -math.pi / 2)
    assert ps.propagated(s, c).to_dict() == {"YZ": -1.0}


def test_rz_matches_weight_one_pauli_rotation():
    s = ps.PauliSum.from_strings({"XIZ": 1.0, "ZYI": 0.25}, num_qubits=3)
    a, b = ps.Circuit(3), ps.Circuit(3)
    a.pauli_rotation("Z", [0], -0.37)
    b.rz(-0.37, 0)
    assert ps.propagated(s, a).to_dict() == ps.propagated(s, b).to_dict()


def test_heisenberg_round_trip_is_identity():
    c = ps.Circuit(3)
    c.pauli_rotation("XY", [0, 2], 0.3)
    c.rz(1.1, 1)
    c.pauli_rotation("YYZ", [0, 1, 2], -0.7)
    s = ps.PauliSum.from_strings({"XZY": 0.5}, num_qubits=3)
    s.propagate(c, direction="forward")
    s.propagate(c, direction="heisenberg")
    d = s.to_dict()
    assert d["XZY"] == pytest.approx(0.5, abs=1e-15)
    assert all(abs(v) < 1e-15 for k, v in d.items() if k != "XZY")


# --- golden fixtures from the reference ------------------------------------------------------------

XXZ = load_golden("xxz_statevector.json")["cases"]


@pytest.mark.parametrize("case", [c for c in XXZ if c["final_terms"] <= 200_000],
                         ids=lambda c: f"n{c['n']}-Jz{c['Jz']}-s{c['steps']}-o{len(c['observable_z'])}")
def test_xxz_statevector_fixture_bit_exact(case):
    n = case["n"]
    lab = ["I"] * n
    for q in case["observable_z"]:
        lab[q] = "Z"
    x, z, c = labels_to_arrays({"".join(lab): 1.0}, n)
    circ = circuit_from_gates(n, case["gates"])
    pol = truncation.coeff(case["epsilon"])
    got, want, la, lb, g, _ = run_both(n, x, z, c, circ, pol, "heisenberg")
    assert la == lb
    assert_same_terms(got, want, what="xxz")
    assert len(got[2]) == case["final_terms"]
    assert abs(g.expectation(case["state"]) - case["expectation"]) <= 1e-14


JL = load_golden("jl_parity.json")["workloads"]


@pytest.mark.parametrize(
    "key,point",
    [(k, p) for k, w in JL.items() for p in w["points"] if p["final_terms"] <= 80_000],
    ids=lambda v: v if isinstance(v, str) else f"eps{v['epsilon']:.3g}-w{v['max_weight']}",
)
def test_jl_parity_fixture_bit_exact(key, point):
    w = JL[key]
    n = w["n_qubits"]
    lab = ["I"] * n
    for q in w["observable_z"]:
        lab[q] = "Z"
    x, z, c = labels_to_arrays({"".join(lab): 1.0}, n)
    pol = truncation.coeff(point["epsilon"])
    if point["max_weight"] is not None:
        pol = truncation.weight(point["max_weight"]) & pol
    got, want, la, lb, g, _ = run_both(n, x, z, c, circuit_from_gates(n, w["gates"]), pol, "heisenberg")
    assert la == lb
    assert_same_terms(got, want, what=key)
    assert len(got[2]) == point["final_terms"]
    if point["expectation"] is not None:
        assert abs(g.expectation(w["state"]) - point["expectation"]) <= 1e-13


# --- the measured configurations at oracle-sized scales ---------------------------------------------


def test_tfim_6x6_threshold_per_layer_counts_and_bit_exact():
    circ = workloads.tfim_2d(6, 5, J=1.0, h=1.0, dt=0.1)
    x, z, c = labels_to_arrays(workloads.tfim_magnetization(6, "X"), 36)
    got, want, la, lb, g, o = run_both(36, x, z, c, circ, truncation.coeff(1e-5), "heisenberg")
    assert la == lb
    assert_same_terms(got, want, what="tfim6")
    assert g.expectation("z+") == pytest.approx(o.expectation("z+"), rel=1e-12, abs=1e-15)


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_noisy_tfim_bit_exact_per_dtype(dtype):
    circ = workloads.tfim_2d(6, 2, J=1.0, h=1.0, dt=0.1, noise_p=1e-3)
    x, z, c = labels_to_arrays(workloads.tfim_magnetization(6, "X"), 36)
    got, want, la, lb, g, o = run_both(36, x, z, c, circ, truncation.coeff(1e-5), "heisenberg", dtype)
    assert la == lb
    assert_same_terms(got, want, what=f"noisy-{dtype}")
    assert g.expectation("z+") == pytest.approx(o.expectation("z+"), rel=1e-12, abs=1e-15)


def test_random_pair_layers_with_topn_and_threshold_bit_exact():
    circ = workloads.random_pair_layers(16, 2)
    x, z, c = workloads.random_observable(16, 400)
    pol = truncation.topn(3000) & truncation.coeff(1e-10)
    got, want, la, lb, _, _ = run_both(16, x, z, c, circ, pol, "heisenberg")
    assert la == lb
    assert max(la) == 3000
    assert_same_terms(got, want, what="pairs-topn")


def test_config1_shape_first_layers_no_truncation_bit_exact():
    full = workloads.random_pair_layers(64, 1)
    circ = ps.Circuit(64)
    for ch in list(full)[:10]:
        circ.append(ch)
    x, z, c = workloads.random_observable(64, 65536)
    got, want, la, lb, _, _ = run_both(64, x, z, c, circ, truncation.coeff(1e-10), "heisenberg")
    assert la == lb
    assert_same_terms(got, want, what="config1-prefix")


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_wide_rotations_and_word_boundaries_bit_exact(seed):
    rng = np.random.default_rng(seed)
    for n in (10, 100, 200):
        circ = ps.Circuit(n)
        for _ in range(12):
            w = int(rng.integers(1, 7))
            qs = [int(q) for q in rng.choice(n, size=w, replace=False)]
            circ.pauli_rotation("".join(rng.choice(list("XYZ"), size=w)), qs, float(rng.uniform(-3.2, 3.2)))
        x, z, c = workloads.random_observable(n, 300, seed=seed)
        got, want, la, lb, _, _ = run_both(n, x, z, c, circ, truncation.coeff(1e-9), "forward")
        assert la == lb
        assert_same_terms(got, want, what=f"wide-{n}")


def test_weight_and_or_keep_programs_bit_exact():
    circ = workloads.random_pair_layers(12, 1)
    x, z, c = workloads.random_observable(12, 200)
    pol = truncation.weight(3) | truncation.coeff(0.05)
    got, want, la, lb, _, _ = run_both(12, x, z, c, circ, pol, "forward")
    assert la == lb
    assert_same_terms(got, want, what="or-program")


# --- ingest, edge cases, errors ----------------------------------------------------------------------


def test_upload_sums_duplicates_in_order_and_drops_zeros():
    W = 1
    x = np.array([[1], [2], [1], [3], [3]], np.uint64)
    z = np.array([[0], [2], [0], [1], [1]], np.uint64)
    c = np.array([0.1, 0.5, 0.2, 0.25, -0.25])
    s = ps.PauliSum.from_arrays(x, z, c, num_qubits=2)
    assert s.x_array().tolist() == [[1], [2]]
    assert s.z_array().tolist() == [[0], [2]]
    assert s.coefficients_array().tolist() == [0.1 + 0.2, 0.5]
    o = oracle_sum(2, x, z, c)
    assert_same_terms((s.x_array(), s.z_array(), s.coefficients_array()), oracle_arrays(o), what="ingest")


def test_upload_rejects_bits_beyond_num_qubits():
    g = ps.GpuPauliSum(3)
    with pytest.raises(ValueError):
        g.upload(np.array([[8]], np.uint64), np.array([[0]], np.uint64), np.array([1.0]))


def test_empty_sum_and_identity_layers():
    g = ps.GpuPauliSum(4)
    g.upload(np.zeros((0, 1), np.uint64), np.zeros((0, 1), np.uint64), np.zeros(0))
    c = ps.Circuit(4)
    c.pauli_rotation("XY", [0, 1], 0.3)
    g.propagate(c)
    assert len(g) == 0
    s = ps.PauliSum.from_strings({"XIII": 1.0, "IZII": -2.0}, num_qubits=4)
    c = ps.Circuit(4)
    c.pauli_rotation("ZZ", [2, 3], 0.0)
    c.pauli_rotation("ZZ", [0, 1], math.pi)
    out = ps.propagated(s, c).to_dict()
    assert out == {"XIII": -1.0, "IZII": -2.0}


def test_layer_api_matches_propagate():
    circ = workloads.random_pair_layers(10, 1)
    x, z, c = workloads.random_observable(10, 100)
    g1 = ps.GpuPauliSum(10)
    g1.upload(x, z, c)
    for ch in circ:
        g1.apply_layer(ch, truncation.coeff(1e-6))
    g2 = ps.GpuPauliSum(10)
    g2.upload(x, z, c)
    g2.propagate(circ, truncation.coeff(1e-6))
    assert_same_terms(g1.download(), g2.download(), what="layer-api")


def test_invalid_channel_leaves_store_untouched():
    s = ps.PauliSum.from_strings({"XI": 1.0}, num_qubits=2)
    g = s.to_device()
    c = ps.Circuit(2)
    c.pauli_rotation("ZZ", [0, 1], 0.1)
    c._channels.append(ps.PauliRotation("Z", (5,), 0.1))
    with pytest.raises(ValueError):
        g.propagate(c)
    assert g.download()[2].tolist() == [1.0]


# --- full-size properties (no oracle) ---------------------------------------------------------------


def test_large_rotation_layers_preserve_norm_and_order():
    x, z, c = workloads.random_observable(64, 1 << 16)
    g = ps.GpuPauliSum(64)
    g.upload(x, z, c)
    circ = workloads.random_pair_layers(64, 1)
    g.propagate(circ, None, "heisenberg")
    gx, gz, gc = g.download()
    assert len(gc) > 1_000_000
    keys = np.concatenate([gx, gz], axis=1)
    # strictly increasing in (x, z) lexicographic order: sorted and unique
    lex = np.lexsort(keys.T[::-1])
    assert np.array_equal(lex, np.arange(len(gc)))
    diff = np.any(keys[1:] != keys[:-1], axis=1)
    assert diff.all()
    # orthogonal layers preserve the 2-norm (no truncation)
    assert np.sum(gc * gc) == pytest.approx(1.0, rel=1e-12)


def test_topn_nan_and_boundary_ties_match_the_oracle():
    labels = ["XI", "YI", "ZI", "IX", "IY", "IZ"]
    x, z, c = labels_to_arrays(dict(zip(labels, [0.5, -0.5, 0.1, 0.5, 0.9, float("nan")])), 2)
    circ = ps.Circuit(2)
    circ.rz(0.0, 0)
    for n_keep in (0, 1, 2, 3, 4, 5, 6, 7):
        got, want, la, lb, _, _ = run_both(2, x, z, c, circ, truncation.topn(n_keep))
        assert la == lb, n_keep
        assert_same_terms(got, want, what=f"topn{n_keep}")


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_topn_many_ties_bit_exact(dtype):
    # coefficients from a small set of values, so whole blocks tie at the boundary
    rng = np.random.default_rng(7)
    x, z, _ = workloads.random_observable(20, 5000, seed=11)
    c = rng.choice([0.25, -0.25, 0.5, 0.125, -0.0625], size=len(x))
    circ = workloads.random_pair_layers(20, 1)
    pol = truncation.topn(2500) & truncation.coeff(1e-12)
    got, want, la, lb, _, _ = run_both(20, x, z, c, circ, pol, "heisenberg", dtype)
    assert la == lb
    assert_same_terms(got, want, what=f"ties-{dtype}")


def test_upload_fast_path_and_fallback_agree():
    x, z, c = workloads.random_observable(64, 20000, seed=5)
    g = ps.GpuPauliSum(64)
    g.upload(x, z, c)  # unsorted: radix sort + dedup
    sx, sz, sc = g.download()
    g2 = ps.GpuPauliSum(64)
    g2.upload(sx, sz, sc)  # already in store form: no sort
    assert_same_terms(g2.download(), (sx, sz, sc), what="fast-path")
    # sorted but with a zero coefficient and a duplicate: must take the general path
    sc2 = sc.copy()
    sc2[3] = 0.0
    dx = np.concatenate([sx[:10], sx[9:10]])
    dz = np.concatenate([sz[:10], sz[9:10]])
    dc = np.concatenate([sc2[:10], sc2[9:10]])
    g2.upload(dx, dz, dc)
    o = oracle_sum(64, dx, dz, dc)
    assert_same_terms(g2.download(), oracle_arrays(o), what="fallback")
    assert len(g2) == 9


# --- light-cone skip: layers that act only where no term lives ---------------------------------


def test_light_cone_layers_are_skipped_and_stay_bit_exact():
    """The XXZ chain from Z on the middle site: most bond gates of the first steps act outside
    the operator's support, change nothing and launch nothing; the result is the oracle's."""
    n = 40
    circ = workloads.xxz_chain(n, 3, Jz=0.5, dt=0.1)
    x, z, c = labels_to_arrays({"I" * 20 + "Z" + "I" * 19: 1.0}, n)
    g = ps.GpuPauliSum(n, "f64")
    g.upload(x, z, c)
    st = g.propagate(circ, truncation.coeff(1e-8), "heisenberg", with_stats=True)
    got = g.download()
    o = oracle_sum(n, x, z, c)
    after = o.propagate(oracle_channels(circ), {"keep": [("coeff", 1e-8)]}, "heisenberg")
    assert st.terms_after == [int(v) for v in after]
    assert_same_terms(got, oracle_arrays(o), what="light-cone")
    assert st.layers_skipped > len(circ) // 2, st.layers_skipped
    assert g.expectation(workloads.neel_state(n)) == pytest.approx(o.expectation(workloads.neel_state(n)),
                                                                   rel=1e-12, abs=1e-15)


def test_first_layer_after_an_upload_is_never_skipped():
    """Uploaded terms have not met the keep program: the first layer drops the one below the
    threshold even though the gate acts elsewhere; the next layer, also elsewhere, is skipped."""
    n = 16
    labels = {"Z" + "I" * 15: 1.0, "IX" + "I" * 14: 1e-9}
    x, z, c = labels_to_arrays(labels, n)
    circ = ps.Circuit(n)
    circ.pauli_rotation("XX", [10, 11], 0.3)
    circ.pauli_rotation("YY", [12, 13], 0.3)
    g = ps.GpuPauliSum(n, "f64")
    g.upload(x, z, c)
    st = g.propagate(circ, truncation.coeff(1e-8), "forward", with_stats=True)
    assert st.terms_after == [1, 1]
    assert st.layers_skipped == 1
    got = g.download()
    o = oracle_sum(n, x, z, c)
    o.propagate(oracle_channels(circ), {"keep": [("coeff", 1e-8)]}, "forward")
    assert_same_terms(got, oracle_arrays(o), what="first-layer")


def test_skip_covers_noise_and_general_tables_outside_the_support():
    """Depolarizing noise and a CNOT on qubits no term touches are skipped too; a CNOT whose
    control is in the support is not, and the support grows by its target."""
    n = 12
    x, z, c = labels_to_arrays({"XZ" + "I" * 10: 0.6, "ZY" + "I" * 10: 0.8}, n)
    circ = ps.Circuit(n)
    circ.depolarize(1e-3, [5])
    circ.cnot(6, 7)
    circ.cnot(1, 8)
    circ.pauli_rotation("XX", [8, 9], 0.4)
    circ.depolarize(1e-3, [10])
    g = ps.GpuPauliSum(n, "f64")
    g.upload(x, z, c)
    g.propagate(ps.Circuit(n), truncation.coeff(1e-12))  # nothing: the store has not met the program
    first = ps.Circuit(n)
    first.pauli_rotation("ZZ", [0, 1], 0.2)  # acts on the support: runs and cleans the store
    g.propagate(first, truncation.coeff(1e-12))
    st = g.propagate(circ, truncation.coeff(1e-12), "forward", with_stats=True)
    assert st.layers_skipped == 3, st.layers_skipped  # depolarize(5), cnot(6, 7), depolarize(10)
    got = g.download()
    o = oracle_sum(n, x, z, c)
    o.propagate(oracle_channels(first), {"keep": [("coeff", 1e-12)]}, "forward")
    o.propagate(oracle_channels(circ), {"keep": [("coeff", 1e-12)]}, "forward")
    assert_same_terms(got, oracle_arrays(o), what="skip-noise-general")


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("ties", [False, True])
def test_topn_compaction_lists_the_next_layers_partners(dtype, ties):
    """A TopN pass followed by a rotation layer writes that layer's partner list while it
    compacts (the layer then launches no classify pass) when every key equal to the boundary is
    kept; when the quota cuts the ties it compacts plainly and the layer classifies itself.
    Either way every layer is bit-exact against the oracle."""
    nq = 20
    x, z, c = workloads.random_observable(nq, 5000, seed=13)
    if ties:
        c = np.random.default_rng(3).choice([0.25, -0.25, 0.5, 0.125, -0.0625], size=len(x))
    circ = workloads.random_pair_layers(nq, 2, seed=9)
    pol = truncation.topn(4000)
    g = ps.GpuPauliSum(nq, dtype)
    g.upload(x, z, c)
    g.set_profiling(True)
    st = g.propagate(circ, pol, "heisenberg", with_stats=True)
    prof = g.read_profile()
    o = oracle_sum(nq, x, z, c, dtype)
    after = o.propagate(oracle_channels(circ), oracle_policy(pol), "heisenberg")
    assert st.terms_after == [int(v) for v in after]
    assert_same_terms(g.download(), oracle_arrays(o), what=f"listed-partners-{dtype}-{ties}")
    classify = prof["k_classify"]["launches"]
    assert classify > 0  # the first layer classifies for itself
    if not ties:
        # the layers after a TopN pass take their partner lists from its compaction
        assert classify < len(circ) // 2, (classify, len(circ))


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_layer_within_the_cap_keeps_every_row_on_the_device(dtype):
    """A sum at its TopN cap meets a rotation that commutes with every term (no partners): the
    layer does not wait for its counts, so the select finds on the device that the live rows fit
    the quota and keeps them all; the next layer, which does split terms, takes its partner list
    from that compaction.  Bit-exact against the oracle throughout."""
    nq = 20
    rng = np.random.default_rng(17)
    W = ps.width_for(nq)
    zs = set()
    while len(zs) < 3000:
        zs.add(int(rng.integers(1, 1 << nq)))
    x = np.zeros((len(zs), W), np.uint64)
    z = np.array(sorted(zs), np.uint64).reshape(-1, W)
    c = rng.standard_normal(len(zs))
    pol = truncation.topn(3000)
    circ = ps.Circuit(nq)
    circ.pauli_rotation("ZZ", [0, 1], 0.3)   # commutes with every Z string: no partners
    circ.pauli_rotation("XY", [2, 3], 0.4)   # splits the terms with Z on exactly one of 2, 3
    circ.pauli_rotation("ZZ", [4, 5], 0.2)
    g = ps.GpuPauliSum(nq, dtype)
    g.upload(x, z, c)
    st = g.propagate(circ, pol, "heisenberg", with_stats=True)
    o = oracle_sum(nq, x, z, c, dtype)
    after = o.propagate(oracle_channels(circ), oracle_policy(pol), "heisenberg")
    assert st.terms_after == [int(v) for v in after]
    assert_same_terms(g.download(), oracle_arrays(o), what=f"keep-all-{dtype}")
