"""General one- and two-qubit tables: the Clifford gates, general unitaries and the PTM noise
channels (crates/paulistrings/src/channel/ptm.rs, ptm/{clifford,unitary,noise}.rs).

CPU tests pin the oracle's restatement to the reference's known answers
(crates/paulistrings/tests/propagate.rs:78-160, python/paulistrings/tests/test_general_unitary.py,
python/paulistrings/tests/test_pauli_channel.py), check that the library's table builder and
the oracle's agree bit for bit on every channel kind, and mirror the reference's argument
validation.  GPU tests run the layers through the C ABI and compare with the oracle bit for
bit: rotation-shaped tables on the partner path, the rest on the sort path (branch records,
radix sort, run-summing dedup), whose sums of up to sixteen contributions follow the naive
layer's order exactly.
"""

from __future__ import annotations

import cmath
import ctypes
import math

import numpy as np
import pytest

import paulistrings_b200 as ps
from oracle.oracle import OracleSum, pauli_key, prepare_table
from paulistrings_b200 import _lib, truncation
from paulistrings_b200.circuit import Circuit, gates, noise

from _util import assert_same_terms, oracle_arrays, oracle_channels, oracle_policy, oracle_sum

R = 1.0 / math.sqrt(2.0)
H = np.array([[R, R], [R, -R]], dtype=complex)
S = np.array([[1.0, 0.0], [0.0, 1.0j]], dtype=complex)
T = np.array([[1.0, 0.0], [0.0, cmath.exp(1j * math.pi / 4)]], dtype=complex)
CNOT = np.array([[1, 0, 0, 0], [0, 1, 0, 0], [0, 0, 0, 1], [0, 0, 1, 0]], dtype=complex)
CZ = np.diag([1.0, 1.0, 1.0, -1.0]).astype(complex)
SWAP = np.array([[1, 0, 0, 0], [0, 0, 1, 0], [0, 1, 0, 0], [0, 0, 0, 1]], dtype=complex)


def random_unitary(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    q, r = np.linalg.qr(a)
    return q * (np.diag(r) / np.abs(np.diag(r)))


def all_channels(q0, q1, seed=7):
    """One channel of every kind on (q0, q1)."""
    return [
        gates.h(q0), gates.s(q0), gates.sdg(q0), gates.x(q0), gates.y(q0), gates.z(q0),
        gates.cnot(q0, q1), gates.cnot(q1, q0), gates.cz(q0, q1), gates.swap(q0, q1),
        gates.unitary_1q(q0, T), gates.unitary_1q(q1, random_unitary(2, seed)),
        gates.unitary_2q(q0, q1, random_unitary(4, seed + 1)), gates.unitary_2q(q1, q0, random_unitary(4, seed + 2)),
        gates.unitary_2q(q0, q1, CNOT),
        noise.dephase(0.1, q0), noise.pauli_channel(0.05, 0.1, 0.15, q1), noise.depolarize2(0.2, q0, q1),
        noise.amplitude_damping(0.3, q0), noise.depolarize(0.05, q1),
    ]


def oracle_single(num_qubits, label_coeffs, dtype="f64"):
    s = OracleSum(num_qubits, dtype)
    keys = np.stack([pauli_key(lab, s.W) for lab, _ in label_coeffs])
    s.set(keys, np.array([c for _, c in label_coeffs], np.float64))
    return s


def oracle_terms(s: OracleSum):
    keys, c = s.get()
    out = {}
    for i in range(len(c)):
        lab = []
        for q in range(s.num_qubits):
            xb = (int(keys[i, q // 64]) >> (q % 64)) & 1
            zb = (int(keys[i, s.W + q // 64]) >> (q % 64)) & 1
            lab.append("IXZY"[xb | (zb << 1)])
        out["".join(lab)] = float(c[i])
    return out


def apply_oracle(num_qubits, terms, channel, adjoint=False):
    s = oracle_single(num_qubits, list(terms.items()))
    circ = Circuit(num_qubits)
    circ.append(channel)
    s.apply(oracle_channels(circ)[0], adjoint=adjoint)
    return oracle_terms(s)


# ---------------------------------------------------------------------------
# oracle known answers
# ---------------------------------------------------------------------------

@pytest.mark.parametrize("gate,inp,want", [
    (gates.h(0), "Z", {"X": 1.0}),
    (gates.h(0), "X", {"Z": 1.0}),
    (gates.h(0), "Y", {"Y": -1.0}),
    (gates.s(0), "X", {"Y": 1.0}),
    (gates.s(0), "Y", {"X": -1.0}),
    (gates.sdg(0), "X", {"Y": -1.0}),
    (gates.x(0), "Z", {"Z": -1.0}),
    (gates.y(0), "X", {"X": -1.0}),
    (gates.z(0), "Y", {"Y": -1.0}),
])
def test_oracle_single_qubit_cliffords(gate, inp, want):
    assert apply_oracle(1, {inp: 1.0}, gate) == want


def test_oracle_cnot_generators_in_one_word_and_across_words():
    # CNOT(0,1): I(x)Z -> Z(x)Z, X(x)I -> X(x)X (crates/paulistrings/tests/propagate.rs:121-169)
    assert apply_oracle(4, {"IZII": 1.0}, gates.cnot(0, 1)) == {"ZZII": 1.0}
    assert apply_oracle(4, {"XIII": 1.0}, gates.cnot(0, 1)) == {"XXII": 1.0}
    lab = ["I"] * 100
    lab[64] = "Z"
    want = ["I"] * 100
    want[63], want[64] = "Z", "Z"
    assert apply_oracle(100, {"".join(lab): 1.0}, gates.cnot(63, 64)) == {"".join(want): 1.0}


def test_oracle_cz_and_swap():
    assert apply_oracle(2, {"XI": 1.0}, gates.cz(0, 1)) == {"XZ": 1.0}
    assert apply_oracle(2, {"IX": 1.0}, gates.cz(0, 1)) == {"ZX": 1.0}
    assert apply_oracle(3, {"XIY": 2.0}, gates.swap(0, 2)) == {"YIX": 2.0}


def test_oracle_t_gate_maps_x_to_two_terms():
    out = apply_oracle(4, {"XIII": 1.0}, gates.unitary_1q(0, T))
    assert set(out) == {"XIII", "YIII"}
    for v in out.values():
        assert abs(abs(v) - R) < 1e-10


def test_oracle_amplitude_damping_both_directions():
    g = 0.3
    fwd = apply_oracle(1, {"I": 1.0, "X": 1.0}, noise.amplitude_damping(g, 0))
    assert fwd == {"I": 1.0, "Z": g, "X": math.sqrt(1 - g)}
    back = apply_oracle(1, {"Z": 1.0}, noise.amplitude_damping(g, 0), adjoint=True)
    assert back == {"I": g, "Z": 1 - g}


def test_oracle_pauli_channel_and_depolarize2_scales():
    px, py, pz = 0.05, 0.1, 0.15
    out = apply_oracle(1, {"X": 1.0, "Y": 1.0, "Z": 1.0}, noise.pauli_channel(px, py, pz, 0))
    assert out == {"X": 1 - 2 * (py + pz), "Y": 1 - 2 * (px + pz), "Z": 1 - 2 * (px + py)}
    out = apply_oracle(2, {"ZZ": 1.0, "XI": 1.0}, noise.depolarize2(0.3, 0, 1))
    assert out == {"ZZ": 1 - 16 * 0.3 / 15, "XI": 1 - 16 * 0.3 / 15}
    assert apply_oracle(2, {"ZZ": 1.0, "II": 1.0}, noise.depolarize2(15 / 16, 0, 1)) == {"II": 1.0}
    assert apply_oracle(1, {"X": 1.0}, noise.dephase(0.25, 0)) == {"X": 0.5}


def test_oracle_unitary_matches_the_named_cliffords():
    init = {"ZIII": 1.0, "XIII": 0.5, "YIII": -0.25, "IXII": 0.5, "YYII": -0.25}
    for u, named in [(H, gates.h(0)), (S, gates.s(0))]:
        a = apply_oracle(4, init, gates.unitary_1q(0, u))
        b = apply_oracle(4, init, named)
        assert set(a) == set(b) and all(abs(a[k] - b[k]) < 1e-10 for k in a)
    for u, named in [(CNOT, gates.cnot(0, 1)), (CZ, gates.cz(0, 1)), (SWAP, gates.swap(0, 1))]:
        assert apply_oracle(4, init, gates.unitary_2q(0, 1, u)) == apply_oracle(4, init, named)


def test_oracle_t_gate_round_trip():
    init = {"XIII": 1.0, "ZIII": 0.3}
    s = oracle_single(4, list(init.items()))
    circ = Circuit(4)
    circ.unitary_1q(0, T)
    s.propagate(oracle_channels(circ), direction="forward")
    s.propagate(oracle_channels(circ), direction="heisenberg")
    out = oracle_terms(s)
    assert set(k for k, v in out.items() if abs(v) > 1e-12) == set(init)
    for k, v in init.items():
        assert abs(out[k] - v) < 1e-10


# ---------------------------------------------------------------------------
# the library's table builder against the oracle's (host code, no device)
# ---------------------------------------------------------------------------

def library_table(channel, num_qubits, adjoint):
    circ = Circuit(num_qubits)
    circ.append(channel)
    arr, n, keep = circ.to_c()
    t = _lib.Table()
    status = _lib.lib().ps_prepare_channel(num_qubits, _lib.PS_F64, arr, int(adjoint), ctypes.byref(t))
    if status != _lib.PS_OK:
        raise ValueError(f"library declined {channel}")
    if t.mode == _lib.PS_TABLE_ROTATION:
        return None
    ents = [(int(t.entries[e].local_delta), [float(t.entries[e].amplitude[s]) for s in range(16)])
            for e in range(t.num_entries)]
    return tuple(int(t.qubits[j]) for j in range(t.k)), ents


@pytest.mark.parametrize("num_qubits,q0,q1", [(8, 2, 5), (8, 6, 1), (100, 63, 64), (100, 70, 3)])
@pytest.mark.parametrize("adjoint", [False, True])
def test_table_builders_agree_bit_for_bit(num_qubits, q0, q1, adjoint):
    for ch in all_channels(q0, q1):
        circ = Circuit(num_qubits)
        circ.append(ch)
        got = library_table(ch, num_qubits, adjoint)
        want = prepare_table(oracle_channels(circ)[0], num_qubits, adjoint)
        assert got[0] == want[0], ch
        gd = {d: a for d, a in got[1]}
        wd = {d: a for d, a in want[1]}
        # the oracle keeps the Clifford residue rule's zeroed identity slots; compare values
        assert set(gd) == set(wd), (ch, sorted(gd), sorted(wd))
        for d in gd:
            ga, wa = np.array(gd[d]), np.array(wd[d])
            assert np.array_equal(ga.view(np.uint64) * (ga != 0), wa.view(np.uint64) * (wa != 0)) or \
                np.array_equal(ga, wa), (ch, d, ga, wa)


def test_adjoint_flag_composes_with_the_layer_direction():
    for ch in all_channels(1, 4):
        a = library_table(ch.adjoint(), 6, False)
        b = library_table(ch, 6, True)
        assert a == b, ch
        assert library_table(ch.adjoint(), 6, True) == library_table(ch, 6, False), ch


# ---------------------------------------------------------------------------
# argument validation (python/paulistrings/tests/test_general_unitary.py,
# test_pauli_channel.py)
# ---------------------------------------------------------------------------

def test_unitary_validation():
    with pytest.raises(ValueError, match="2x2"):
        gates.unitary_1q(0, np.eye(3, dtype=complex))
    with pytest.raises(ValueError, match="4x4"):
        gates.unitary_2q(0, 1, np.eye(2, dtype=complex))
    with pytest.raises(ValueError, match="not unitary"):
        gates.unitary_1q(0, np.array([[1.0, 1.0], [0.0, 1.0]], dtype=complex))
    off = CNOT.copy()
    off[0, 0] *= 1.0 + 1e-9
    with pytest.raises(ValueError, match=r"not unitary .*tolerance 1e-10"):
        gates.unitary_2q(0, 1, off)
    with pytest.raises(ValueError, match="must differ"):
        gates.unitary_2q(1, 1, CNOT)


@pytest.mark.parametrize("args", [(-0.1, 0.0, 0.0), (0.0, -0.1, 0.0), (0.0, 0.0, -0.1)])
def test_pauli_channel_rejects_a_negative_probability(args):
    with pytest.raises(ValueError, match="non-negative"):
        noise.pauli_channel(*args, 0)


def test_pauli_channel_bounds():
    with pytest.raises(ValueError, match="at most 1"):
        noise.pauli_channel(0.5, 0.3, 0.3, 0)
    with pytest.raises(ValueError):
        noise.pauli_channel(float("nan"), 0.0, 0.0, 0)
    noise.pauli_channel(0.5, 0.25, 0.25, 0)


@pytest.mark.parametrize("p", [-0.01, 1.01])
def test_depolarize2_and_single_qubit_noise_ranges(p):
    with pytest.raises(ValueError):
        noise.depolarize2(p, 0, 1)
    for make in (noise.depolarize, noise.dephase, noise.amplitude_damping):
        with pytest.raises(ValueError):
            make(p, 0)
    with pytest.raises(ValueError, match="must differ"):
        noise.depolarize2(0.1, 2, 2)
    with pytest.raises(ValueError, match="must differ"):
        gates.cnot(3, 3)


def test_out_of_range_qubits_are_rejected_at_append():
    c = Circuit(4)
    with pytest.raises(ValueError):
        c.cnot(0, 4)
    with pytest.raises(ValueError):
        c.amplitude_damping(0.1, [5])


def test_circuit_broadcast_methods():
    c = Circuit(4)
    c.pauli_channel(0.1, 0.0, 0.0, [0, 1, 2])
    c.depolarize2(0.1, [(0, 1), (2, 3)])
    c.dephase(0.1, [3])
    assert len(c) == 6
    assert c[0] == noise.pauli_channel(0.1, 0.0, 0.0, 0)
    assert c[3] == noise.depolarize2(0.1, 0, 1)
    assert gates.sdg(2).debug_name == "phase_gate_adjoint"
    assert gates.sdg(2).adjoint() == gates.s(2)


# ---------------------------------------------------------------------------
# device parity
# ---------------------------------------------------------------------------

def random_sum(num_qubits, count, seed, max_weight=4):
    rng = np.random.default_rng(seed)
    W = ps.width_for(num_qubits)
    x = np.zeros((count, W), np.uint64)
    z = np.zeros((count, W), np.uint64)
    for i in range(count):
        w = int(rng.integers(1, max_weight + 1))
        for q in rng.choice(num_qubits, size=w, replace=False):
            p = int(rng.integers(1, 4))
            bit = np.uint64(1) << np.uint64(int(q) % 64)
            if p & 1:
                x[i, int(q) // 64] |= bit
            if p & 2:
                z[i, int(q) // 64] |= bit
    c = rng.normal(size=count)
    return x, z, c


def run_both(num_qubits, circuit, x, z, c, policy=None, direction="forward", dtype="f64", compensated=False):
    g = ps.GpuPauliSum(num_qubits, dtype)
    if compensated:
        assert _lib.lib().ps_set_compensated_sums(g._h, 1) == _lib.PS_OK
    g.upload(x, z, c)
    stats = g.propagate(circuit, policy, direction, with_stats=True)
    got = g.download()
    o = oracle_sum(num_qubits, x, z, c, dtype)
    o.propagate(oracle_channels(circuit), oracle_policy(policy), direction)
    return got, oracle_arrays(o), stats


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("num_qubits,q0,q1", [(64, 5, 40), (100, 63, 64), (100, 90, 2)])
@pytest.mark.parametrize("direction", ["forward", "heisenberg"])
def test_every_channel_kind_matches_the_oracle_bit_for_bit(dtype, num_qubits, q0, q1, direction):
    x, z, c = random_sum(num_qubits, 3000, seed=q0 * 131 + q1)
    # make the support qubits busy so every pattern occurs
    rng = np.random.default_rng(q1)
    for q in (q0, q1):
        bit = np.uint64(1) << np.uint64(q % 64)
        x[rng.random(len(c)) < 0.5, q // 64] |= bit
        z[rng.random(len(c)) < 0.5, q // 64] |= bit
    for ch in all_channels(q0, q1):
        circ = Circuit(num_qubits)
        circ.append(ch)
        got, want, _ = run_both(num_qubits, circ, x, z, c, truncation.coeff(1e-9), direction, dtype)
        assert_same_terms(got, want, what=f"{ch} {direction} {dtype}")


@pytest.mark.gpu
def test_layer_paths():
    num_qubits = 16
    x, z, c = random_sum(num_qubits, 2000, seed=1)
    expect = [(gates.cnot(0, 1), _lib.PS_PATH_SORT), (gates.unitary_2q(2, 3, random_unitary(4, 3)), _lib.PS_PATH_SORT),
              (gates.h(0), _lib.PS_PATH_ROTATION), (gates.s(1), _lib.PS_PATH_ROTATION),
              (noise.amplitude_damping(0.2, 2), _lib.PS_PATH_ROTATION), (noise.dephase(0.1, 3), _lib.PS_PATH_RESCALE),
              (noise.depolarize2(0.1, 4, 5), _lib.PS_PATH_RESCALE), (gates.x(3), _lib.PS_PATH_RESCALE)]
    for ch, path in expect:
        g = ps.GpuPauliSum(num_qubits)
        g.upload(x, z, c)
        st = g.apply_layer(ch)
        assert st.path == path, ch


@pytest.mark.gpu
@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("direction", ["forward", "heisenberg"])
def test_random_clifford_t_noise_circuit_matches_the_oracle(dtype, direction):
    num_qubits = 12
    rng = np.random.default_rng(11)
    circ = Circuit(num_qubits)
    for layer in range(6):
        for q in range(num_qubits):
            pick = int(rng.integers(0, 5))
            if pick == 0:
                circ.h(q)
            elif pick == 1:
                circ.unitary_1q(q, T)
            elif pick == 2:
                circ.rz(float(rng.uniform(-3, 3)), q)
            elif pick == 3:
                circ.s(q)
        perm = rng.permutation(num_qubits)
        for k in range(0, num_qubits - 1, 2):
            a, b = int(perm[k]), int(perm[k + 1])
            pick = int(rng.integers(0, 4))
            if pick == 0:
                circ.cnot(a, b)
            elif pick == 1:
                circ.cz(a, b)
            elif pick == 2:
                circ.unitary_2q(a, b, random_unitary(4, 100 * layer + k))
            else:
                circ.swap(a, b)
        circ.amplitude_damping(0.02, [int(rng.integers(0, num_qubits))])
        circ.depolarize2(0.01, [(0, num_qubits - 1)])
    x, z, c = random_sum(num_qubits, 200, seed=5, max_weight=3)
    got, want, stats = run_both(num_qubits, circ, x, z, c, truncation.coeff(1e-6), direction, dtype)
    assert stats.final_terms == len(got[2])
    assert_same_terms(got, want, what=f"random circuit {direction} {dtype}")


@pytest.mark.gpu
def test_named_and_matrix_gates_agree_on_the_device():
    init = ps.PauliSum.from_strings({"ZIII": 1.0, "IXII": 0.5, "YYII": -0.25, "XIII": 0.5, "YIII": -0.25},
                                    num_qubits=4)
    for u, name, args in [(H, "h", (0,)), (S, "s", (0,)), (CNOT, "cnot", (0, 1)), (CZ, "cz", (0, 1)),
                          (SWAP, "swap", (0, 1))]:
        a, b = Circuit(4), Circuit(4)
        if len(args) == 1:
            a.unitary_1q(args[0], u)
        else:
            a.unitary_2q(args[0], args[1], u)
        getattr(b, name)(*args)
        da = ps.propagated(init, a).to_dict()
        db = ps.propagated(init, b).to_dict()
        assert set(da) == set(db), name
        for k in da:
            assert abs(da[k] - db[k]) < 1e-10, (name, k)


@pytest.mark.gpu
def test_t_gate_round_trips_on_the_device():
    init = ps.PauliSum.from_strings({"XIII": 1.0, "ZIII": 0.3}, num_qubits=4)
    c = Circuit(4)
    c.unitary_1q(0, T)
    fwd = ps.propagated(init, c, direction="forward")
    assert len(fwd) == 3
    back = ps.propagated(fwd, c, direction="heisenberg").to_dict()
    back = {k: v for k, v in back.items() if abs(v) > 1e-12}
    assert set(back) == {"XIII", "ZIII"}
    assert abs(back["XIII"] - 1.0) < 1e-10 and abs(back["ZIII"] - 0.3) < 1e-10


@pytest.mark.gpu
def test_dense_layers_in_f32_with_compensated_sums_stay_close_to_f64():
    num_qubits = 10
    circ = Circuit(num_qubits)
    for layer in range(4):
        for k in range(0, num_qubits - 1, 2):
            circ.unitary_2q((k + layer) % num_qubits, (k + layer + 1) % num_qubits, random_unitary(4, 7 * layer + k))
    x, z, c = random_sum(num_qubits, 300, seed=9, max_weight=3)
    ref = oracle_sum(num_qubits, x, z, c, "f64")
    ref.propagate(oracle_channels(circ), None, "forward")
    rx, rz, rc = oracle_arrays(ref)
    errs = {}
    for comp in (False, True):
        got, want, _ = run_both(num_qubits, circ, x, z, c, None, "forward", "f32", compensated=comp)
        if not comp:
            assert_same_terms(got, want, what="plain f32 vs oracle f32")
        gx, gz, gc = got
        ref_map = {(tuple(a), tuple(b)): v for a, b, v in zip(rx, rz, rc)}
        err = max(abs(v - ref_map.get((tuple(a), tuple(b)), 0.0)) for a, b, v in zip(gx, gz, gc))
        errs[comp] = err
    scale = float(np.max(np.abs(rc)))
    assert errs[True] <= 2e-5 * scale
    assert errs[True] <= errs[False] * 1.01 + 1e-12
