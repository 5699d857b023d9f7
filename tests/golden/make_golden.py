"""Regenerate the golden fixtures in this directory from the reference repository.

Run where a checkout of the reference is available (it is never read at test time), giving
the path of that checkout:

    python tests/golden/make_golden.py <path to the reference checkout>

What it writes, and where each number comes from (paths inside the reference):

* ``xxz_statevector.json`` -- ``examples/xxz_chain/results/statevector.json``: the open
  XXZ chain (``examples/common/circuits.py:292-339``, dt = 0.1, even-odd bonds),
  Heisenberg picture, ``coeff(1e-12)``, domain-wall state, observable ``Z_c`` or
  ``Z_c Z_{c+1}`` at ``c = n // 2`` (``examples/xxz_chain/run_benchmark_d.py:151-169``).
  Per case: the reference's own expectation value, the statevector value, and the
  final term count.
* ``jl_parity.json`` -- ``benchmarks/python/jl_performance/post-optimization/summary.json``:
  the XXZ n = 100 workload (6 steps, Jz = 0.5) and the 127-qubit kicked-Ising workload
  (5 steps, theta_h = 5 pi / 16, theta_zz = -pi / 2), each per cutoff with the
  reference's final term count and expectation value.

Each case carries its gate list, recorded by running the reference's own circuit
builders (``examples/common/circuits.py``) against a stub ``paulistrings`` module
that records ``Circuit`` calls.  Gates are ``[kind, paulis, qubits, param]`` with
kind ``"rotation"`` (``exp(-i param P / 2)``).
"""

from __future__ import annotations

import json
import math
import sys
import types
from pathlib import Path

HERE = Path(__file__).resolve().parent


class _RecordingCircuit:
    def __init__(self, num_qubits):
        self.num_qubits = num_qubits
        self.gates = []

    def rx(self, theta, qubit):
        self.gates.append(["rotation", "X", [int(qubit)], float(theta)])

    def ry(self, theta, qubit):
        self.gates.append(["rotation", "Y", [int(qubit)], float(theta)])

    def rz(self, theta, qubit):
        self.gates.append(["rotation", "Z", [int(qubit)], float(theta)])

    def pauli_rotation(self, pauli, qubits, theta):
        self.gates.append(["rotation", str(pauli), [int(q) for q in qubits], float(theta)])

    def append(self, channel):
        self.gates.append(channel)


def _load_builders(reference: Path):
    stub = types.ModuleType("paulistrings")
    stub.Circuit = _RecordingCircuit
    stub.gates = types.SimpleNamespace()
    sys.modules["paulistrings"] = stub
    sys.path.insert(0, str(reference / "examples"))
    from common import circuits  # noqa: E402  (the reference's own builders)

    return circuits


def _domain_wall(n):
    return "0" * (n // 2) + "1" * (n - n // 2)


def main(reference: Path) -> None:
    circuits = _load_builders(reference)

    sv = json.loads((reference / "examples/xxz_chain/results/statevector.json").read_text())
    assert sv["truncation"] == {"min_abs_coeff": 1e-12}
    cases = []
    for row in sv["rows"]:
        n, jz, steps, kind = row["n"], row["Jz"], row["steps"], row["observable"]
        c = n // 2
        obs = [c] if kind == "z1" else [c, c + 1]
        circ = circuits.xxz_chain_trotter(n, steps, Jz=jz, dt=0.1)
        cases.append(
            {
                "n": n,
                "Jz": jz,
                "steps": steps,
                "observable_z": obs,
                "state": _domain_wall(n),
                "epsilon": 1e-12,
                "direction": "heisenberg",
                "expectation": row["paulistrings"],
                "statevector": row["statevector"],
                "final_terms": row["final_terms"],
                "gates": circ.gates,
            }
        )
    (HERE / "xxz_statevector.json").write_text(json.dumps({"source": "examples/xxz_chain/results/statevector.json", "cases": cases}))

    summ = json.loads(
        (reference / "benchmarks/python/jl_performance/post-optimization/summary.json").read_text()
    )
    workloads = {}
    for curve in summ["curves"]:
        key = curve["workload"]
        if key == "xxz":
            circ = circuits.xxz_chain_trotter(100, 6, Jz=0.5, dt=0.1)
            obs_q = 50
        elif key == "kicked_ising":
            circ = circuits.heavy_hex_kicked_ising(127, trotter_steps=5, theta_h=5.0 * math.pi / 16.0)
            obs_q = 62
        else:
            continue
        (label,) = list(curve["observable"].keys())
        assert label[obs_q] == "Z" and label.count("I") == len(label) - 1
        points = []
        for cfg in curve["configs"]:
            parity = cfg["parity"]
            if cfg.get("disqualified") or not parity.get("ok"):
                continue
            points.append(
                {
                    "epsilon": cfg["truncation"]["min_abs_coeff"],
                    "max_weight": cfg["truncation"].get("max_weight"),
                    "final_terms": parity["rust_final_terms"],
                    "expectation": parity.get("expectation_rust"),
                }
            )
        workloads[key] = {
            "n_qubits": curve["n_qubits"],
            "state": curve["state"],
            "observable_z": [obs_q],
            "direction": "heisenberg",
            "points": points,
            "gates": circ.gates,
        }
        assert len(circ.gates) == parity["n_layers"]
    (HERE / "jl_parity.json").write_text(
        json.dumps({"source": "benchmarks/python/jl_performance/post-optimization/summary.json", "workloads": workloads})
    )


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path to the reference checkout>")
    main(Path(sys.argv[1]))
