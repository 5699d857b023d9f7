"""Benchmark of the per-layer Pauli-propagation path on B200.

Workload (the configuration the headline metric is quoted on): 64 qubits, 30 layers of
random dense two-qubit rotations -- per layer a seeded random matching of the qubits into 32
pairs, each pair exp(-i theta P(x)Q / 2) with P, Q uniform over {X, Y, Z}, theta uniform in
[0, 2 pi), then RZ(phi) on every qubit -- applied in the Heisenberg picture to 65,536
distinct random Pauli strings of weight 1-4 with N(0, 1) coefficients normalised to unit
2-norm; float64 coefficients; policy TopN(2^26) & coeff(1e-10) after every channel.
Synthetic data from one splitmix64 stream (seed 0xC0FFEE); the reference measures on its
own synthetic circuits, so nothing external stands in here.

A step is one circuit layer (96 channels).  The warm-up steps are the first layers, which
also grow the store to the 2^26-term cap; the timed steps continue the same run at the cap.
``value`` is terms/s per layer: the terms entering each channel, summed over the timed
channels, divided by their device time (CUDA events on the library's stream).  The store
(>= 1.6 GB) is larger than L2, so no flush is needed between steps.

``e2e`` is the same metric through the public C-ABI calls with host buffers: each step
uploads the state from pinned host memory, runs the layer and downloads the result into
pinned host memory, all inside the timed region.

``--impl reference`` times the reference's CPU path: the reference is Rust and cannot be
built in this image, so its restatement (oracle/, OpenMP over every host thread) runs a
bounded sample of the same workload's capped channels on the host.

Multi-GPU (torchrun): the path does not shard, so each rank runs an independent replica with
its own seed; value is the terms of all ranks over the slowest rank's time.
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

# The CPU baselines run the oracle's OpenMP engine on every host thread; its idle workers sleep
# after a short spin instead of spinning on the cores the device's host thread needs in the
# device timings that follow (read when the OpenMP runtime starts, so set before any import).
os.environ.setdefault("GOMP_SPINCOUNT", "10000")

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT), str(ROOT / "paulistrings-rs_b200")]

METRIC = "terms/s per layer"
TERM_CAP = 1 << 26
NUM_QUBITS = 64
LAYERS = 30
PROFILED_LAYERS = 2  # layers after the timed ones that carry per-kernel CUDA events
EPS = 1e-10
SEED = 0xC0FFEE


def workload_config(k, w, cap=None):
    cap = cap or TERM_CAP
    return {
        "workload": "random two-qubit rotation layers: 64 qubits, 30 layers x (32 pair rotations + 64 RZ), "
        "65,536-term random observable, Heisenberg, TopN(2^26) & coeff(1e-10), f64",
        "num_qubits": NUM_QUBITS,
        "layers": LAYERS,
        "channels_per_layer": 96,
        "term_cap": cap,
        "initial_terms": 65536,
        "timed_layers": k,
        "warmup_layers": w,
        "seed": SEED,
        "l2": "inputs larger than L2 (store >= 1.6 GB at the cap), no flush",
    }


def layer_circuits(seed):
    from paulistrings_b200 import Circuit, workloads

    full = workloads.random_pair_layers(NUM_QUBITS, LAYERS, seed)
    chans = list(full)
    out = []
    # Heisenberg order: the last layer first; each sub-circuit is propagated with
    # direction="heisenberg", which reverses it and applies adjoints.
    for layer in reversed(range(LAYERS)):
        c = Circuit(NUM_QUBITS)
        for ch in chans[96 * layer : 96 * (layer + 1)]:
            c.append(ch)
        out.append(c)
    return out


class ClockSampler:
    """SM clock and throttle-reason samples during the timed region.

    Sampled in-process through NVML on a background thread (the device found by its UUID, so
    CUDA_VISIBLE_DEVICES cannot point it at another GPU), every `period` seconds: an
    `nvidia-smi -lms` process polling beside the timed steps measurably delays the host's
    stream synchronizations, which this path does twice per channel.  Falls back to
    `nvidia-smi` when NVML is not importable.
    """

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    REASONS = (("hw_slowdown", 0x8), ("hw_thermal_slowdown", 0x40), ("sw_thermal_slowdown", 0x20),
               ("sw_power_cap", 0x4))

    def __init__(self, device, period=0.25):
        self.device = device
        self.period = period
        self.proc = None
        self.thread = None
        self.stop = threading.Event()
        self.lines = []
        self.samples = []  # (sm MHz, max sm MHz, reason bits)

    def __enter__(self):
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            uuid = uuid if uuid.startswith("GPU-") else "GPU-" + uuid
            h = pynvml.nvmlDeviceGetHandleByUUID(uuid)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._poll_nvml, args=(pynvml, h, mx), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", str(int(self.period * 1000))], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _poll_nvml(self, pynvml, h, mx):
        while True:
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((float(sm), float(mx), int(bits)))
            except Exception:
                pass
            if self.stop.wait(self.period):
                return

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        self.stop.set()
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread:
            self.thread.join(timeout=5)

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        for s, m, bits in self.samples:
            sm.append(s)
            mx = max(mx, m)
            for nm, bit in self.REASONS:
                if bits & bit:
                    reasons.add(nm)
        names = [nm for nm, _ in self.REASONS]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        src = "nvml" if self.samples else ("nvidia-smi" if self.lines else None)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "source": src}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": src, "period_s": self.period}


def measured_peaks():
    try:
        d = json.loads((ROOT / "MEASURED_PEAKS.json").read_text())
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic():
    """Per-launch DRAM bytes of the dominant kernel from a committed ncu summary, if any."""
    try:
        return json.loads((ROOT / "profiles" / "traffic.json").read_text())
    except (OSError, ValueError):
        return {}


def cpu_baseline(seconds: float):
    """The reference's CPU path on this host's cores: the oracle's sorted-store engine (the
    reference host engine's shape -- rotation scan, linear partner order, merge-join with the
    keep program -- restated in C with OpenMP over all host threads; bit-identical to the naive
    checker) on a bounded sample of the capped channels: the same circuit from the same initial
    observable runs untimed until the 2^26-term cap binds (channel 184), then the following
    channels, each entering with 2^26 terms as the device's timed channels do, are timed until
    `seconds` of wall time."""
    import numpy as np

    from oracle.oracle import OracleSum
    from paulistrings_b200 import workloads

    threads = os.cpu_count() or 1
    x, z, c = workloads.random_observable(NUM_QUBITS, 65536, SEED + 1)
    o = OracleSum(NUM_QUBITS, "f64")
    o.set(np.concatenate([x, z], axis=1), c)
    pol = {"keep": [("coeff", EPS)], "passes": [("topn", TERM_CAP)]}
    terms = channels = grown = 0
    t_grow = time.perf_counter()
    t0 = None
    done = False
    for circ in layer_circuits(SEED):
        for ch in reversed(list(circ)):
            if t0 is None and len(o) >= TERM_CAP:
                t0 = time.perf_counter()
            if t0 is not None:
                terms += len(o)
                channels += 1
            else:
                grown += 1
            o.apply(("rotation", ch.paulis, list(ch.qubits), ch.theta), adjoint=True, policy=pol,
                    sorted_engine=True, threads=threads)
            if t0 is not None and time.perf_counter() - t0 > seconds:
                done = True
                break
        if done:
            break
    dt = time.perf_counter() - (t0 if t0 is not None else t_grow)
    return {
        "value": terms / dt if terms else 0.0,
        "unit": METRIC,
        "cores": threads,
        "kind": "port",
        "sample": f"{channels} capped channels (channels {grown + 1}-{grown + channels} of the same workload, each "
        f"entering with {TERM_CAP} terms; the first {grown} channels grew the sum to the cap untimed, "
        f"{time.perf_counter() - t_grow - dt:.1f} s), {dt:.1f} s timed, sorted-store engine on {threads} host threads",
    }


def dist_setup(n_gpus):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    return world, rank, local


def _reduce(v, world, op):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def dist_max(v, world):
    import torch.distributed as dist

    return _reduce(v, world, dist.ReduceOp.MAX if world > 1 else None)


def dist_sum(v, world):
    import torch.distributed as dist

    return _reduce(v, world, dist.ReduceOp.SUM if world > 1 else None)


def replica_throughput(terms: float, device_ms: float, world: int) -> tuple:
    """Whole-job terms/s over independent replicas: every rank's terms over the slowest rank's
    device time (weak scaling).  Returns (value, max_ms, all_terms)."""
    max_ms = dist_max(device_ms, world)
    all_terms = dist_sum(terms, world)
    return all_terms / (max_ms * 1e-3), max_ms, all_terms


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def run_reference(args, world, rank):
    if rank != 0:
        return
    cb = cpu_baseline(args.cpu_seconds)
    line = {
        "impl": "reference",
        "metric": METRIC,
        "value": cb["value"],
        "unit": METRIC,
        "n_gpus": args.gpus,
        "steps": args.steps,
        "warmup": args.warmup,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": dict(workload_config(args.steps, args.warmup), parallelism=f"replicas{world}"),
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is Rust (no cargo in this image); its host engine restated in C with OpenMP "
        "(oracle/, bit-identical to the naive checker) is timed instead",
    }
    print(json.dumps(line))


def run_ours(args, world, rank, local):
    import numpy as np
    import torch

    import paulistrings_b200 as ps
    from paulistrings_b200 import truncation, workloads

    seed = SEED + 7919 * rank
    cap = args.term_cap
    policy = truncation.topn(cap) & truncation.coeff(EPS)
    layers = layer_circuits(seed)
    assert args.warmup + args.steps <= LAYERS, "warmup + steps must fit in the 30-layer circuit"
    x0, z0, c0 = workloads.random_observable(NUM_QUBITS, 65536, seed + 1)

    # --- device-resident timing (value, roofline) --------------------------------------------------
    g = ps.GpuPauliSum(NUM_QUBITS, "f64", device=local)
    g.upload(x0, z0, c0)
    for li in range(args.warmup):
        g.propagate(layers[li], policy, "heisenberg")
    barrier(world)
    terms = 0
    terms_out = 0
    dev_ms = 0.0
    launches = 0
    torch.cuda.synchronize()
    # ncu --profile-from-start off captures exactly the timed steps
    torch.cuda.cudart().cudaProfilerStart()
    with ClockSampler(local) as clocks:
        for li in range(args.warmup, args.warmup + args.steps):
            st = g.propagate(layers[li], policy, "heisenberg", with_stats=True)
            terms += st.total_terms_in
            terms_out += sum(st.terms_after)
            dev_ms += st.device_ms
            launches += st.kernel_launches
    torch.cuda.cudart().cudaProfilerStop()
    barrier(world)
    state_after = g.download()
    # per-kernel CUDA-event times and algorithmic bytes for the roofline, from the layers that
    # follow the timed ones (events around every launch would add host work to the timed steps)
    g.set_profiling(True)
    first = args.warmup + args.steps
    for li in range(first, min(LAYERS, first + PROFILED_LAYERS)):
        g.propagate(layers[li], policy, "heisenberg")
    prof = g.read_profile()
    prof_ms = sum(r["total_ms"] for r in prof.values())
    g.set_profiling(False)
    g.close()
    del g

    value, max_ms, all_terms = replica_throughput(terms, dev_ms, world)

    # --- end to end through the C ABI with pinned host buffers ---------------------------------
    if args.no_e2e:
        e2e_value, h2d, d2h = None, 0, 0
        return finish(args, world, rank, value, max_ms, launches, prof, dev_ms, clocks, state_after, cap,
                      e2e_value, h2d, d2h, terms, terms_out)
    rows = cap + 1024
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True).numpy()
    hx = pin((rows, 1), torch.int64).view(np.uint64)
    hz = pin((rows, 1), torch.int64).view(np.uint64)
    hc = pin((rows,), torch.float64)
    ox = pin((rows, 1), torch.int64).view(np.uint64)
    oz = pin((rows, 1), torch.int64).view(np.uint64)
    oc = pin((rows,), torch.float64)
    # the e2e run restarts from the state the warm-up reached, held in pinned host memory
    g = ps.GpuPauliSum(NUM_QUBITS, "f64", device=local)
    g.upload(x0, z0, c0)
    for li in range(args.warmup):
        g.propagate(layers[li], policy, "heisenberg")
    n = len(g)
    g.download(out=(hx, hz, hc))
    h2d = d2h = 0
    e2e_terms = 0
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for li in range(args.warmup, args.warmup + args.steps):
        g.upload(hx[:n], hz[:n], hc[:n])
        h2d += n * (16 + 8)
        st = g.propagate(layers[li], policy, "heisenberg", with_stats=True)
        e2e_terms += st.total_terms_in
        _, _, cc = g.download(out=(ox, oz, oc))
        n = cc.shape[0]
        d2h += n * (16 + 8)
        hx, ox = ox, hx
        hz, oz = oz, hz
        hc, oc = oc, hc
    torch.cuda.synchronize()
    e2e_s = dist_max(time.perf_counter() - t0, world)
    barrier(world)
    e2e_value = dist_sum(e2e_terms, world) / e2e_s
    g.close()
    return finish(args, world, rank, value, max_ms, launches, prof, dev_ms, clocks, state_after, cap, e2e_value,
                  h2d, d2h, terms, terms_out)


def finish(args, world, rank, value, max_ms, launches, prof, dev_ms, clocks, state_after, cap, e2e_value, h2d, d2h,
           terms_in, terms_out):
    if rank != 0:
        return
    peak, peak_kind = measured_peaks()
    dom = max(prof.items(), key=lambda kv: kv[1]["total_ms"])
    name, rec = dom
    per_launch_bytes = rec["algorithmic_bytes"] / max(1, rec["timed_launches"])
    per_launch_ms = rec["total_ms"] / max(1, rec["timed_launches"])
    achieved = per_launch_bytes / (per_launch_ms * 1e-3) / 1e9
    traffic = ncu_traffic().get(name)
    roofline = {
        "bound": "hbm",
        "kernel": name,
        "achieved": round(achieved, 1),
        "peak": peak,
        "peak_kind": peak_kind,
        "unit": "GB/s",
        "frac": round(achieved / peak, 4),
        "traffic": traffic,
        "launches_timed": rec["timed_launches"],
        "share_of_device_time": round(rec["total_ms"] / max(1e-9, sum(r["total_ms"] for r in prof.values())), 4),
    }
    all_bytes = sum(r["algorithmic_bytes"] for r in prof.values())
    all_ms = sum(r["total_ms"] for r in prof.values())
    chans = NUM_QUBITS // 2 + NUM_QUBITS  # channels per layer: the pair rotations and the RZ sweep
    prof_channels = max(1, min(PROFILED_LAYERS, LAYERS - args.warmup - args.steps)) * chans
    bytes_per_channel = all_bytes / prof_channels
    timed_ms_per_channel = dev_ms / max(1, args.steps * chans)
    # the layer's algorithmic bytes over the timed channels' device time, and over the kernels' own time
    layer_frac = bytes_per_channel / (timed_ms_per_channel * 1e-3) / 1e9 / peak
    kernel_layer_frac = all_bytes / (all_ms * 1e-3) / 1e9 / peak
    # the least a channel can move: read every input row once and write every output row once
    min_frac = (terms_in + terms_out) * (16 + 8) / (dev_ms * 1e-3) / 1e9 / peak
    line = {
        "metric": METRIC,
        "value": value,
        "unit": METRIC,
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": max_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": dict(workload_config(args.steps, args.warmup, cap), parallelism=f"replicas{world}"),
        "e2e": None if e2e_value is None else {"value": e2e_value, "unit": METRIC,
                                              "h2d_bytes_per_step": h2d // args.steps,
                                              "d2h_bytes_per_step": d2h // args.steps},
        "gpu_launches": launches,
        "roofline": roofline,
        "layer_roofline_frac": round(layer_frac, 4),
        "min_traffic_frac": round(min_frac, 4),
        "kernel_profile": {k: {"launches": v["timed_launches"], "ms": round(v["total_ms"], 3),
                               "GB": round(v["algorithmic_bytes"] / 1e9, 3)} for k, v in prof.items() if v["launches"]},
        "ms_per_channel": {"timed": round(timed_ms_per_channel, 4),
                           "kernels_only": round(all_ms / prof_channels, 4)},
        "kernel_layer_roofline_frac": round(kernel_layer_frac, 4),
        "final_terms": int(state_after[2].shape[0]),
        "clocks": clocks.summary(),
    }
    # the other configurations run on one GPU (rank 0 of an N = 1 run); replicas add nothing.
    # They run before the CPU baseline, whose host threads would otherwise share the cores the
    # device's host thread needs in their timings.
    line["configs"] = run_configs(args) if world == 1 else "measured by the N=1 run"
    line["cpu_baseline"] = cpu_baseline(args.cpu_seconds) if world == 1 and args.cpu_seconds > 0 else None
    print(json.dumps(line))


# ---------------------------------------------------------------------------------------------
# the other configurations: one object each under "configs" on the bench line
# ---------------------------------------------------------------------------------------------

def _labels(terms, num_qubits):
    import numpy as np

    import paulistrings_b200 as ps

    W = ps.width_for(num_qubits)
    x = np.array([ps.parse_label(k, W)[0] for k in terms], np.uint64).reshape(-1, W)
    z = np.array([ps.parse_label(k, W)[1] for k in terms], np.uint64).reshape(-1, W)
    c = np.array(list(terms.values()), np.float64)
    return x, z, c


def _timed_propagation(num_qubits, x, z, c, circuit, policy, dtype, compensated=False, repeats=3):
    """Device terms/s per layer of one propagation (the best of `repeats` identical runs, each
    from a fresh upload), over the layers that ran kernels."""
    import torch

    import paulistrings_b200 as ps
    from paulistrings_b200 import _lib

    best = None
    for _ in range(repeats):
        g = ps.GpuPauliSum(num_qubits, dtype)
        if compensated:
            _lib.check(_lib.lib().ps_set_compensated_sums(g._h, 1), g._h, "compensated")
        g.upload(x, z, c)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = g.propagate(circuit, policy, "heisenberg", with_stats=True)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        if best is None or st.device_ms < best[0].device_ms:
            best = (st, wall, g)
        else:
            g.close()
    st, wall, g = best
    run = {
        "terms_per_s_per_layer": (st.total_terms_in - st.skipped_terms_in) / (st.device_ms * 1e-3),
        "device_ms": round(st.device_ms, 3),
        "wall_ms": round(wall * 1e3, 3),
        "layers": st.layers,
        "layers_skipped": st.layers_skipped,
        "peak_terms": st.peak_terms,
        "final_terms": st.final_terms,
        "gpu_launches": st.kernel_launches,
    }
    return run, g


def _cpu_propagation(num_qubits, x, z, c, circuit, policy_dict, dtype="f64", seconds=15.0):
    """The oracle's sorted-store engine (all host threads) on the same circuit, channel by channel
    (Heisenberg order), until `seconds`: terms/s per layer over the channels it finished."""
    import numpy as np

    from oracle.oracle import OracleSum
    from paulistrings_b200.circuit import Depolarizing, PauliRotation

    threads = os.cpu_count() or 1
    o = OracleSum(num_qubits, dtype)
    o.set(np.concatenate([x, z], axis=1), c)
    terms = done = 0
    t0 = time.perf_counter()
    chans = list(circuit)
    for ch in reversed(chans):
        if isinstance(ch, PauliRotation):
            spec = ("rotation", ch.paulis, list(ch.qubits), ch.theta)
        elif isinstance(ch, Depolarizing):
            spec = ("depolarize", "", [ch.qubit], ch.p)
        else:
            raise TypeError(ch)
        terms += len(o)
        o.apply(spec, adjoint=True, policy=policy_dict, sorted_engine=True, threads=threads)
        done += 1
        if time.perf_counter() - t0 > seconds:
            break
    dt = time.perf_counter() - t0
    return {"value": terms / dt, "unit": METRIC, "cores": threads, "kind": "port",
            "sample": f"{done} of {len(chans)} channels, {dt:.1f} s, sorted-store engine on {threads} host threads"}, \
        (o if done == len(chans) else None)


def config_tfim6(args):
    """6 x 6 periodic transverse-field Ising Trotter circuit (36 qubits): observable
    (1/36) sum X_i, Heisenberg, 5 steps of RZZ(-2 J dt) on the 72 bonds (horizontal then
    vertical, row-major) and RX(2 h dt) on every qubit, J = h = 1, dt = 0.1; coeff(1e-5) after
    every channel; f64; readout in |0...0>."""
    from paulistrings_b200 import truncation, workloads

    circ = workloads.tfim_2d(6, 5, J=1.0, h=1.0, dt=0.1)
    x, z, c = _labels(workloads.tfim_magnetization(6, "X"), 36)
    run, g = _timed_propagation(36, x, z, c, circ, truncation.coeff(1e-5), "f64")
    run["expectation"] = g.expectation("0" * 36)
    g.close()
    cb, o = _cpu_propagation(36, x, z, c, circ, {"keep": [("coeff", 1e-5)]}, seconds=args.cpu_seconds)
    if o is not None:  # the CPU engine finished the circuit: its readout beside the device's
        run["cpu_expectation"] = o.expectation("0" * 36)
    run["cpu_baseline"] = cb
    run["workload"] = "config 0: 6x6 TFIM, 5 Trotter steps (540 channels), coeff(1e-5), f64, Heisenberg"
    return run


def config_noisy_tfim6(args):
    """The precision form: the 6 x 6 circuit above with depolarizing p = 1e-3 on every qubit
    after each Trotter step, run in f64 and in f32 with compensated sums; the <O> error in
    |0...0> and the largest coefficient error over the strings both runs keep."""
    import numpy as np

    from paulistrings_b200 import truncation, workloads

    circ = workloads.tfim_2d(6, 5, J=1.0, h=1.0, dt=0.1, noise_p=1e-3)
    x, z, c = _labels(workloads.tfim_magnetization(6, "X"), 36)
    out, states = {}, {}
    for dtype in ("f64", "f32"):
        run, g = _timed_propagation(36, x, z, c, circ, truncation.coeff(1e-5), dtype, compensated=dtype == "f32")
        run["expectation"] = g.expectation("0" * 36)
        states[dtype] = g.download()
        g.close()
        out[dtype] = run
    a, b = states["f64"], states["f32"]
    ka = np.concatenate([a[0], a[1]], axis=1)
    kb = np.concatenate([b[0], b[1]], axis=1)
    va = ka.view([("", ka.dtype)] * ka.shape[1]).ravel()
    vb = kb.view([("", kb.dtype)] * kb.shape[1]).ravel()
    _, ia, ib = np.intersect1d(va, vb, assume_unique=True, return_indices=True)
    e64, e32 = out["f64"]["expectation"], out["f32"]["expectation"]
    return {
        "workload": "config 2: config 0 + depolarizing(1e-3) on every qubit after each step (720 channels), "
        "f64 vs f32 with compensated sums",
        "f64": out["f64"], "f32": out["f32"],
        "abs_error": abs(e32 - e64), "rel_error": abs(e32 - e64) / abs(e64) if e64 else None,
        "terms_f64": int(len(a[2])), "terms_f32": int(len(b[2])), "common_terms": int(len(ia)),
        "max_coeff_abs_error_common": float(np.max(np.abs(a[2][ia] - b[2][ib]))) if len(ia) else 0.0,
        "max_abs_coeff_f64": float(np.max(np.abs(a[2]))) if len(a[2]) else 0.0,
    }


def _max_error(values, ref):
    return float(max(abs(a - b) for a, b in zip(values[1:], ref[1:])))


def _time_to_error(plain, learned):
    """For each plain f64 budget, the error it reached and the cheapest learned run (by wall time)
    whose error is at most that: the learned form's time to the same <O> error and the ratio."""
    out = []
    for b, p in sorted(plain.items()):
        hits = [(r["wall_s"], lb) for lb, r in learned.items() if r["max_error"] <= p["max_error"]]
        row = {"plain_budget_log2": b, "error": p["max_error"], "plain_wall_s": round(p["wall_s"], 4)}
        if hits:
            t, lb = min(hits)
            row.update({"learned_budget_log2": lb, "learned_wall_s": round(t, 4), "ratio": round(p["wall_s"] / t, 3)})
        else:
            row.update({"learned_budget_log2": None, "learned_wall_s": None, "ratio": None})
        out.append(row)
    return out


def config_learned_tfim8(args):
    """Learned truncation against plain TopN on the 8 x 8 periodic TFIM quench (64 qubits):
    observable (1/64) sum X_i, per Trotter step RZZ(-2 J dt) on the 128 bonds (horizontal then
    vertical, row-major) and RX(2 h dt) on every qubit, J = 1, dt = 0.05, 20 steps, <X>(t) read in
    |+...+> after every step (the reference's quench protocol).  Reference: f64 with
    coeff(LEARN_REF_EPS) & TopN(2^LEARN_REF_CAP).  Plain: f64 TopN at 2^20 / 2^22 / 2^24.
    Learned: f32 scored TopN with a scorer trained (on this GPU, by this library's kernels) on
    attribution rows from coeff(LEARN_TRAIN_EPS) runs at h in {0.75, 1.5, 2.5}, at budgets down to
    2^16.  Error: max over t of |<X>(t) - <X>_ref(t)|.  Time to error: for each plain budget, the
    cheapest learned run reaching its error."""
    import numpy as np

    from paulistrings_b200 import learned, truncation, workloads

    L, steps, dt = 8, 20, 0.05
    nq = L * L
    obs = workloads.tfim_magnetization(L, "X")

    def step(h):
        return workloads.tfim_2d(L, 1, J=1.0, h=h, dt=dt)

    sc, losses, rows, t_data, t_train = learned.train_scorer(
        obs, nq, step, (0.75, 1.5, 2.5), steps, "x+", args.learn_train_eps, samples_per_step=args.learn_samples,
        every=4, chunk=256, epochs=40, batch=1024, lr=1e-3)
    result = {
        "workload": "config 3: 8x8 TFIM quench, J=1, dt=0.05, 20 steps (3,840 channels), <X>(t) in |+...+>; plain "
        "f64 TopN vs f32 + learned (scored) TopN",
        "reference": f"f64 coeff({args.learn_ref_eps:g}) & TopN(2^{args.learn_ref_cap})",
        "scorer": {"train_fields": [0.75, 1.5, 2.5], "attribution_threshold": args.learn_train_eps, "rows": rows,
                   "data_s": round(t_data, 2), "train_s": round(t_train, 2),
                   "loss_first_last": [float(losses[0]), float(losses[-1])]},
        "fields": {},
    }
    ref_pol = truncation.coeff(args.learn_ref_eps) & truncation.topn(1 << args.learn_ref_cap)
    for h in args.learn_fields:
        ref = learned.trotter_series(obs, nq, step(h), steps, ref_pol, "f64", "x+")
        plain, scored = {}, {}
        for b in args.learn_plain_budgets:
            r = learned.trotter_series(obs, nq, step(h), steps, truncation.topn(1 << b), "f64", "x+")
            r["max_error"] = _max_error(r["values"], ref["values"])
            plain[b] = r
        for b in args.learn_budgets:
            r = learned.trotter_series(obs, nq, step(h), steps,
                                       truncation.scored_topn(1 << b, sc, rescore_every=args.learn_rescore or len(step(h))),
                                       "f32", "x+")
            r["max_error"] = _max_error(r["values"], ref["values"])
            scored[b] = r
        slim = lambda d: {str(k): {"max_error": v["max_error"], "wall_s": round(v["wall_s"], 4),
                                   "device_ms": round(v["device_ms"], 2), "peak_terms": v["peak_terms"],
                                   "terms_per_s_per_layer": v["terms_in"] / max(1e-9, v["device_ms"] * 1e-3)}
                          for k, v in d.items()}
        result["fields"][str(h)] = {
            "reference": {"wall_s": round(ref["wall_s"], 3), "peak_terms": ref["peak_terms"],
                          "X_final": ref["values"][-1]},
            "plain_f64": slim(plain), "learned_f32": slim(scored),
            "time_to_error": _time_to_error(plain, scored),
        }
    sc.close()
    ratios = [r["ratio"] for f in result["fields"].values() for r in f["time_to_error"] if r["ratio"]]
    result["ratio_median"] = float(np.median(ratios)) if ratios else None
    return result


def config_learned_xxz256(args):
    """Learned truncation on the open XXZ chain, L = 256 (W = 4): observable Z_128, per Trotter
    step RXX(2 dt), RYY(2 dt), RZZ(2 Jz dt) on every bond, even bonds then odd (the reference's
    examples/common/circuits.py:326-338), Jz = 0.5, dt = 0.1, read out in the Neel state
    |0101...> after every step.  Plain: f64 TopN at 2^XXZ_BUDGET.  Learned: f32 scored TopN with
    the config-3 architecture retrained on attribution rows of the L = 64 chain (observable Z_32)
    and applied to L = 256 through a site map (a 64-site window centred on the observable's site,
    the sites beyond it clamped to the window's edge rows).  Error: against a plain f64 run at
    4x the budget (the tightest this measurement affords)."""
    import numpy as np

    from paulistrings_b200 import learned, truncation, workloads

    L, steps, dt, jz = 256, args.xxz_steps, 0.1, 0.5
    obs = {"I" * 128 + "Z" + "I" * 127: 1.0}
    state = workloads.neel_state(L)
    step = workloads.xxz_chain(L, 1, Jz=jz, dt=dt)
    # scorer: attribution rows of the 64-site chain
    obs64 = {"I" * 32 + "Z" + "I" * 31: 1.0}
    sc, losses, rows, t_data, t_train = learned.train_scorer(
        obs64, 64, lambda _h: workloads.xxz_chain(64, 1, Jz=jz, dt=dt), (jz,), steps, workloads.neel_state(64),
        args.learn_train_eps, samples_per_step=args.xxz_samples, every=5, chunk=256, epochs=40, batch=1024,
        lr=1e-3)
    sc.set_site_map(np.clip(np.arange(L) - 128 + 32, 0, 63))
    b = args.xxz_budget
    ref = learned.trotter_series(obs, L, step, steps, truncation.topn(1 << (b + 2)), "f64", state)
    plain = learned.trotter_series(obs, L, step, steps, truncation.topn(1 << b), "f64", state)
    runs = {"plain_f64": {b: plain}, "learned_f32": {}}
    for lb in (b - 2, b):
        runs["learned_f32"][lb] = learned.trotter_series(
            obs, L, step, steps, truncation.scored_topn(1 << lb, sc, rescore_every=args.learn_rescore or len(step)), "f32",
            state)
    sc.close()
    out = {
        "workload": f"config 4: open XXZ chain L=256, Jz=0.5, dt=0.1, {steps} steps ({765 * steps} channels), Z_128 "
        "in the Neel state; plain f64 TopN vs f32 + learned (scored) TopN",
        "reference": f"f64 TopN(2^{b + 2})",
        "scorer": {"trained_on": "XXZ L=64, Z_32", "attribution_threshold": args.learn_train_eps, "rows": rows,
                   "data_s": round(t_data, 2), "train_s": round(t_train, 2),
                   "site_map": "sites 96..159 -> rows 0..63, beyond clamped to the edge rows",
                   "loss_first_last": [float(losses[0]), float(losses[-1])]},
        "reference_run": {"wall_s": round(ref["wall_s"], 3), "peak_terms": ref["peak_terms"],
                          "Z_final": ref["values"][-1], "layers_skipped": ref["layers_skipped"]},
    }
    for form, d in runs.items():
        out[form] = {}
        for k, r in d.items():
            r["max_error"] = _max_error(r["values"], ref["values"])
            out[form][str(k)] = {"max_error": r["max_error"], "wall_s": round(r["wall_s"], 3),
                                 "device_ms": round(r["device_ms"], 1), "peak_terms": r["peak_terms"],
                                 "layers_skipped": r["layers_skipped"],
                                 "terms_per_s_per_layer": r["terms_in"] / max(1e-9, r["device_ms"] * 1e-3)}
    out["time_to_error"] = _time_to_error(runs["plain_f64"], runs["learned_f32"])
    return out


CONFIGS = {"tfim6": config_tfim6, "noisy": config_noisy_tfim6, "learned": config_learned_tfim8,
           "xxz": config_learned_xxz256}


def run_configs(args):
    out = {}
    for name in [c for c in args.configs.split(",") if c and c != "none"]:
        t0 = time.perf_counter()
        try:
            out[name] = CONFIGS[name](args)
        except Exception as exc:  # one failed configuration must not hide the others' numbers
            out[name] = {"error": f"{type(exc).__name__}: {exc}"}
        out[name]["bench_s"] = round(time.perf_counter() - t0, 1)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--term-cap", type=int, default=TERM_CAP,
                    help="TopN cap; smaller values give the small cases profiled under ncu")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--configs", default="tfim6,noisy,learned,xxz",
                    help="the other configurations measured after the headline (comma list of "
                         f"{','.join(CONFIGS)}; 'none' for the headline alone)")
    ap.add_argument("--configs-only", action="store_true", help="print only the configurations' object")
    # the learned comparisons: config 3's fields and plain budgets, the learned form from 2^16 up;
    # config 4 at 50 steps and 2^20 terms against a 2^22 reference (--xxz-budget 22: about five
    # minutes; the 2^28 budget of its definition: --xxz-budget 28, much longer)
    ap.add_argument("--learn-fields", type=float, nargs="+", default=[0.5, 1.0, 2.0, 3.0])
    ap.add_argument("--learn-plain-budgets", type=int, nargs="+", default=[20, 22, 24], help="log2 TopN budgets")
    ap.add_argument("--learn-budgets", type=int, nargs="+", default=[16, 18, 20, 22],
                    help="log2 budgets of the learned form")
    ap.add_argument("--learn-ref-eps", type=float, default=1e-7)
    ap.add_argument("--learn-ref-cap", type=int, default=28, help="log2 TopN cap of the reference run")
    ap.add_argument("--learn-train-eps", type=float, default=1e-5, help="threshold of the attribution runs")
    ap.add_argument("--learn-samples", type=int, default=1024, help="attribution samples per step boundary")
    ap.add_argument("--learn-rescore", type=int, default=0,
                    help="layers between the learned pass's fresh predictions (0: one Trotter step)")
    ap.add_argument("--xxz-budget", type=int, default=20, help="log2 TopN budget of the L=256 XXZ comparison")
    ap.add_argument("--xxz-steps", type=int, default=50)
    ap.add_argument("--xxz-samples", type=int, default=256,
                    help="attribution samples per step boundary of the L=64 XXZ training runs")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("at least 3 warm-up steps")
    if args.configs_only:
        print(json.dumps({"configs": run_configs(args)}))
        return
    world, rank, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
