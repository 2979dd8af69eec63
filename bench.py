#!/usr/bin/env python
"""Benchmark of the Heisenberg-picture PauliSum path on B200.

Metric: term-gate updates/s = sum over the gates of a circuit of the live terms entering
each gate (reference semantics: merge after every gate, truncate at the list's TRUNCATE ops),
divided by the time.  A step is one complete propagation of the observable through the
workload's gate list plus the <O> readout.

Workloads of one sum (synthetic inputs: the circuits are generated):
  kicked_ising_2d (default)  open 12x12 lattice, 20 layers, RX(0.6) on every qubit then
                             RZZ(-pi/2) on all 264 bonds per layer, observable Z at (6,6),
                             |c| < 1e-5 truncation and weight cap 10
  tfim_1d                    open chain, n=20, J=h=1, dt=0.1, 10 Trotter steps, obs Z(10),
                             |c| < 1e-4
  clifford_t                 the first 26 Heisenberg layers of the random Clifford+T
                             brickwork (n=64, 1000 layers, seed 0, T = RZ(pi/4) with p=0.05),
                             |c| < 1e-6; the full depth outgrows any memory

Arms:
  default           the CUDA engine through its C ABI (ppvm_b200.PauliSum)
  --impl reference  the CPU restatement of the reference PauliSum (oracle/) in the
                    reference's multi-threaded configuration (DashMap + rayon, restated with a
                    pool of host threads) on every host core: one propagation of the same
                    full workload per step (rank 0 only)

Multi-GPU (torchrun): every rank propagates its own replica of the circuit (the path has
no cross-sum exchange at one sum per GPU); value = all ranks' updates / max rank time.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from ppvm_b200 import circuits as C  # noqa: E402
from ppvm_b200 import gates as G  # noqa: E402

METRIC = "term-gate updates/s"
L2_NOTE = "flushed between steps (256 MB write)"
SINGLE_SUM = ("kicked_ising_2d", "tfim_1d", "clifford_t")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ppvm_b200", choices=["ppvm_b200", "reference"])
    ap.add_argument("--layers", type=int, default=20, help="kicked_ising_2d: layers of the circuit")
    ap.add_argument("--workload", default="kicked_ising_2d",
                    choices=[*SINGLE_SUM, "batched_tfim", "learned_kicked_ising", "layer_bandwidth",
                             "kernel_families"],
                    help="kicked_ising_2d: one 12x12 sum (headline); tfim_1d: one 20-qubit TFIM chain; "
                         "clifford_t: the first 26 layers of the n=64 Clifford+T brickwork; "
                         "batched_tfim: 256 independent 1D TFIM "
                         "instances through the batched engine; learned_kicked_ising: time to <O> within 1e-3 "
                         "with learned vs plain term-budget truncation on a 10x10 kicked-Ising circuit; "
                         "layer_bandwidth: the 12x12 circuit at --thr/--max-weight, one line per layer with "
                         "each kernel family's time and algorithmic bandwidth (sums larger than L2); "
                         "kernel_families: one op per kernel family on a copy of a sum larger than L2")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--thr", type=float, default=1e-7, help="layer_bandwidth: coefficient threshold")
    ap.add_argument("--max-weight", type=int, default=12, help="layer_bandwidth: weight cap")
    ap.add_argument("--stop-terms", type=float, default=4e7, help="layer_bandwidth: stop past this many terms")
    ap.add_argument("--family-terms", type=float, default=3e6,
                    help="kernel_families: grow the sums past this many terms")
    return ap.parse_args()


def workload(name: str = "kicked_ising_2d", layers: int = 20) -> C.Workload:
    """The single-sum workload ``name`` (``layers``: kicked-Ising layers)."""
    if name == "tfim_1d":
        return C.tfim_1d(n=20, J=1.0, h=1.0, dt=0.1, steps=10, thr=1e-4)
    if name == "clifford_t":
        return C.clifford_t(n=64, layers=1000, seed=0, p_t=0.05, thr=1e-6, heisenberg_layers=26)
    return C.kicked_ising_2d(L=12, layers=layers, theta_h=0.6, thr=1e-5, max_weight=10)


def describe(wl: C.Workload) -> str:
    if wl.name.startswith("tfim1d"):
        m = wl.meta
        return (f"tfim_1d open chain, n={wl.n_qubits}, J={m['J']}, h={m['h']}, dt={m['dt']}, {m['steps']} Trotter "
                f"steps, obs Z({wl.n_qubits // 2}), thr {wl.min_abs_coeff:g}, no weight cap")
    if wl.name.startswith("clifford_t"):
        m = wl.meta
        return (f"clifford_t n={wl.n_qubits} brickwork ({m['layers']} layers, seed {m['seed']}, T = RZ(pi/4) "
                f"with p=0.05): its first {m['heisenberg_layers']} Heisenberg layers, random weight-4 observable, "
                f"thr {wl.min_abs_coeff:g}, no weight cap")
    return (f"kicked_ising_2d 12x12 open lattice, {wl.meta['layers']} layers, RX(0.6) + RZZ(-pi/2) on 264 bonds, "
            f"obs Z(6,6), thr 1e-5, weight cap 10")


def config_dict(wl, n_gpus):
    """The workload's description, the same in both arms' lines."""
    return {"workload": describe(wl), "n_qubits": wl.n_qubits, "gates_per_step": wl.n_gates,
            "layers": wl.meta.get("heisenberg_layers", wl.meta.get("layers", wl.meta.get("steps"))),
            "parallelism": f"replicas x{n_gpus}" if n_gpus > 1 else "single sum", "l2": L2_NOTE}


# ---------------------------------------------------------------------------------------------
def oracle_run(wl, threads=None):
    """One propagation on the oracle: the IndexMap configuration on one thread (threads None),
    or the DashMap configuration on ``threads`` host threads (0: all).  Returns (term-gate
    updates, seconds, <O>, peak live terms)."""
    from oracle.pyoracle import OracleSum

    o = OracleSum(wl.n_qubits, wl.min_abs_coeff, wl.max_weight, wl.clifford_angles, threads=threads)
    x, z = G.parse_word(wl.observable[0][0], wl.n_qubits)
    o.add_terms(x[None], z[None], np.array([wl.observable[0][1]]))
    t = time.perf_counter()
    cnt = o.run_ops(wl.ops, counts=True)
    val = o.overlap_with_zero()
    dt = time.perf_counter() - t
    return C.term_gate_updates(cnt, wl.ops), dt, val, max(int(cnt.max()), len(o))


# Single-thread CPU samples: the whole workload, except for clifford_t, whose single-thread
# propagation takes minutes; there the sample is its first 24 layers (a tenth of the updates).
CPU_SAMPLE_LAYERS = {"clifford_t": 24}


def cpu_baseline(name, layers):
    """The IndexMap oracle (the reference's Python-binding configuration), one thread."""
    sub = CPU_SAMPLE_LAYERS.get(name)
    wl = workload(name, layers)
    if sub is not None:
        wl = C.clifford_t(n=64, layers=1000, seed=0, p_t=0.05, thr=1e-6, heisenberg_layers=sub)
    tgu, dt, val, peak = oracle_run(wl)
    what = "the whole workload" if sub is None else f"the first {sub} Heisenberg layers of the workload"
    return ({"value": tgu / dt, "unit": METRIC, "cores": 1, "kind": "port",
             "sample": f"{what}, one propagation, single-thread C++ restatement of the reference's IndexMap "
                       f"PauliSum ({dt:.1f} s)"},
            None if sub is not None else {"term_gate_updates_per_step": tgu, "expectation": val,
                                          "peak_live_terms": peak})


def cpu_all_cores(name, layers):
    """The DashMap oracle (the reference's multi-threaded configuration) on every host core."""
    threads = os.cpu_count() or 1
    tgu, dt, val, peak = oracle_run(workload(name, layers), threads=threads)
    return ({"value": tgu / dt, "unit": METRIC, "cores": threads, "kind": "port",
             "sample": f"the whole workload, one propagation, C++ restatement of the reference's DashMap + rayon "
                       f"PauliSum on {threads} host threads ({dt:.1f} s)"},
            {"term_gate_updates_per_step": tgu, "expectation": val, "peak_live_terms": peak})


def flush_host_caches(buf):
    """Writes a 256 MB host buffer: the CPU's caches hold nothing of the previous step."""
    buf += 1


def run_reference(args):
    """The reference arm: the oracle in the reference's DashMap configuration on every host
    thread.  A step is one propagation of the full workload (the GPU arm's step); value = the
    steps' term-gate updates / their summed wall time.  Host caches are flushed between steps."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    wl = workload(args.workload, args.layers)
    threads = os.cpu_count() or 1
    buf = np.zeros(256 * 1024 * 1024 // 8, dtype=np.float64)
    res = None
    for _ in range(args.warmup):
        flush_host_caches(buf)
        oracle_run(wl, threads=threads)
    tot_u, tot_t = 0, 0.0
    for _ in range(args.steps):
        flush_host_caches(buf)
        u, dt, val, peak = oracle_run(wl, threads=threads)
        tot_u += u
        tot_t += dt
        res = {"term_gate_updates_per_step": u, "expectation": val, "peak_live_terms": peak}
    v = tot_u / tot_t
    sample = (f"per step, one propagation of the whole workload by the C++ restatement of the reference's "
              f"DashMap + rayon PauliSum on {threads} host threads")
    line = {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (generated circuit)", "config": config_dict(wl, 1), "result": res,
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------------
class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region, every 20 ms, through
    NVML in this process (the library nvidia-smi reads them with): the SM clock, its maximum
    and the clock-event reason bits, nothing else.  NVML is initialised before the warm-up.
    Spawning nvidia-smi during the timed region stalled the GPU for milliseconds; an NVML
    clock read does not.  Without NVML, one nvidia-smi process looping every 100 ms (-lms)."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.times = []
        self._p = None
        self._nvml = None
        self._stop = threading.Event()
        self._first = threading.Event()
        self._t = threading.Thread(target=self._loop, daemon=True)

    def _nvml_handle(self):
        import pynvml as nv

        nv.nvmlInit()
        try:  # the CUDA device's own GPU: NVML may number GPUs differently from CUDA
            import torch

            pr = torch.cuda.get_device_properties(self.index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return nv, nv.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return nv, nv.nvmlDeviceGetHandleByIndex(self.index)

    def _loop(self):
        if self._nvml is not None:
            nv, h = self._nvml
            bits = [nv.nvmlClocksEventReasonHwSlowdown, nv.nvmlClocksEventReasonHwThermalSlowdown,
                    nv.nvmlClocksEventReasonSwThermalSlowdown, nv.nvmlClocksEventReasonSwPowerCap]
            while not self._stop.is_set():
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    mx = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
                    rs = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    flags = ["Active" if rs & b else "Not Active" for b in bits]
                    self.rows.append([str(self.index), str(sm), str(mx), "", hex(rs)] + flags)
                    self.times.append(time.perf_counter())
                except Exception:
                    pass
                self._first.set()
                self._stop.wait(0.02)
            return
        for line in self._p.stdout:
            line = line.strip()
            if line:
                self.rows.append([c.strip() for c in line.split(",")])
                self.times.append(time.perf_counter())
                self._first.set()

    def window(self, t0: float, t1: float) -> None:
        """Keeps the samples taken in [t0, t1] (or the one nearest to it if none was)."""
        keep = [i for i, t in enumerate(self.times) if t0 <= t <= t1]
        if not keep and self.times:
            keep = [min(range(len(self.times)), key=lambda i: min(abs(self.times[i] - t0), abs(self.times[i] - t1)))]
        self.rows = [self.rows[i] for i in keep]

    def __enter__(self):
        try:
            self._nvml = self._nvml_handle()
        except Exception:
            self._nvml = None
            try:
                self._p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                            "--format=csv,noheader,nounits", "-lms", "100"],
                                           stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            except OSError:
                return self  # neither NVML nor nvidia-smi: summary() reports the clocks as unavailable
        self._t.start()
        self._first.wait(timeout=10)  # the first query, and its stall, before anything is timed
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._nvml is not None:
            self._t.join(timeout=10)
        if self._p is not None:
            self._p.terminate()  # the process this sampler started
            try:
                self._p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self._p.kill()
            self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[j] for r in self.rows for j in range(4) if len(r) > 5 + j and r[5 + j] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def over_ranks(values, device, op: str = "max") -> list[float]:
    """The elementwise max (or sum) of ``values`` over all ranks; the values themselves on one
    rank.  ``device`` is the rank's CUDA device under NCCL, the CPU under gloo."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()]


def batched_shard_seed(rank: int) -> int:
    """Rank r of the batched workload propagates the 256 instances of seed 1 + r: the ranks'
    shards are independent instances, and rank 0's shard is the single-GPU batch."""
    return 1 + rank


# DRAM bytes (read + write) per launch of the dominant kernel, per workload: the mean over the
# kernel's launches in one step, from an ncu capture of this code (dram__bytes_read.sum +
# dram__bytes_write.sum of every launch of the kernel in the step).  Filled from a capture of
# the current kernels; a workload or kernel without an entry reports null.
CAPTURED_TRAFFIC: dict = {
    "kicked_ising_2d": {"run_groups": 66548 + 402, "tableau": 237986 + 0},          # 21 and 19 launches
    "clifford_t": {"run_groups": 7685530 + 5397443, "tableau": 8022518 + 3209472},  # 25 and 25 launches
}
TRAFFIC_SOURCE = ("ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none over one step "
                  "of this workload (every launch of the kernel), mean per launch")


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def one_instance_batch(wl, steps, warmup, updates):
    """The same workload through the batched engine as its only instance: one CTA holds the
    whole sum in shared memory and runs the whole gate list in one launch
    (ppvm_batch_run_persistent).  For sums of a few thousand terms this avoids the per-gate
    launches and L2 round trips of the single-sum engine."""
    import torch

    from ppvm_b200.batch import Instance, PauliSumBatch
    from ppvm_b200.paulisum import ops_array

    inst = [Instance(wl.n_qubits, list(wl.observable), ops_array(wl.ops), wl.min_abs_coeff, wl.max_weight)]
    b = PauliSumBatch(inst)
    stream = torch.cuda.current_stream()
    b.set_stream(stream.cuda_stream)
    for _ in range(max(warmup, 3)):
        b.run_persistent()
        b.overlap_with_zero()
    _, tgu = b.term_gate_updates()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    torch.cuda.synchronize()
    for i in range(steps):
        flush.fill_(float(i))
        ev[i][0].record(stream)
        b.run_persistent()
        b.overlap_with_zero()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    dev_s = sum(a.elapsed_time(c) for a, c in ev) / 1e3
    e2e_s = 0.0
    for i in range(steps):  # a new batch from the host circuit each step, <O> read back
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t = time.perf_counter()
        b2 = PauliSumBatch(inst)
        b2.run_persistent()
        b2.overlap_with_zero()
        e2e_s += time.perf_counter() - t
        del b2
    return {"engine": "PauliSumBatch with one instance, resident in shared memory, one launch per step",
            "value": tgu * steps / dev_s, "unit": METRIC, "ms_per_step": 1e3 * dev_s / steps,
            "e2e": {"value": tgu * steps / e2e_s, "ms_per_step": 1e3 * e2e_s / steps},
            "term_gate_updates_per_step": tgu, "updates_equal": tgu == updates}


def run_gpu(args):
    import torch
    import torch.distributed as dist

    from ppvm_b200.paulisum import PauliSum, ops_array

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    wl = workload(args.workload, args.layers)
    obs_word, obs_c = wl.observable[0]

    def make(capacity=0):
        s = PauliSum([obs_word], wl.n_qubits, [obs_c], min_abs_coeff=wl.min_abs_coeff,
                     max_pauli_weight=wl.max_weight, clifford_angles=wl.clifford_angles, device=local,
                     capacity=capacity)
        s.set_stream(stream.cuda_stream)
        return s

    clk = ClockSampler(local)  # started before the warm-up: its first query is not in the timed region
    clk.__enter__()
    # warm-up: also learns the peak live count so timed steps never grow storage
    peak = 0
    for _ in range(max(args.warmup, 1)):
        s = make(peak * 2)
        s.run(wl.ops)
        s.overlap_with_zero()
        counts = s.live_counts()
        peak = max(peak, int(counts.max()), len(s))
        del s
    updates = C.term_gate_updates(counts, wl.ops)
    cap = max(4 * peak, 1 << 16)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    # ---- device-resident timing: inputs already in HBM (sums created up front) -----------
    gate_list = ops_array(wl.ops)  # the circuit, packed once as ppvm_op records
    # warm-up, continued: a sum's handle sizes its op log and upload arena on its first run
    # (allocations that synchronise), and destroyed sums leave their handles to the library's
    # cache.  So every handle the timed steps will use runs the circuit once here.
    warm = [make(cap) for _ in range(args.steps)]
    for s in warm:
        s.run(gate_list)
        s.overlap_with_zero()
    del warm, s

    def timed_pass(per_launch_events: bool):
        sums = [make(cap) for _ in range(args.steps)]
        for s in sums:
            s.profile(per_launch_events)
        l0 = sum(s.launch_count() for s in sums)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        res = []
        tw0 = time.perf_counter()
        for i, s in enumerate(sums):
            flush.fill_(float(i))
            ev[i][0].record(stream)
            s.run(gate_list)
            res.append(s.overlap_with_zero())
            ev[i][1].record(stream)
        torch.cuda.synchronize()
        tw1 = time.perf_counter()
        if world > 1:
            dist.barrier()
        prof = {}
        for s in sums:
            for k, v in s.profile_read().items():
                p = prof.setdefault(k, {"ms": 0.0, "launches": 0, "bytes": 0})
                p["ms"] += v["ms"]
                p["launches"] += v["launches"]
                p["bytes"] += v["bytes"]
        nl = sum(s.launch_count() for s in sums) - l0
        del sums
        return sum(a.elapsed_time(b) for a, b in ev) / 1e3, res, prof, nl, tw0, tw1

    # pass 1 (`value`): no per-launch events; pass 2: the same steps with CUDA events around
    # every launch, for the per-kernel breakdown and the roofline
    dev_s, results, _, launches, t0_wall, t1_wall = timed_pass(False)
    t_wall = t1_wall - t0_wall
    clk.__exit__(None, None, None)
    clk.window(t0_wall, t1_wall)
    prof_s, _, prof, _, _, _ = timed_pass(True)

    # ---- end to end through the public API with host buffers ---------------------------------
    e2e_ms = []
    h2d = d2h = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    for i in range(args.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t = time.perf_counter()
        s = make(cap)  # host observable -> device
        s.run(gate_list)  # the packed host gate list -> device, live-count log back
        v = s.overlap_with_zero()  # result back to host
        e2e_ms.append(1e3 * (time.perf_counter() - t))
        h2d, d2h = s.transfer_counters()  # bytes this step copied each way
        del s
    e2e_s = sum(e2e_ms) / 1e3

    # ---- max over ranks (each rank propagates a replica of the sum) ----------------------------
    dev_s, e2e_s = over_ranks([dev_s, e2e_s], dev, "max")
    total_updates = updates * args.steps * world
    value = total_updates / dev_s
    e2e_value = total_updates / e2e_s

    if rank == 0:
        peak_gbs, peak_kind = measured_peak()
        fams = {k: v for k, v in prof.items() if v["launches"]}
        dom = max(fams, key=lambda k: fams[k]["ms"]) if fams else None
        roof = None
        if dom:
            d = fams[dom]
            achieved = d["bytes"] / (d["ms"] / 1e3) / 1e9
            roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
                    "frac": achieved / peak_gbs, "peak_kind": peak_kind,
                    "traffic": CAPTURED_TRAFFIC.get(args.workload, {}).get(dom),
                    "traffic_source": TRAFFIC_SOURCE if dom in CAPTURED_TRAFFIC.get(args.workload, {}) else None,
                    "bytes_per_launch": d["bytes"] / d["launches"],
                    "avg_launch_us": 1e3 * d["ms"] / d["launches"],
                    "share_of_device_time": d["ms"] / (1e3 * prof_s) if prof_s else None,
                    "timing": "per-launch CUDA events on the sum's stream, in a second timed pass of the same steps "
                              f"({1e3 * prof_s / args.steps:.3f} ms per step with the events)"}
        result = {"peak_live_terms": peak, "term_gate_updates_per_step": updates, "expectation": results[-1]}
        line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated circuit)",
                "config": config_dict(wl, world),
                "result": result,
                "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                        "ms_per_step": 1e3 * e2e_s / args.steps,
                        "per_step": "sum created from the host observable string, the host gate list (ppvm_op "
                                    "records, packed once from Python tuples before timing) uploaded and run, "
                                    "the per-op log and <O> read back"},
                "gpu_launches": launches,
                "roofline": roof,
                "kernel_breakdown": {k: {"ms": round(v["ms"], 3), "launches": v["launches"], "bytes": v["bytes"]}
                                     for k, v in fams.items()},
                "clocks": clk.summary(),
                "wall_s_timed_region": t_wall}
        if world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"], one = cpu_baseline(args.workload, args.layers)
            line["cpu_baseline_all_cores"], allc = cpu_all_cores(args.workload, args.layers)
            # the oracle's figures for the same workload: the term-gate updates and the live
            # peak must be equal, <O> within 1e-10
            ref = one or allc
            line["parity_vs_oracle"] = {
                "updates_equal": ref["term_gate_updates_per_step"] == updates,
                "peak_equal": ref["peak_live_terms"] == peak,
                "expectation_abs_diff": abs(ref["expectation"] - results[-1]),
                "oracle_expectation": ref["expectation"]}
        if world == 1 and args.workload == "tfim_1d":
            line["one_instance_batch"] = one_instance_batch(wl, args.steps, args.warmup, updates)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


BATCH_CPU_SAMPLE = 64  # instances of the batched workload timed on the host CPU
_WORKER_CACHE = {}  # per spawned process: the batched circuits, built once outside the timed rounds


def _batched_circuits():
    if "batched" not in _WORKER_CACHE:
        _WORKER_CACHE["batched"] = C.batched_tfim()
    return _WORKER_CACHE["batched"]


def _cpu_batch_worker(idx):
    """The oracle over the given instances of the batched workload (spawned process)."""
    wls = _batched_circuits()
    return batched_cpu([wls[i] for i in idx])


def _warm_worker(_):
    """Builds a worker's circuits before the timed rounds."""
    _batched_circuits()
    return 0


def cpu_map_all_cores(fn, tasks):
    """Runs fn over tasks on every host core (spawned processes: none inherits a CUDA context).
    Returns (sum of term-gate updates, wall seconds of the parallel map, workers)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    cores = max(1, min(len(tasks), os.cpu_count() or 1))
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_warm_worker, range(cores)))  # start the workers outside the timed map
        t = time.perf_counter()
        out = list(ex.map(fn, tasks))
        dt = time.perf_counter() - t
    return sum(u for u, _ in out), dt, cores


def batched_config(n_inst, world):
    """The batched workload's description, the same in both arms' lines."""
    return {"workload": f"batched_tfim: {n_inst} independent 1D TFIM instances (seed 1), n ~ U[16,128], "
                        "steps ~ U[5,30], h ~ U[0.5,1.5], J=1, dt=0.05, obs Z(n/2), thr 1e-5",
            "instances": n_inst,
            "parallelism": (f"{world} shards of {n_inst} instances: rank r holds seed 1 + r" if world > 1
                            else "one batch"),
            "l2": L2_NOTE}


def batched_cpu(wls):
    from oracle.pyoracle import OracleSum

    t0 = time.perf_counter()
    tgu = 0
    for w in wls:
        o = OracleSum(w.n_qubits, w.min_abs_coeff, w.max_weight)
        x, z = G.parse_word(w.observable[0][0], w.n_qubits)
        o.add_terms(x[None], z[None], np.array([w.observable[0][1]]))
        tgu += C.term_gate_updates(o.run_ops(w.ops, counts=True), w.ops)
        o.overlap_with_zero()
    return tgu, time.perf_counter() - t0


def run_batched_reference(args):
    """The batched reference arm: the oracle over all 256 instances per step, the instances
    spread over every host core (spawned processes, each single-threaded)."""
    import concurrent.futures as cf
    import multiprocessing as mp

    if int(os.environ.get("RANK", "0")) != 0:
        return
    n = len(C.batched_tfim())
    cores = max(1, min(n, os.cpu_count() or 1))
    chunks = [list(range(i, n, cores)) for i in range(cores)]
    tot_u, tot_t = 0, 0.0
    buf = np.zeros(256 * 1024 * 1024 // 8, dtype=np.float64)
    with cf.ProcessPoolExecutor(max_workers=cores, mp_context=mp.get_context("spawn")) as ex:
        list(ex.map(_warm_worker, range(4 * cores)))  # workers started, circuits built
        for _ in range(args.warmup):
            list(ex.map(_cpu_batch_worker, chunks))
        for _ in range(args.steps):
            flush_host_caches(buf)
            t = time.perf_counter()
            out = list(ex.map(_cpu_batch_worker, chunks))
            tot_t += time.perf_counter() - t
            tot_u += sum(u for u, _ in out)
    v = tot_u / tot_t
    line = {"metric": METRIC, "value": v, "unit": METRIC, "impl": "reference", "n_gpus": 0, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (generated circuits)",
            "config": batched_config(n, 1), "result": {"term_gate_updates_per_step": tot_u // max(args.steps, 1)},
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": cores, "kind": "port",
                             "sample": f"all {n} instances per step over {cores} spawned single-thread processes"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_batched(args):
    import torch
    import torch.distributed as dist

    from ppvm_b200.batch import PauliSumBatch
    from ppvm_b200.paulisum import PauliSum

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    wls = C.batched_tfim(seed=batched_shard_seed(rank))
    b = PauliSumBatch.from_workloads(wls, device=local)
    b.set_stream(stream.cuda_stream)
    clk = ClockSampler(local)  # started before the warm-up: its first query is not in the timed region
    clk.__enter__()
    tune = b.autotune()  # warm-up: sizes every region, captures the layer graphs, picks the launch config
    for _ in range(max(args.warmup, 1)):
        b.run()
    per, tgu = b.term_gate_updates()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0_wall = time.perf_counter()
    for i in range(args.steps):
        flush.fill_(float(i))
        ev[i][0].record(stream)
        b.run()
        owz = b.overlap_with_zero()
        ev[i][1].record(stream)
    torch.cuda.synchronize()
    clk.__exit__(None, None, None)
    clk.window(t0_wall, time.perf_counter())
    dev_s = sum(a.elapsed_time(c) for a, c in ev) / 1e3
    # end to end: a new batch from the host circuits (each gate list packed once as ppvm_op
    # records, as a serving caller holds its circuits), run, <O> of every instance read back
    from ppvm_b200.batch import Instance
    from ppvm_b200.paulisum import ops_array

    packed = [Instance(w.n_qubits, list(w.observable), ops_array(w.ops), w.min_abs_coeff, w.max_weight) for w in wls]
    caps = b.capacities()
    e2e_s = 0.0
    h2d = d2h = 0
    for i in range(args.steps):
        flush.fill_(float(i))
        torch.cuda.synchronize()
        t = time.perf_counter()
        b2 = PauliSumBatch(packed, device=local, capacity=caps)
        b2.set_config(tune["block"], tune["items"], tune["table_factor"])
        b2.run()
        b2.overlap_with_zero()
        e2e_s += time.perf_counter() - t
        h2d, d2h = b2.transfer_counters()
        del b2
    # the same instances one after another through the plain single-sum engine
    seq = None
    if rank == 0 and not args.no_cpu_baseline:
        t = time.perf_counter()
        for w in wls:
            s = PauliSum([w.observable[0][0]], w.n_qubits, [1.0], min_abs_coeff=w.min_abs_coeff, device=local)
            s.run(w.ops)
            s.overlap_with_zero()
        seq_s = time.perf_counter() - t
        seq = {"value": tgu / seq_s, "unit": METRIC, "ms_to_all_O": 1e3 * seq_s,
               "what": "the 256 instances one after another through the plain single-sum engine (PauliSum)"}
    # each rank propagates its own shard of instances: the job's updates are the sum over ranks,
    # its time the max
    dev_s, e2e_s = over_ranks([dev_s, e2e_s], dev, "max")
    tgu_job = int(over_ranks([tgu], dev, "sum")[0])
    if rank == 0:
        peak_gbs, peak_kind = measured_peak()
        # algorithmic bytes: every term-gate update reads the X and Z word holding the gate's qubit
        achieved = 16.0 * tgu * args.steps / dev_s / 1e9
        line = {"metric": METRIC, "value": tgu_job * args.steps / dev_s, "unit": METRIC, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_s / args.steps,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (generated circuits)",
                "config": batched_config(len(wls), world),
                "result": {"term_gate_updates_per_step": tgu, "launch_config": tune,
                           "max_live_terms": int(max(b.len_of(j) for j in range(len(wls))))},
                "e2e": {"value": tgu_job * args.steps / e2e_s, "unit": METRIC, "h2d_bytes_per_step": h2d,
                        "d2h_bytes_per_step": d2h, "ms_per_step": 1e3 * e2e_s / args.steps},
                "time_to_all_O_ms": 1e3 * dev_s / args.steps,
                "sequential_plain_gpu": seq,
                "gpu_launches": (max(w.meta["steps"] for w in wls) + 1 + 1) * args.steps,
                "roofline": {"bound": "latency", "kernel": "k_batch", "achieved": achieved, "peak": peak_gbs,
                             "unit": "GB/s", "frac": achieved / peak_gbs, "peak_kind": peak_kind, "traffic": None,
                             "note": "16 B per term-gate update; one CTA per instance, the largest instance sets the time"},
                "clocks": clk.summary()}
        if world == 1 and not args.no_cpu_baseline:
            u, dt = batched_cpu(wls[:BATCH_CPU_SAMPLE])
            line["cpu_baseline"] = {"value": u / dt, "unit": METRIC, "cores": 1, "kind": "port",
                                    "sample": f"first {BATCH_CPU_SAMPLE} of the 256 instances, single-thread C++ "
                                              f"restatement of the reference PauliSum ({dt:.1f} s)"}
            ncores = os.cpu_count() or 1
            chunks = [list(range(i, len(wls), ncores)) for i in range(min(ncores, len(wls)))]
            u, dt, used = cpu_map_all_cores(_cpu_batch_worker, chunks)
            line["cpu_baseline_all_cores"] = {"value": u / dt, "unit": METRIC, "cores": used, "kind": "port",
                                              "ms_to_all_O": 1e3 * dt,
                                              "sample": f"all 256 instances over {used} spawned processes"}
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_learned(args):
    """Time to <O> at |err| <= 1e-3: learned vs plain term-budget truncation (one GPU)."""
    import torch

    from ppvm_b200 import learned

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if rank != 0:
        return
    torch.cuda.set_device(local)
    res = learned.compare_budgets(device=local)  # training set, training, reference, one pass per budget
    # the timed passes: every (budget, kind) again, args.steps times each, median kept
    wl = C.kicked_ising_random_h(L=10, layers=4, seed=2, thr=1e-7)
    net = res.pop("net")
    for r in res["rows"]:
        ts = []
        for _ in range(args.steps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            learned.run_with_budget(wl, r["budget"], net if r["kind"] == "learned" else None, 10, device=local)
            ts.append(time.perf_counter() - t)
        r["s"] = statistics.median(ts)
    ok = {k: [r for r in res["rows"] if r["kind"] == k and r["err"] <= 1e-3] for k in ("plain", "learned")}
    best = {k: (min(v, key=lambda r: r["s"]) if v else None) for k, v in ok.items()}
    ref_t = []
    for _ in range(args.steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        learned.run_with_budget(wl, None, device=local)
        ref_t.append(time.perf_counter() - t)
    val = best["learned"]["s"] if best["learned"] else None
    ref_s = statistics.median(ref_t)

    def at_tolerance(tol):  # fastest run of each kind within tol; the unbudgeted run always is
        out = {}
        for k in ("plain", "learned"):
            within = [r for r in res["rows"] if r["kind"] == k and r["err"] <= tol and r["budget"] < 1_000_000]
            r = min(within, key=lambda r: r["s"]) if within else None
            out[k] = {"budget": r["budget"], "s": r["s"], "err": r["err"]} if r else {"budget": None, "s": ref_s,
                                                                                    "err": 0.0}
        return out
    line = {"metric": "time to <O> at |err|<=1e-3", "value": val, "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (generated circuits)",
            "config": {"workload": "kicked Ising 10x10 open lattice, 4 layers, theta_h ~ U[0.4,0.8] (seed 2), "
                                   "RZZ(-pi/2) bonds, obs Z(5,5); reference: plain |c| < 1e-7, no budget",
                       "network": "8-64-64-1 GELU, BF16 tensor cores, trained on 6x6 circuits (seeds 11-18)",
                       "budgets": sorted({r["budget"] for r in res["rows"]})},
            "learned": best["learned"], "plain": best["plain"],
            "reference": {"O": res["reference"]["O"], "s": statistics.median(ref_t), "peak": res["reference"]["peak"]},
            "rows": res["rows"], "train": res["train"],
            "speedup_vs_plain_budget": (best["plain"]["s"] / val) if (val and best["plain"]) else None,
            "speedup_vs_reference": (ref_s / val) if val else None,
            "by_tolerance": {"1e-3": at_tolerance(1e-3), "1e-4": at_tolerance(1e-4),
                             "note": "budget None: no budget within the tolerance, the unbudgeted run's time"}}
    print(json.dumps(line), flush=True)


def run_layer_bandwidth(args):
    """Kicked Ising 12x12 at a looser truncation, layer by layer: per kernel family, the
    per-launch CUDA-event time and the algorithmic bytes (from the per-op log), for layers
    entering with more than 2e6 terms.  Not a bench line: a measurement of the kernels on
    sums far larger than L2."""
    import torch

    from ppvm_b200 import learned
    from ppvm_b200.paulisum import PauliSum, ops_array

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    wl = C.kicked_ising_2d(L=12, layers=20, theta_h=0.6, thr=args.thr, max_weight=args.max_weight)
    lay = [ops_array(p) for p in learned.split_layers(wl.ops)]
    s = PauliSum([wl.observable[0][0]], wl.n_qubits, [1.0], min_abs_coeff=args.thr,
                 max_pauli_weight=args.max_weight, clifford_angles=True, capacity=1 << 20)
    for li, a in enumerate(lay):
        n_in = len(s)
        big = n_in > 2_000_000
        s.profile(big)
        torch.cuda.synchronize()
        t = time.perf_counter()
        s.run(a)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t
        line = {"layer": li, "terms_in": n_in, "terms_out": len(s), "wall_ms": 1e3 * wall}
        if big:
            line["families"] = {k: {"ms": v["ms"], "bytes": v["bytes"], "gb_s": v["bytes"] / 1e6 / max(v["ms"], 1e-9)}
                                for k, v in s.profile_read().items() if v["launches"]}
        print(json.dumps(line), flush=True)
        if len(s) > args.stop_terms or n_in > args.stop_terms:
            break


def run_kernel_families(args):
    """Every kernel family of the single-sum engine, one op at a time, on sums larger than L2.

    The 12x12 kicked-Ising circuit at --thr / --max-weight is propagated until the sum holds
    more than --family-terms terms, three times: in the reference's term order (per-gate
    rotation path), as a lossy sum (loss channels) and as a term set (fused runs).  Each op
    below then runs on a fresh device copy of that sum, after an L2 flush, with the per-op
    profile on: per kernel family the launches, CUDA-event time, algorithmic bytes (the
    engine's per-op log) and their rate against the measured copy bandwidth.  Each op sits in
    an NVTX range "kf:<op>", so that an ncu capture can select exactly its launches.  One
    JSON line per op; not a bench line."""
    import torch

    from ppvm_b200 import gates as G
    from ppvm_b200 import learned
    from ppvm_b200.paulisum import LossyPauliSum, PauliSum, ops_array

    if int(os.environ.get("RANK", "0")) != 0:
        return
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    peak, peak_kind = measured_peak()
    wl = C.kicked_ising_2d(L=12, layers=20, theta_h=0.6, thr=args.thr, max_weight=args.max_weight)
    lay = [ops_array(p) for p in learned.split_layers(wl.ops)]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def grown(cls, exact):
        s = cls([wl.observable[0][0]], wl.n_qubits, [1.0], min_abs_coeff=args.thr,
                max_pauli_weight=args.max_weight, clifford_angles=True, exact_order=exact, capacity=1 << 22)
        for a in lay:
            if len(s) > args.family_terms:
                break
            s.run(a)
        return s

    n = wl.n_qubits
    rzz_layer = [op for op in wl.ops if op[0] == G.RZZ][:264]  # the 264 RZZ(-pi/2) bonds of one layer
    cases = [
        ("exact", "rx", [G.r1(G.RX, 66, 0.6)]),
        ("exact", "rzz", [G.r2(G.RZZ, 66, 67, 0.3)]),
        ("exact", "truncate", [G.truncate()]),
        ("exact", "clifford_h_x4", [G.g1(G.H, q) for q in (10, 40, 70, 100)]),
        ("exact", "pauli_error_x4", [G.pauli_error(q, (0.01, 0.02, 0.03)) for q in (10, 40, 70, 100)]),
        ("exact", "amplitude_damping", [G.amplitude_damping(66, 0.05)]),
        ("exact", "tableau_rzz_layer", rzz_layer),
        ("lossy", "loss_channel", [G.loss_channel(66, 0.05)]),
        ("set", "rx_run_layer", [G.r1(G.RX, q, 0.6) for q in range(n)] + [G.truncate()]),
        ("exact", "overlap_with_zero", None),
        ("exact", "truncate_budget_half", None),
    ]
    cases.sort(key=lambda c: ("exact", "lossy", "set").index(c[0]))
    base, base_mode = None, None
    for mode, name, ops in cases:  # grouped by mode: one base sum on the device at a time
        if mode != base_mode:
            base = None
            base = grown(LossyPauliSum if mode == "lossy" else PauliSum, mode != "set")
            base_mode = mode
        s = base.copy()
        gl = ops_array(ops) if ops is not None else None
        flush.fill_(1.0)
        torch.cuda.synchronize()
        s.profile(True)
        n_in = len(s)
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.nvtx.range(f"kf:{name}"):
            t0.record()
            if name == "overlap_with_zero":
                s.overlap_with_zero()
            elif name == "truncate_budget_half":
                s.truncate_budget(n_in // 2)
            else:
                s.run(gl)
            t1.record()
            torch.cuda.synchronize()
        fam = {k: {"launches": v["launches"], "ms": v["ms"], "bytes": v["bytes"],
                   "gb_s": v["bytes"] / 1e6 / max(v["ms"], 1e-9),
                   "frac": v["bytes"] / 1e6 / max(v["ms"], 1e-9) / peak}
               for k, v in s.profile_read().items() if v["launches"]}
        print(json.dumps({"op": name, "mode": mode, "terms_in": n_in, "terms_out": len(s),
                          "call_ms": t0.elapsed_time(t1), "families": fam, "peak_gb_s": peak,
                          "peak_kind": peak_kind}), flush=True)
        del s


def main():
    args = parse()
    if args.workload == "layer_bandwidth":
        run_layer_bandwidth(args)
        return
    if args.workload == "kernel_families":
        run_kernel_families(args)
        return
    if args.workload == "learned_kicked_ising":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no learned truncation"}))
        else:
            run_learned(args)
        return
    if args.workload == "batched_tfim":
        run_batched_reference(args) if args.impl == "reference" else run_batched(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
