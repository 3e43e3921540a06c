"""Benchmark: PaMO stage-2 simplification on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl product|reference]
                    [--workload c2|c1] [--no-cpu-baseline]

Workload (default "c2"): 1024x1024 noisy torus (1,048,576 verts / 2,097,152
faces, fp32/int32, seeded) simplified with ratio 0.01 (~20,971 faces) by the
stage-2 loop of PaMO.run (centring, init permutation, collapse rounds with the
self-intersection undo, compaction) -- the path this library implements.

One step = one whole simplification of the mesh.  `value` = input Mfaces/s with
the inputs already resident in HBM (device-timed with CUDA events around the
steps); `e2e` = the same metric through the public C ABI entry points with host
buffers: pinned host -> device copy of the mesh, the run, device -> host copy of
the result, all inside the timed region.  The working set per round is far
larger than the 126 MB L2 at 2M faces (several hundred MB), so no explicit L2
flush is done between steps.

`--impl reference` times the reference's algorithm on the host cores (the CPU
restatement under oracle/, all threads) on a bounded sample of the same workload:
the first rounds of the same run, extrapolated to the whole run by the face
counts of the rounds (identical to the device run's rounds).

With --gpus N > 1 (torchrun, one rank per GPU) every rank simplifies its own
copy of the mesh (replicas; there is no data exchange), timed as the max over
ranks; value = N * faces / time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """SM clocks and throttle reasons sampled through NVML during the timed region
    (in-process, every 100 ms)."""

    REASONS = {  # nvmlClocksEventReason bits
        "sw_power_cap": 0x4,
        "hw_slowdown": 0x8,
        "sw_thermal_slowdown": 0x20,
        "hw_thermal_slowdown": 0x40,
        "hw_power_brake_slowdown": 0x80,
    }

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self.error = None

    def start(self):
        def run():
            try:
                import pynvml as N

                N.nvmlInit()
                h = N.nvmlDeviceGetHandleByIndex(self.index)
                mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
                while not self._stop.is_set():
                    sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                    try:
                        rs = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                    except Exception:
                        rs = N.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                    self.samples.append((sm, mx, rs))
                    self._stop.wait(0.1)
            except Exception as e:  # no NVML: report that instead of clocks
                self.error = repr(e)

        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0, "error": self.error}
        sm = [s[0] for s in self.samples]
        reasons = sorted({k for s in self.samples for k, bit in self.REASONS.items() if s[2] & bit})
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(s[1] for s in self.samples)),
                "reasons": reasons, "samples": len(self.samples)}


def workload(name):
    from pamo_b200 import meshgen as mg

    if name == "c1":
        V, F = mg.displaced_icosphere(5, 0)
        return V, F, 0.05, "icosphere-L5-sh8 (10,242 v / 20,480 f) ratio 0.05"
    V, F = mg.noisy_torus(1024, 1024, 0)
    return V, F, 0.01, "torus-1024x1024-noise (1,048,576 v / 2,097,152 f) ratio 0.01"


def dist_init(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def reference_arm(args):
    """CPU restatement of the reference's stage 2 on the host cores."""
    ws, rank, _ = dist_init(args)
    if rank != 0:
        return 0
    from oracle import oracle as O

    V, F, ratio, desc = workload(args.workload)
    target = int(ratio * len(F))
    tm = O.tris_mean(V, F)
    Vc = (V - tm).astype(np.float32)
    Fs = O.shuffle_faces(F)
    # bounded sample: the first rounds of the run
    sample_rounds = args.sample_rounds
    step_s = []
    face_rounds = None
    for _ in range(args.warmup + args.steps):
        o = O.Stage2Oracle()
        t0 = time.perf_counter()
        v, f, rounds = o.run(Vc, Fs, target, 4, 1e-3, sample_rounds)
        step_s.append(time.perf_counter() - t0)
    t = float(np.median(step_s[args.warmup:]))
    # faces entering each round of the full run, to extrapolate the sample
    frac = _sample_fraction(args, sample_rounds)
    total_s = t / frac if frac else float("nan")
    value = len(F) / 1e6 / total_s
    cores = O.lib().s2o_num_threads()
    line = {"metric": "input Mfaces/s", "value": value, "unit": "Mfaces/s", "impl": "reference", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc},
            "cpu_baseline": {"value": value, "unit": "Mfaces/s", "cores": cores, "kind": "port",
                             "sample": f"first {sample_rounds} rounds ({frac * 100:.1f}% of the run's face-rounds), "
                                       f"extrapolated by face-rounds"},
            "e2e": {"value": value, "unit": "Mfaces/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def cpu_baseline_sample(args, V, F, ratio):
    """The CPU restatement (oracle/, OpenMP on all host threads) on the first
    `sample_rounds` rounds of the same run, extrapolated by face-rounds."""
    from oracle import oracle as O

    target = int(ratio * len(F))
    tm = O.tris_mean(V, F)
    Vc = (V - tm).astype(np.float32)
    Fs = O.shuffle_faces(F)
    o = O.Stage2Oracle()
    t0 = time.perf_counter()
    o.run(Vc, Fs, target, 4, 1e-3, args.sample_rounds)
    t = time.perf_counter() - t0
    frac = _sample_fraction(args, args.sample_rounds)
    total = t / frac if frac else float("nan")
    return {"value": len(F) / 1e6 / total, "unit": "Mfaces/s", "cores": O.lib().s2o_num_threads(), "kind": "port",
            "sample": f"first {args.sample_rounds} rounds ({(frac or 0) * 100:.1f}% of the run's face-rounds, "
                      f"{t:.1f} s), extrapolated by face-rounds"}


def _sample_fraction(args, sample_rounds):
    """Share of face-rounds covered by the first `sample_rounds` rounds, from the
    recorded round sizes of the same workload (tests/golden/<workload>_round_faces.json)."""
    path = os.path.join(ROOT, "tests", "golden", f"{args.workload}_round_faces.json")
    try:
        sizes = json.load(open(path))["faces_in"]
    except Exception:
        return None
    tot = float(sum(sizes))
    return float(sum(sizes[:sample_rounds])) / tot if tot else None


def roofline_edge_cost(phases, round_faces, peaks):
    """HBM roofline of the edge-cost kernel (one launch per round).

    Algorithmic bytes per round with F faces (closed mesh: E = 1.5 F edges,
    V = 0.5 F vertices), each array read or written once: edges 8 B/edge,
    cost write 4 B/edge, CSR offsets 4 B/vertex, CSR entries 12 B/face, faces
    (int4) 16 B/face, points (float4) 16 B/vertex, quadrics 48 B/vertex,
    invalid flags 1 B/vertex, per-vertex key minimum read+write 16 B/vertex:
    12 E + 85 V + 28 F = 88.5 B/face."""
    ph = phases.get("edge_cost")
    if not ph or not ph["ms"] or not round_faces:
        return None
    total_bytes = sum(88.5 * f for f in round_faces)
    t = ph["ms"] / 1e3
    achieved = total_bytes / t / 1e9
    peak = peaks.get("hbm_gbs") or 6650.0
    return {"bound": "hbm", "kernel": "k_edge_cost", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": None, "launches": ph["calls"],
            "avg_launch_ms": ph["ms"] / max(ph["calls"], 1),
            "bytes_per_launch_avg": total_bytes / max(ph["calls"], 1),
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks.get("hbm_gbs") else "fallback"}


def product_arm(args):
    import torch

    import pamo_b200
    from pamo_b200 import _lib

    ws, rank, local = dist_init(args)
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    V, F, ratio, desc = workload(args.workload)
    target = int(ratio * len(F))
    nF = len(F)
    ctx = pamo_b200.Context(local)
    L = _lib.lib()
    s = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(s.cuda_stream)
    Pd = torch.from_numpy(V).to(dev)
    Fd = torch.from_numpy(F).to(dev)
    on, om, rr = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()

    def run_resident():
        _lib.check("pamo_stage2_run", L.pamo_stage2_run(ctx.handle, Pd.data_ptr(), Fd.data_ptr(), len(V), nF, target,
                                                        4, 1e-3, 1000000, sp, ctypes.byref(on), ctypes.byref(om),
                                                        ctypes.byref(rr)))

    # pinned host buffers for the end-to-end leg
    Ph = torch.from_numpy(V).pin_memory()
    Fh = torch.from_numpy(F).pin_memory()
    Pe = torch.empty_like(Pd)
    Fe = torch.empty_like(Fd)
    out_v = torch.empty((len(V), 3), dtype=torch.float32).pin_memory()
    out_f = torch.empty((nF, 3), dtype=torch.int32).pin_memory()

    def run_e2e():
        Pe.copy_(Ph, non_blocking=True)
        Fe.copy_(Fh, non_blocking=True)
        _lib.check("pamo_stage2_run", L.pamo_stage2_run(ctx.handle, Pe.data_ptr(), Fe.data_ptr(), len(V), nF, target,
                                                        4, 1e-3, 1000000, sp, ctypes.byref(on), ctypes.byref(om),
                                                        ctypes.byref(rr)))
        _lib.check("pamo_stage2_fetch", L.pamo_stage2_fetch(ctx.handle, out_v.data_ptr(), out_f.data_ptr(), 1, sp))
        return on.value * 12 + om.value * 12

    for _ in range(args.warmup):
        run_resident()
    torch.cuda.synchronize()
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
    clk = ClockSampler(local)
    clk.start()
    for _ in range(100):  # NVML initialisation stalls the device briefly: let it finish first
        if clk.samples or clk.error:
            break
        time.sleep(0.05)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(s)
    for _ in range(args.steps):
        run_resident()
    ev1.record(s)
    torch.cuda.synchronize()
    dev_ms = ev0.elapsed_time(ev1) / args.steps
    # end-to-end leg with host buffers, per-step latencies
    lat = []
    d2h = 0
    for _ in range(max(args.steps, 3)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        d2h = run_e2e()
        torch.cuda.synchronize()
        lat.append(time.perf_counter() - t0)
    clocks = clk.stop()
    # one more run with per-phase CUDA events (outside the timed region)
    L.pamo_profile_enable(ctx.handle, 1)
    run_resident()
    torch.cuda.synchronize()
    ph_ms = (ctypes.c_double * 16)()
    ph_calls = (ctypes.c_longlong * 16)()
    nph = L.pamo_profile_read(ctx.handle, ph_ms, ph_calls, 16)
    L.pamo_profile_enable(ctx.handle, 0)
    phases = {_lib.PHASES[i]: {"ms": ph_ms[i], "calls": ph_calls[i]} for i in range(min(nph, len(_lib.PHASES)))}
    sizes = (ctypes.c_int * 4096)()
    nr = L.pamo_stage2_round_sizes(ctx.handle, sizes, 4096)
    round_faces = [sizes[i] for i in range(min(nr, 4096))]
    ms_max = dev_ms
    e2e_ms = float(np.mean(lat)) * 1e3
    if ws > 1:
        import torch.distributed as dist
        t = torch.tensor([dev_ms, e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max, e2e_ms = float(t[0]), float(t[1])
    rounds = rr.value
    stats = (ctypes.c_longlong * 8)()
    L.pamo_stage2_last_round_stats(ctx.handle, stats)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_sample(args, V, F, ratio)
    if rank == 0:
        value = ws * nF / 1e6 / (ms_max / 1e3)
        e2e = ws * nF / 1e6 / (e2e_ms / 1e3)
        peaks = _peaks()
        line = {
            "metric": "input Mfaces/s", "value": value, "unit": "Mfaces/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "stages": "2 (stage-2 loop of PaMO.run)", "faces_out": om.value,
                       "verts_out": on.value, "rounds": rounds, "l2": "inputs/working set > L2, no flush",
                       "parallelism": f"replicas x{ws}"},
            "latency_ms": {"p50": float(np.percentile(lat, 50)) * 1e3, "p99": float(np.percentile(lat, 99)) * 1e3},
            "e2e": {"value": e2e, "unit": "Mfaces/s", "h2d_bytes_per_step": int(nF * 12 + len(V) * 12),
                    "d2h_bytes_per_step": int(d2h)},
            "clocks": clocks,
            "cpu_baseline": cpu,
            "phases_ms": {k: round(v["ms"], 3) for k, v in phases.items()},
            "roofline": roofline_edge_cost(phases, round_faces, peaks),
            "round_faces": round_faces if args.dump_rounds else None,
        }
        print(json.dumps(line))
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--workload", default="c2", choices=["c1", "c2"])
    ap.add_argument("--sample-rounds", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--dump-rounds", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)
    return product_arm(args)


if __name__ == "__main__":
    sys.exit(main())
