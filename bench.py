#!/usr/bin/env python
"""MBD energies/s on one B200 (replicas on N GPUs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode MODE]

Workload (one step): the MBD@rsSCS energy of three isolated {H,C,N,O}
clusters of N = 500, 1000 and 2000 atoms (seeded random sequential packing at
0.1 atoms/A^3, Hirshfeld ratios U(0.6,1.0); synthetic stand-ins, no dataset),
each with all 21 imaginary frequencies.  Working set per step: 0.38 / 1.5 /
6.1 GB of relay matrices, far larger than the 126 MB L2, so no L2 flush is
inserted between steps.

value : energies/s with inputs resident in HBM (mbd_rsscs_compute only),
        device-timed with CUDA events on the library's stream, max over ranks.
e2e   : the same metric through mbd_rsscs_energy_batch with host buffers
        (upload + compute + download every step), wall-clock.
Multi-GPU: replicas only (each rank runs the whole workload on its GPU;
value = all ranks' energies / max time).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MBD energies/s, mixed+batched+learned vs plain FP64 on 1 B200, |dE|<=1e-6 Ha"
SIZES = (500, 1000, 2000)
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12   # 148 SMs x 64 DFMA/clk x 2 x 1965 MHz


def workload():
    from mbd_b200 import synthetic as sy
    return [sy.cluster(n, seed=k) for k, n in enumerate(SIZES)]


def relay_flops(n_atoms):
    n = 3 * n_atoms
    return 21 * n ** 3 / 3.0


def eig_flops(n_atoms, nsl=1):
    n = 3 * n_atoms * nsl
    return 4.0 / 3.0 * n ** 3


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [ln for ln in out.splitlines() if ln.strip()]

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in getattr(self, "lines", []):
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(reps=1):
    """The FP64 oracle (numpy + LAPACK, all host threads) on a bounded sample:
    one energy of the N=500 and N=1000 clusters; the N=2000 term of a step is
    extrapolated from N=1000 by the n^3 scaling of its dense LAPACK work."""
    from oracle import mbd_oracle as mo
    geos = workload()
    times = {}
    for (geo, st), n in zip(geos[:2], SIZES[:2]):
        og = mo.Geometry(list(geo.names), geo.coords, geo.hirshfeld, geo.lattice, geo.n_periodic)
        t0 = time.perf_counter()
        for _ in range(reps):
            mo.mbd_at_rsscs(og, mo.Settings())
        times[n] = (time.perf_counter() - t0) / reps
    t_step = times[500] + times[1000] + times[1000] * 8.0
    return {"value": len(SIZES) / t_step, "unit": "energies/s", "cores": os.cpu_count(), "kind": "port",
            "sample": (f"oracle energies of the N=500 ({times[500]:.2f} s) and N=1000 ({times[1000]:.2f} s) "
                       f"clusters; N=2000 extrapolated x8 from N=1000"),
            "seconds_per_step": t_step}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    for _ in range(args.warmup if args.warmup < 1 else 1):
        pass
    vals = []
    cb = None
    for _ in range(max(1, args.steps)):
        cb = cpu_baseline()
        vals.append(cb["seconds_per_step"])
    t = sum(vals)
    value = len(SIZES) * len(vals) / t
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "energies/s", "n_gpus": args.gpus,
            "steps": len(vals), "warmup": 0, "ms_per_step": 1000 * t / len(vals), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "isolated {H,C,N,O} clusters N in {500,1000,2000} (seeds 0,1,2), 21 freqs"},
            "cpu_baseline": {**{k: cb[k] for k in ("unit", "cores", "kind", "sample")}, "value": value},
            "e2e": {"value": value, "unit": "energies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="plain")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--sizes", default=None,
                    help="comma-separated cluster sizes replacing 500,1000,2000 (profiling runs only)")
    args = ap.parse_args()
    if args.sizes:
        global SIZES
        SIZES = tuple(int(x) for x in args.sizes.split(","))

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import torch
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)

    from mbd_b200 import Engine
    geos = workload()
    eng = Engine(local)
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=torch.device("cuda", local))
    code = eng.upload([g for g, _ in geos], [s for _, s in geos])
    if code != 0:
        raise SystemExit(f"upload failed: {code}")
    # warm-up (W full steps, results checked)
    for _ in range(max(3, args.warmup)):
        if eng.compute(args.mode) != 0:
            raise SystemExit("compute failed")
        code, res = eng.download()
        if code != 0:
            raise SystemExit(f"compute failed with status {code}")
    plain_ref = None
    if args.mode != "plain":
        eng.compute("plain")
        _, plain_ref = eng.download()
        eng.compute(args.mode)
        eng.download()

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        start.record(stream)
        for _ in range(args.steps):
            if eng.compute(args.mode) != 0:
                raise SystemExit("compute failed")
        stop.record(stream)
        stop.synchronize()
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    stats = eng.stats()
    code, res = eng.download()
    stage = eng.timings()
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    value = world * len(SIZES) * args.steps / (ms / 1000.0)

    # roofline of the dominant stage (device time of the last step, per stage)
    peaks, peak_src = load_peaks()
    stages = {k: v for k, v in stage.items() if k != "total"}
    dom = max(stages, key=stages.get)
    if dom == "relay_factor":
        flops = sum(relay_flops(n) for n in SIZES)
        achieved = flops / (stages[dom] / 1000.0) / 1e12
        roof = {"bound": "tensor", "kernel": "syrk_lower/trsm_panel/potrf_diag (FP64 DFMA)",
                "achieved": achieved, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                "frac": achieved / FP64_NOMINAL_TFLOPS, "traffic": None,
                "peak_source": "nominal FP64 (148 SM x 64 DFMA/clk x 1965 MHz); MEASURED_PEAKS.json has no FP64 entry",
                "algorithmic": "21*(3N)^3/3 flops per energy"}
    elif dom == "tridiag":
        flops = sum(eig_flops(n) for n in SIZES)
        achieved = flops / (stages[dom] / 1000.0) / 1e12
        roof = {"bound": "tensor", "kernel": "tridiag_kernel (FP64)", "achieved": achieved,
                "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s", "frac": achieved / FP64_NOMINAL_TFLOPS,
                "traffic": None, "peak_source": "nominal FP64", "algorithmic": "(4/3)(3N)^3 flops per energy"}
    else:
        roof = {"bound": "hbm", "kernel": dom, "achieved": None, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": None, "traffic": None, "peak_source": peak_src}
    roof["stage_ms"] = stages

    line = {"metric": METRIC, "value": value, "unit": "energies/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.mode == "plain" else "tf32x3+f64",
            "data": "synthetic",
            "config": {"workload": "isolated {H,C,N,O} clusters N in {500,1000,2000} (seeds 0,1,2), 21 freqs",
                       "mode": args.mode, "parallelism": f"replicas{world}" if world > 1 else "1gpu",
                       "l2": "working set 0.38-6.1 GB per geometry > 126 MB L2; no flush"},
            "gpu_launches": stats["launches"] * args.steps,
            "roofline": roof,
            "energies": [r.energy for r in res]}
    if plain_ref is not None:
        line["max_abs_dE_vs_plain_fp64"] = max(abs(a.energy - b.energy) for a, b in zip(res, plain_ref))
    if rank == 0:
        line["clocks"] = clk.summary()

    # end-to-end through the C ABI with host buffers
    if not args.no_e2e:
        if dist:
            dist.barrier()
        gl = [g for g, _ in geos]
        sl = [s for _, s in geos]
        for _ in range(1):
            eng.energy_batch(gl, sl, args.mode)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            rr = eng.energy_batch(gl, sl, args.mode)
        t_e2e = time.perf_counter() - t0
        st2 = eng.stats()
        if dist:
            t = torch.tensor([t_e2e], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_e2e = float(t.item())
        line["e2e"] = {"value": world * len(SIZES) * args.steps / t_e2e, "unit": "energies/s",
                       "h2d_bytes_per_step": st2["h2d_bytes"], "d2h_bytes_per_step": st2["d2h_bytes"],
                       "status": [r.status for r in rr]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline()
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
