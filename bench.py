#!/usr/bin/env python
"""MBD energies/s on one B200 (replicas on N GPUs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--mode MODE]
                    [--workload clusters|batched|boxes]

Workload (one step, default): the MBD@rsSCS energy of three isolated
{H,C,N,O} clusters of N = 500, 1000 and 2000 atoms (seeded random sequential
packing at 0.1 atoms/A^3, Hirshfeld ratios U(0.6,1.0); synthetic stand-ins,
no dataset), each with all 21 imaginary frequencies.  Working set per step:
0.38 / 1.5 / 6.1 GB of relay matrices, far larger than the 126 MB L2, so no
L2 flush is inserted between steps.  --workload batched: 256 clusters of
N ~ U{20..600} in one batch; --workload boxes: periodic boxes of 2000, 4000
and 6000 atoms.

value : energies/s of the headline mode (mixed_learned: block-CG relay solve
        started from the network's prediction, preconditioned by 64-row tile
        inverses, FP64 eigensolve; the network is trained before timing) with
        inputs resident in HBM (mbd_rsscs_compute only), device-timed with
        CUDA events on the library's stream, max over ranks.
plain_fp64 : the same workload in the plain FP64 mode, timed the same way;
mixed_direct / learned_no_network : the 3xTF32 direct relay solve and the
        block-CG without the network, timed the same way.
e2e   : the headline mode through mbd_rsscs_energy_batch with host buffers
        (upload + compute + download every step), wall clock.  Each step
        uploads the batch anew, so its compute launches kernel by kernel.
Multi-GPU: replicas only (each rank runs the whole workload on its GPU;
value = all ranks' energies / max time).
"""
from __future__ import annotations

import argparse
import json

import numpy as np
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MBD energies/s, mixed+batched+learned vs plain FP64 on 1 B200, |dE|<=1e-6 Ha"
SIZES = (500, 1000, 2000)
BOX_SIZES = (2000, 4000, 6000)
FP64_NOMINAL_TFLOPS = 148 * 64 * 2 * 1.965e9 / 1e12   # 148 SMs x 64 DFMA/clk x 2 x 1965 MHz
TWO_STAGE_MAX_N = 1152 * 16 + 32   # largest Hamiltonian the two-stage reduction takes (panel rows x cluster CTAs + a panel)


WORKLOADS = {
    "clusters": "isolated {H,C,N,O} clusters N in {500,1000,2000} (seeds 0,1,2), 21 freqs",
    "batched": "256 isolated {H,C,N,O} clusters N ~ U{20..600} (seed 0), 21 freqs, one batch",
    "boxes": "periodic cubic {H,C,N,O} boxes N in {2000,4000,6000} (seeds 0,1,2) at 0.1 atoms/A^3, "
             "cut-offs 120/100/25 A, 21 freqs",
    "sheet": "periodic graphene sheet: hexagonal C, a = 2.46 A, 8x8 cells (128 atoms), 20 A along z with "
             "vacuum axis z, cut-offs 120/100/25 A (2x2x1 supercell, Hamiltonian 1536 wide), 21 freqs",
}
WORKLOAD = "clusters"


def workload():
    from mbd_b200 import synthetic as sy
    if WORKLOAD == "batched":
        return sy.cluster_batch(256)
    if WORKLOAD == "boxes":
        return [sy.periodic_box(n, seed=k) for k, n in enumerate(BOX_SIZES)]
    if WORKLOAD == "sheet":
        return [sy.graphene_sheet()]
    return [sy.cluster(n, seed=k) for k, n in enumerate(SIZES)]


def workload_name():
    if WORKLOAD == "clusters" and SIZES != (500, 1000, 2000):
        return f"isolated {{H,C,N,O}} clusters N in {{{','.join(map(str, SIZES))}}}, 21 freqs"
    return WORKLOADS[WORKLOAD]


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return json.load(fh), "measured"
    except OSError:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# DRAM traffic (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# the workload's dominant kernels, from ncu captures of this bench command on
# a B200: a profile constant, not measured by the run that prints it.
PROFILED_TRAFFIC = {
    "clusters": {"sb2st_kernel": 7881000, "tridiag_kernel": 210234000000},
}


def load_traffic():
    return PROFILED_TRAFFIC.get(WORKLOAD, {})


def fp64_step_flops(results):
    """Algorithmic FP64 work of the reference's method per step: for each
    energy 21 (3N)^3/3 (Cholesky of the relay matrices) + 126 (3N)^2 (their
    3-RHS solves) + (4/3) (3N n_SL)^3 (reduction of the CFDM Hamiltonian)."""
    fl = 0.0
    for r in results:
        n = 3.0 * len(r.alpha_eff)
        nsl = float(np.prod(r.supercell))
        fl += 21.0 * n ** 3 / 3.0 + 126.0 * n * n + (4.0 / 3.0) * (n * nsl) ** 3
    return fl


def _supercell_cells(geo, st):
    """Cells of the supercell (get_supercell, UTILS.f90:1252-1283): the
    Hamiltonian has 3 N times this many rows."""
    if not geo.n_periodic:
        return 1
    bohr = 0.52917721
    cells = 1
    for k in range(3):
        if not st.mbd_scs_vacuum_axis[k]:
            cells *= int(np.ceil((st.mbd_supercell_cutoff / bohr) / np.linalg.norm(geo.lattice[k] / bohr)))
    return cells


def image_terms(geo, st):
    """(pair, image) terms of the reference's image sums for one energy:
    short-range (scs_*_block, UTILS.f90:561-579, 610-631: atom pairs i >= j,
    images in the box +-ceil(cut/|a_k|) with 0 < r <= cut), once per
    frequency; long-range (supercell_*_block/cfdm_*_block, UTILS.f90:883-1094:
    lower-triangle (atom, cell) pairs of the supercell, supercell images with
    r <= cut).  Counted here from the geometry (numpy), for the throughput
    figure of the periodic sheet workload."""
    bohr = 0.52917721
    lat = geo.lattice / bohr
    xyz = geo.coords / bohr

    def box(cut, L, vac):
        rng = [0 if (vac[k] or geo.n_periodic == 0) else int(np.ceil(cut / np.linalg.norm(L[k]))) for k in range(3)]
        g = np.stack(np.meshgrid(*[np.arange(-m, m + 1) for m in rng], indexing="ij"), -1).reshape(-1, 3)
        return g @ L

    vac = tuple(bool(v) for v in st.mbd_scs_vacuum_axis)
    scut = st.mbd_scs_dip_cutoff / bohr
    sh = box(scut, lat, vac)
    ii, jj = np.tril_indices(len(xyz), 0)
    sr = 0
    for s0 in range(0, len(ii), 4096):
        d = (xyz[ii[s0:s0 + 4096]] - xyz[jj[s0:s0 + 4096]])[:, None, :] + sh[None]
        r = np.sqrt((d * d).sum(-1))
        sr += int(np.count_nonzero((r <= scut) & (r > 0.0)))
    sl = np.array([1 if (vac[k] or geo.n_periodic == 0) else int(np.ceil((st.mbd_supercell_cutoff / bohr)
                                                                          / np.linalg.norm(lat[k])))
                   for k in range(3)])
    cells = np.stack(np.meshgrid(*[np.arange(m) for m in sl], indexing="ij"), -1).reshape(-1, 3) @ lat
    big = (xyz[:, None, :] + cells[None]).reshape(-1, 3)
    lcut = st.mbd_cfdm_dip_cutoff / bohr
    shl = box(lcut, lat * sl[:, None], vac)
    ii, jj = np.tril_indices(len(big), 0)
    lr = 0
    for s0 in range(0, len(ii), 4096):
        d = (big[ii[s0:s0 + 4096]] - big[jj[s0:s0 + 4096]])[:, None, :] + shl[None]
        r = np.sqrt((d * d).sum(-1))
        lr += int(np.count_nonzero((r <= lcut) & (r > 0.0)))
    return 21 * sr, lr


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
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
        for ln in self.lines:
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


def _oracle_energy(geo, st):
    from oracle import mbd_oracle as mo
    og = mo.Geometry(list(geo.names), geo.coords, geo.hirshfeld, geo.lattice, geo.n_periodic)
    os_ = mo.Settings(xc=st.xc, mbd_supercell_cutoff=st.mbd_supercell_cutoff,
                      mbd_cfdm_dip_cutoff=st.mbd_cfdm_dip_cutoff, mbd_scs_dip_cutoff=st.mbd_scs_dip_cutoff,
                      mbd_scs_vacuum_axis=tuple(st.mbd_scs_vacuum_axis))
    t0 = time.perf_counter()
    mo.mbd_at_rsscs(og, os_)
    return time.perf_counter() - t0


def cpu_baseline():
    """The FP64 oracle (numpy + LAPACK, all host threads) on the workload, every
    energy timed (nothing extrapolated).  clusters / sheet: one oracle energy of
    every geometry of the step.  batched: the first geometries of the batch
    (a random sample of its size distribution) until about 20 s of CPU time,
    energies/s over that sample."""
    geos = workload()
    if WORKLOAD == "batched":
        t, done = 0.0, 0
        for geo, st in geos:
            t += _oracle_energy(geo, st)
            done += 1
            if t >= 20.0:
                break
        return {"value": done / t, "unit": "energies/s", "cores": os.cpu_count(), "kind": "port",
                "sample": f"oracle energies of the first {done} of the batch's {len(geos)} geometries "
                          f"(N ~ U{{20..600}}), {t:.1f} s"}
    times = [_oracle_energy(geo, st) for geo, st in geos]
    sizes = ",".join(str(len(g.names)) for g, _ in geos)
    return {"value": len(geos) / sum(times), "unit": "energies/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"one oracle energy of each geometry of the step (N = {sizes}): "
                      + ", ".join(f"{t:.2f} s" for t in times)}


def run_reference(args, rank, world):
    """Reference arm: the reference (Fortran/MPI/ScaLAPACK) cannot be built in
    this image, so its CPU path is the FP64 oracle port on the host cores.
    Each step is one oracle energy, cycling through the workload's geometries
    in order; energies/s = the workload's energies over the summed mean time
    of each of its geometries (every energy timed, nothing extrapolated)."""
    if rank != 0:
        return 0
    if WORKLOAD == "boxes":
        print(json.dumps({"impl": "reference", "metric": METRIC, "config": {"workload": workload_name()},
                          "unavailable": "the FP64 oracle needs hours per 2000-atom box at these cut-offs "
                                         "(its long-range image sums are numpy loops); not timed"}), flush=True)
        return 0
    geos = workload()
    steps = max(1, args.steps)
    per = {}
    t_all = 0.0
    for k in range(steps):
        g = k % len(geos)
        t = _oracle_energy(*geos[g])
        per.setdefault(g, []).append(t)
        t_all += t
    if WORKLOAD == "batched":
        value = steps / t_all
        sample = f"oracle energies of the batch's first {min(steps, len(geos))} geometries (N ~ U{{20..600}})"
    else:
        mean = [statistics.mean(per[g]) for g in sorted(per)]
        value = len(per) / sum(mean)
        sample = ("one oracle energy per step, cycling through the step's geometries: "
                  + ", ".join(f"N={len(geos[g][0].names)} {len(per[g])}x mean {statistics.mean(per[g]):.2f} s"
                              for g in sorted(per)))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "energies/s", "n_gpus": args.gpus,
            "steps": steps, "warmup": 0, "ms_per_step": 1000 * t_all / steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name()},
            "cpu_baseline": {"unit": "energies/s", "cores": os.cpu_count(), "kind": "port", "sample": sample,
                             "value": value},
            "e2e": {"value": value, "unit": "energies/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks_of(x, dist, device):
    """The largest x over the ranks of the process group (x itself without
    one): every replica times its own copy of the workload, the job takes as
    long as the slowest."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world, energies_per_step, steps, ms):
    """Whole-job energies/s of `world` replicas that each compute
    energies_per_step energies per step, `steps` steps in `ms` (max over ranks)."""
    return world * energies_per_step * steps / (ms / 1000.0)


def time_mode(eng, stream, mode, steps, warmup, clocks=None, flush=None):
    """Device time of `steps` back-to-back mbd_rsscs_compute calls after
    warm-up.  With `flush` (a device buffer larger than L2) the buffer is
    rewritten before every step, outside the timed events, and the steps are
    timed one by one."""
    import torch
    for _ in range(warmup):
        if eng.compute(mode) != 0:
            raise SystemExit(f"compute({mode}) failed")
        code, _ = eng.download()
        if code != 0:
            raise SystemExit(f"compute({mode}) returned status {code}")
    torch.cuda.synchronize()
    ctx = clocks if clocks is not None else _Null()
    with ctx:
        if flush is None:
            start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            start.record(stream)
            for _ in range(steps):
                if eng.compute(mode) != 0:
                    raise SystemExit(f"compute({mode}) failed")
            stop.record(stream)
            stop.synchronize()
            ms = start.elapsed_time(stop)
        else:
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                   for _ in range(steps)]
            with torch.cuda.stream(stream):
                for a, b in evs:
                    flush.add_(1.0)
                    a.record(stream)
                    if eng.compute(mode) != 0:
                        raise SystemExit(f"compute({mode}) failed")
                    b.record(stream)
            evs[-1][1].synchronize()
            ms = sum(a.elapsed_time(b) for a, b in evs)
    stats = eng.stats()
    code, res = eng.download()
    if code != 0:
        raise SystemExit(f"compute({mode}) returned status {code}")
    return ms, stats, res, eng.timings()


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def roofline(stage_ms, sizes, mode):
    """Roofline of the dominant stage of the last timed step."""
    peaks, src = load_peaks()
    sub = ("total", "tridiag_dense_to_band", "tridiag_to_tridiagonal", "tridiag_one_stage_launch",
           "tridiag_band_chase_launch")
    stages = {k: v for k, v in stage_ms.items() if k not in sub}
    dom = max(stages, key=stages.get)
    one_ms = stage_ms.get("tridiag_one_stage_launch", 0.0)
    chase_ms = stage_ms.get("tridiag_band_chase_launch", stage_ms.get("tridiag_to_tridiagonal", 0.0))
    two_stage = stage_ms.get("tridiag_dense_to_band", 0.0) > 0.0
    if two_stage and one_ms > 0.05:
        # both launches ran: the matrices above the two-stage limit took the one-stage one
        big = [n for n in sizes if 3 * n > TWO_STAGE_MAX_N]
        sizes_two = [n for n in sizes if 3 * n <= TWO_STAGE_MAX_N]
        if one_ms >= chase_ms:
            two_stage, sizes, stages["tridiag"] = False, big, one_ms
        else:
            sizes = sizes_two
    if dom == "tridiag" and two_stage:
        # two-stage path: the batch-wide bulge-chasing launch (timed alone by
        # the stage events).  Per task it reads and writes its diagonal block and
        # the block below it (2 x 32 x 32 FP64 each way); sweep i of an n x n
        # band has ceil((n - i - 1) / 32) tasks, sweeps i = 0 .. n - 3.
        def tasks(n):
            return sum((n - i - 1 + 31) // 32 for i in range(0, n - 2))
        t_ms = chase_ms
        nbytes = sum(tasks(3 * n) for n in sizes) * 4 * 32 * 32 * 8.0
        achieved = nbytes / (t_ms / 1000.0) / 1e9
        return {"bound": "hbm", "kernel": "sb2st_kernel (band -> tridiagonal bulge chasing, one launch per batch)",
                "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": achieved / peaks.get("hbm_gbs"), "traffic": load_traffic().get("sb2st_kernel"),
                "traffic_source": "ncu capture of one launch of this workload (a profile constant)",
                "kernel_ms": t_ms,
                "peak_source": f"{src} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic": "per bulge-chasing task 2 x 32x32 FP64 blocks read + written; "
                               "sum over sweeps i of ceil((n-i-1)/32) tasks, n = 3N",
                "note": "latency-bound: the 2n-task dependency chain between consecutive sweeps sets the time; "
                        "the band stays in L2 (measured DRAM traffic far below the algorithmic bytes)",
                "stage_ms": stages}
    if dom == "tridiag":
        # one read of the trailing lower triangle per column: sum_m m^2/2 * 8 B = n^3/6 * 8 B
        nbytes = sum((3.0 * n) ** 3 / 6.0 * 8.0 for n in sizes)
        achieved = nbytes / (stages[dom] / 1000.0) / 1e9
        traffic = load_traffic().get("tridiag_kernel")
        return {"bound": "hbm", "kernel": "tridiag_kernel (FP64 Householder; one cooperative launch reduces every Hamiltonian of the batch)",
                "achieved": achieved, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
                "frac": achieved / peaks.get("hbm_gbs"), "traffic": traffic,
                "peak_source": f"{src} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)",
                "algorithmic": "(3N)^3/6 * 8 B per energy (SYMV reads of the trailing lower triangle)",
                "stage_ms": stages}
    if dom == "relay_factor":
        fl = sum(21 * (3.0 * n) ** 3 / 3.0 for n in sizes)
        if mode == "plain":
            achieved = fl / (stages[dom] / 1000.0) / 1e12
            return {"bound": "tensor", "kernel": "syrk_lower/trsm_panel/potrf_diag (FP64 DFMA)",
                    "achieved": achieved, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                    "frac": achieved / FP64_NOMINAL_TFLOPS, "traffic": None,
                    "peak_source": "nominal FP64 (148 SM x 64 DFMA/clk x 1965 MHz); no FP64 entry in MEASURED_PEAKS.json",
                    "algorithmic": "21*(3N)^3/3 flop per energy", "stage_ms": stages}
        achieved = 3 * fl / (stages[dom] / 1000.0) / 1e12
        peak = peaks.get("bf16_tflops") / 2.0
        return {"bound": "tensor", "kernel": "tc3_gemm_kernel (3xTF32 tcgen05) + potrf_diag_f32",
                "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak, "traffic": None,
                "peak_source": f"{src} bf16 cuBLAS / 2 (dense TF32 rate)",
                "algorithmic": "3 x 21*(3N)^3/3 TF32 flop per energy", "stage_ms": stages}
    note = None
    if dom == "relay_solve" and mode == "mixed_learned":
        note = ("block-CG over the slots' overlapping streams (the stage time is summed over geometries); no "
                "per-launch timing of its matrix pass cg_tile_kernel here (ncu: 4.72 TB/s, 72 % of the measured "
                "copy bandwidth on an n = 3000 relay batch)")
    return {"bound": "hbm", "kernel": dom, "achieved": None, "peak": peaks.get("hbm_gbs"), "unit": "GB/s",
            "frac": None, "traffic": None, "peak_source": src, "note": note, "stage_ms": stages}


def main():
    global SIZES, WORKLOAD
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="mixed_learned", choices=["plain", "mixed", "mixed_learned"])
    ap.add_argument("--train-geoms", type=int, default=None,
                    help="geometries (N ~ U{50..400}, clusters or, for --workload boxes, periodic boxes) the "
                         "learned warm start is trained on before timing (default 160; 2000 for boxes)")
    ap.add_argument("--train-epochs", type=int, default=12)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison run")
    ap.add_argument("--workload", default="clusters", choices=sorted(WORKLOADS),
                    help="clusters: the three-cluster headline workload; batched: 256 uneven clusters; "
                         "boxes: three periodic boxes of 2000-6000 atoms")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the untuned launch shapes (profiling runs: the autotuner's own launches "
                         "would swamp a launch list)")
    ap.add_argument("--sizes", default=None,
                    help="comma-separated cluster sizes replacing 500,1000,2000 (profiling runs only)")
    args = ap.parse_args()
    WORKLOAD = args.workload
    if args.train_geoms is None:
        args.train_geoms = 2000 if WORKLOAD == "boxes" else 160
    if args.sizes:
        SIZES = tuple(int(x) for x in args.sizes.split(","))
    warmup = max(3, args.warmup)

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
    learned = None
    if args.mode == "mixed_learned":
        # the network is trained once, before any timing, on direct relay
        # solutions of clusters from the same generator (other seeds)
        from mbd_b200 import synthetic as sy
        rng = np.random.default_rng(12345)
        gen = sy.periodic_box if WORKLOAD == "boxes" else sy.cluster
        train = [gen(int(n), seed=100000 + k) for k, n in
                 enumerate(rng.integers(50, 401, size=args.train_geoms))]
        t0 = time.perf_counter()
        loss = eng.learned_train([g for g, _ in train], [s for _, s in train], epochs=args.train_epochs, lr=1e-3,
                                 seed=7)
        learned = {"train_geoms": args.train_geoms,
                   "train_sizes": ("periodic boxes" if WORKLOAD == "boxes" else "clusters") + " N ~ U{50..400}",
                   "epochs": args.train_epochs, "train_seconds": time.perf_counter() - t0,
                   "loss_first_epoch": float(loss[0]), "loss_last_epoch": float(loss[-1])}
    # launch shapes of the eigen stages tuned for this workload's Hamiltonian
    # sizes before anything is timed (the network's training above used the
    # defaults; the choices apply to the computes below)
    t0 = time.perf_counter()
    tuned = [] if args.no_autotune else eng.autotune(max(3 * len(g.names) * _supercell_cells(g, s) for g, s in geos))
    tune_s = time.perf_counter() - t0
    stream = torch.cuda.ExternalStream(eng.stream_handle(), device=torch.device("cuda", local))
    # the sheet's working set (25 MB of relay matrices) fits in the 126 MB L2:
    # a 512 MB buffer is rewritten before every timed step
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float64, device=torch.device("cuda", local)) \
        if WORKLOAD == "sheet" else None
    code = eng.upload([g for g, _ in geos], [s for _, s in geos])
    if code != 0:
        raise SystemExit(f"upload failed: {code}")

    def max_over_ranks(x):
        return max_over_ranks_of(x, dist, "cuda")

    plain = None
    extra = {}
    if args.mode == "mixed_learned" and not args.no_plain:
        # the same relay solve without the network (block-CG from zero) and the
        # direct tensor-core relay solve, for comparison
        for name, mode in (("mixed_direct", "mixed"), ("learned_no_network", "mixed_learned")):
            if dist:
                dist.barrier()
            if name == "learned_no_network":
                eng.use_network(False)
            xms, _, xres, xstage = time_mode(eng, stream, mode, args.steps, warmup, flush=flush)
            eng.use_network(True)
            xms = max_over_ranks(xms)
            extra[name] = {"value": replica_rate(world, len(geos), args.steps, xms), "ms_per_step": xms / args.steps,
                           "stage_ms": dict(xstage), "refine_iters": [r.refine_iters for r in xres][:8]}
    if args.mode != "plain" and not args.no_plain:
        if dist:
            dist.barrier()
        pms, _, pres, pstage = time_mode(eng, stream, "plain", args.steps, warmup, flush=flush)
        plain_res = pres
        pms = max_over_ranks(pms)
        plain = {"value": replica_rate(world, len(geos), args.steps, pms), "ms_per_step": pms / args.steps,
                 "energies": [r.energy for r in pres][:8], "stage_ms": {k: v for k, v in pstage.items()}}
    if dist:
        dist.barrier()
    clk = ClockSampler(local)
    ms, stats, res, stage = time_mode(eng, stream, args.mode, args.steps, warmup, clocks=clk, flush=flush)
    ms = max_over_ranks(ms)
    value = replica_rate(world, len(geos), args.steps, ms)

    step_fl = fp64_step_flops(res)
    step_tf = step_fl / (ms / args.steps / 1000.0) / 1e12
    line = {"metric": METRIC, "value": value, "unit": "energies/s", "n_gpus": world, "steps": args.steps,
            "warmup": warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": {"plain": "f64", "mixed": "tf32x3+f64", "mixed_learned": "f64 (CG) + f32 (network)"}[args.mode],
            "data": "synthetic (seeded {H,C,N,O} " + ("periodic boxes" if WORKLOAD == "boxes" else "clusters")
                    + "; no dataset exists for this path)",
            "config": {"workload": workload_name(),
                       "mode": args.mode, "parallelism": f"replicas{world}" if world > 1 else "1gpu",
                       "l2": {"clusters": "working set 0.38-6.1 GB per geometry > 126 MB L2; no flush",
                              "batched": "working set up to 0.54 GB per geometry, 25 GB per batch > 126 MB L2; "
                                         "no flush",
                              "boxes": "working set 6.1-54 GB per geometry > 126 MB L2; no flush",
                              "sheet": "working set 25 MB < L2: a 512 MB buffer is rewritten before every timed "
                                       "step (outside the timed events)"}[WORKLOAD]},
            "gpu_launches": stats["launches"] * args.steps,
            "roofline": roofline(stage, [len(g.names) for g, _ in geos], args.mode),
            "roofline_step": {"bound": "fp64", "achieved": step_tf, "peak": FP64_NOMINAL_TFLOPS, "unit": "TFLOP/s",
                              "frac": step_tf / FP64_NOMINAL_TFLOPS, "flop_per_step": step_fl,
                              "algorithmic": "per energy 21 (3N)^3/3 + 126 (3N)^2 + (4/3)(3N n_SL)^3 FP64 flop "
                                             "(the reference's Cholesky, solves and Hamiltonian reduction) / "
                                             "device time of the whole step",
                              "peak_source": "nominal FP64 (148 SM x 64 DFMA/clk x 2 x 1965 MHz); "
                                             "MEASURED_PEAKS.json has no FP64 entry",
                              # the same work against a split-precision (3xTF32) tensor-core rate:
                              # the measured bf16 burst rate / 2 (TF32) / 3 (three products)
                              "frac_of_tf32_split": step_tf / (load_peaks()[0].get("bf16_tflops", 1590.0) / 6.0),
                              "tf32_split_peak": load_peaks()[0].get("bf16_tflops", 1590.0) / 6.0},
            "energies": [r.energy for r in res][:8],
            "refine_iters": [r.refine_iters for r in res][:8],
            "stage_ms": dict(stage)}
    line["autotune"] = {"seconds": tune_s, "choices": tuned}
    if learned is not None:
        line["learned"] = learned
    if WORKLOAD == "sheet":
        sr, lr = image_terms(*geos[0])
        build_ms = stage.get("relay_build", 0.0) + stage.get("cfdm_build", 0.0)
        line["image_sums"] = {"sr_terms_per_energy": sr, "lr_terms_per_energy": lr,
                              "build_ms": build_ms,
                              "build_ms_plain_fp64": (pstage.get("relay_build", 0.0) + pstage.get("cfdm_build", 0.0))
                              if plain is not None else None,
                              "build_ms_mixed_direct": (extra["mixed_direct"]["stage_ms"].get("relay_build", 0.0)
                                                        + extra["mixed_direct"]["stage_ms"].get("cfdm_build", 0.0))
                              if "mixed_direct" in extra else None,
                              "terms_per_s": (sr + lr) / (build_ms / 1000.0) if build_ms > 0 else None,
                              "note": "reference-equivalent (pair, image) terms of the short-range (x 21 "
                                      "frequencies) and long-range image sums / device time of the relay and "
                                      "CFDM tensor builds"}
    line.update(extra)
    if plain is not None:
        line["plain_fp64"] = plain
        line["speedup_vs_plain_fp64"] = value / plain["value"]
        line["max_abs_dE_vs_plain_fp64"] = max(abs(a.energy - b.energy) for a, b in zip(res, plain_res))
    if rank == 0:
        line["clocks"] = clk.summary()

    # end-to-end through the C ABI with host buffers
    if not args.no_e2e:
        if dist:
            dist.barrier()
        gl = [g for g, _ in geos]
        sl = [s for _, s in geos]
        eng.energy_batch(gl, sl, args.mode)
        torch.cuda.synchronize()
        with ClockSampler(local) as eclk:
            t0 = time.perf_counter()
            for _ in range(args.steps):
                rr = eng.energy_batch(gl, sl, args.mode)
            t_e2e = max_over_ranks(time.perf_counter() - t0)
        st2 = eng.stats()
        line["e2e"] = {"value": replica_rate(world, len(geos), args.steps, 1000.0 * t_e2e), "unit": "energies/s",
                       "h2d_bytes_per_step": st2["h2d_bytes"], "d2h_bytes_per_step": st2["d2h_bytes"],
                       "status": [r.status for r in rr], "clocks": eclk.summary(),
                       # how the last step's compute ran: kernel by kernel, or (with
                       # MBD_B200_GRAPH_UPDATE=1) as a graph of the batch's shape
                       "first_compute_graph": st2["first_compute_graph"], "graph_updates": st2["graph_updates"]}
    if WORKLOAD == "boxes":
        # one 200-atom box with these cut-offs already takes the oracle about
        # five minutes (its periodic image sums are numpy loops)
        line["cpu_baseline"] = {"value": None, "unit": "energies/s", "cores": os.cpu_count(), "kind": "port",
                                "sample": "not timed: the oracle needs minutes per 200-atom box at these cut-offs"}
    elif rank == 0 and world == 1 and not args.no_cpu_baseline and not args.sizes:
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
