"""Benchmark: F[rho] + dF/drho evaluations per second at 128^3 on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--precision fp64|mixed]

Workload (one "step" = one full F + dF/drho evaluation, functionals::total of
the reference): the 128^3 DDFT state of the LJ-fluid configuration --
periodic 128^3 grid, dx = 0.125 sigma, kT = 0.8, single species White-Bear-II
FMT with the WCA hard-sphere diameter of a cut LJ (sigma = eps = 1,
r_c = 2.5, QF weights), mean density 0.35 with seeded 1% white noise.  Inputs
are synthetic (seeded); no dataset is involved.

Timing: inputs resident in HBM, W untimed warm-up steps, then K steps, each
bracketed by CUDA events on the engine's stream with an L2 flush between
steps, outside the events: a write of a 256 MiB buffer, then a read of a
second one, so that no dirty line of the flush is written back inside the
timed region; barrier + synchronize on both sides; the max over ranks.  Each rank evaluates its own replica
(one grid does not shard: every transform of the evaluation is global), so `value` = N * K / max time.

`e2e` repeats the metric through the public host API with pinned host
buffers, H2D of every state's rho and D2H of its force and scalars inside the
timed region: `value` through cdft_total_stream (a sequence of states per
call, the copies of one state overlapping the evaluation of the next),
`per_call` through cdft_total (one state per call, copies and evaluation in
series), and `copy_bound` the same page-locked copies alone (the PCIe rate
the streamed number is measured against).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SHAPE = (128, 128, 128)
DX = 0.125
KT = 0.8
RHO_BAR = 0.35
SEED = 20261204
METRIC = "F+dF/drho evals/s at 128^3"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0


def workload_profile():
    rng = np.random.default_rng(SEED)
    return RHO_BAR * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, SHAPE[0] * SHAPE[1] * SHAPE[2]))


def hbm_peak():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


def stage_bytes(info, S=1, M=1, has_vext=False, fused=False):
    """Compulsory HBM bytes of each stage of one evaluation: one read and one
    write of every array the stage touches (each FFT counted as one read of its
    input and one write of its output), FP64 I/O for rho, V_ext and the force.
    Keys follow the engine's stage order (Engine.stage_names)."""
    N, Nk = info["N"], info["Nk"]
    C, D = info["channels"], info["deriv_channels"]
    s = 4 if info["precision"] == 1 else 8
    Br, Bc, Bio = N * s, 2 * Nk * s, 8 * N
    pointwise = C * Br + S * Bio * (2 if has_vext else 1) + D * Br + S * Bio
    if fused:
        return {
            "-0": 0,
            "plane_fwd_rho": S * Bio + S * Bc,  # the plane means re-read rho from L2
            "col_fwd": S * Bc + M * 4 * Nk + C * Bc,  # (+ MF weight, FP32 real)
            "plane_inv_channels": C * (Bc + Br),
            "pointwise": pointwise,
            "plane_fwd_derivatives": D * (Br + Bc),
            "col_bwd": D * Bc + S * Bc,
            "plane_inv_epilogue": S * Bc + 2 * S * Bio,
            "-8": 0,
            "-9": 0,
        }
    return {
        "split": (S * Bio + S * Br) if info["precision"] == 1 else 0,   # rho -> fp32 fluctuation
        "r2c_rho": S * Br + S * Bc,
        "k_forward": S * Bc + M * 8 * Nk + C * Bc,                     # (+ MF weight, FP64 real)
        "c2r_channels": C * (Bc + Br),
        "pointwise": pointwise,
        "r2c_derivatives": D * (Br + Bc),
        "k_backward": D * Bc + S * Bc,
        "c2r_force": S * (Bc + Br),
        "epilogue": S * Br + 2 * S * Bio,
        "reduce": 0,
    }


def algorithmic_bytes(info, S=1, M=1, has_vext=False, fused=False):
    """Compulsory HBM bytes of one evaluation (the sum over its stages)."""
    return sum(stage_bytes(info, S, M, has_vext, fused).values())


def unfused_bytes(N, Nk, s, S=1, C=11, M=1):
    """Compulsory HBM bytes of the unfused 25-transform decomposition of one
    evaluation (the reference's own pass structure: hard_sphere.hpp:50-136,
    mean_field.hpp:234-281, functionals.hpp:64-95): one read and one write per
    FFT pass and per pointwise pass, C FMT channels per species (eta, n2, v2
    and the six tensor components), M mean-field interactions, transforms in
    s-byte reals, rho and the force FP64.  128^3 mixed (s = 4): 0.934 GB."""
    Br, Bc, Bio = N * s, 2 * Nk * s, 8 * N
    SC = S * C
    return (S * Bio + 2 * S * Bc + M * Bc / 2 + 2 * (SC + M) * Bc + (SC + M) * Br + SC * Br + M * Br
            + 2 * S * Bio + SC * Br + S * Bio + SC * Br + 2 * SC * Bc + 2 * S * Bc + 2 * S * Br + 2 * S * Bio)


class L2Flush:
    """Between timed steps: write a 256 MiB buffer (more than the 126 MB L2),
    then read another, leaving L2 clean and cold."""

    def __init__(self, torch, dev):
        n = 256 * 1024 * 1024 // 4
        self.w = torch.empty(n, dtype=torch.float32, device=dev)
        self.r = torch.ones(n, dtype=torch.float32, device=dev)
        self.acc = torch.empty((), dtype=torch.float32, device=dev)
        self.torch = torch

    def __call__(self, i):
        self.w.fill_(float(i))
        self.torch.sum(self.r, 0, out=self.acc)


# DRAM bytes per launch of each fused-path stage, measured by ncu
# (dram__bytes_read.sum + dram__bytes_write.sum, 128^3 mixed, middle stages
# in one plane chunk).  The table is the text file below, written from the ncu
# CSV by `python bench.py --traffic-table <ncu.csv>`; a stage missing from it
# reports traffic null.
TRAFFIC_TABLE = os.path.join(ROOT, "profiles", "traffic_128cubed_mixed.txt")
FUSED_KERNELS = {  # kernel-name prefix in the ncu list -> stage (bool arguments print as 0 / 1)
    "k_rplane_fwd<128, 128, double": "plane_fwd_rho", "k_rcol_fwd1": "col_fwd",
    "k_rplane_inv<128, 128, 0": "plane_inv_channels", "k_rplane_inv<128, 128, false": "plane_inv_channels",
    "k_pointwise1_tma": "pointwise", "k_pointwise_tma": "pointwise",
    "k_rplane_fwd<128, 128, float": "plane_fwd_derivatives", "k_rcol_bwd1": "col_bwd",
    "k_rplane_inv<128, 128, 1": "plane_inv_epilogue", "k_rplane_inv<128, 128, true": "plane_inv_epilogue"}


def measured_traffic():
    """{stage: DRAM bytes per launch} from the traffic table (empty if absent)."""
    out = {}
    try:
        with open(TRAFFIC_TABLE) as f:
            for line in f:
                parts = line.split()
                if len(parts) >= 2 and not line.startswith("#"):
                    out[parts[0]] = float(parts[1])
    except OSError:
        pass
    return out


def _short_kernel_name(name):
    """ "void ns::k_x<1, 2>(args)" -> "k_x<1, 2>" """
    name = name.split("(")[0].replace("void ", "").strip()
    head, lt, tail = name.partition("<")
    return head.rsplit("::", 1)[-1] + lt + tail


def traffic_table(csv_path):
    """Reduce an ncu --csv launch list with dram__bytes_read.sum and
    dram__bytes_write.sum of the fused-path kernels to one line per stage:
    `<stage> <mean DRAM bytes per launch> <launches>`."""
    import csv
    scale = {"byte": 1.0, "Kbyte": 1e3, "Mbyte": 1e6, "Gbyte": 1e9, "KB": 1e3, "MB": 1e6, "GB": 1e9}
    with open(csv_path) as f:
        rows = [r for r in csv.reader(f)]
    head = next(i for i, r in enumerate(rows) if "Kernel Name" in r and "Metric Name" in r)
    h = rows[head]
    ki, mi, vi, ii = h.index("Kernel Name"), h.index("Metric Name"), h.index("Metric Value"), h.index("ID")
    ui = h.index("Metric Unit") if "Metric Unit" in h else None
    per = {}
    for r in rows[head + 1:]:
        if len(r) <= vi or r[mi] not in ("dram__bytes_read.sum", "dram__bytes_write.sum"):
            continue
        name = _short_kernel_name(r[ki])
        stage = next((st for pre, st in FUSED_KERNELS.items() if name.startswith(pre)), None)
        if stage is None:
            continue
        unit = scale.get(r[ui], 1.0) if ui is not None else 1.0
        per[(stage, r[ii])] = per.get((stage, r[ii]), 0.0) + float(r[vi].replace(",", "")) * unit
    acc = {}
    for (stage, _), b in per.items():
        acc.setdefault(stage, []).append(b)
    print("# stage  DRAM_bytes_per_launch  launches   (from " + os.path.basename(csv_path) + ")")
    for stage in dict.fromkeys(FUSED_KERNELS.values()):
        if stage in acc:
            v = acc[stage]
            print(f"{stage} {sum(v) / len(v):.4e} {len(v)}")


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def setup_dist(args):
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if ws > 1:
        import datetime
        import torch.distributed as d
        backend = "nccl" if (args.impl == "ours" and torch.cuda.is_available()) else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        d.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        dist = d
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return ws, rank, local, dist


def run_reference(args, ws, rank, dist):
    """--impl reference: the CPU restatement of the reference path (the oracle)
    on all host cores, same workload, bounded sample per step."""
    if rank != 0:
        return
    from oracle import fmt as ofmt
    from oracle import potentials as opot
    from oracle.functional import Model, Species, make_weights, total
    from oracle.grid import Grid, WORKERS
    lj = opot.make_lennard_jones(1.0, 1.0, 2.5)
    d = opot.hard_sphere_diameter(lj, KT, opot.WCA)
    g = Grid(dx=DX, box_size=tuple(n * DX for n in SHAPE), shape=SHAPE)
    model = Model(g, [Species("LJ", d)], [opot.Interaction(0, 0, lj)], KT)
    w = make_weights(ofmt.FMTModel("WhiteBearII"), model)
    rho = workload_profile()
    for _ in range(args.warmup):
        total(model, [rho], w, [0.0])
    budget = 150.0
    t0 = time.perf_counter()
    done = 0
    for _ in range(args.steps):
        total(model, [rho], w, [0.0])
        done += 1
        if time.perf_counter() - t0 > budget:
            break
    el = time.perf_counter() - t0
    v = done / el
    line = {"metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": ws, "steps": done, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / done, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": "128^3 LJ-fluid DDFT state, WhiteBearII + cut LJ (QF), 1 species",
                       "grid": list(SHAPE), "dx": DX, "kT": KT},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": WORKERS, "kind": "port",
                             "sample": f"{done} evaluations of the 128^3 workload (NumPy/SciPy FP64 oracle)"},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(seconds=12.0):
    """The oracle on the host cores, bounded to ~`seconds` of work."""
    from oracle import fmt as ofmt
    from oracle import potentials as opot
    from oracle.functional import Model, Species, make_weights, total
    from oracle.grid import Grid, WORKERS
    lj = opot.make_lennard_jones(1.0, 1.0, 2.5)
    d = opot.hard_sphere_diameter(lj, KT, opot.WCA)
    g = Grid(dx=DX, box_size=tuple(n * DX for n in SHAPE), shape=SHAPE)
    model = Model(g, [Species("LJ", d)], [opot.Interaction(0, 0, lj)], KT)
    w = make_weights(ofmt.FMTModel("WhiteBearII"), model)
    rho = workload_profile()
    total(model, [rho], w, [0.0])  # warm-up
    t0 = time.perf_counter()
    n = 0
    while True:
        ref = total(model, [rho], w, [0.0])
        n += 1
        if time.perf_counter() - t0 > seconds:
            break
    el = time.perf_counter() - t0
    return {"value": n / el, "unit": "evals/s", "cores": WORKERS, "kind": "port",
            "sample": f"{n} evaluations of the 128^3 workload (NumPy/SciPy FP64 oracle, scipy.fft workers={WORKERS})"}, ref


def _build_engine(cd, precision):
    lj = cd.make_lennard_jones(1.0, 1.0, 2.5)
    d = lj.hard_sphere_diameter(KT, cd.WEEKS_CHANDLER_ANDERSEN)
    g = cd.Grid(dx=DX, box_size=tuple(n * DX for n in SHAPE), shape=SHAPE)
    model = cd.Model(g, [cd.Species("LJ", d)], [cd.Interaction(0, 0, lj)], KT)
    return cd.Engine(cd.WhiteBearII(), model, precision), d


def _time_device(torch, eng, rho, force, scal, flush, stream, steps, warmup, sampler=None):
    """Per-step CUDA-event timing on the engine's stream, L2 flushed between steps."""
    sp = stream.cuda_stream

    def step():
        eng.total_device(rho.data_ptr(), None, [0.0], force.data_ptr(), scal.data_ptr(), sp)

    with torch.cuda.stream(stream):
        for _ in range(max(warmup, 3)):
            step()
    torch.cuda.synchronize()
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    if sampler:
        sampler.start()
        time.sleep(0.3)
    with torch.cuda.stream(stream):
        for i in range(steps):
            flush(i)
            starts[i].record(stream)
            step()
            ends[i].record(stream)
    torch.cuda.synchronize()
    clocks = sampler.stop() if sampler else None
    return float(np.sum([a.elapsed_time(b) for a, b in zip(starts, ends)])), clocks


def stage_breakdown(torch, eng, rho, force, scal, flush, stream, n, peak):
    """Live per-stage durations (CUDA events between the stages, on the
    evaluation's stream) and the HBM roofline fraction of each stage."""
    eng.stage_timing(True)
    eng.stage_times()
    with torch.cuda.stream(stream):
        for i in range(n):
            flush(i)
            eng.total_device(rho.data_ptr(), None, [0.0], force.data_ptr(), scal.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize()
    ms, count = eng.stage_times()
    eng.stage_timing(False)
    sb = stage_bytes(eng.info, fused=eng.transforms == "fused")
    out = {}
    for k, v in ms.items():
        if k.startswith("-"):
            continue  # a stage this path does not have (two adjacent events)
        t = v / max(count, 1)
        gbs = sb[k] / (t * 1e-3) / 1e9 if t > 0 and sb[k] else None
        out[k] = {"ms": t, "algorithmic_bytes": sb[k], "achieved_gbs": gbs,
                  "frac": (gbs / peak) if gbs else None,
                  "kind": "cuFFT" if k.startswith(("r2c", "c2r")) else "engine kernel"}
    return out


SWEEP_SHAPES = (48, 64, 96)
SWEEP_BATCH = 16


def batched_headline(torch, cd, dev, precision, rho, flush, stream, steps):
    """The headline state (128^3) as B = 2, 4 and 8 problems of one batched
    engine per launch (independent states sharing the launches: the
    throughput of evaluating many states, not the latency of one), in
    problem evaluations per second, L2 flushed between steps; and the FP64
    path batched the same way at B = 4 (fp64_B4), its like-for-like
    reference."""
    lj = cd.make_lennard_jones(1.0, 1.0, 2.5)
    d = lj.hard_sphere_diameter(KT, cd.WEEKS_CHANDLER_ANDERSEN)
    g = cd.Grid(dx=DX, box_size=tuple(n * DX for n in SHAPE), shape=SHAPE)
    model = cd.Model(g, [cd.Species("LJ", d)], [cd.Interaction(0, 0, lj)], KT)
    out = {}
    other = cd.FP64 if precision == cd.MIXED else cd.MIXED
    for B, prec in ((2, precision), (4, precision), (8, precision), (4, other)):
        eng = cd.Engine(cd.WhiteBearII(), model, prec, batch=B)
        rb = rho.repeat(B).contiguous()
        f = torch.empty_like(rb)
        sc = torch.empty((B, 10), dtype=torch.float64, device=dev)
        mus = [0.0] * B
        if eng.transforms == "fused":
            eng.autotune_ex(rb.data_ptr(), mu=mus, stream=stream.cuda_stream, reps=5)
        with torch.cuda.stream(stream):
            for _ in range(3):
                eng.total_device(rb.data_ptr(), None, mus, f.data_ptr(), sc.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        with torch.cuda.stream(stream):
            for i in range(steps):
                flush(i)
                evs[i][0].record(stream)
                eng.total_device(rb.data_ptr(), None, mus, f.data_ptr(), sc.data_ptr(), stream.cuda_stream)
                evs[i][1].record(stream)
        torch.cuda.synchronize()
        t = sum(a.elapsed_time(b) for a, b in evs) / steps
        key = f"B{B}" if prec == precision else ("fp64" if other == cd.FP64 else "mixed") + f"_B{B}"
        out[key] = {"problem_evals_per_s": B / (t * 1e-3), "ms_per_launch": t}
        eng.close()
    if "fp64_B4" in out:
        out["B4_vs_fp64_B4"] = out["B4"]["problem_evals_per_s"] / out["fp64_B4"]["problem_evals_per_s"]
    return out


def sweep_throughput(torch, cd, dev, precision, flush, stream, steps):
    """Batched evaluation of 16 problems of each grid of the parameter sweep
    (48^3, 64^3, 96^3 at dx = 0.1, kT = 1, WhiteBearII + cut LJ), as problem
    evaluations per second, against the same problems one engine call each."""
    lj = cd.make_lennard_jones(1.0, 1.0, 2.5)
    d = lj.hard_sphere_diameter(1.0, cd.WEEKS_CHANDLER_ANDERSEN)
    rng = np.random.default_rng(SEED + 4)
    out = {}
    for n in SWEEP_SHAPES:
        g = cd.Grid(dx=0.1, box_size=(0.1 * n,) * 3, shape=(n, n, n))
        model = cd.Model(g, [cd.Species("LJ", d)], [cd.Interaction(0, 0, lj)], 1.0)
        N = g.total_points
        rho = torch.tensor(0.6 * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, (SWEEP_BATCH, N))), device=dev)
        mus = list(np.linspace(-1.0, 2.0, SWEEP_BATCH))
        res = {}
        for B in (SWEEP_BATCH, 1):
            eng = cd.Engine(cd.WhiteBearII(), model, precision, batch=B)
            f = torch.empty((B, N), dtype=torch.float64, device=dev)
            sc = torch.empty((B, 10), dtype=torch.float64, device=dev)
            if eng.transforms == "fused":
                eng.autotune(rho[0].data_ptr(), mu=mus[:B], stream=stream.cuda_stream, reps=5)
            calls = SWEEP_BATCH // B

            def step():
                for c in range(calls):
                    eng.total_device(rho[c * B].data_ptr(), None, mus[c * B:(c + 1) * B], f.data_ptr(), sc.data_ptr(),
                                     stream.cuda_stream)
            with torch.cuda.stream(stream):
                for _ in range(3):
                    step()
            torch.cuda.synchronize()
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
            with torch.cuda.stream(stream):
                for i in range(steps):
                    flush(i)
                    evs[i][0].record(stream)
                    step()
                    evs[i][1].record(stream)
            torch.cuda.synchronize()
            t = sum(a.elapsed_time(b) for a, b in evs) / steps
            res[B] = SWEEP_BATCH / (t * 1e-3)
            eng.close()
        out[f"{n}^3"] = {"batched_problem_evals_per_s": res[SWEEP_BATCH], "one_by_one_problem_evals_per_s": res[1],
                         "speedup": res[SWEEP_BATCH] / res[1]}
    return out


def fire_step_rates(torch, cd, precision, steps=200):
    """FIRE minimisation steps per second (problem-steps: problems x steps),
    each step replayed as a captured CUDA graph and launched kernel by
    kernel: 16 problems at 48^3 on one batched engine, and one 16^3 problem
    (launch-bound).  Host-driven loop, timed by the wall clock around it."""
    import time
    lj = cd.make_lennard_jones(1.0, 1.0, 2.5)
    d = lj.hard_sphere_diameter(1.0, cd.WEEKS_CHANDLER_ANDERSEN)
    rng = np.random.default_rng(SEED + 5)
    out = {}
    for n, B in ((48, SWEEP_BATCH), (16, 1)):
        g = cd.Grid(dx=0.1, box_size=(0.1 * n,) * 3, shape=(n, n, n))
        model = cd.Model(g, [cd.Species("LJ", d)], [cd.Interaction(0, 0, lj)], 1.0)
        w = cd.make_weights(cd.FMTModel("WhiteBearII"), model, precision, batch=B)
        rho0 = 0.6 * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, (B, g.total_points)))
        mus = list(np.linspace(-1.0, 2.0, B))
        fire = cd.Fire(dt=0.01, dt_max=0.05, alpha_start=0.1, f_alpha=0.99, force_tolerance=1e-30, max_steps=steps)
        rate = {}
        try:
            for on in (True, False, True, False):
                cd.set_step_graphs(on)
                mz = cd.Minimizer(fire=fire, check_interval=50)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                if B > 1:
                    it = mz.grand_potential_batch(model, w, rho0, mus)[0].iterations
                else:
                    it = mz.grand_potential(model, w, rho0[0], mus[0]).iterations
                torch.cuda.synchronize()
                rate[on] = B * it / (time.perf_counter() - t0)  # the second run of each mode is kept
        finally:
            cd.set_step_graphs(True)
        out[f"{n}^3 x{B}"] = {"graph_problem_steps_per_s": rate[True], "direct_problem_steps_per_s": rate[False],
                              "speedup": rate[True] / rate[False]}
    return out


# ------------------------------------------------------------- config runs
#
# The other configurations of the workload family, each run once at N = 1 and
# reported beside the headline: the drivers at their stated sizes, mixed
# precision with FP64 refinement against FP64.


def _lj_model(cd, n, dx, kT, diameter=None, rc=2.5, batch_shape=None):
    lj = cd.make_lennard_jones(1.0, 1.0, rc)
    d = diameter if diameter is not None else lj.hard_sphere_diameter(kT, cd.WEEKS_CHANDLER_ANDERSEN)
    shape = batch_shape or (n, n, n)
    g = cd.Grid(dx=dx, box_size=tuple(k * dx for k in shape), shape=shape)
    return cd.Model(g, [cd.Species("LJ", d)], [cd.Interaction(0, 0, lj)], kT)


def _smoothed_gaussian_noise(shape, dx, width, rng):
    """Unit-normal white noise convolved with a normalised Gaussian of the
    given width (sigma units), rescaled to unit variance."""
    w = rng.standard_normal(shape)
    k = [2.0 * np.pi * np.fft.fftfreq(n, d=dx) for n in shape]
    K2 = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    f = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-0.5 * width * width * K2)))
    return (f / f.std()).reshape(-1)


def config_wall(cd, torch):
    """64^3, dx = 0.1, kT = 1, WBII (d = 1) + cut LJ (WCA, QF): rho = 0.5 (1 +
    0.05 G) with G seeded unit-normal noise smoothed over 0.5 sigma; a hard
    wall at x = 0 as rho = 0 and V_ext = 50 kT on the planes x < d/2.  FIRE
    grand-potential minimisation at the bulk mu of rho = 0.5 to tolerance
    1e-10 in FP64, and in mixed precision with the FP64 refine engine."""
    n, dx = 64, 0.1
    model = _lj_model(cd, n, dx, 1.0, diameter=1.0)
    rng = np.random.default_rng(SEED + 1)
    rho0 = 0.5 * (1.0 + 0.05 * _smoothed_gaussian_noise((n, n, n), dx, 0.5, rng))
    ix = np.repeat(np.arange(n), n * n)
    wall = ix * dx < 0.5
    rho0[wall] = 0.0
    vext = np.where(wall, 50.0, 0.0)
    w64 = cd.make_weights(cd.WhiteBearII(), model, cd.FP64)
    wmx = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)
    mu = cd.make_bulk_thermodynamics(model.species, w64).chemical_potential([0.5], 0)
    fire = cd.Fire(dt=0.1, dt_max=1.0, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-10, max_steps=50000)
    out = {"workload": "64^3 WBII + cut LJ, hard wall at x = 0, grand potential at the mu of rho = 0.5",
           "tolerance": "rms force 1e-10 (periodic box, no boundary treatment)"}
    res = {}
    for label, w, ref in (("fp64", w64, None), ("mixed_refined", wmx, w64)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = cd.Minimizer(fire=fire, refine=ref, refine_switch=1e3, use_homogeneous_boundary=False,
                         use_monitor=False).grand_potential(model, w, rho0, mu, external_field=vext)
        torch.cuda.synchronize()
        res[label] = r
        # the converged residual: max |dOmega/drho| over the fluid
        chk = cd.total(model, [r.densities[0]], w64, [mu], [vext])
        resid = float(np.max(np.abs(chk.forces[0][~wall]))) / model.grid.cell_volume
        out[label] = {"iterations": r.iterations, "converged": r.converged, "wall_s": time.perf_counter() - t0,
                      "grand_potential": r.grand_potential, "max_dOmega_drho_fluid": resid}
    a, b = res["fp64"], res["mixed_refined"]
    out["mixed_vs_fp64"] = {"max_drho": float(np.max(np.abs(a.densities[0] - b.densities[0]))),
                            "dOmega_over_Omega": abs(a.grand_potential - b.grand_potential) / abs(a.grand_potential)}
    # two profiles that both meet rms 1e-10 differ by up to ~1e-8 (the
    # criterion's tolerance ball); both converged to 1e-11 they agree closer
    tight = cd.Fire(dt=0.1, dt_max=1.0, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-11, max_steps=50000)
    tr = {}
    for label, w, ref in (("fp64", w64, None), ("mixed_refined", wmx, w64)):
        tr[label] = cd.Minimizer(fire=tight, refine=ref, refine_switch=1e3, use_homogeneous_boundary=False,
                                 use_monitor=False).grand_potential(model, w, rho0, mu, external_field=vext)
    out["mixed_vs_fp64_at_1e-11"] = {
        "iterations": [tr["fp64"].iterations, tr["mixed_refined"].iterations],
        "converged": tr["fp64"].converged and tr["mixed_refined"].converged,
        "max_drho": float(np.max(np.abs(tr["fp64"].densities[0] - tr["mixed_refined"].densities[0])))}
    for w in (w64, wmx):
        w.engine.close()
    return out


def config_ddft(cd, torch, n_steps=2000):
    """The headline state (128^3, dx = 0.125, kT = 0.8, rho = 0.35 (1 + 0.01 U))
    relaxed by 2000 integrating-factor DDFT steps at dt = 1e-4 (dt_max = dt),
    fixed-point tolerance 1e-8: FP64, and mixed precision with two FP64
    refinement iterations per step; the difference every 100 steps."""
    model = _lj_model(cd, 128, DX, KT)
    rho0 = workload_profile()
    w64 = cd.make_weights(cd.WhiteBearII(), model, cd.FP64)
    wmx = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)
    runs, times = {}, {}
    # mixed: FP32 transforms, FP64 Phi and sums; mixed_fp64_energy: the same
    # steps with each step's final compute (its energy and forces) in FP64
    for label, w, ref in (("fp64", w64, None), ("mixed", wmx, None), ("mixed_fp64_energy", wmx, w64)):
        sim = cd.Simulation(step=cd.StepConfig(dt=1e-4, dt_max=1e-4, fp_tolerance=1e-8), n_steps=n_steps,
                            snapshot_interval=100, log_interval=100, refine=ref, refine_iterations=0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        runs[label] = sim.run([rho0], w, 0.0)
        torch.cuda.synchronize()
        times[label] = time.perf_counter() - t0
    out = {"workload": f"128^3 LJ fluid, {n_steps} IF steps at dt = 1e-4, fp_tolerance 1e-8"}
    for label in ("fp64", "mixed", "mixed_fp64_energy"):
        out[label] = {"s": times[label], "steps_per_s": n_steps / times[label]}
    for label in ("mixed", "mixed_fp64_energy"):
        per = []
        for a, b in zip(runs["fp64"]["snapshots"], runs[label]["snapshots"]):
            per.append([a.step, float(np.max(np.abs(a.densities[0] - b.densities[0]))),
                        abs(a.energy - b.energy) / abs(a.energy)])
        out[label].update({"vs_fp64_per_100_steps": {"columns": ["step", "max_drho", "dF_over_F"], "rows": per},
                           "max_drho": max(r[1] for r in per), "max_dF_over_F": max(r[2] for r in per),
                           "speedup_vs_fp64": times["fp64"] / times[label]})
    for w in (w64, wmx):
        w.engine.close()
    return out


def config_nucleus(cd, torch):
    """Critical vapour-liquid nucleus: 128^3, dx = 0.1 (L = 12.8), LJ (rc = 3)
    at kT = 0.7, WBII; vapour at S = 1.5 times the coexisting vapour density,
    a tanh droplet of radius 3 sigma and width 0.5 of the coexisting liquid;
    the fixed-mass FP64 FIRE cluster, then the saddle search (eigenvector
    following at fixed mass, the lowest mode by block Lanczos, block 2, on
    batched FP64 Hessian-vector products) in FP64 and in mixed precision with
    the FP64 refine engine, both from that cluster.  The barrier is Omega at
    the saddle minus Omega of the uniform background at its chemical
    potential."""
    n, dx, kT = 128, 0.1, 0.7
    model = _lj_model(cd, n, dx, kT, rc=3.0)
    w64 = cd.make_weights(cd.WhiteBearII(), model, cd.FP64)
    wmx = cd.make_weights(cd.WhiteBearII(), model, cd.MIXED)
    hw = cd.make_weights(cd.WhiteBearII(), model, cd.FP64, batch=2)
    eos = cd.make_bulk_thermodynamics(model.species, w64)
    co = cd.PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_coexistence(eos)
    rout = 1.5 * co.rho_vapor
    mu = eos.chemical_potential([rout], 0)
    x = np.arange(n) * dx - n * dx / 2
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X ** 2 + Y ** 2 + Z ** 2).ravel()
    rho0 = rout + (co.rho_liquid - rout) * 0.5 * (1.0 - np.tanh((r - 3.0) / 0.5))
    dv = model.grid.cell_volume
    tm = float(rho0.sum()) * dv
    out = {"workload": "128^3 LJ nucleus at kT = 0.7, S = 1.5, tanh R = 3 sigma (WBII)",
           "rho_vapor": co.rho_vapor, "rho_liquid": co.rho_liquid}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    cl = cd.Minimizer(fire=cd.Fire(dt=0.1, dt_max=1.0, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-9,
                                   max_steps=50000), param=cd.Unbounded(1e-99)).fixed_mass(model, w64, rho0, mu, tm)
    torch.cuda.synchronize()
    rc = np.asarray(cl.densities[0])
    faces = model.grid.boundary_mask().astype(bool)
    bg = float(rc[faces].mean())
    mubg = eos.chemical_potential([bg], 0)
    omega_bg = cd.total(model, [np.full(rc.size, bg)], w64, [mubg]).grand_potential
    out["cluster"] = {"iterations": cl.iterations, "converged": cl.converged, "s": time.perf_counter() - t0,
                      "background": bg, "max_density": float(rc.max())}
    res = {}
    for label, w, kw in (("fp64", w64, {}), ("mixed_refined", wmx, {"refine": w64})):
        se = cd.Search(fire=cd.Fire(dt=1e-3, dt_max=1.0, alpha_start=0.01, f_alpha=1.0, force_tolerance=1e-10,
                                    max_steps=20000),
                       eigenvalue=cd.EigenvalueSolver(1e-6, 300, exact_hvp=True, method="lanczos", block=2),
                       omega_tolerance=1e-9, tolerance_start=1e-6, max_outer_iterations=12, hvp_weights=hw, **kw)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s_ = se.find(model, w, rc, mubg, tm)
        torch.cuda.synchronize()
        res[label] = s_
        out[label] = {"barrier": s_.grand_potential - omega_bg, "grand_potential": s_.grand_potential,
                      "eigenvalue": s_.eigenvalue, "converged": s_.converged,
                      "outer_iterations": s_.outer_iterations, "fire_steps": s_.fire_steps,
                      "lanczos_products": s_.eigen_iterations, "s": time.perf_counter() - t0}
    a, b = out["fp64"], out["mixed_refined"]
    out["mixed_vs_fp64"] = {"barrier_rel": abs(a["barrier"] - b["barrier"]) / abs(a["barrier"]),
                            "eigenvalue_rel": abs(a["eigenvalue"] - b["eigenvalue"]) / abs(a["eigenvalue"]),
                            "max_drho": float(np.max(np.abs(res["fp64"].density - res["mixed_refined"].density)))}
    for w in (w64, wmx, hw):
        w.engine.close()
    return out


def config_solid(cd, torch, cells=8, reps=5):
    """The binary hard-sphere FCC solid: 256^3 on 8 x 8 x 8 cells (a = 1.55,
    dx = 0.0484375), large spheres (d = 1) as Gaussian peaks (alpha = 50, 0.8
    particles per site) on FCC(001) sites, small spheres (d = 0.5) uniform at
    0.1, esFMT A = 1 B = 0.  At the crystal and 1% off it (the crystal times
    1 + 0.01 G, G smoothed unit noise, seeded): FP64, mixed with the mean
    split, and mixed with the anchored split at the crystal (FP64 channels
    of the anchor, FP32 transforms of the difference).  The FP64 engine is
    pinned to the oracle at 64^3 on the same solid."""
    import math
    from classicaldft_b200 import crystal as cc
    a_fcc, dx, alpha, occ = 1.55, 0.0484375, 50.0, 0.8
    n = int(round(cells * a_fcc / dx))
    lat = cc.build_lattice(cc.Structure.FCC, cc.Orientation._001, (cells,) * 3)
    sites = lat.scaled_positions(a_fcc / math.sqrt(2.0))
    grid = cd.Grid(dx=dx, box_size=(n * dx,) * 3, shape=(n,) * 3)
    rho1 = cc.gaussian_peaks(grid, sites, alpha, occ * (alpha / math.pi) ** 1.5, 0.0)
    N = grid.total_points
    rho2 = torch.full((N,), 0.1, dtype=torch.float64, device=rho1.device)
    model = cd.Model(grid, [cd.Species("large", 1.0), cd.Species("small", 0.5)], [], 1.0)
    fmt = cd.FMTModel("esFMT", 1.0, 0.0)
    gen = torch.Generator(device=rho1.device).manual_seed(SEED + 5)
    noise = torch.randn(2, n, n, n, dtype=torch.float64, device=rho1.device, generator=gen)
    k = torch.fft.fftfreq(n, device=rho1.device, dtype=torch.float64)
    K2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    g = torch.fft.ifftn(torch.fft.fftn(noise, dim=(1, 2, 3)) * torch.exp(-2.0 * (math.pi * 2.0) ** 2 * K2),
                        dim=(1, 2, 3)).real
    g = (g / g.std(dim=(1, 2, 3), keepdim=True)).reshape(2, N)
    crystal = torch.cat([rho1, rho2]).contiguous()
    near = torch.cat([rho1 * (1.0 + 0.01 * g[0]), rho2 * (1.0 + 0.01 * g[1])]).contiguous()
    del noise, g, K2
    w64 = cd.make_weights(fmt, model, cd.FP64)
    wmx = cd.make_weights(fmt, model, cd.MIXED)
    force = torch.empty_like(crystal)
    scal = torch.zeros(10, dtype=torch.float64, device=crystal.device)
    mu = [0.0, 0.0]

    def run(w, x):
        w.engine.total_device(x.data_ptr(), None, mu, force.data_ptr(), scal.data_ptr(), 0)
        torch.cuda.synchronize()
        return float(scal[0]), force.clone()

    def rate(w, x):
        run(w, x)
        t0 = time.perf_counter()
        for _ in range(reps):
            w.engine.total_device(x.data_ptr(), None, mu, force.data_ptr(), scal.data_ptr(), 0)
        torch.cuda.synchronize()
        return reps / (time.perf_counter() - t0)

    out = {"workload": f"{n}^3 binary hard-sphere FCC solid ({cells}^3 cells, a = 1.55), esFMT A = 1 B = 0",
           "states": {"crystal": "Gaussian peaks alpha = 50, 0.8 per site; small spheres 0.1",
                      "near": "the crystal times 1 + 0.01 G (G smoothed unit noise, seeded)"}}
    res = {}
    for label, x in (("crystal", crystal), ("near", near)):
        f64, F64 = run(w64, x)
        fmx, Fmx = run(wmx, x)
        res[label] = (f64, F64, fmx, Fmx)
    wmx.engine.set_anchor(w64.engine, crystal)
    for label, x in (("crystal", crystal), ("near", near)):
        f64, F64, fmx, Fmx = res[label]
        fan, Fan = run(wmx, x)
        den = float(F64.abs().max())
        out[label] = {"F_fp64": f64,
                      "mixed_mean_split": {"dF_over_F": abs(fmx - f64) / abs(f64),
                                           "max_dforce_over_max_force": float((Fmx - F64).abs().max()) / den},
                      "mixed_anchored": {"dF_over_F": abs(fan - f64) / abs(f64),
                                         "max_dforce_over_max_force": float((Fan - F64).abs().max()) / den}}
    out["evals_per_s"] = {"fp64": rate(w64, near), "mixed_anchored": rate(wmx, near)}
    wmx.engine.clear_anchor()
    out["evals_per_s"]["mixed_mean_split"] = rate(wmx, near)
    for w in (w64, wmx):
        w.engine.close()
    return out


def config_sweep(cd, torch):
    """16 state points each on 48^3, 64^3 and 96^3 grids (dx = 0.1, kT = 1,
    WBII + cut LJ), mu evenly spaced over the liquid branch (from the bulk
    coexistence to 1.5 above it), seeded 1% noise around the bulk liquid
    density: FIRE grand-potential minimisations as one group minimisation
    (one graph launch per step for all 48), against the three per-size
    batched minimisations one after another."""
    per = 16
    lj = cd.make_lennard_jones(1.0, 1.0, 2.5)
    rng = np.random.default_rng(SEED + 4)
    fire = cd.Fire(dt=0.05, dt_max=0.5, alpha_start=0.01, f_alpha=0.99, force_tolerance=1e-10, max_steps=4000)
    members, ws = [], []
    eos = None
    for n in SWEEP_SHAPES:
        model = _lj_model(cd, n, 0.1, 1.0)
        w = cd.make_weights(cd.WhiteBearII(), model, cd.FP64, batch=per)
        if eos is None:
            eos = cd.make_bulk_thermodynamics(model.species, w)
            co = cd.PhaseSearch(rho_max=1.0, rho_scan_step=0.005).find_coexistence(eos)
            mu_coex = eos.chemical_potential([co.rho_liquid], 0)
            mus = np.linspace(mu_coex, mu_coex + 1.5, per)
            rl = [cd.density_from_chemical_potential(m, co.rho_liquid, eos) for m in mus]
        N = model.grid.total_points
        rhos = np.stack([rl[b] * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, N)) for b in range(per)])
        members.append((w, rhos, mus, None))
        ws.append(w)
    mz = cd.Minimizer(fire=fire)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = mz.minimize_group(members)
    torch.cuda.synchronize()
    t_group = time.perf_counter() - t0
    t0 = time.perf_counter()
    seq = [mz.grand_potential_batch(None, w, rhos, mus) for (w, rhos, mus, _) in members]
    torch.cuda.synchronize()
    t_seq = time.perf_counter() - t0
    steps = sum(r.iterations for rs in res for r in rs)
    same = all(np.array_equal(a.densities[0], b.densities[0]) for ra, rb in zip(res, seq) for a, b in zip(ra, rb))
    for w in ws:
        w.engine.close()
    return {"workload": "16 each of 48^3 / 64^3 / 96^3 grand-potential minimisations (WBII + cut LJ, kT = 1)",
            "converged": int(sum(r.converged for rs in res for r in rs)), "problems": 3 * per,
            "problem_steps": steps, "group_s": t_group, "per_size_batches_s": t_seq,
            "group_problem_steps_per_s": steps / t_group, "per_size_problem_steps_per_s": steps / t_seq,
            "speedup": t_seq / t_group, "identical_to_per_size_runs": bool(same)}


def run_ours(args, ws, rank, local, dist):
    import ctypes
    import torch
    import classicaldft_b200 as cd
    dev = torch.device("cuda", local)
    precision = cd.MIXED if args.precision == "mixed" else cd.FP64
    eng, d = _build_engine(cd, precision)
    rho_h = workload_profile()
    rho = torch.tensor(rho_h, dtype=torch.float64, device=dev)
    tuned = None
    if args.plane_chunks:
        eng.set_plane_chunks(args.plane_chunks)
        if args.pointwise >= 0:
            eng.set_pointwise(args.pointwise)
        if args.pointwise_spread >= 0:
            eng.set_pointwise_spread(args.pointwise_spread)
    elif eng.transforms == "fused":
        # the engine's autotuner picks the plane-chunk count and the pointwise
        # kernel variant on this state
        (k, v, tq, sp), ms = eng.autotune_ex(rho.data_ptr(), mu=[0.0], reps=10)
        pw_kept = eng.plane_width
        tuned = {"chosen": {"plane_chunks": k, "pointwise_variant": v, "column_tile": tq, "pointwise_spread": sp,
                            "plane_width": pw_kept},
                 "ms_per_eval": {f"t{tt}_v{vv}_k{c}_d{dd}": round(t, 5) for (tt, vv, c, dd), t in ms.items()}}
        # back-to-back evaluations, CUDA events: programmatic dependent launch
        # between the passes off against on (the timed run uses on), and the
        # two middle plane widths at the chosen configuration
        f_tmp = torch.empty_like(rho)
        s_tmp = torch.zeros(10, dtype=torch.float64, device=dev)

        def per_eval():
            for _ in range(3):
                eng.total_device(rho.data_ptr(), None, [0.0], f_tmp.data_ptr(), s_tmp.data_ptr(), 0)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(50):
                eng.total_device(rho.data_ptr(), None, [0.0], f_tmp.data_ptr(), s_tmp.data_ptr(), 0)
            e1.record()
            torch.cuda.synchronize()
            return round(e0.elapsed_time(e1) / 50, 5)

        dl, pw = {}, {}
        for on in (False, True, False, True):
            eng.set_dependent_launch(on)
            dl.setdefault("on_ms" if on else "off_ms", []).append(per_eval())
        for wide in (0, 1, 0, 1):
            eng.set_plane_width(wide)
            pw.setdefault(f"width{wide}_ms", []).append(per_eval())
        eng.set_plane_width(pw_kept)
        tuned["dependent_launch"] = dl
        tuned["plane_width"] = pw
    force = torch.empty_like(rho)
    scal = torch.zeros(10, dtype=torch.float64, device=dev)
    flush = L2Flush(torch, dev)
    stream = torch.cuda.Stream(device=dev)
    sampler = ClockSampler(torch.cuda.current_device() if "CUDA_VISIBLE_DEVICES" not in os.environ else local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    t_ms, clocks = _time_device(torch, eng, rho, force, scal, flush, stream, args.steps, args.warmup, sampler)
    if dist:
        dist.barrier()
        tt = torch.tensor([t_ms], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_ms = float(tt.item())
    value = ws * args.steps / (t_ms * 1e-3)
    ms_step = t_ms / args.steps
    f_main = force.clone()
    s_main = scal.clone()

    # the other precision on the same input: throughput and the accuracy of mixed vs FP64
    other = cd.FP64 if precision == cd.MIXED else cd.MIXED
    eng2, _ = _build_engine(cd, other)
    force2 = torch.empty_like(rho)
    scal2 = torch.zeros(10, dtype=torch.float64, device=dev)
    t2, _ = _time_device(torch, eng2, rho, force2, scal2, flush, stream, max(args.steps // 2, 10), args.warmup)
    if dist:
        tt = torch.tensor([t2], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t2 = float(tt.item())
    n2 = max(args.steps // 2, 10)
    f64, f32 = (force2, f_main) if precision == cd.MIXED else (f_main, force2)
    s64, s32 = (scal2, s_main) if precision == cd.MIXED else (s_main, scal2)
    dF = abs(float(s32[0]) - float(s64[0])) / abs(float(s64[0]))
    dforce = float((f32 - f64).abs().max() / f64.abs().max())
    eng2.close()

    # e2e through the host API with pinned buffers: one cdft_total per state,
    # and cdft_total_stream over a sequence of states (copies of one state
    # overlapping the evaluation of the next)
    rho_pin = torch.tensor(rho_h, dtype=torch.float64).pin_memory()
    f_pin = torch.empty_like(rho_pin).pin_memory()
    sc_pin = torch.empty(10, dtype=torch.float64).pin_memory()
    L = cd.lib()
    mu = (ctypes.c_double * 1)(0.0)

    def e2e_step():
        st = L.cdft_total(eng.handle, rho_pin.data_ptr(), None, mu, f_pin.data_ptr(),
                          ctypes.cast(sc_pin.data_ptr(), ctypes.POINTER(ctypes.c_double)))
        if st != 0:
            raise RuntimeError(L.cdft_last_error().decode())

    def timed_max(fn, reps):
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            fn()
        el = time.perf_counter() - t0
        if dist:
            tt = torch.tensor([el], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            el = float(tt.item())
        return el

    for _ in range(3):
        e2e_step()
    n_e2e = max(10, min(args.steps, 200))
    e2e_call_val = ws * n_e2e / timed_max(e2e_step, n_e2e)

    ring = 4  # distinct page-locked states and force buffers, reused round robin
    rho_ring = [torch.tensor(rho_h * (1.0 + 1e-3 * i), dtype=torch.float64).pin_memory() for i in range(ring)]
    f_ring = [torch.empty_like(rho_pin).pin_memory() for _ in range(ring)]
    n_stream = max(20, min(args.steps, 200))
    rptr = [rho_ring[i % ring].data_ptr() for i in range(n_stream)]
    fptr = [f_ring[i % ring].data_ptr() for i in range(n_stream)]
    mus_stream = np.zeros((n_stream, 1))
    eng.total_stream_ptrs(rptr[:ring], mus_stream[:ring], fptr[:ring])  # warm-up (device slots)
    e2e_val = ws * n_stream / timed_max(lambda: eng.total_stream_ptrs(rptr, mus_stream, fptr), 1)
    # the PCIe bound of that number: the same page-locked copies alone, the
    # state in on one stream and the force out on another
    d_in = torch.empty(rho_pin.numel(), dtype=torch.float64, device=dev)
    d_out = torch.zeros_like(d_in)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def copies_only():
        for i in range(n_stream):
            with torch.cuda.stream(s_in):
                d_in.copy_(rho_ring[i % ring], non_blocking=True)
            with torch.cuda.stream(s_out):
                f_ring[i % ring].copy_(d_out, non_blocking=True)
        s_in.synchronize()
        s_out.synchronize()

    copies_only()
    copy_val = ws * n_stream / timed_max(copies_only, 1)

    info = eng.info
    fused = eng.transforms == "fused"
    nbytes = algorithmic_bytes(info, S=1, M=1, fused=fused)
    ub = unfused_bytes(info["N"], info["Nk"], 4 if precision == cd.MIXED else 8)
    peak, peak_kind = hbm_peak()
    achieved = nbytes / (ms_step * 1e-3) / 1e9
    names = {cd.MIXED: "mixed", cd.FP64: "fp64"}
    stages = stage_breakdown(torch, eng, rho, force, scal, flush, stream, max(10, min(args.steps, 100)), peak)
    mine = {k: v for k, v in stages.items() if v["kind"] == "engine kernel" and v["algorithmic_bytes"]}
    top = max(mine, key=lambda k: mine[k]["ms"])
    traffic = measured_traffic()
    sweep = None if args.no_sweep else sweep_throughput(torch, cd, dev, precision, flush, stream, 20)
    batched = None if args.no_sweep else batched_headline(torch, cd, dev, precision, rho, flush, stream, 20)
    fire_rates = None if args.no_sweep else fire_step_rates(torch, cd, precision)
    line = {
        "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": ws, "steps": args.steps,
        "warmup": max(args.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 FFT+k-space / f64 Phi+sums" if precision == cd.MIXED else "f64",
        "data": "synthetic",
        "config": {"workload": "128^3 LJ-fluid DDFT state, WhiteBearII + cut LJ (QF), 1 species",
                   "grid": list(SHAPE), "dx": DX, "kT": KT, "rho_bar": RHO_BAR, "noise": "1% uniform, seeded",
                   "hs_diameter": d, "precision": names[precision], "parallelism": f"replicas x{ws}",
                   "l2": "flushed between timed steps (256 MiB write + 256 MiB read, outside the events)",
                   "transforms": eng.transforms, "plane_chunks": (info["kernels_per_eval"] - 4) // 3 if fused else None,
                   "autotune": tuned},
        # the dominant kernel (the longest stage of the evaluation): its
        # algorithmic bytes over its live duration; the whole evaluation beside it
        "roofline": {"bound": "hbm", "kernel": top, "achieved": mine[top]["achieved_gbs"], "peak": peak,
                     "unit": "GB/s", "frac": mine[top]["frac"],
                     "traffic": traffic.get(top) if fused and precision == cd.MIXED else None,
                     "algorithmic_bytes": mine[top]["algorithmic_bytes"], "ms": mine[top]["ms"],
                     "peak_source": peak_kind,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch, "
                                       "profiles/traffic_128cubed_mixed.txt",
                     "evaluation": {
                         "achieved": achieved, "frac": achieved / peak, "algorithmic_bytes": nbytes,
                         "traffic": (sum(traffic[k] for k in FUSED_KERNELS.values())
                                     if fused and precision == cd.MIXED and all(k in traffic for k in
                                                                                 FUSED_KERNELS.values())
                                     else None),
                         "scope": ("one full evaluation (the seven fused-path kernels)" if fused
                                   else "one full evaluation (cuFFT transforms + engine kernels)"),
                         # the same time against the bytes of the unfused 25-transform
                         # decomposition (what a pass-per-transform evaluation must move)
                         "unfused_count": {"algorithmic_bytes": ub, "achieved": ub / (ms_step * 1e-3) / 1e9,
                                           "frac": ub / (ms_step * 1e-3) / 1e9 / peak}}},
        "stages": stages,
        "sweep": sweep,
        "batched_128": batched,
        "fire_steps": fire_rates,
        names[other]: {"value": ws * n2 / (t2 * 1e-3), "ms_per_step": t2 / n2},
        "mixed_vs_fp64": {"dF_over_F": dF, "max_dforce_over_max_force": dforce},
        "e2e": {"value": e2e_val, "unit": "evals/s", "h2d_bytes_per_step": 8 * info["N"],
                "d2h_bytes_per_step": 8 * info["N"] + 80,
                "api": f"cdft_total_stream: {n_stream} host states per call, page-locked, copies overlapped",
                "per_call": {"value": e2e_call_val, "unit": "evals/s",
                             "api": "cdft_total: one host state per call, page-locked"},
                "copy_bound": {"value": copy_val, "unit": "evals/s", "frac": e2e_val / copy_val,
                               "what": "the same page-locked H2D and D2H copies alone, one stream each way"}},
        "clocks": clocks,
        "gpu_launches": int(info["kernels_per_eval"]) * args.steps,
    }
    if ws == 1 and not args.no_configs:
        # the other configurations at their own sizes (N = 1 only)
        for key, fn in (("config_wall_64", config_wall), ("config_ddft_128", config_ddft),
                        ("config_nucleus_128", config_nucleus), ("config_sweep_48_64_96", config_sweep),
                        ("config_solid_256", config_solid)):
            try:
                line[key] = fn(cd, torch)
            except Exception as exc:  # reported, not hidden
                line[key] = {"error": f"{type(exc).__name__}: {exc}"}
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cb, ref = cpu_baseline_sample(args.cpu_seconds)
        line["cpu_baseline"] = cb
        # the timed runs' outputs against the oracle's evaluation of the same state
        f_ref = ref.forces[0]
        fmax = float(np.max(np.abs(f_ref)))
        for key, f_dev, s_dev in (("oracle_vs_mixed", f32, s32), ("oracle_vs_fp64", f64, s64)):
            line[key] = {"dF_over_F": abs(float(s_dev[0]) - ref.free_energy) / abs(ref.free_energy),
                         "dOmega_over_Omega": abs(float(s_dev[1]) - ref.grand_potential) / abs(ref.grand_potential),
                         "max_dforce_over_max_force": float(np.max(np.abs(f_dev.cpu().numpy() - f_ref))) / fmax}
    if rank == 0:
        print(json.dumps(line), flush=True)
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-sweep", action="store_true", help="skip the batched 48/64/96^3 sweep measurement")
    ap.add_argument("--plane-chunks", type=int, default=0,
                    help="plane chunks of the fused path's middle stages (0: the engine's default; 1 runs them "
                         "back to back, as a profiler's serialised launch list sees them)")
    ap.add_argument("--pointwise", type=int, default=-1,
                    help="with --plane-chunks: the pointwise kernel variant (0 generic, 1 / 2 one species at 5 / 6 "
                         "CTAs per SM, 3 branch-free, 4 / 5 branch-free with two points per thread at 3 / 4 "
                         "CTAs per SM; -1: the engine's default)")
    ap.add_argument("--pointwise-spread", type=int, default=-1,
                    help="with --plane-chunks: divisor of the pointwise grid per chunk (0: the chunk count)")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the runs of the other configurations (wall, DDFT, nucleus, uneven sweep)")
    ap.add_argument("--traffic-table", metavar="NCU_CSV",
                    help="print the per-stage DRAM traffic table from an ncu --csv launch list and exit")
    args = ap.parse_args()
    if args.traffic_table:
        traffic_table(args.traffic_table)
        return
    ws, rank, local, dist = setup_dist(args)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank, dist)
        else:
            run_ours(args, ws, rank, local, dist)
    finally:
        if dist:
            dist.barrier()
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
