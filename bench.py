#!/usr/bin/env python
"""Benchmark of the FP64 GPU time step (cell-steps/s at 257^3).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): the 257^3-node grid on [-1,1]^3 (h = 1/128, the "256^3"
of the headline metric), Douglas-ADI + MIB-L2, torus R=0.5 r=0.2, beta 1:1000,
exact solution e^{-t}(...) (eq 8), dt = h, FP64.  A "step" is one time step
of that problem, computed by the fast FP64 form (MTS_PRECISION_FAST: FP64
throughout, equal to the reference up to rounding); the bit-exact plain form
is timed beside it.  Each field is 136 MB and a step streams ~1 GB, larger
than the 126 MB L2, so no explicit L2 flush is needed between steps.

Multi-GPU: one independent replica per rank (the path does not shard; no
collective on the data path), weak scaling; value = all ranks' cell-steps over
the max-over-ranks device time.

Prints one JSON line (rank 0).
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "matched-time-splitting-3d_b200"))

WORKLOAD = dict(n=(257, 257, 257), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=1000.0, eq=8,
                method="adi", mib=2, dt=2.0 / 256)
METRIC = "cell-steps/s @256^3 plain FP64"
# Algorithmic bytes per node and step of the fast FP64 form: the residual
# with the x solve (read u^n 8 + tag 1, write d* 8), the y solve in place
# (read 8, write 8), the z solve with the update (read d** 8, read u^n 8,
# write u^{n+1} 8).
FAST_BYTES = {0: 17, 1: 16, 2: 24}
FAST_NAMES = ["fast_x_residual_and_solve", "fast_y_solve", "fast_z_solve_and_update"]
REF_MAX_STEPS = 3  # timed steps per reference process (CPU arm)
# Algorithmic bytes per node and step of the mixed ADI form: residual (read
# u^n 8 + tag 1, write rho 4), x and y FP32 solves (read 4, write 4 each),
# and the z solve with the accumulation (read 4, read u^n 8, write u^{n+1}
# 8).  The per-node coefficients that crossing lines read (12 bytes a node
# of those lines) are the factorisation, not counted, as in the plain model.
MIXED_BYTES = 13 + 8 + 8 + 20
CONTRACT_BYTES = {"adi": 67, "lod-ie": 51, "lod-cn": 51, "ts": 102}
PEAKS_PATH = os.path.join(ROOT, "MEASURED_PEAKS.json")


def peak_hbm() -> float:
    """Measured copy bandwidth of this pool's B200s (GB/s), else the fallback."""
    if os.path.exists(PEAKS_PATH):
        with open(PEAKS_PATH) as f:
            return float(json.load(f)["hbm_gbs"])
    return 6650.0

# Algorithmic HBM bytes per grid node per launch of each kernel slot
# (field reads/writes at 8 B plus the 1-byte node tag; scratch excluded).
ALG_BYTES = {
    "adi": {1: 17, 2: 16, 3: 24, 4: 24},
    "lod-ie": {1: 17, 2: 17, 3: 17},
    "lod-cn": {1: 17, 2: 17, 3: 17},
    "ts": {1: 17, 2: 17, 3: 17, 4: 17, 5: 17},
}
SLOT_NAMES = {
    # ADI: the jumps (with the MIB rows of the first right-hand side) run on
    # a side stream beside the pointwise pass; that slot's time overlaps the next
    "adi": ["jumps_side_stream", "adi_rhs", "adi_x_sweep", "adi_y_sweep", "adi_z_sweep"],
    "lod-ie": ["jumps", "lod_x_sweep", "lod_y_sweep", "lod_z_sweep"],
    "lod-cn": ["jumps", "lod_x_sweep", "lod_y_sweep", "lod_z_sweep"],
    "ts": ["jumps", "ts_explicit_x", "ts_explicit_y", "ts_z_sweep", "ts_y_sweep", "ts_x_sweep"],
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=257, help="nodes per axis")
    ap.add_argument("--method", default="adi", choices=["adi", "lod-ie", "lod-cn", "ts"])
    ap.add_argument("--surface", default="torus", choices=["torus", "ellipsoid"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--ref-procs", type=int, default=0, help="reference processes (0: auto)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default sweep shapes")
    ap.add_argument("--precision", default="auto", choices=["auto", "fast", "plain"],
                    help="arithmetic of the headline step: fast (FP64, reordered; Douglas-ADI) or plain "
                         "(bit-identical to the reference); auto = fast where the form applies")
    ap.add_argument("--no-exact", action="store_true", help="skip the bit-exact plain form run beside the fast one")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision run (ADI only)")
    ap.add_argument("--shapes", default="", help="sweep shapes of the three sweeps, e.g. 4,4,4 (no autotune)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-form run")
    ap.add_argument("--no-served", action="store_true", help="skip the served-form run")
    ap.add_argument("--batch-problems", type=int, default=512)
    ap.add_argument("--batch-steps", type=int, default=50)
    ap.add_argument("--served-requests", type=int, default=10000, help="requests per arrival rate")
    ap.add_argument("--served-rates", default="1000,2000", help="Poisson arrival rates, requests/s")
    ap.add_argument("--workload", default="step", choices=["step", "precision", "batched", "served"],
                    help="step: the headline line (default); precision / batched / served: the full sweep of "
                         "that form alone, one JSON line")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# Batched and served forms (wall-clock: the unit is whole solves, setup of the
# device state and host work included; the GPU is synchronized at both ends).

def run_precision(grids=(257, 385), betas=(1e-3, 1.0, 1e3), steps: int = 20) -> dict:
    """The precision form against both FP64 forms: Douglas-ADI + MIB-L2,
    torus, beta_out / beta_in in `betas`, dt = h, `steps` steps of each from
    the same start; cell-steps/s of each (CUDA events), L-infinity of each
    against the exact solution, and the mixed solution's difference from the
    bit-exact one."""
    import numpy as np
    import torch

    import mts_b200 as M

    out = {}
    for n in grids:
        for b in betas:
            spec = M.Spec(n=(n, n, n), surface="torus", surface_params=(0.5, 0.2), beta_in=1.0, beta_out=b,
                          method="adi", mib=2, dt=2.0 / (n - 1), setup="device")
            res = {}
            for prec in ("plain", "fast", "mixed"):
                with M.Solver(spec) as s:
                    s.set_precision(prec)
                    if prec == "plain":
                        s.autotune(1)
                    s.initialize()
                    s.advance(2)
                    s.synchronize()
                    s.time = 0.0
                    s.initialize()
                    st = torch.cuda.ExternalStream(s.stream())
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record(st)
                    s.advance(steps)
                    e1.record(st)
                    s.synchronize()
                    ms = e0.elapsed_time(e1)
                    lmax, l2, _ = s.norms()
                    res[prec] = (ms, lmax, l2, s.solution())
            up, uf, um = res["plain"][3], res["fast"][3], res["mixed"][3]
            nodes = n ** 3
            out[f"{n}^3 beta {b:g}"] = {
                "plain_cell_steps_per_s": nodes * steps / (res["plain"][0] / 1e3),
                "fast_cell_steps_per_s": nodes * steps / (res["fast"][0] / 1e3),
                "mixed_cell_steps_per_s": nodes * steps / (res["mixed"][0] / 1e3),
                "speedup": res["plain"][0] / res["mixed"][0],
                "speedup_vs_fast": res["fast"][0] / res["mixed"][0],
                "fast_speedup": res["plain"][0] / res["fast"][0],
                "fast_rel_maxdiff": float(np.abs(uf - up).max() / np.abs(up).max()),
                "linf_exact_plain": res["plain"][1], "linf_exact_mixed": res["mixed"][1],
                "linf_ratio": res["mixed"][1] / res["plain"][1],
                "linf_vs_plain_fp64": float(np.abs(um - up).max()),
                "rel_maxdiff_vs_plain": float(np.abs(um - up).max() / np.abs(up).max()),
            }
            del up, uf, um, res
    return {"workload": "precision form: 257^3 and 385^3 Douglas-ADI MIB-L2 torus, beta 1e-3/1/1e3, dt = h, "
                        f"{steps} steps", "steps": steps, "cases": out}


def run_batched(count: int, steps: int, seed: int = 0) -> dict:
    """`count` independent problems of the batched family, `steps` steps each:
    one problem after another (plain FP64, mts_advance per problem) against
    all of them in one batch (mts_batch_advance).  Results must agree bit for
    bit; the solves/s ratio is the batching speed-up."""
    import torch

    import mts_b200 as M
    from mts_b200.workloads import batched_problems

    specs = batched_problems(count, seed)
    # the host setup alone (tags, crossings, MIB weights on host threads), for
    # comparison with the device setup the run uses
    t_host = time.perf_counter()
    for sp in specs:
        M.setup_host(sp)
    t_host = time.perf_counter() - t_host
    specs = [dataclasses.replace(sp, setup="device") for sp in specs]
    t_setup = time.perf_counter()
    solvers = [M.Solver(sp) for sp in specs]
    t_setup = time.perf_counter() - t_setup
    nodes = sum(sp.n[0] * sp.n[1] * sp.n[2] for sp in specs)
    for s in solvers:
        s.initialize()
    torch.cuda.synchronize()
    # sequential: one problem at a time, each to completion
    t0 = time.perf_counter()
    for s in solvers:
        s.advance(steps)
        s.synchronize()
    seq = time.perf_counter() - t0
    ref = [s.norms() for s in solvers]
    for s in solvers:
        s.time = 0.0
        s.initialize()
    torch.cuda.synchronize()
    # batched: every problem in one graph per step pair
    M.batch_advance(solvers, 1)  # warm: module loading, first graph
    for s in solvers:
        s.time = 0.0
        s.initialize()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("batched_steps")  # lets a profiler select the batched launches
    t0 = time.perf_counter()
    M.batch_advance(solvers, steps)
    bat = time.perf_counter() - t0
    torch.cuda.nvtx.range_pop()
    same = all(s.norms() == r for s, r in zip(solvers, ref))
    # the same mix with its Douglas-ADI problems in the mixed form (FP32
    # segmented line solves inside the multi-problem launches; the other
    # methods have no mixed form and stay plain): alone, then batched
    adi = [i for i, sp in enumerate(specs) if sp.method == "adi"]
    for i in adi:
        solvers[i].set_precision("mixed")
    for s in solvers:
        s.time = 0.0
        s.initialize()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for s in solvers:
        s.advance(steps)
        s.synchronize()
    seq_m = time.perf_counter() - t0
    ref_m = [s.norms() for s in solvers]
    for s in solvers:
        s.time = 0.0
        s.initialize()
    M.batch_advance(solvers, 1)
    for s in solvers:
        s.time = 0.0
        s.initialize()
    torch.cuda.synchronize()
    torch.cuda.nvtx.range_push("batched_steps_mixed")
    t0 = time.perf_counter()
    M.batch_advance(solvers, steps)
    bat_m = time.perf_counter() - t0
    torch.cuda.nvtx.range_pop()
    same_m = all(s.norms() == r for s, r in zip(solvers, ref_m))
    ratios = [ref_m[i][0] / ref[i][0] for i in adi if ref[i][0] > 0]
    mixed = {
        "adi_problems_mixed": len(adi), "batched_solves_per_s": count / bat_m, "speedup": seq / bat_m,
        "batched_cell_steps_per_s": nodes * steps / bat_m, "sequential_same_forms_s": seq_m, "batched_s": bat_m,
        "results_identical_alone_vs_batched": same_m, "linf_ratio_max": max(ratios) if ratios else None,
        "linf_ratio_min": min(ratios) if ratios else None,
        "speedup_basis": "sequential plain FP64 solves of the same 512 problems",
    }
    for s in solvers:
        s.close()
    return {
        "mixed_adi": mixed,
        "problems": count, "steps": steps, "seed": seed, "nodes_total": nodes,
        "sequential_solves_per_s": count / seq, "batched_solves_per_s": count / bat,
        "speedup": seq / bat, "batched_cell_steps_per_s": nodes * steps / bat,
        "sequential_s": seq, "batched_s": bat, "create_s": t_setup, "host_setup_only_s": t_host,
        "setup": "device (mts_create with setup = device: tags, crossing scan, rtsafe and MIB weight LU on the GPU; "
                 "create_s also holds the upload of every problem)",
        "results_identical": same,
        "timing": "wall clock between synchronizations (launch and graph overheads included)",
        "family": "grids U{17,25,33,49,65}^3, shifted ellipsoids, beta_out log-uniform [1e-3,1e3], "
                  "methods U{ADI,LOD-IE,LOD-CN,TS} x MIB-L1/L2, dt = min h, plain FP64, numpy PCG64 seed 0",
    }


def run_served(count: int, rates: list[float], seed: int = 0, budget: float = 120e9) -> dict:
    """Poisson streams of `count` requests per rate through the continuous-
    batching server, against the sequential plain solver on the same stream.
    Both use the device setup.  The sequential service time is measured on a
    stratified sample of the stream (by grid class: the batched family's
    grids, 129^3, 257^3), weighted by each class's share of the stream; its
    latencies come from one FIFO solver fed the stream's arrivals with
    service times drawn from the measured ones of each request's class."""
    import numpy as np

    from mts_b200 import serve, setup_device
    from mts_b200.workloads import served_requests, size_class

    def on_device(reqs):
        for q in reqs:
            q.spec = dataclasses.replace(q.spec, setup="device")
        return reqs

    out = {"requests_per_rate": count, "hbm_budget_bytes": budget, "setup": "device",
           "server_forms": "Douglas-ADI requests in the mixed form (FP32 segmented solves, batched), the others "
                           "plain FP64; the sequential arm solves every request in plain FP64",
           "rates": {}}
    t_gen = time.perf_counter()
    stream = on_device(served_requests(count, 1000.0, seed, validate=setup_device))
    out["stream_generation_s"] = time.perf_counter() - t_gen
    classes = {}
    for q in stream:
        classes.setdefault(size_class(q.spec), []).append(q)
    share = {c: len(v) / len(stream) for c, v in classes.items()}
    per_class = {"small": 48, "129": 16, "257": 6}
    rs = np.random.default_rng(seed + 1)
    svc = {}
    serve.solve_alone(stream[0])  # module loading and first-launch costs, not timed
    plain_lmax = {}  # request id -> L-infinity error of its plain solve (the sample's Douglas-ADI requests)
    for c, v in classes.items():
        pick = rs.choice(len(v), min(per_class.get(c, 8), len(v)), replace=False)
        times = []
        for i in pick:
            t0 = time.perf_counter()
            r = serve.solve_alone(v[int(i)])
            times.append(time.perf_counter() - t0)
            if v[int(i)].spec.method == "adi":
                plain_lmax[r.id] = r.lmax
        svc[c] = np.array(times)
    mean_svc = sum(share[c] * svc[c].mean() for c in svc)
    out["sequential_solves_per_s"] = float(1.0 / mean_svc)
    out["sequential_sample"] = {c: {"share": share[c], "sampled": int(len(svc[c])), "mean_s": float(svc[c].mean())}
                                for c in svc}
    rng = np.random.default_rng(seed + 2)
    for rate in rates:
        reqs = on_device(served_requests(count, rate, seed, validate=setup_device))
        srv = serve.Server(hbm_budget=budget, setup="device", precision="mixed")
        t0 = time.perf_counter()
        res = srv.run(reqs)
        span = time.perf_counter() - t0
        ratios = [r.lmax / plain_lmax[r.id] for r in res if r.id in plain_lmax and plain_lmax[r.id] > 0]
        lat = np.array([r.latency for r in res])
        arr = np.array([q.arrival for q in reqs])
        seq_svc = np.array([rng.choice(svc[size_class(q.spec)]) for q in reqs])
        seq_lat = serve.fifo_latencies(arr, seq_svc)
        out["rates"][str(rate)] = {
            "solves_per_s": len(res) / span, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "sequential_p50_s": float(np.percentile(seq_lat, 50)),
            "sequential_p99_s": float(np.percentile(seq_lat, 99)), "peak_active": srv.peak_active,
            "peak_budget_bytes": srv.peak_bytes, "batches": srv.batches,
            "loop_batch_s": srv.batch_s, "loop_retire_s": srv.retire_s,
            "solves_per_s_vs_sequential": len(res) / span / out["sequential_solves_per_s"],
            "adi_linf_ratio_vs_plain_max": max(ratios) if ratios else None, "adi_linf_ratio_samples": len(ratios),
        }
    out["timing"] = ("wall clock from the first arrival to the last completion; latency = completion - arrival; "
                     "sequential: service times measured per grid class on a stratified sample, latencies from a "
                     "FIFO queue over the same arrivals")
    return out


def workload(a):
    w = dict(WORKLOAD)
    w["n"] = (a.n, a.n, a.n)
    w["dt"] = 2.0 / (a.n - 1)
    w["method"] = a.method
    if a.surface == "ellipsoid":
        w["surface"] = "ellipsoid"
        w["surface_params"] = (0.7001, 0.4999, 0.4001, 1.0, 0.0, 0.0, 0.0)
    return w


def config_of(w, world, form="plain"):
    return {
        "workload": f"{w['n'][0]}^3 {w['method']} MIB-L{w['mib']} {w['surface']}{tuple(w['surface_params'])} "
                    f"beta {w['beta_in']}:{w['beta_out']} eq{w['eq']} dt=h plain FP64 ({form} form)",
        "grid": list(w["n"]),
        "method": w["method"],
        "mib": w["mib"],
        "surface": w["surface"],
        "surface_params": list(w["surface_params"]),
        "beta": [w["beta_in"], w["beta_out"]],
        "dt": w["dt"],
        "replicas": world,
        "parallelism": f"replicas x{world}",
        "l2_flush": "not needed: inputs larger than L2 (136 MB per field, ~1 GB streamed per step)",
    }


# ---------------------------------------------------------------------------
# clocks sampled during the timed region

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        rows = []
        with open(self.path) as f:
            for ln in f:
                parts = [p.strip() for p in ln.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the reference's own code on the host cores

def reference_binary():
    for name in ("mts_ref_noaux", "mts_ref"):
        p = os.path.join(ROOT, "oracle", "_ref", name)
        if os.path.exists(p):
            return p
    return None


def mem_available_gb() -> float:
    try:
        with open("/proc/meminfo") as f:
            for ln in f:
                if ln.startswith("MemAvailable:"):
                    return int(ln.split()[1]) / 1e6
    except OSError:
        pass
    return 16.0


def run_reference_sample(w, procs: int, steps_per_proc: int, timeout: float = 900):
    """Runs `procs` independent copies of the reference binary on the
    workload, each for `steps_per_proc` time steps, concurrently on the host
    cores.  Returns (cell-steps/s, cores, sample text, kind) from the binaries'
    own step timers (setup excluded)."""
    binary = reference_binary()
    n = w["n"]
    sp = list(w["surface_params"])
    if binary is None:
        return None
    args = [binary, "--n", *map(str, n), "--surface", w["surface"], *map(repr, sp), "--beta", repr(w["beta_in"]),
            repr(w["beta_out"]), "--eq", str(w["eq"]), "--method", w["method"], "--mib", str(w["mib"]), "--dt",
            repr(w["dt"]), "--steps", str(steps_per_proc)]
    ps = [subprocess.Popen(args, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for _ in range(procs)]
    secs = []
    for p in ps:
        out, _ = p.communicate(timeout=timeout)
        line = [ln for ln in out.splitlines() if ln.startswith("{")]
        if not line:
            raise RuntimeError("reference run produced no result line")
        secs.append(json.loads(line[-1])["step_seconds"])
    nodes = n[0] * n[1] * n[2]
    value = procs * nodes * steps_per_proc / max(secs)
    sample = (f"{procs} concurrent single-threaded reference processes ({os.path.basename(binary)}), each "
              f"{steps_per_proc} step(s) of the {n[0]}^3 workload; per-process timed seconds "
              f"{min(secs):.2f}-{max(secs):.2f} s (setup excluded)")
    return value, procs, sample, "reference"


def auto_procs(w) -> int:
    nodes = w["n"][0] * w["n"][1] * w["n"][2]
    per_proc_gb = 1.5 * nodes / 257 ** 3 + 0.05
    cores = os.cpu_count() or 1
    return max(1, min(cores, 16, int(mem_available_gb() * 0.6 / per_proc_gb)))


# ---------------------------------------------------------------------------

def max_over_ranks(values, dist=None):
    """Element-wise max of per-rank timings over all ranks (every rank takes
    part; a device tensor under NCCL, a host tensor under gloo)."""
    import torch

    if dist is None:
        return [float(v) for v in values]
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor(list(values), dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def job_value(world: int, nodes: int, steps: int, ms_max: float) -> float:
    """Whole-job throughput: every rank advances its own replica of `nodes`
    cells by `steps` steps; the job takes the slowest rank's time."""
    return world * nodes * steps / (ms_max / 1e3)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def main():
    a = parse()
    world, rank, local = dist_setup()
    w = workload(a)
    nodes = w["n"][0] * w["n"][1] * w["n"][2]

    if a.workload != "step":
        # one form's full workload on one GPU, one JSON line (rank 0 only)
        if rank != 0:
            return 0
        import torch

        torch.cuda.set_device(local)
        if a.workload == "precision":
            res = run_precision()
        elif a.workload == "batched":
            res = run_batched(a.batch_problems, a.batch_steps)
        else:
            res = run_served(a.served_requests, [float(v) for v in a.served_rates.split(",") if v])
        print(json.dumps({"workload": a.workload, **res}))
        return 0

    if a.impl == "reference":
        if rank != 0:
            return 0
        # The reference is single-threaded: the host's cores run independent
        # copies of it (replicas, like the GPU ranks), the K timed steps spread
        # over them, at most REF_MAX_STEPS each so that the run stays within a
        # few minutes (one 257^3 step takes ~7-10 s on one core).  No warm-up
        # steps: compiled CPU code has nothing to warm that its setup (excluded
        # from the timing) has not already touched.
        procs = a.ref_procs or auto_procs(w)
        per_proc = max(1, min(REF_MAX_STEPS, -(-a.steps // procs)))
        res = run_reference_sample(w, procs, per_proc)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference build oracle/_ref missing"}))
            return 0
        value, cores, sample, kind = res
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": a.gpus,
            "steps": procs * per_proc, "warmup": 0, "ms_per_step": 1e3 * nodes / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (analytic exact solution)", "config": config_of(w, 1),
            "cpu_baseline": {"value": value, "unit": "cell-steps/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    import mts_b200 as M

    spec = M.Spec(**w)
    prec = a.precision
    if prec == "auto":
        prec = "fast" if w["method"] == "adi" else "plain"
    solver = M.Solver(spec)
    solver.set_precision(prec)
    solver.initialize()

    def plain_shapes(sv):
        if a.shapes:
            sh = tuple(int(v) for v in a.shapes.split(","))
            for k, v in enumerate(sh):
                sv.set_sweep_shape(k, v)
            return sh
        if a.no_autotune:
            return ("default",)
        return sv.autotune(2)

    shapes = plain_shapes(solver) if prec == "plain" else ("none: the fast form has no sweep shapes",)
    solver.advance(a.warmup)
    solver.synchronize()

    stream = torch.cuda.ExternalStream(solver.stream())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(torch.cuda.current_device())
    launches0 = solver.launch_count()
    solver.set_profiling(True)
    solver.profile_read()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks.start()
    torch.cuda.nvtx.range_push("timed_steps")  # lets a profiler select the timed launches
    ev0.record(stream)
    solver.advance(a.steps)
    ev1.record(stream)
    torch.cuda.nvtx.range_pop()
    solver.synchronize()
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    kms, kn = solver.profile_read()
    solver.set_profiling(False)
    launches = solver.launch_count() - launches0
    lmax, l2, _ = solver.norms()
    t_head = solver.time
    u_head = solver.solution() if w["method"] == "adi" and (not a.no_mixed or (prec == "fast" and not a.no_exact)) \
        else None

    # end to end through the C ABI with host buffers: the field goes up and
    # comes back every step (the reference's Solve_2nd contract on a host
    # CubicDoub), pinned host memory.
    e2e_steps = max(1, a.e2e_steps)
    hu = torch.empty(nodes, dtype=torch.float64, pin_memory=True)
    hu.copy_(torch.from_numpy(solver.solution()))
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    solver.advance_host_ptr(hu.data_ptr(), hu.data_ptr(), 1)
    if dist:
        dist.barrier()
    e0.record(stream)
    for _ in range(e2e_steps):
        solver.advance_host_ptr(hu.data_ptr(), hu.data_ptr(), 1)
    e1.record(stream)
    solver.synchronize()
    e2e_ms = e0.elapsed_time(e1)

    ms_max, e2e_max = max_over_ranks([ms, e2e_ms], dist)
    value = job_value(world, nodes, a.steps, ms_max)
    e2e_value = job_value(world, nodes, e2e_steps, e2e_max)

    def timed_run(precision):
        """Another handle on the same workload: warm-up, then the same K
        steps from the same start, so that its solution is compared with the
        headline's at the same time.  Returns (ms, kernel ms, launches,
        norms, solution, shapes)."""
        sv = M.Solver(spec)
        sv.set_precision(precision)
        sv.initialize()
        sh = plain_shapes(sv) if precision == "plain" else None
        sv.advance(a.warmup)
        sv.synchronize()
        st_ = torch.cuda.ExternalStream(sv.stream())
        m0 = torch.cuda.Event(enable_timing=True)
        m1 = torch.cuda.Event(enable_timing=True)
        sv.set_profiling(True)
        sv.profile_read()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push(f"timed_steps_{precision}")
        m0.record(st_)
        sv.advance(a.steps)
        m1.record(st_)
        torch.cuda.nvtx.range_pop()
        sv.synchronize()
        ms_ = m0.elapsed_time(m1)
        km, kc = sv.profile_read()
        sv.set_profiling(False)
        nr = sv.norms()
        u_ = sv.solution()
        assert sv.time == t_head
        sv.close()
        (ms_,) = max_over_ranks([ms_], dist)
        return ms_, km, kc, nr, u_, sh

    def rel(u_, ref):
        return float(abs(u_ - ref).max() / max(1e-300, abs(ref).max()))

    # The bit-exact plain form on the same workload (the drop-in arithmetic,
    # bit-identical to the reference), beside the fast form.
    exact = None
    if prec == "fast" and not a.no_exact and u_head is not None:
        ms_e, km_e, kc_e, (le, l2e, _), ue, sh_e = timed_run("plain")
        v_e = job_value(world, nodes, a.steps, ms_e)
        exact = {
            "value": v_e, "unit": "cell-steps/s", "ms_per_step": ms_e / a.steps, "sweep_shapes": list(sh_e),
            "fast_speedup": value / v_e, "lmax": le, "l2": l2e,
            "fast_rel_maxdiff": rel(u_head, ue), "fast_lmax_rel_diff": abs(lmax - le) / le,
            "kernels": {nm: {"ms_per_launch": km_e[k] / kc_e[k], "launches": int(kc_e[k])}
                        for k, nm in enumerate(SLOT_NAMES["adi"]) if kc_e[k] > 0},
            "form": "MTS_PRECISION_PLAIN: the reference's operations in the reference's order (bit-identical); "
                    "fast_rel_maxdiff = max|u_fast - u_exact| / max|u_exact| after the same warm-up + timed steps",
        }
        del ue

    # The mixed-precision form (FP32 line solves on the increment, FP64
    # residual and state) on the same workload, same steps from the same
    # start, so its error is compared at the same time.
    mixed = None
    if u_head is not None and not a.no_mixed:
        ms_m, kms_m, kn_m, (lm, l2m, _), um, _ = timed_run("mixed")
        v_m = job_value(world, nodes, a.steps, ms_m)
        # the jumps and the residual's MIB rows run on a side stream beside
        # the pointwise residual: the first slot is that stream's jumps
        # launch (its time overlaps the second), the second the residual
        # up to the join
        names_m = ["jumps_side_stream", "residual_fp64", "x_solve_fp32", "y_solve_fp32", "z_solve_fp32_and_accumulate"]
        mixed = {
            "value": v_m, "unit": "cell-steps/s", "ms_per_step": ms_m / a.steps,
            "speedup_vs_plain": v_m / value,
            "speedup_vs_exact_plain": (v_m / exact["value"]) if exact else None,
            "lmax": lm, "l2": l2m, "lmax_plain": lmax, "l2_plain": l2, "lmax_ratio": lm / lmax,
            "rel_maxdiff_vs_plain": rel(um, u_head), "t": t_head,
            "bytes_per_node_step": MIXED_BYTES,
            "step_roofline_frac": MIXED_BYTES * nodes * a.steps / (ms_m / 1e3) / 1e9 / peak_hbm(),
            "kernels": {n: {"ms_per_launch": kms_m[k] / kn_m[k], "launches": int(kn_m[k])}
                        for k, n in enumerate(names_m) if kn_m[k] > 0},
            "form": "residual dt(A_x+A_y+A_z)u^n + dt src in FP64, three segmented FP32 line solves of the "
                    "increment (warp per line, lane segments joined by shuffle scans), FP64 state += increment "
                    "in the z solve; speedup_vs_plain is against the headline (fast FP64) form",
        }
        del um

    method = w["method"]
    if prec == "fast":
        names, alg = FAST_NAMES, FAST_BYTES
    else:
        names, alg = SLOT_NAMES[method], ALG_BYTES[method]
    kernels = {}
    for k, name in enumerate(names):
        if kn[k] > 0:
            kernels[name] = {"ms_per_launch": kms[k] / kn[k], "launches": int(kn[k]),
                             "share": kms[k] / max(1e-12, kms[: len(names)].sum())}
    dom = max((k for k in alg), key=lambda k: kms[k])
    peak, peak_src = peak_hbm(), ("measured" if os.path.exists(PEAKS_PATH) else "fallback")
    per_launch_ms = kms[dom] / kn[dom]
    achieved = alg[dom] * nodes / (per_launch_ms / 1e3) / 1e9
    step_bytes = sum(alg.values())
    roofline = {
        "bound": "hbm", "kernel": names[dom], "achieved": achieved, "peak": peak, "unit": "GB/s",
        "frac": achieved / peak, "peak_source": f"hbm_gbs of MEASURED_PEAKS.json ({peak_src})",
        "traffic": None,
        "algorithmic_bytes_per_node": alg[dom],
        # the contract's step model: 67 B per node-step for ADI (51 LOD, 102 TS)
        "step_contract": {"bytes_per_node_step": CONTRACT_BYTES[method],
                          "frac": CONTRACT_BYTES[method] * nodes * a.steps / (ms / 1e3) / 1e9 / peak},
        "step": {"bytes_per_node_step": step_bytes,
                 "achieved": step_bytes * nodes * a.steps / (ms / 1e3) / 1e9,
                 "frac": step_bytes * nodes * a.steps / (ms / 1e3) / 1e9 / peak},
    }
    traffic_path = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(traffic_path):
        with open(traffic_path) as f:
            tr = json.load(f).get(f"{method}:{names[dom]}")
        if tr:
            roofline["traffic"] = tr["bytes_per_node"] * nodes
            roofline["traffic_source"] = tr["source"]

    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (analytic exact solution, seeded geometry)",
        "precision_form": prec,
        "config": config_of(w, world, prec), "gpu_launches": int(launches), "kernels": kernels,
        "roofline": roofline, "sweep_shapes": list(shapes),
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": 8 * nodes,
                "d2h_bytes_per_step": 8 * nodes, "steps": e2e_steps,
                "api": "mts_advance_host (field uploaded and downloaded every step, pinned host memory)"},
        "clocks": clk, "accuracy": {"lmax": lmax, "l2": l2, "t": t_head},
    }
    if exact is not None:
        line["exact_plain"] = exact
    if mixed is not None:
        line["mixed"] = mixed
    if rank == 0 and world == 1 and not a.no_mixed and w["method"] == "adi":
        # the precision form's second grid of its config, 385^3, one beta ratio
        line["precision_385"] = run_precision(grids=(385,), betas=(1e3,), steps=10)
    if rank == 0 and world == 1 and not a.no_batched:
        line["batched"] = run_batched(a.batch_problems, a.batch_steps)
    if rank == 0 and world == 1 and not a.no_served:
        line["served"] = run_served(a.served_requests, [float(v) for v in a.served_rates.split(",") if v])
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            res = run_reference_sample(w, a.ref_procs or auto_procs(w), 1)
        except Exception as e:  # the baseline is reported, never required
            res = None
            line["cpu_baseline_error"] = str(e)[:200]
        if res is not None:
            v, cores, sample, kind = res
            line["cpu_baseline"] = {"value": v, "unit": "cell-steps/s", "cores": cores, "kind": kind,
                                    "sample": sample}
    solver.close()
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
