#!/usr/bin/env python
"""bench.py -- node*layer*steps/s of SHYFEM's semi-implicit step on B200.

Default workload at N=1 (the batched ensemble): 64 independent basins with
node counts log-uniform in 5k..100k (2.1M nodes, 4.2M triangles in total),
each made like the 2D tidal channel (100 m jittered triangle mesh at a
seeded aspect ratio, depth 10 m +- 2 m, M2 0.5 m level boundary, quadratic
friction) with 10 z-layers, and a uniform wind of 10 m/s plus a seeded
per-basin perturbation of sigma 3 m/s, dt = 60 s; seeded synthetic input of
that shape (no dataset ships with the reference).  All basins advance in
one CUDA-graph step.  One bench "step" is one model time step (hydro, the
body of shyfem_run's loop) of every basin.  Beside it the line reports the
plain single-run form: the same basins advanced one model at a time (each
with the default launch plan), and the accuracy of the timed run: the
first `--check-steps` steps of its smallest, median and largest basins
against the FP64 oracle.  The timed model's launch shapes are chosen first
by the library's autotuner (shygpu_autotune) on the same basins.

`--workload basin3d` times the 3D baroclinic basin instead (~20k nodes, 20
z-layers, temperature and salinity transported, dt = 120 s); `--workload
lagoon` the 250k-node lagoon on 30 sigma layers with three tracers (dt =
30 s); `--workload serve` a Poisson stream of forecast requests through the
serving loop (latency p50/p99).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl shygpu|reference]
                  [--workload ensemble|basin3d|lagoon|serve]

N > 1 runs one process per GPU, each advancing its own replica (replicas
only: the step has no exchange between basins), value = all ranks' units /
max-over-ranks time.  `--impl reference` times the CPU restatement of the
reference's algorithm (the oracle) on all host cores.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "shyfemcm-ismar_b200"))

METRIC = "node*layer*steps/s"
PEAKS_FILE = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM = 6650.0


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=400)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="shygpu", choices=["shygpu", "reference"])
    p.add_argument("--workload", default="ensemble", choices=["ensemble", "basin3d", "lagoon", "serve"])
    p.add_argument("--serve-requests", type=int, default=30,
                   help="serve workload: requests of the Poisson stream (20/min)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain", action="store_true")
    p.add_argument("--check-steps", type=int, default=None,
                   help="steps of the accuracy check against the oracle (0: none; default 60, on the lagoon 8, "
                        "where an oracle step of its 250k nodes and 30 layers takes about 12 s)")
    p.add_argument("--no-tune", action="store_true", help="keep the default launch plan (no shygpu_autotune)")
    a = p.parse_args()
    if a.check_steps is None:
        a.check_steps = 8 if a.workload == "lagoon" else 60
    return a


def make_cases(workload, rank=0, first=None):
    from shygpu import cases
    if workload == "basin3d":
        return [cases.basin3d_case(nkn_target=20000, seed=2 + 1000 * rank)]
    if workload == "lagoon":
        return [cases.lagoon_case(nkn_target=250000, nlv=30, seed=7 + 1000 * rank)]
    if workload == "serve":
        return [c for _, c, _ in cases.serve_requests(first or 30, seed=5 + 1000 * rank)]
    return cases.ensemble_cases(64, seed=4 + 1000 * rank, first=first)


def case_specs(workload, rank=0):
    """The cases of make_cases as specs the oracle's worker processes build
    themselves (name of the constructor in shygpu.cases, its arguments)."""
    if workload == "basin3d":
        return [("basin3d_case", dict(nkn_target=20000, seed=2 + 1000 * rank))]
    if workload == "lagoon":
        return [("lagoon_case", dict(nkn_target=250000, nlv=30, seed=7 + 1000 * rank))]
    if workload == "ensemble":
        return [("ensemble_cases", dict(n=64, seed=4 + 1000 * rank, only=[i])) for i in range(64)]
    raise ValueError(workload)


def check_members(workload, case_list):
    """Indices of the basins the accuracy check compares: the smallest, the
    median and the largest of the ensemble; the one basin otherwise."""
    if len(case_list) == 1:
        return [0]
    order = np.argsort([c["nkn"] for c in case_list], kind="stable")
    return sorted({int(order[0]), int(order[len(order) // 2]), int(order[-1])})


def units_per_step(case_list):
    return sum(c["nkn"] * c["nlv"] for c in case_list)


def active_units_per_step(case_list):
    """Node-layers that hold water: the layers above each node's bottom."""
    return sum(int(c["ilhkv"].sum()) for c in case_list)


def reduce_over_ranks(x, world, op="max", device="cuda"):
    """x reduced over the ranks of the job (max for times, sum for work);
    the value itself on one rank."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def replica_throughput(units, steps, seconds, world, device="cuda"):
    """Whole-job units per second of replicas: every rank's own units (its
    replica's ensemble) summed, over the slowest rank's time."""
    total = reduce_over_ranks(units * steps, world, "sum", device)
    return total / reduce_over_ranks(seconds, world, "max", device)


L2_NOTE = "inputs larger than L2; the GPU arm also writes 256 MiB between timed steps"


def workload_config(workload, case_list, world=1):
    """The workload as both arms report it (the same dict for the same
    cases)."""
    act = {"active_node_layers": active_units_per_step(case_list),
           "active_fraction": active_units_per_step(case_list) / units_per_step(case_list),
           "l2": L2_NOTE, "parallelism": f"replicas{world}"}
    if workload == "lagoon":
        c = case_list[0]
        return dict({"workload": "lagoon_sigma_tracers", "nkn": c["nkn"], "nel": c["nel"],
                     "nlv": c["nlv"], "layers": "sigma", "dt_s": c["params"]["dt"], "tracers": 3,
                     "forcing": "M2 0.5 m + S2 0.3 m"}, **act)
    if workload == "basin3d":
        c = case_list[0]
        return dict({"workload": "basin3d_baroclinic_ts", "nkn": c["nkn"], "nel": c["nel"],
                     "nlv": c["nlv"], "dt_s": c["params"]["dt"], "tracers": "T,S",
                     "forcing": "10 m/s wind, M2 0.3 m"}, **act)
    return dict({"workload": "ensemble_64_basins_5k_100k_nodes", "basins": len(case_list),
                 "nkn_total": sum(c["nkn"] for c in case_list),
                 "nel_total": sum(c["nel"] for c in case_list), "nlv": case_list[0]["nlv"],
                 "depth_m": "10 +- 2", "layers": "z: 2 m surface layer, 1 m below",
                 "dt_s": case_list[0]["params"]["dt"], "forcing": "10 +- 3 m/s wind, M2 0.5 m",
                 "seed": 4}, **act)


def plain_gpu(case_list, steps, lib):
    """The plain single-run GPU form: each basin in a model of its own,
    advanced alone (CUDA-graph step), one basin after the other; device
    time summed over the basins."""
    import torch
    import shygpu
    total_ms = 0.0
    units = 0
    for c in case_list:
        m = shygpu.Model([c])
        m.set_state_all()
        m.run(3)
        st = torch.cuda.ExternalStream(m.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(st):
            e0.record(st)
            lib.shygpu_enqueue(m.h, steps)
            e1.record(st)
        torch.cuda.synchronize()
        shygpu.check(lib.shygpu_sync(m.h), "plain step")
        total_ms += e0.elapsed_time(e1)
        units += c["nkn"] * c["nlv"] * steps
        m.close()
    return units / (total_ms / 1000.0), total_ms / steps


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.rows = []
        self.stop_flag = False
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append((time.time(), line.strip()))

    def summary(self, t0, t1):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        sel = [r for t, r in self.rows if t0 - 0.15 <= t <= t1 + 0.15] or [r for _, r in self.rows]
        for r in sel:
            parts = [x.strip() for x in r.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of each kernel (FP32 state, compulsory traffic)
# ---------------------------------------------------------------------------
def algorithmic_bytes(case_list, infos, nsc, cor=False):
    nkn = sum(c["nkn"] for c in case_list)
    nel = sum(c["nel"] for c in case_list)
    NL = sum(int(c["ilhv"].sum()) for c in case_list)          # active element-layers
    NK = sum(int(c["ilhkv"].sum()) for c in case_list)         # active node-layers
    NI = sum(c["nkn"] * (c["nlv"] + 1) for c in case_list)     # node interfaces
    nnz = 7 * nkn
    # Krylov traffic per basin: its own iterations over its own rows
    kry = sum(i.krylov_iters * (8 * 7 * c["nkn"] + 48 * c["nkn"])
              + max(i.refinements, 1) * (12 * 7 * c["nkn"] + 20 * c["nkn"])
              for c, i in zip(case_list, infos))
    b = {}
    # the zeta solve counted as the survey of the path counts its compulsory
    # traffic: assembly and right-hand side about 100 B per node, then per
    # Krylov iteration about 80 B per node for CG (two vector streams of
    # eight bytes, the matrix row, ~7 entries) or 150 B for BiCGStab
    b_it = 150 if cor else 80
    b["zeta_survey"] = sum(c["nkn"] * (100 + b_it * i.krylov_iters) for c, i in zip(case_list, infos))
    b["column"] = NL * (24 + (4 if cor else 0)) + nel * (12 + 32 + 16 + 8 + 48) + NK * 4 + NI * 4 + nkn * 12
    b["zeta"] = nel * (48 + 36 + 12) + nnz * (4 + 12 + 4) + nkn * (4 + 4 + 4 + 4 + 20) + kry
    b["final"] = NL * (24 + (4 if cor else 0)) + nel * (12 + 32 + 16 + 16 + 4 + 8 + 12) + nkn * 4
    b["node"] = NL * 16 + nel * (12 + 32 + 16 + 4) + NK * 12 + nkn * 20 + NI * 4
    b["stab"] = NL * 24 + nel * (36 + 32 + 16 + 4 + 12) + NK * 8 + NI * 8
    b["reduce"] = nkn * 8
    b["conz"] = NL * 28 + nel * (32 + 16 + 4 + 12) + NK * (8 * nsc + 8 + 8) + NI * 8
    b["rho"] = NK * (8 + 4 + 4)     # T, S read, layer depth read, rho written
    return b


def load_peak():
    try:
        d = json.loads(PEAKS_FILE.read_text())
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


# ---------------------------------------------------------------------------
# CPU baseline / reference arm: the oracle on host cores
# ---------------------------------------------------------------------------
def oracle_pool():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_pool as op
    return op


def cpu_timing(workload, case_list, nsteps, warm, nproc, rank=0):
    """The oracle advancing the workload's own basins: each process takes a
    share of the basins (largest first to the least loaded), advances them
    `warm` untimed and `nsteps` timed steps; units over the slowest
    process's time."""
    op = oracle_pool()
    specs = case_specs(workload, rank)
    units, secs, used = op.time_steps(specs, [c["nkn"] * c["nlv"] for c in case_list], nsteps, warm, nproc)
    return units / secs, secs, used


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    if a.workload == "serve":
        print(json.dumps({"impl": "reference", "unavailable": "the serving workload has no CPU arm"}), flush=True)
        return
    nproc = os.cpu_count() or 1
    # each bench step: one time step of every basin of the workload
    steps = max(1, a.steps if a.steps <= 40 else 20)
    warm = min(max(a.warmup, 1), 2)
    case_list = make_cases(a.workload, 0)
    value, tmax, used = cpu_timing(a.workload, case_list, steps, warm, nproc)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
            "n_gpus": a.gpus, "steps": steps, "warmup": warm,
            "ms_per_step": 1000.0 * tmax / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(a.workload, case_list, world),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": used, "kind": "port",
                             "host_cpu": host_cpu(),
                             "sample": f"{steps} time steps of every basin of the workload (the GPU arm's "
                                       f"basins), dealt over {used} processes, one per host core; FP64 C++ "
                                       "restatement of the reference step (oracle/shyref.cpp, -O3)"},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def host_cpu():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def accuracy(case_list, picks, gpu_states, gpu_volumes, oracle_results):
    """Largest differences of the checked basins from the oracle: water
    level [m], transports relative to the largest transport component, tracers
    relative to theirs (None without tracers), volume relative."""
    dz = du = dv = 0.0
    dc = None
    for i, sg, vg, o in zip(picks, gpu_states, gpu_volumes, oracle_results):
        c, so = case_list[i], o["state"]
        dz = max(dz, float(np.abs(sg["znv"] - so["znv"]).max()))
        me = np.arange(c["nlv"])[None, :] < c["ilhv"][:, None]
        umax = max(np.abs(so["utlnv"][me]).max(), np.abs(so["vtlnv"][me]).max(), 1e-30)
        for f in ("utlnv", "vtlnv"):
            du = max(du, float(np.abs(sg[f] - so[f])[me].max() / umax))
        mk = np.arange(c["nlv"])[None, :] < c["ilhkv"][:, None]
        p = c["params"]
        fs = (["tempv"] if p["itemp"] else []) + (["saltv"] if p["isalt"] else []) + \
             (["conzv"] if p["nconz"] > 0 else [])
        for f in fs:
            a, b = sg[f], so[f]
            m = mk if a.ndim == 2 else np.broadcast_to(mk, a.shape)
            r = float(np.abs(a - b)[m].max() / max(np.abs(b[m]).max(), 1e-30))
            dc = r if dc is None else max(dc, r)
        dv = max(dv, abs(vg - o["volume"]) / o["volume"])
    return {"zeta_err_m": dz, "transport_rel_err": du, "tracer_rel_err": dc, "volume_rel_err": dv}


# ---------------------------------------------------------------------------
# the serving workload: a Poisson stream of forecast requests
# ---------------------------------------------------------------------------
def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = min(len(xs) - 1, max(0, int(math.ceil(q / 100.0 * len(xs))) - 1))
    return xs[k]


def run_serve(a):
    """Requests arrive at their (seeded) Poisson times in wall-clock time and
    are served by shygpu.Server; latency = finish - submit on the server's
    clock.  Beside it the plain path: one run at a time in arrival order,
    each run's service time measured alone (create + set_state + steps) on
    a 288-step sample scaled to its horizon, queued FIFO on the same
    arrival times."""
    import torch
    import shygpu
    from shygpu import cases
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    os.environ.setdefault("SHYGPU_NO_BUILD", "1")
    reqs = cases.serve_requests(a.serve_requests, seed=5 + 1000 * rank)
    lib = shygpu.lib()
    # warm the library and the CUDA context on a small run
    w = shygpu.Model(cases.channel_case())
    w.set_state(0)
    w.run(3)
    w.close()
    free, _ = torch.cuda.mem_get_info()
    srv = shygpu.Server(int(0.8 * free), max_active=16, quantum_steps=60)
    sampler = ClockSampler(local)
    launches0 = lib.shygpu_launch_count()
    pending = list(reqs)
    ids = []
    t_wall0 = time.time()
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        while pending and pending[0][0] <= now:
            arr, c, n = pending.pop(0)
            ids.append((srv.submit(c, n), c, n, arr))
        act, queued, _ = srv.progress(block=False)
        if not pending and act == 0 and queued == 0:
            break
        if act == 0 and queued == 0:
            time.sleep(min(0.01, max(0.0, pending[0][0] - now)))
        else:
            time.sleep(0.0005)
    t_wall1 = time.time()
    clocks = sampler.summary(t_wall0, t_wall1)
    launches = lib.shygpu_launch_count() - launches0
    lat, units, t_first, t_last, failed = [], 0, None, None, 0
    for rid, c, n, arr in ids:
        st, steps, ts, ta, td = srv.status(rid)
        if st != shygpu.Server.DONE:
            failed += 1
            continue
        lat.append(td - ts)
        units += c["nkn"] * c["nlv"] * n
        t_first = ts if t_first is None else min(t_first, ts)
        t_last = td if t_last is None else max(t_last, td)
        srv.result(rid)
    srv.close()
    span = t_last - t_first
    value = units / span
    # plain path: each run alone, FIFO on the same arrival times
    service = []
    for arr, c, n in reqs:
        t_c = time.perf_counter()
        m = shygpu.Model(c)
        m.set_state(0)
        torch.cuda.synchronize()
        t_create = time.perf_counter() - t_c
        m.run(3)
        st = torch.cuda.ExternalStream(m.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            e0.record(st)
            lib.shygpu_enqueue(m.h, 288)
            e1.record(st)
        torch.cuda.synchronize()
        shygpu.check(lib.shygpu_sync(m.h), "plain run")
        service.append(t_create + e0.elapsed_time(e1) / 1000.0 * n / 288.0)
        m.close()
    finish, plain_lat = 0.0, []
    for (arr, c, n), sv in zip(reqs, service):
        finish = max(arr, finish) + sv
        plain_lat.append(finish - arr)
    plain_value = units / (finish - reqs[0][0])
    h2d = sum(c["nkn"] * 4 + 2 * c["nel"] * c["nlv"] * 4 for _, c, _ in reqs)
    d2h = h2d
    steps_total = sum(n for _, _, n in reqs)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": steps_total, "warmup": 3, "ms_per_step": 1000.0 * span / steps_total,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": "serve_poisson_20_per_min", "requests": len(reqs),
                   "nkn_range": [2000, 200000], "nlv": 10, "horizon_steps": 2880, "dt_s": 60.0,
                   "admission": "HBM footprint, 80% of free memory, 16 slots, 60-step quanta",
                   "l2": "inputs larger than L2", "parallelism": f"replicas{world}"},
        "latency_s": {"p50": pct(lat, 50), "p99": pct(lat, 99), "max": max(lat) if lat else None},
        "failed": failed,
        "plain_gpu": {"value": plain_value, "unit": METRIC,
                      "latency_s": {"p50": pct(plain_lat, 50), "p99": pct(plain_lat, 99)},
                      "form": "one run at a time in arrival order; service time measured alone "
                              "(create + set_state + 288 steps, scaled to the horizon)"},
        "served_over_plain": value / plain_value,
        "gpu_launches": int(launches),
        "clocks": clocks,
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": h2d / steps_total,
                "d2h_bytes_per_step": d2h / steps_total,
                "path": "shygpu_serve_submit + shygpu_serve_progress + shygpu_serve_result (host arrays in and out)"},
        "roofline": None,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# the GPU arm
# ---------------------------------------------------------------------------
def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
        return
    if a.workload == "serve":
        run_serve(a)
        return
    import torch
    import torch.distributed as dist
    import shygpu

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=300))
    torch.cuda.set_device(local)
    os.environ.setdefault("SHYGPU_NO_BUILD", "1")
    os.environ["CUDA_VISIBLE_DEVICES_HINT"] = str(local)

    # The accuracy check of the timed run: the oracle advances the checked
    # basins in spawned processes while the GPU runs (rank 0 only).
    check_pool = None
    if rank == 0 and a.check_steps > 0:
        op = oracle_pool()
        picks_spec = case_specs(a.workload, rank)
        case_list = make_cases(a.workload, rank)
        picks = check_members(a.workload, case_list)
        check_pool = op.run_states([picks_spec[i] for i in picks], a.check_steps, wait=False)
    else:
        case_list = make_cases(a.workload, rank)
    model = shygpu.Model(case_list)
    model.set_state_all()
    stream = torch.cuda.ExternalStream(model.stream())
    # the launch shapes chosen by the library's autotuner on these basins
    # (its trials start from the initial state and leave it unchanged)
    tuning = None
    if not a.no_tune:
        t0 = time.perf_counter()
        choice, tms = model.autotune(steps=4)
        tuning = {"choice": choice, "ms_per_step": tms, "seconds": time.perf_counter() - t0,
                  "by": "shygpu_autotune (trials of the candidate plans on the timed basins)"}
    check_gpu = None
    if check_pool is not None:
        # the first steps of the timed run itself, read back before timing
        model.run(a.check_steps)
        check_gpu = ([model.get_state(i) for i in picks], [model.info(i).volume for i in picks])
    units = units_per_step(case_list)
    L2_FLUSH = 256 << 20
    flush = torch.empty(L2_FLUSH // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            dist.barrier()

    # ---- warm-up ----
    model.run(max(a.warmup, 3))
    # ---- device-timed region: K single steps, L2 flushed between them ----
    sampler = ClockSampler(local)
    time.sleep(1.0)
    ev0 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    ev1 = [torch.cuda.Event(enable_timing=True) for _ in range(a.steps)]
    lib = shygpu.lib()
    launches0 = lib.shygpu_launch_count()
    barrier()
    torch.cuda.synchronize()
    t_wall0 = time.time()
    with torch.cuda.stream(stream):
        for i in range(a.steps):
            flush.fill_(float(i))
            ev0[i].record(stream)
            lib.shygpu_enqueue(model.h, 1)
            ev1[i].record(stream)
    torch.cuda.synchronize()
    t_wall1 = time.time()
    shygpu.check(lib.shygpu_sync(model.h), "step")
    launches = lib.shygpu_launch_count() - launches0
    ms_total = sum(e0.elapsed_time(e1) for e0, e1 in zip(ev0, ev1))
    barrier()
    clocks = sampler.summary(t_wall0, t_wall1)
    value = replica_throughput(units, a.steps, ms_total / 1000.0, world)
    ms_total = 1000.0 * reduce_over_ranks(ms_total / 1000.0, world, "max")
    ms_step = ms_total / a.steps

    check = None
    if check_pool is not None:
        pl, res = check_pool
        try:
            results = res.get()
        finally:
            pl.close()
            pl.join()
        check = dict(accuracy(case_list, picks, check_gpu[0], check_gpu[1], results),
                     steps=a.check_steps, basins=picks, nkn=[case_list[i]["nkn"] for i in picks],
                     against="FP64 oracle (oracle/shyref.cpp), the same basins from the same initial state")

    # ---- end to end through the public API: forcing in from pinned host
    #      memory and the water level of every basin out, every step ----
    # Headline form: the whole-model calls of a pipelined forecast service
    # (shygpu_set_forcing_all, shygpu_enqueue, shygpu_get_levels): every
    # step's wind goes up and its levels come down in one copy each,
    # enqueued without waiting; shygpu_sync at the end checks every step.
    # The levels land in a ring of four pinned buffers.
    c0 = case_list[0]
    nb = len(case_list)
    taux_all = torch.from_numpy(np.concatenate([np.ascontiguousarray(c["tauxnv"]) for c in case_list])).pin_memory()
    tauy_all = torch.from_numpy(np.concatenate([np.ascontiguousarray(c["tauynv"]) for c in case_list])).pin_memory()
    nkn_all = sum(c["nkn"] for c in case_list)
    ring = [torch.empty(nkn_all, dtype=torch.float32).pin_memory() for _ in range(4)]
    h2d = nkn_all * 8
    d2h = nkn_all * 4
    e2e_steps = min(a.steps, 200)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        shygpu.check(lib.shygpu_set_forcing_all(model.h, taux_all.data_ptr(), tauy_all.data_ptr(), None, None),
                     "set_forcing_all")
        shygpu.check(lib.shygpu_enqueue(model.h, 1), "enqueue")
        shygpu.check(lib.shygpu_get_levels(model.h, ring[i % 4].data_ptr()), "get_levels")
    shygpu.check(lib.shygpu_sync(model.h), "sync")
    e2e_s = time.perf_counter() - t0
    e2e_value = replica_throughput(units, e2e_steps, e2e_s, world)

    # The reference-style form, basin by basin with a wait after each call
    # (shygpu_set_forcing per basin, shygpu_run(1), shygpu_get_state per
    # basin), reported beside it.
    taux = [torch.from_numpy(np.ascontiguousarray(c["tauxnv"])).pin_memory() for c in case_list]
    tauy = [torch.from_numpy(np.ascontiguousarray(c["tauynv"])).pin_memory() for c in case_list]
    outs = [torch.empty(c["nkn"], dtype=torch.float32).pin_memory() for c in case_list]
    from shygpu import abi
    import ctypes as C
    states = []
    for o in outs:
        st = abi.ShyState()
        st.znv = C.cast(C.c_void_p(o.data_ptr()), abi.f32p)
        states.append(st)
    pb_steps = min(a.steps, 50)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(pb_steps):
        for b in range(nb):
            lib.shygpu_set_forcing(model.h, b, taux[b].data_ptr(), tauy[b].data_ptr(), None, None)
        shygpu.check(lib.shygpu_run(model.h, 1), "run")
        for b in range(nb):
            shygpu.check(lib.shygpu_get_state(model.h, b, C.byref(states[b])), "get_state")
    pb_s = time.perf_counter() - t0
    pb_value = replica_throughput(units, pb_steps, pb_s, world)

    # ---- live per-kernel times for the roofline (eager launches with events) ----
    prof = model.profile_steps(20)
    infos = [model.info(b) for b in range(nb)]
    nsc = int(c0["params"]["itemp"]) + int(c0["params"]["isalt"]) + int(c0["params"]["nconz"])
    algo = algorithmic_bytes(case_list, infos, nsc)
    tot_ms = sum(v[0] for v in prof.values())
    dom = max(prof, key=lambda k: prof[k][0])
    dom_ms, dom_n = prof[dom]
    peak, peak_kind = load_peak()
    dom_bytes = algo["zeta_survey"] if dom == "zeta" else algo[dom]
    achieved = dom_bytes / (dom_ms / dom_n / 1000.0) / 1e9
    traffic = None
    tf = ROOT / "profiles" / "traffic.json"
    if tf.exists():
        try:
            traffic = json.loads(tf.read_text()).get(a.workload, {}).get(dom)
        except Exception:
            traffic = None
    kernels = {k: {"ms_per_launch": (v[0] / v[1] if v[1] else 0.0), "share": v[0] / tot_ms if tot_ms else 0,
                   "launches": v[1], "algorithmic_bytes": algo[k],
                   "gbs": (algo[k] / (v[0] / v[1] / 1000.0) / 1e9) if v[1] and v[0] > 0 else 0.0}
               for k, v in prof.items()}

    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": workload_config(a.workload, case_list, world),
        "gpu_launches": int(launches),
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "steps": e2e_steps,
                "path": "shygpu_set_forcing_all(wind) + shygpu_enqueue(1) + shygpu_get_levels(znv) every step, "
                        "pinned host buffers, shygpu_sync at the end",
                "per_basin": {"value": pb_value, "steps": pb_steps,
                              "path": "shygpu_set_forcing(wind) + shygpu_run(1) + shygpu_get_state(znv), "
                                      "every basin, waiting after each call"}},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "algorithmic_bytes_per_launch": dom_bytes,
                     "bytes_model": ("zeta: 100 B per node for assembly + 80 B per node per CG "
                                     "iteration, each basin with its own iteration count")
                     if dom == "zeta" else "compulsory traffic of the kernel's arrays",
                     "achieved_design_bytes": (algo["zeta"] / (dom_ms / dom_n / 1000.0) / 1e9)
                     if dom == "zeta" else None},
        "accuracy": check,
        "tuning": tuning,
        "kernels": kernels,
        "solver": {"krylov_iters_last_step": infos[0].krylov_iters,
                   "refinements": infos[0].refinements, "resid": infos[0].resid},
    }
    if a.workload == "ensemble" and not a.no_plain:
        psteps = min(a.steps, 40)
        pv, pms = plain_gpu(case_list, psteps, lib)
        line["plain_gpu"] = {"value": pv, "unit": METRIC, "ms_per_step": pms, "steps": psteps,
                             "form": "one model per basin, basins advanced one after the other"}
        line["batched_over_plain"] = value / pv
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        # a bounded sample: about 20 s of CPU work at the oracle's ~1.8e6
        # node*layer*steps/s per core, over every basin of the workload
        nproc = os.cpu_count() or 1
        csteps = int(max(1, min(20, round(20 * 1.8e6 / units))))
        v, tmax, used = cpu_timing(a.workload, case_list, csteps, 1, nproc)
        line["cpu_baseline"] = {"value": v, "unit": METRIC, "cores": used, "kind": "port",
                                "host_cpu": host_cpu(),
                                "sample": f"{csteps} time steps of every basin of the timed workload, "
                                          f"dealt over {used} processes, one per host core; FP64 C++ "
                                          "restatement of the reference step (oracle/shyref.cpp, -O3)"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    model.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
