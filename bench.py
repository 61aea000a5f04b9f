"""Benchmark: site-updates/s of the leapfrog evolution on B200 (headline: SM 256^3, mixed form).

Contract: ``python bench.py --gpus N --steps K --warmup W`` (torchrun for N > 1)
prints ONE JSON line on rank 0.  A "step" is one leapfrog time step of the
whole lattice (the body of GFTEvolver's Lattice::evolve time loop), with the
Energy and GaugeCondition analysers logging every 10 steps as in the
reference's shipped analyser configuration.

  value      site-updates/s of the mixed form over all ranks, fields resident
             in HBM (device-timed with CUDA events on the library's stream,
             max over ranks).  State (2.55 GB at 256^3) >> L2 (126 MB): no L2
             flush needed.
  e2e        the same metric through the C ABI with host buffers: upload of the
             initial fields from pinned host memory, K steps, download of the
             final fields and the observable rows, all inside the timed region.
  roofline   step kernel: algorithmic bytes per site-update (228 B for SM in
             FP32 storage: both time levels read once, one level written)
             x sites / average step-kernel duration, vs measured HBM copy
             bandwidth.
  cpu_baseline  the reference itself (oracle/_ref/ref32, compiled from its own
             sources) on the host cores, a bounded sample; forms.fp64 carries the
             same for its double-storage build (oracle/_ref/ref64).
  precision  the mixed form against the FP64 form on the same initial data
             over --precision-steps steps (default 1000): field deviation,
             energy drift and Gauss-law residual.

``--impl reference`` times the reference CPU evolver on the host cores
instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

B_ALG = {  # algorithmic bytes per site-update: 2 levels read once + 1 level written
    ("sm", 4): 57 * 4, ("sm", 8): 57 * 8,
    ("2hdm", 4): 69 * 4, ("2hdm", 8): 69 * 8,
}
LOG_EVERY = 10


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=256)
    ap.add_argument("--model", choices=["sm", "2hdm"], default="sm")
    ap.add_argument("--form", choices=["mixed", "fp64", "ref32", "ref64"], default="mixed")
    ap.add_argument("--fp64-steps", type=int, default=None, help="steps for the FP64 comparison run")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--exchange", choices=["library", "python"], default="library",
                    help="x-slabs (--slab, N > 1): ghost-plane exchange posted by the library over NCCL and "
                         "overlapped with the interior planes, or a per-step callback through torch.distributed")
    ap.add_argument("--fp64-kernel", choices=["auto", "global", "tiled"], default="auto",
                    help="step kernel of the FP64 form (its own line with --form fp64, or the comparison leg)")
    ap.add_argument("--kernel", choices=["auto", "global", "tiled", "pair", "split"], default="auto",
                    help="step kernel of the throughput forms")
    ap.add_argument("--tile", type=int, default=0, help="tiled kernel: tile shape index (0: 8x32, 1: 4x32, 2: 4x16, 3: 16x16)")
    ap.add_argument("--march", type=int, default=32, help="tiled kernel: planes per CTA along x")
    ap.add_argument("--precision-table", type=int, default=0,
                    help="steps of a run of every form (mixed, ref32, fp64) against the FP64 form (0: skip)")
    ap.add_argument("--precision-steps", type=int, default=1000,
                    help="steps of the mixed-vs-FP64 precision run (0: skip)")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-form comparison run")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other benchmark configurations (SM 32^3 FP64, 2HDM 192^3, 2HDM 448^3 wall)")
    ap.add_argument("--slab", action="store_true",
                    help="N = 1: run the x-slab path (ghost planes refreshed by the exchange callback) on one GPU")
    ap.add_argument("--ensemble-steps", type=int, default=500,
                    help="steps of the 64-member ensemble run (0: skip)")
    ap.add_argument("--ensemble-tile", type=int, default=-1,
                    help="ensemble: tile shape index (0: 8x32, 1: 4x32, 2: 4x16, 3: 16x16); -1: the autotuner's choice")
    ap.add_argument("--ensemble-march", type=int, default=64, help="ensemble: planes per tile along x with --ensemble-tile")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def workload_params(model: str, n: int):
    from gftevolver_b200 import GFT_MODEL_2HDM, GFT_MODEL_SM, InitialData, LatticeParams
    if model == "sm":
        p = LatticeParams(model=GFT_MODEL_SM, nx=n, ny=n, nz=n, dt=0.05, g=0.65, gp=0.35, lam=0.13, eta_sqr=1.0,
                          energy_every=LOG_EVERY, gauss_every=LOG_EVERY)
        ic = InitialData(seed=20240101, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    else:
        p = LatticeParams(model=GFT_MODEL_2HDM, nx=n, ny=n, nz=n, dt=0.05, g=0.65, gp=0.35,
                          m1=0.5, m2=0.5, l1=0.065, l2=0.065, l3=0.2, m12r=0.2, l4p5=-0.1,
                          energy_every=LOG_EVERY, gauss_every=LOG_EVERY)
        ic = InitialData(seed=20240102, mean=[0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
    return p, ic


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="gft_clocks_", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.out, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                t = [x.strip() for x in line.split(",")]
                if len(t) >= 9:
                    rows.append(t)
        os.unlink(self.out.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def measured_peaks():
    """HBM copy bandwidth (GB/s) measured on this pool's B200s, else the recipe's fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            with open(path) as f:
                d = json.load(f)
            return float(d["hbm_gbs"]), "measured"
        except (OSError, ValueError, KeyError, TypeError):
            pass  # an unreadable file: the fallback, named as such in the line
    return 6650.0, "fallback"


def committed_traffic(kernel: str):
    """Per-launch DRAM bytes from the committed ncu summary, if any (profiles/*.json)."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(kernel)


# ---------------------------------------------------------------------------
# CPU baseline: the reference binary (or the oracle port) on the host cores
# ---------------------------------------------------------------------------
def cpu_reference_throughput(model: str, n: int, steps: int, procs: int, fp64: bool = False):
    """Run `procs` independent reference processes, each n^3 for `steps` steps; aggregate site-updates/s.
    fp64: the reference built with double storage (oracle/_ref/ref64) instead of its float build."""
    import numpy as np
    from oracle import oracle as orc
    from oracle import refrun

    op = orc.Params(model=orc.MODEL_SM if model == "sm" else orc.MODEL_2HDM, nx=n, ny=n, nz=n,
                    energy_every=LOG_EVERY, gauss_every=LOG_EVERY)
    ic = orc.ICSpec(seed=7, mean=[1.0 if model == "sm" else 0.7] * 8, sigma=[0.1] * 8, theta_sigma=0.1,
                    eps_sigma=0.1)
    sc, ve = orc.init_fields(op, ic, np.float32)
    if refrun.available(fp64):
        results = [None] * procs

        def one(k):
            results[k] = refrun.run(op, sc, ve, steps, fp64=fp64)[3]

        ths = [threading.Thread(target=one, args=(k,)) for k in range(procs)]
        t0 = time.perf_counter()
        for t in ths:
            t.start()
        for t in ths:
            t.join()
        wall = time.perf_counter() - t0
        per = [op.nsite * steps / s for s in results]
        agg = procs * op.nsite * steps / max(results)
        return {"value": agg, "unit": "site-updates/s", "cores": procs, "kind": "reference",
                "per_process": statistics.median(per), "wall_s": wall,
                "sample": f"{procs} independent processes of the reference "
                          f"(oracle/_ref/{'ref64' if fp64 else 'ref32'}, -O3) "
                          f"each {n}^3 x {steps} steps, analysers every {LOG_EVERY}"}
    if fp64:
        return None  # the FP64 figure is reported only for the reference itself
    # oracle port (single thread per process)
    t0 = time.perf_counter()
    orc.evolve(op, sc, ve, steps)
    secs = time.perf_counter() - t0
    return {"value": op.nsite * steps / secs, "unit": "site-updates/s", "cores": 1, "kind": "port",
            "sample": f"C oracle, 1 thread, {n}^3 x {steps} steps"}


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def run_reference_arm(args, rank, world):
    """--impl reference: the reference CPU evolver on the host cores (rank 0 only).

    One reference process per host core, each evolving its own n^3 lattice for
    W + K steps (the reference is single-threaded and not reentrant, so the
    cores run independent lattices); n is chosen so the run takes about a
    minute.  Site-updates/s of this per-site loop does not depend on n.
    """
    if rank != 0:
        return
    procs = host_cores()
    total = args.warmup + args.steps
    n = int(round((60.0 * 1.9e5 / max(total, 1)) ** (1.0 / 3.0)))
    n = max(8, min(n, 64))
    r = cpu_reference_throughput(args.model, n, total, procs)
    value = r["value"]
    line = {
        "impl": "reference", "metric": "site-updates/s", "value": value, "unit": "site-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 storage, f64 arithmetic", "data": "synthetic",
        "config": {"workload": f"{args.model.upper()} periodic leapfrog, {n}^3 per process (bounded sample of the "
                               f"{args.size}^3 workload; site-updates/s is size-independent for this per-site loop), "
                               f"analysers every {LOG_EVERY}",
                   "lattice": [n, n, n], "log_every": LOG_EVERY, "processes": procs},
        "cpu_baseline": {"value": value, "unit": "site-updates/s", "cores": r["cores"], "kind": r["kind"],
                         "sample": r["sample"]},
        "e2e": {"value": value, "unit": "site-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Precision of the mixed form against the FP64 form
# ---------------------------------------------------------------------------
def precision_report(p, ic, steps: int, device: int) -> dict:
    """Evolve the same initial data in the mixed and the FP64 form and compare.

    Both forms generate the initial fields on the device from the same seed
    (the mixed form stores them rounded to float).  Reported: the largest
    absolute deviation of any stored word after `steps` steps (both levels,
    reference layout), the relative energy drift of each form over the run and
    the largest relative difference of the mixed energy from the FP64 energy
    at the logging steps, and the Gauss-law residual (largest |violation| over
    sites, constraint equations and logging steps) of each form.
    """
    import torch

    from gftevolver_b200 import Evolver

    evs = {f: Evolver(p, form=f, device=device) for f in ("mixed", "fp64")}
    rows = {}
    for f, ev in evs.items():
        ev.init_fields(ic)
        rows[f] = ev.evolve(steps)
    fields = {}
    for f, ev in evs.items():
        dt = torch.float64 if f == "fp64" else torch.float32
        sc = torch.empty((2, p.nx, p.ny, p.nz, p.nsc), dtype=dt, device=f"cuda:{device}")
        ve = torch.empty((2, p.nx, p.ny, p.nz, 15), dtype=dt, device=f"cuda:{device}")
        ev.download_device(sc.data_ptr(), ve.data_ptr(), f == "fp64")
        fields[f] = (sc, ve)
        ev.close()
    dev_sc = (fields["mixed"][0].double() - fields["fp64"][0]).abs().max().item()
    dev_ve = (fields["mixed"][1].double() - fields["fp64"][1]).abs().max().item()
    del fields
    torch.cuda.empty_cache()

    def energies(rs):
        return [(r["time_iter"], r["energy"]) for r in rs if r["has_energy"]]

    e32, e64 = energies(rows["mixed"]), energies(rows["fp64"])
    def drift(es):
        e0 = es[0][1]
        return max(abs(e - e0) for _, e in es) / abs(e0)
    rel_e = max(abs(a[1] - b[1]) / abs(b[1]) for a, b in zip(e32, e64))
    def gauss(rs):
        g = [max(r["gauss_max"]) for r in rs if r["has_gauss"]]
        return max(g) if g else None
    def gauss_int(rs):
        g = [max(r["gauss_int"]) for r in rs if r["has_gauss"]]
        return max(g) if g else None
    return {
        "steps": steps, "lattice": [p.nx, p.ny, p.nz], "log_every": LOG_EVERY,
        "field_max_abs_dev": {"scalars": dev_sc, "links": dev_ve},
        "energy_drift_rel": {"mixed": drift(e32), "fp64": drift(e64)},
        "energy_mixed_vs_fp64_rel": rel_e,
        "gauss_max": {"mixed": gauss(rows["mixed"]), "fp64": gauss(rows["fp64"])},
        "gauss_int": {"mixed": gauss_int(rows["mixed"]), "fp64": gauss_int(rows["fp64"])},
        "energy_t0": e64[0][1],
    }


def precision_table(p, ic, steps: int, device: int) -> dict:
    """Every form on the same device initial data for `steps` steps, against the FP64 form:
    storage bytes per site-update, the largest Gauss residual (over sites, constraints and
    logging steps), the largest relative energy difference from the FP64 form at the logging
    steps, the largest |stored word - FP64| after the run, and site-updates/s of the run.

    ref32 is the reference's own design: float storage with every per-site operation in FP64
    (renormalisation and momentum accumulation included), in the reference's order."""
    import torch

    from gftevolver_b200 import Evolver

    out, fields, rows = {}, {}, {}
    for form in ("fp64", "mixed", "ref32"):
        ev = Evolver(p, form=form, device=device)
        ev.init_fields(ic)
        st = torch.cuda.ExternalStream(ev.stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        rows[form] = ev.evolve(steps)
        e1.record(st)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        dt = torch.float64 if form == "fp64" else torch.float32
        sc = torch.empty((2, p.nx, p.ny, p.nz, p.nsc), dtype=dt, device=f"cuda:{device}")
        ve = torch.empty((2, p.nx, p.ny, p.nz, p.nve), dtype=dt, device=f"cuda:{device}")
        ev.download_device(sc.data_ptr(), ve.data_ptr(), form == "fp64")
        torch.cuda.synchronize()
        ev.close()
        if form == "fp64":
            fields["fp64"] = (sc, ve)
        else:
            dev = max((sc.double() - fields["fp64"][0]).abs().max().item(),
                      (ve.double() - fields["fp64"][1]).abs().max().item())
            del sc, ve
        g = [max(r["gauss_max"]) for r in rows[form] if r["has_gauss"]]
        out[form] = {"bytes_per_site_update": B_ALG[("sm" if p.model == 1 else "2hdm", 8 if form == "fp64" else 4)],
                     "gauss_max": max(g) if g else None, "value": p.nsite * steps / (ms / 1e3),
                     "field_max_abs_dev_vs_fp64": 0.0 if form == "fp64" else dev}
    del fields
    torch.cuda.empty_cache()
    e64 = [r["energy"] for r in rows["fp64"] if r["has_energy"]]
    for form in out:
        e = [r["energy"] for r in rows[form] if r["has_energy"]]
        out[form]["energy_vs_fp64_rel"] = max(abs(a - b) / abs(b) for a, b in zip(e, e64))
        out[form]["energy_drift_rel"] = max(abs(a - e[0]) for a in e) / abs(e[0])
    return {"steps": steps, "lattice": [p.nx, p.ny, p.nz], "log_every": LOG_EVERY, "forms": out}


# ---------------------------------------------------------------------------
# Ensemble: 64 SM realisations of uneven sizes in one persistent launch per step
# ---------------------------------------------------------------------------
def ensemble_report(steps: int, device: int, tile: int = -1, march: int = 64) -> dict:
    """64 SM members, edges drawn uniformly from {32, 48, 64, 96} (seeded), distinct
    seeds, mixed form, analysers every LOG_EVERY steps; tile and march depth from
    the autotuner (or `tile` >= 0 and `march`); whole logging periods replayed
    from a CUDA graph."""
    import random

    import numpy as np

    from gftevolver_b200 import GFT_MODEL_SM, Ensemble, InitialData, LatticeParams

    rng = random.Random(4)
    edges = [rng.choice((32, 48, 64, 96)) for _ in range(64)]
    ps = [LatticeParams(model=GFT_MODEL_SM, nx=n, ny=n, nz=n, dt=0.05, g=0.65, gp=0.35, lam=0.13, eta_sqr=1.0,
                        energy_every=LOG_EVERY, gauss_every=LOG_EVERY) for n in edges]
    ics = [InitialData(seed=1000 + k, mean=[1.0] * 8, sigma=[0.1] * 8, theta_sigma=0.1, eps_sigma=0.1)
           for k in range(64)]
    with Ensemble(ps, device=device) as ens:
        ens.init_fields(ics)
        if tile < 0:
            tile, march = ens.autotune(4)
        else:
            ens.set_kernel(tile, march)
        ens.evolve(2 * LOG_EVERY)  # warm-up (builds the graph)
        l0 = ens.launch_count
        sampler = ClockSampler(device)
        sampler.start()
        rows = ens.evolve(steps)
        clocks = sampler.stop()
        ms = ens.last_ms
        launches = ens.launch_count - l0
        nsite = ens.nsite
        bad = [r for m in rows for r in m if r["has_energy"] and not np.isfinite(r["energy"])]
    return {
        "workload": "64 SM members, edges uniform in {32,48,64,96} (seeded), random links eps~N(0,0.1^2), "
                    "theta_Y~N(0,0.1^2), Higgs N(1,0.1^2), distinct seeds, mixed form, analysers every "
                    f"{LOG_EVERY} steps",
        "members": 64, "sites": nsite, "edges_histogram": {str(e): edges.count(e) for e in (32, 48, 64, 96)},
        "steps": steps, "value": nsite * steps / (ms / 1e3), "unit": "site-updates/s",
        "ms_per_step": ms / steps,
        # 228 B per site-update (the single lattice's algorithmic bytes) over the whole step, launches included
        "roofline_frac": B_ALG[("sm", 4)] * nsite * steps / (ms / 1e3) / 1e9 / measured_peaks()[0],
        "tile": ["8x32", "4x32", "4x16", "16x16"][tile], "march": march, "graphs": True,
        "kernel_launches_per_step": launches / steps, "nonfinite_rows": len(bad),
        # SM clocks of this leg (it follows the other legs' seconds of load; a power cap lowers them)
        "clocks": clocks,
        "ms_x_sm_mhz": (ms / steps * clocks["sm_mhz"]) if clocks.get("sm_mhz") else None,
    }


# ---------------------------------------------------------------------------
# The other benchmark configurations, measured at their own sizes
# ---------------------------------------------------------------------------
def _timed_config(p, ic, form, steps, device):
    import torch

    from gftevolver_b200 import Evolver
    ev = Evolver(p, form=form, device=device)
    ev.init_fields(ic)
    ev.evolve(3)
    ev.step_kernel_ms()
    st = torch.cuda.ExternalStream(ev.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    rows = ev.evolve(steps)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    kms, _ = ev.step_kernel_ms()
    name = ev.step_kernel_name
    ev.close()
    sbytes = 8 if form in ("fp64", "ref64") else 4
    model = "sm" if p.model == 1 else "2hdm"
    balg = B_ALG[(model, sbytes)]
    peak = measured_peaks()[0]
    e = [r for r in rows if r["has_energy"]]
    g = [max(r["gauss_max"]) for r in rows if r["has_gauss"]]
    return {
        "form": form, "steps": steps, "value": p.nsite * steps / (ms / 1e3), "unit": "site-updates/s",
        "ms_per_step": ms / steps, "kernel": name, "step_kernel_ms": kms,
        "roofline_frac": balg * p.nsite / (kms / 1e3) / 1e9 / peak if kms > 0 else None,
        "energy_first": e[0]["energy"] if e else None, "energy_last": e[-1]["energy"] if e else None,
        "gauss_max": max(g) if g else None, "plaq_su2_last": e[-1]["plaq_su2"] if e else None,
    }


def configs_report(device: int) -> dict:
    """SM 32^3 FP64 identity links (1000 steps); 2HDM 192^3 FP64 and mixed (100 of the 500
    steps, which the timing does not depend on); 2HDM 448^3 mixed bubble wall (2000 steps,
    analysers every 50).  Initial data are generated on the device from fixed seeds."""
    import dataclasses

    from gftevolver_b200 import InitialData
    out = {}
    p, _ = workload_params("sm", 32)
    ic = InitialData(seed=7, mean=[0.0] * 8, sigma=[0.1] * 8)  # identity links, Higgs N(0, 0.1^2)
    r = _timed_config(p, ic, "fp64", 1000, device)
    r["workload"] = "SM 32^3 FP64, identity links, Higgs N(0,0.1^2), dt=0.05, analysers every 10"
    out["sm_32_fp64"] = r
    p, ic = workload_params("2hdm", 192)
    for form in ("fp64", "mixed"):
        r = _timed_config(p, ic, form, 100, device)
        r["workload"] = ("2HDM 192^3, m11^2=m22^2=-0.5, m12^2=0.1, l1=l2=0.13, l3=0.2, l4=l5=-0.05, random links, "
                         "doublets N(0.7,0.1^2), dt=0.05")
        out[f"2hdm_192_{form}"] = r
    out["2hdm_192_mixed"]["mixed_over_fp64"] = out["2hdm_192_mixed"]["value"] / out["2hdm_192_fp64"]["value"]
    p, _ = workload_params("2hdm", 448)
    p = dataclasses.replace(p, energy_every=50, gauss_every=50)
    ic = InitialData(seed=5, mean=[0.0] * 8, sigma=[0.05] * 8, wall_width=5.0, wall_value=1.0)
    r = _timed_config(p, ic, "mixed", 2000, device)
    r["workload"] = ("2HDM 448^3 mixed, doublet 1 component 0 a periodic tanh double wall along z (width 5, "
                     "value 1) + N(0,0.05^2), doublet 2 N(0,0.05^2), identity links, dt=0.05, analysers every 50")
    out["2hdm_448_wall_mixed"] = r
    return out


# ---------------------------------------------------------------------------
def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import numpy as np
    import torch

    from gftevolver_b200 import Evolver

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    p, ic = workload_params(args.model, args.size)
    form = args.form
    sbytes = 8 if form in ("fp64", "ref64") else 4
    balg = B_ALG[(args.model, sbytes)]

    kind = {"auto": 0, "global": 1, "tiled": 2, "pair": 3, "split": 4}[args.kernel]
    kind64 = {"auto": 0, "global": 1, "tiled": 2}[args.fp64_kernel]

    def make_runner(form_):
        """N = 1: the whole lattice.  N > 1: this rank's x-slab of an (N * n) x n x n lattice
        (ghost planes exchanged over NCCL after every step; rows combined over ranks)."""
        if world > 1 or args.slab:
            import dataclasses

            from gftevolver_b200.slab import SlabEvolver
            s = SlabEvolver(dataclasses.replace(p, nx=p.nx * world), form=form_, device=local,
                            exchange=args.exchange)
            return s, s.local
        e = Evolver(p, form=form_, device=local)
        return e, e

    def timed_run(form_, steps, warmup, sampler=None):
        runner, ev = make_runner(form_)
        if form_ == "mixed" and (kind != 0 or args.tile != 0 or args.march != 32):
            ev.set_kernel(kind, args.tile, args.march)
        if form_ == "fp64" and kind64 != 0:
            ev.set_kernel(kind64, args.tile if kind64 == 2 else 0, args.march)
        runner.init_fields(ic)
        if warmup:
            runner.evolve(warmup)
        ev.step_kernel_ms()  # reset
        launches0 = ev.launch_count
        stream = torch.cuda.ExternalStream(ev.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        barrier()
        if sampler:
            sampler.start()
        e0.record(stream)
        rows = runner.evolve(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        clocks = sampler.stop() if sampler else None
        barrier()
        ms = e0.elapsed_time(e1)
        kms, nk = ev.step_kernel_ms()
        ev.timed_launches = ev.launch_count - launches0
        ev.runner = runner
        return ev, ms, kms, nk, rows, clocks

    sampler = ClockSampler(local)
    ev, ms, kms, nk, rows, clocks = timed_run(form, args.steps, args.warmup, sampler)
    kernel_name = ev.step_kernel_name
    ms_max = max_over_ranks(ms)
    value = world * p.nsite * args.steps / (ms_max / 1e3)
    launches = ev.timed_launches  # the library's own count of kernels launched in the timed region

    # FP64 plain form for the mixed-vs-FP64 ratio
    fp64 = None
    if form == "mixed" and not args.no_fp64:
        ev.runner.close()
        fsteps = args.fp64_steps or args.steps  # the same step count (and logging steps) as the mixed form
        ev64, ms64, kms64, nk64, _, _ = timed_run("fp64", fsteps, min(args.warmup, 3))
        ms64 = max_over_ranks(ms64)
        v64 = world * p.nsite * fsteps / (ms64 / 1e3)
        fp64 = {"value": v64, "steps": fsteps, "step_kernel_ms": kms64,
                "roofline_frac": (B_ALG[(args.model, 8)] * p.nsite / (kms64 / 1e3)) / 1e9 / measured_peaks()[0],
                "mixed_over_fp64": value / v64}
        ev64.runner.close()
    else:
        ev.runner.close()

    # end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        dt = torch.float32 if sbytes == 4 else torch.float64
        sc_h = torch.empty((2, p.nx, p.ny, p.nz, p.nsc), dtype=dt).pin_memory()
        ve_h = torch.empty((2, p.nx, p.ny, p.nz, 15), dtype=dt).pin_memory()
        runner, ev = make_runner(form)
        if world > 1 or args.slab:  # the slab with its ghost planes
            sc_h = torch.empty((2, p.nx + 2, p.ny, p.nz, p.nsc), dtype=dt).pin_memory()
            ve_h = torch.empty((2, p.nx + 2, p.ny, p.nz, 15), dtype=dt).pin_memory()
        runner.init_fields(ic)
        ev.download_ptr(sc_h.data_ptr(), ve_h.data_ptr(), sbytes == 8)
        ev.upload_ptr(sc_h.data_ptr(), ve_h.data_ptr(), sbytes == 8, 0)  # warm the staging buffer
        runner.evolve(min(args.warmup, 3))
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        ev.upload_ptr(sc_h.data_ptr(), ve_h.data_ptr(), sbytes == 8, 0)
        rows_e2e = runner.evolve(args.steps)
        ev.download_ptr(sc_h.data_ptr(), ve_h.data_ptr(), sbytes == 8)
        torch.cuda.synchronize()
        secs = time.perf_counter() - t0
        barrier()
        secs = max_over_ranks(secs)
        runner.close()
        nbytes = (sc_h.numel() + ve_h.numel()) * sc_h.element_size()
        e2e = {"value": world * p.nsite * args.steps / secs, "unit": "site-updates/s",
               "h2d_bytes_per_step": nbytes / args.steps,
               "d2h_bytes_per_step": (nbytes + len(rows_e2e) * 160) / args.steps,
               "note": "upload of both levels from pinned host memory + K steps (analysers every 10) + download "
                       "of both levels and the observable rows, per rank; bytes per step = per-run bytes / K"}

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # single-GPU properties: measured at N = 1 only
    precision = None
    if args.precision_steps > 0 and form == "mixed" and world == 1:
        precision = precision_report(p, ic, args.precision_steps, local)
    ptable = None
    if args.precision_table > 0 and world == 1:
        ptable = precision_table(p, ic, args.precision_table, local)
    ensemble = None
    if args.ensemble_steps > 0 and world == 1:
        ensemble = ensemble_report(args.ensemble_steps, local, args.ensemble_tile, args.ensemble_march)
    configs = None
    if not args.no_configs and world == 1 and args.size == 256 and args.model == "sm":
        configs = configs_report(local)

    peak, peak_kind = measured_peaks()
    achieved = balg * p.nsite / (kms / 1e3) / 1e9
    traffic = committed_traffic(f"{kernel_name}_{args.model}_{form}_{args.size}")
    cpu = None
    if not args.no_cpu_baseline and world == 1:  # the CPU baselines belong to the N = 1 line
        try:
            # 52^3 x 20 steps per process: about 10 s of each core's time at the reference's ~2.7e5
            # site-updates/s per core
            cpu = cpu_reference_throughput(args.model, 52, 20, host_cores())
        except Exception as ex:  # the baseline is reported, not required
            cpu = {"value": None, "error": str(ex)}
        if fp64 is not None:
            # the reference's double-storage build beside the FP64 form
            try:
                fp64["cpu_reference"] = cpu_reference_throughput(args.model, 52, 20, host_cores(), fp64=True)
            except Exception as ex:
                fp64["cpu_reference"] = {"value": None, "error": str(ex)}
    line = {
        "metric": "site-updates/s", "value": value, "unit": "site-updates/s", "n_gpus": world,
        # the FP64 form on the same workload, up front so that short records of the line keep it
        "fp64_value": fp64["value"] if fp64 else None,
        "mixed_over_fp64": fp64["mixed_over_fp64"] if fp64 else None,
        "fp64_roofline_frac": fp64["roofline_frac"] if fp64 else None,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if sbytes == 4 else "f64", "data": "synthetic",
        "config": {"workload": (f"{args.model.upper()} {world * args.size}x{args.size}x{args.size} periodic leapfrog "
                                f"({args.size}^3 x-slab per GPU)" if world > 1 else
                                f"{args.model.upper()} {args.size}^3 periodic leapfrog") + f", form={form}, random SU(2) "
                               f"links eps~N(0,0.1^2), theta_Y~N(0,0.1^2), Higgs N(1,0.1^2), dt=0.05, "
                               f"energy+Gauss analysers every {LOG_EVERY} steps",
                   "lattice": [p.nx, p.ny, p.nz], "form": form, "log_every": LOG_EVERY,
                   "l2": "inputs larger than L2 (state %.2f GB per level pair)" % (2 * p.nsite * (15 + p.nsc) * sbytes / 1e9),
                   "parallelism": (f"x-slabs x{world}: lattice {world * p.nx}x{p.ny}x{p.nz}, one ghost plane per "
                                   "side exchanged over NCCL send/recv every step ("
                                   + ("posted by the library, overlapped with the interior planes"
                                      if args.exchange == "library" else "after the step, from a callback")
                                   + "), FP64 all-reduce of the analyser rows") if world > 1 else
                                  ("single GPU, one x-slab exchanging with itself" if args.slab else "single GPU"),
                   "kernel": args.kernel, "tile": args.tile, "march": args.march},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic, "peak_kind": peak_kind, "kernel": kernel_name,
                     "bytes_per_site_update": balg, "avg_kernel_ms": kms, "kernel_launches_timed": nk,
                     # clock-normalised step time (ms x median SM MHz under load): compares runs on
                     # boxes whose clocks differ (a power cap lowers them for this issue-bound kernel)
                     "kernel_ms_x_sm_mhz": (kms * clocks["sm_mhz"]) if clocks and clocks.get("sm_mhz") else None},
        "gpu_launches": launches,
        "clocks": clocks,
        "forms": {"fp64": fp64} if fp64 else None,
        "e2e": e2e,
        "cpu_baseline": cpu,
        "precision": precision,
        "precision_table": ptable,
        "ensemble": ensemble,
        "configs": configs,
        "analyser_rows": len(rows),
    }
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
