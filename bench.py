#!/usr/bin/env python
"""Benchmark of the B200 force/integration path (one JSON line on rank 0).

Workload: 33,400 flexible waters (100,200 atoms) in a 10 nm cube, LJ + Ewald
real space at 1.0 nm, PME 96^3 order 4, pair list every 10 steps, leapfrog at
1 fs.  Metric: ns/day (steps * dt * 86400 / time); pairs/s is reported beside
it.  A step is one full MD step (forces + integration); the timed region runs
whole pair-list periods (list rebuild + 10 steps, energies on the last step),
with L2 flushed before each period.  Inputs are seeded synthetic water (no
public dataset is named).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lima|reference]

N > 1 runs under torchrun as independent replicas (a single system has no
decomposition across GPUs: short-range forces would need a halo exchange and
PME a distributed FFT), value = the sum of all ranks' ns/day over the max time.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT_NS = 1e-6
PERIOD = 10                  # steps per pair-list period (nstlist)
CUTOFF = 1.0
GRID = (96, 96, 96)
FLOPS_PER_PAIR = 50          # counting rule of the pair kernel's roofline
WORKLOAD = "water100k_10nm_pme96"


def ns_per_day(step_seconds: float) -> float:
    # the reference prints n_steps*dt/(wall/86400) (code/LIMA/mdrun.h:134-143)
    return DT_NS * 86400.0 / step_seconds


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active," \
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown," \
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
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
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


class NvmlSampler:
    """SM clock and throttle reasons polled through NVML every ~1 ms on a
    thread, so that even a timed region of a few milliseconds holds samples.
    Falls back to the nvidia-smi sampler when NVML is not available."""

    # clocks-event reason bits (nvml.h: nvmlClocksEventReason*)
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, device: int, period_s: float = 0.001):
        self.device = device
        self.period = period_s
        self.samples = []
        self.fallback = None
        self.nv = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(device)
            self.max_mhz = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
        except Exception:
            self.nv = None
            self.fallback = ClockSampler(device)

    def _run(self):
        nv = self.nv
        while not self.stop_flag.is_set():
            try:
                mhz = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                try:
                    rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                except Exception:
                    rs = int(nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h))
                self.samples.append((mhz, rs))
            except Exception:
                pass
            time.sleep(self.period)

    def start(self):
        if self.fallback is not None:
            return self.fallback.start()
        self.stop_flag = threading.Event()
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()

    def stop(self):
        if self.fallback is not None:
            return self.fallback.stop()
        self.stop_flag.set()
        self.t.join(timeout=5)
        sm = [m for m, _ in self.samples]
        reasons = sorted(k for k, b in self.REASONS.items() if any(r & b for _, r in self.samples))
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(sm), "source": "NVML, ~1 ms polling"}


def headline_config(n_atoms: int, world: int) -> dict:
    """The workload's description, identical in both arms' JSON lines."""
    return {"workload": WORKLOAD, "atoms": n_atoms, "pme_grid": list(GRID), "cutoff_nm": CUTOFF, "nstlist": PERIOD,
            "dt_fs": 1.0, "integrator": "leapfrog", "parallelism": "replicas" if world > 1 else "single",
            "l2": "flushed (256 MiB write) before every timed iteration; an iteration is one pair-list "
                  "period: list rebuild + 10 steps, energies evaluated on the last step",
            "accumulation": "int64 fixed point forces/energies, FP64 positions"}


def accuracy_summary():
    """Per-configuration accuracy against the FP64 oracle, from the committed
    report of tests/accuracy_report.py (profiles/accuracy_configs.json): force
    errors over the frames, the worst energy term, and the constant-energy
    drift and variance coefficient at dt = 1 fs."""
    path = os.path.join(ROOT, "profiles", "accuracy_configs.json")
    if not os.path.exists(path):
        return None
    try:
        rep = json.load(open(path))
    except Exception:
        return None
    out = {"source": "profiles/accuracy_configs.json (tests/accuracy_report.py, one B200)", "configs": {}}
    for r in rep:
        sm = r["summary"]
        terms = {k: v["max"] for k, v in sm["energy_rel"].items()}
        worst = max(((k, v) for k, v in terms.items() if k != "potential"), key=lambda x: x[1])
        c = {"atoms": r["atoms"], "frames": sm["frames"], "max_force_err_j_mol_nm": sm["max_abs_err"]["max"],
             "rms_force_err_j_mol_nm": sm["rms_err"]["max"], "rel_rms_force_err": sm["rel_rms"]["max"],
             "worst_energy_term": worst[0], "worst_energy_rel": worst[1], "potential_rel": terms.get("potential")}
        if "rel_rms_outside_band" in sm:
            c["rel_rms_force_err_outside_cutoff_band"] = sm["rel_rms_outside_band"]["max"]
        for d in r.get("drift") or []:
            if abs(d["dt_fs"] - 1.0) < 1e-9:
                c["drift_kj_mol_ns_atom"] = d["drift_kj_mol_per_ns_per_atom"]
                c["drift_per_ns_over_kinetic"] = d["drift_per_ns_over_kinetic"]
                c["variance_coefficient"] = d["variance_coefficient"]
        out["configs"][r["config"]] = c
    return out


def stage_rooflines(ph: dict, s, n_rows: int, hbm_gbs: float) -> dict:
    """Algorithmic bytes per stage (per-unit figures in DESIGN.md section 3) over
    the stage's event-timed average duration, against the measured HBM copy
    bandwidth.  ph: per-phase microseconds (phases serialised)."""
    n = s.n
    pts = GRID[0] * GRID[1] * GRID[2]
    half = (GRID[0] // 2 + 1) * GRID[1] * GRID[2]
    ex = s.exclusions()
    nx = int(((s.charge[ex[:, 0]] != 0) & (s.charge[ex[:, 1]] != 0)).sum())
    work = {
        "integrate": (108 * n, "108 B/atom"),
        "bonded": (96 * len(s.bonds) + 144 * len(s.angles) + 192 * len(s.dihedrals) + 112 * nx,
                   "96 B/bond + 144 B/angle + 192 B/dihedral + 112 B/excluded charged pair (Ewald correction)"),
        "pme": (16 * n + 4 * pts + 2 * 16 * pts + 20 * half + 40 * n,
                "spread 16 B/atom + 4 B/grid point, two 3-D FFTs 16 B/point each, convolution 20 B/half-complex "
                "point, gather 40 B/atom"),
        "nblist": (40 * n + 8 * n_rows, "40 B/atom + 8 B per pair-list row written (per rebuild)"),
    }
    out = {}
    for k, (b, rule) in work.items():
        us = ph.get(k)
        if not us:
            continue
        gbs = b / (us * 1e-6) / 1e9
        out[k] = {"us": us, "bytes": b, "achieved_gbs": gbs, "peak_gbs": hbm_gbs, "frac": gbs / hbm_gbs,
                  "rule": rule}
    if ph.get("pme"):
        out["pme"]["grid_points_per_s"] = pts / (ph["pme"] * 1e-6)
    return out


def cpu_step_time(system, n_steps: int, threads: int, cutoff: float = CUTOFF, grid=GRID, es_mode: int = 2):
    """The CPU oracle port of the same step (FP32 reference-faithful pair loop with
    all host threads, FP64 SPME and bonded terms, leapfrog), seconds per step.
    es_mode 1 (cutoff Coulomb) runs without PME."""
    from oracle import oracle as O
    from lima_b200.systems import ewald_kappa
    O.build()
    kappa = ewald_kappa(cutoff, 1e-5) if es_mode == 2 else 0.0
    s = system
    ex = s.exclusions()
    xp = ex[(s.charge[ex[:, 0]] != 0) & (s.charge[ex[:, 1]] != 0)]
    pos = s.pos.copy()
    vel = s.vel.astype(np.float64).copy()
    fprev = np.zeros_like(pos)
    m = s.mass.astype(np.float64)
    times = []
    for k in range(n_steps + 1):
        t0 = time.perf_counter()
        f, _, _ = O.nonbonded(pos, s.box, s.charge, s.sigma, s.epsilon, ex, cutoff, es_mode, kappa, precision=32,
                              nthreads=threads)
        if es_mode == 2:
            fl, _, _ = O.pme(pos, s.charge, s.box, grid, kappa)
            fx, _ = O.exclusion_correction(pos, s.charge, s.box, xp, kappa)
            f = f + fl + fx
        fb, _ = O.bonded(pos, s.box, s.bonds, s.bond_par, s.angles, s.angle_par, s.dihedrals, s.dihedral_par,
                         s.impropers, s.improper_par, s.pairbonds, s.pair_par)
        O.integrate(pos, vel, fprev, f + fb, m, DT_NS, 0)
        if k > 0:                      # first step is warm-up
            times.append(time.perf_counter() - t0)
    return statistics.median(times)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from lima_b200 import systems
    s = systems.config2()
    threads = os.cpu_count() or 1
    n = max(1, min(args.steps, 3))
    t = cpu_step_time(s, n, threads)
    v = ns_per_day(t)
    line = {
        "impl": "reference", "metric": "ns_per_day", "value": v, "unit": "ns/day", "n_gpus": args.gpus,
        "steps": n, "warmup": 1, "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": headline_config(s.n, int(os.environ.get("WORLD_SIZE", "1"))),
        "cpu_baseline": {"value": v, "unit": "ns/day", "cores": threads, "kind": "port",
                         "sample": f"{n} full MD steps of the {s.n}-atom box on the host (oracle port: FP32 "
                                   f"pair loop, FP64 SPME 96^3 and bonded terms), median"},
        "e2e": {"value": v, "unit": "ns/day", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU force path; the timed reference is the oracle restatement of its formulas",
    }
    print(json.dumps(line), flush=True)
    return 0


def _timed_steps(eng, n, per_step=False):
    """Device time per step (engine's CUDA events on its main stream)."""
    if per_step:
        out = []
        for _ in range(n):
            eng.reset_timings()
            eng.step(1)
            out.append(eng.timings()["step"] * 1e-6)
        return out
    eng.reset_timings()
    eng.step(n)
    t = eng.timings()
    return [t["step"] * 1e-6] * 1, t


def other_configs(args, local):
    """Secondary workloads of the specification, reported beside the headline:
    C0 (1,000 waters, cutoff Coulomb), C1 (chains + water, PME 48x48x80) and C4
    (256 uneven systems stepped together).  Pair-list periods replay as CUDA
    graphs; these working sets are not flushed from L2 between steps (C4's is
    larger than L2)."""
    from lima_b200 import Engine, systems
    from lima_b200 import engine as E
    out = {}
    k = max(args.other_steps, 21)
    # C0
    s0 = systems.config0()
    e0 = Engine(cutoff=1.2, electrostatics=E.ES_CUTOFF, nstlist=10, dt=DT_NS, device=local, use_graphs=1)
    e0.load(s0)
    e0.autotune(2)
    e0.step(20)
    t = _timed_steps(e0, k)[0][0]
    out["c0_water1k_cutoff"] = {"atoms": s0.n, "ns_per_day": ns_per_day(t), "ms_per_step": t * 1e3, "steps": k}
    e0.close()
    if args.cpu_other:
        threads = os.cpu_count() or 1
        tc = cpu_step_time(s0, 5, threads, cutoff=1.2, es_mode=1)
        out["c0_water1k_cutoff"]["cpu_baseline"] = {
            "ns_per_day": ns_per_day(tc), "ms_per_step": tc * 1e3, "cores": threads, "kind": "port",
            "sample": "5 full MD steps of the same box on the host (oracle port: FP32 pair loop, cutoff Coulomb, "
                      "FP64 bonded terms), median"}
    # C1
    s1 = systems.config1()
    e1 = Engine(cutoff=1.2, electrostatics=E.ES_EWALD, ewald_tol=1e-5, nstlist=10, dt=DT_NS, device=local,
                use_graphs=1)
    e1.load(s1, pme_grid=(48, 48, 80))
    e1.minimize(force_tol=1e5, max_steps=300)
    e1.autotune(2)
    e1.step(20)
    t = _timed_steps(e1, k)[0][0]
    out["c1_chains_water_pme48x48x80"] = {"atoms": s1.n, "ns_per_day": ns_per_day(t), "ms_per_step": t * 1e3,
                                          "steps": k, "prep": "300 energy-minimisation steps"}
    if args.cpu_other:
        threads = os.cpu_count() or 1
        p1, v1 = e1.state()
        s1c = dataclasses.replace(s1, pos=p1, vel=v1)
        tc = cpu_step_time(s1c, 3, threads, cutoff=1.2, grid=(48, 48, 80), es_mode=2)
        out["c1_chains_water_pme48x48x80"]["cpu_baseline"] = {
            "ns_per_day": ns_per_day(tc), "ms_per_step": tc * 1e3, "cores": threads, "kind": "port",
            "sample": "3 full MD steps of the minimised box on the host (oracle port: FP32 pair loop, FP64 SPME "
                      "48x48x80, exclusion correction and bonded terms incl. dihedrals), median"}
    e1.close()
    # C4
    if not args.skip_batch:
        import time as _t
        t0 = _t.perf_counter()
        batch = systems.batch_systems(256)
        gen_s = _t.perf_counter() - t0
        # one CUDA graph per 20 steps: two pair-list periods per graph
        e4 = Engine(n_systems=len(batch), cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5, pme_spacing=0.12,
                    nstlist=10, dt=DT_NS, device=local, use_graphs=2)
        for i, sy in enumerate(batch):
            e4.select(i)
            e4.load(sy)
        e4.minimize(force_tol=1e5, max_steps=100)
        e4.autotune(2)
        e4.step(20)
        t = _timed_steps(e4, k)[0][0]
        lat = sorted(_timed_steps(e4, min(k, 60), per_step=True))
        n_at = sum(sy.n for sy in batch)
        out["c4_batch256"] = {"systems": len(batch), "atoms": n_at, "aggregate_ns_per_day": len(batch) * ns_per_day(t),
                              "ms_per_step": t * 1e3, "steps": k,
                              "step_latency_ms_p50": 1e3 * lat[len(lat) // 2],
                              "step_latency_ms_p99": 1e3 * lat[min(len(lat) - 1, int(0.99 * len(lat)))],
                              "note": "every system advances each batched step, so a system's step latency is the "
                                      "batched step time; p50/p99 over eagerly timed steps; blocks of 20 steps "
                                      "(two pair-list periods) replay as one CUDA graph",
                              "generation_s": gen_s}
        e4.close()
    return out


def learned_config(args, local):
    """C3: the headline box with the learned coarse-grid PME correction.  The
    network is trained on the GPU on frames the engine generates (labelled by
    the full 96^3 grid), scored on a later, held-out state, and the step is
    timed with the correction on (coarse 32^3 + network, full-grid check every
    50 steps) against plain 96^3 PME on the same engine."""
    from lima_b200 import Engine, systems
    from lima_b200 import engine as E
    s = systems.config2()
    eng = Engine(cutoff=CUTOFF, electrostatics=E.ES_EWALD, ewald_tol=1e-5, nstlist=10, dt=DT_NS, device=local)
    eng.load(s, pme_grid=GRID)
    lp = E.LearnedPME(eng, coarse_grid=(32, 32, 32), max_frames=args.c3_frames)
    eng.step(20)
    t0 = time.perf_counter()
    for _ in range(args.c3_frames):
        eng.step(20)
        lp.collect()
    collect_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    loss = lp.train(epochs=args.c3_epochs, batch=65536, lr=1e-3, seed=1)
    train_s = time.perf_counter() - t0
    eng.step(100)                      # held-out state, 100 steps after the last frame
    coarse_rel, learned_rel = lp.eval()
    k = max(args.other_steps, 101)
    # plain full-grid PME, eager steps, per-phase times
    eng.phase_timing(True)
    eng.reset_timings()
    eng.step(k)
    t_full = eng.timings()
    # learned path; a loose bound keeps it on so that its cost can be measured
    lp.enable(True, check_interval=50, tolerance=1.0)
    eng.reset_timings()
    eng.step(k)
    t_learned = eng.timings()
    eng.phase_timing(False)
    eng.reset_timings()
    eng.step(k)
    step_learned = eng.timings()["step"] * 1e-6
    lp.enable(False)
    eng.reset_timings()
    eng.step(k)
    step_full = eng.timings()["step"] * 1e-6
    # the specified bound: the first full-grid check decides
    lp.enable(True, check_interval=50, tolerance=1e-3)
    eng.step(60)
    st = lp.status()
    eng.close()
    return {
        "atoms": s.n, "coarse_grid": [32, 32, 32], "full_grid": list(GRID), "frames": args.c3_frames,
        "epochs": args.c3_epochs, "batch": 65536, "final_train_loss": loss,
        "collect_s": collect_s, "train_s": train_s,
        "heldout_rel_rmse_coarse": coarse_rel, "heldout_rel_rmse_learned": learned_rel,
        "meets_1e-3_bound": bool(learned_rel <= 1e-3),
        "fallback_at_1e-3": {"fell_back": st["fell_back"], "last_check_rel": st["last_rel"]},
        "pme_stage_us_full": t_full["pme"], "pme_stage_us_learned": t_learned["pme"],
        "phase_us_full": {q: t_full[q] for q in ("nonbonded", "bonded", "pme", "integrate")},
        "ns_per_day_full_eager": ns_per_day(step_full), "ns_per_day_learned_eager": ns_per_day(step_learned),
        "speedup_learned_vs_full": step_full / step_learned,
        "note": "phase times serialise the streams; ns/day figures are eager steps with the PME stream "
                "overlapping the pair kernel. The learned stage includes a full-grid check every 50 steps "
                "and on the energy step.",
    }


def run_c4(args, world, rank, local, dist):
    """Config 4 across ranks: every rank partitions the whole batch's specs with
    the same longest-processing-time rule (lima_b200.partition), generates only
    its own systems and steps them in one batched engine, each block of 20 steps
    (two pair-list periods) replayed as one CUDA graph.  No collective touches the data path; the
    device-timed step time is reduced with MAX over ranks and the per-rank step
    latencies are gathered for the per-system percentiles."""
    import torch
    from lima_b200 import Engine, systems
    from lima_b200 import engine as E
    from lima_b200.partition import lpt_partition, step_cost

    specs = systems.batch_specs(args.c4_systems)
    costs = [step_cost(sp[1], int(math.ceil(sp[4] / 0.12)) ** 3) for sp in specs]
    mine = lpt_partition(costs, world)[rank]
    t0 = time.perf_counter()
    batch = [systems.batch_system(specs[i]) for i in mine]
    gen_s = time.perf_counter() - t0
    # one CUDA graph per 20 steps (two pair-list periods)
    eng = Engine(n_systems=len(batch), cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5, pme_spacing=0.12,
                 nstlist=PERIOD, dt=DT_NS, device=local, use_graphs=2)
    for i, sy in enumerate(batch):
        eng.select(i)
        eng.load(sy)
    eng.minimize(force_tol=1e5, max_steps=100)
    shape = eng.autotune(1) if args.pair_shape < 0 else args.pair_shape
    if args.pair_shape >= 0:
        eng.set_pair_shape(shape)
    eng.step(max(args.warmup, 3) * PERIOD + 1)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    n_iter = 2 * max(1, (args.steps + 2 * PERIOD - 1) // (2 * PERIOD))   # whole 20-step graph blocks
    sampler = NvmlSampler(local)
    barrier()
    sampler.start()
    eng.reset_timings()
    eng.step(n_iter * PERIOD + 1)   # the last step runs eagerly (it evaluates the energies)
    t = eng.timings()
    barrier()
    clocks = sampler.stop()
    step_s = t["step"] * 1e-6
    launches = t["kernel_launches"]
    lat = [step_s]
    for _ in range(min(20, n_iter * PERIOD)):   # per-step latencies, eager single steps
        eng.reset_timings()
        eng.step(1)
        lat.append(eng.timings()["step"] * 1e-6)
    if dist is not None:
        tt = torch.tensor([step_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        step_max = float(tt.item())
        gathered = [None] * world
        dist.all_gather_object(gathered, {"systems": len(batch), "lat": lat[1:], "atoms": sum(b.n for b in batch)})
    else:
        step_max = step_s
        gathered = [{"systems": len(batch), "lat": lat[1:], "atoms": sum(b.n for b in batch)}]
    # end to end: host states in, one batched step, host states and energies out
    n_e2e = min(args.steps, 20)
    pos_h = [torch.from_numpy(b.pos.astype(np.float64)).pin_memory().numpy() for b in batch]
    vel_h = [torch.from_numpy(b.vel.astype(np.float32)).pin_memory().numpy() for b in batch]
    for i in range(len(batch)):
        eng.select(i)
        eng.state(pos_h[i], vel_h[i])
    barrier()
    te = time.perf_counter()
    for _ in range(n_e2e):
        for i in range(len(batch)):
            eng.select(i)
            eng.set_state(pos_h[i], vel_h[i])
        eng.step(1)
        for i in range(len(batch)):
            eng.select(i)
            eng.state(pos_h[i], vel_h[i])
        eng.energies()
    barrier()
    e2e_s = (time.perf_counter() - te) / n_e2e
    if dist is not None:
        tt = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    n_atoms = sum(b.n for b in batch)
    eng.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    lat_all = sorted(x for g in gathered for x in g["lat"] for _ in range(g["systems"]))
    n_sys = len(specs)
    line = {
        "metric": "ns_per_day", "value": n_sys * ns_per_day(step_max), "unit": "ns/day", "n_gpus": world,
        "steps": n_iter * PERIOD + 1, "warmup": max(args.warmup, 3) * PERIOD, "ms_per_step": step_max * 1e3,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": {"workload": f"batch{n_sys}_water_chains_pme0.12", "systems": n_sys,
                   "atoms": sum(g["atoms"] for g in gathered), "cutoff_nm": 1.0, "pme_spacing_nm": 0.12,
                   "nstlist": PERIOD, "dt_fs": 1.0, "parallelism": f"systems partitioned over {world} ranks (LPT)",
                   "l2": "not flushed: the batch's working set exceeds L2; blocks of 20 steps replay as one CUDA graph"},
        "aggregate": "sum over systems of each system's ns/day; every system advances one step per batched step",
        "step_latency_ms_p50": 1e3 * lat_all[len(lat_all) // 2],
        "step_latency_ms_p99": 1e3 * lat_all[min(len(lat_all) - 1, int(0.99 * len(lat_all)))],
        "systems_per_rank": [g["systems"] for g in gathered], "generation_s_rank0": gen_s,
        "pair_launch_shape": shape,
        "e2e": {"value": n_sys * ns_per_day(e2e_s), "unit": "ns/day", "h2d_bytes_per_step": n_atoms * 36,
                "d2h_bytes_per_step": n_atoms * 36 + 15 * 8,
                "path": "per system lima_set_state(host), one lima_step(1), per system lima_get_state(host), "
                        "lima_get_energies (rank 0's share)"},
        "gpu_launches": launches, "clocks": clocks,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_lima(args):
    import torch
    from lima_b200 import Engine, systems
    from lima_b200 import engine as E

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    if args.workload == "c4":
        return run_c4(args, world, rank, local, dist)

    if args.profile_large:
        # profiling mode for the memory-bound kernels (binning and sort, bonded,
        # exclusion correction, integrator) on a box whose per-atom state is
        # larger than the 126 MB L2: 2.0 M atoms of water with 64 chains (bonds,
        # angles, dihedrals), PME spacing 0.12 nm; set-up plus `profile_large`
        # plain steps
        sl = systems.water_with_chains(2_000_000, 64, seed=7, name="water2M")
        el = Engine(cutoff=CUTOFF, electrostatics=E.ES_EWALD, ewald_tol=1e-5, pme_spacing=0.12, nstlist=10,
                    dt=DT_NS, device=local)
        el.load(sl)
        el.step(args.profile_large)
        torch.cuda.synchronize()
        print(json.dumps({"profile_large_steps": args.profile_large, "atoms": sl.n,
                          "bonds": len(sl.bonds), "angles": len(sl.angles), "dihedrals": len(sl.dihedrals),
                          "timings": el.timings()}), flush=True)
        el.close()
        return 0
    s = systems.config2()
    eng = Engine(cutoff=CUTOFF, electrostatics=E.ES_EWALD, ewald_tol=1e-5, nstlist=10, dt=DT_NS, device=local)
    eng.load(s, pme_grid=GRID)
    if args.profile_learned:
        # profiling mode for the learned correction: one labelled frame, one
        # epoch, then `profile_learned` steps with coarse PME + network
        lp = E.LearnedPME(eng, coarse_grid=(32, 32, 32), max_frames=1)
        eng.step(5)
        lp.collect()
        lp.train(epochs=1, batch=65536)
        lp.enable(True, check_interval=1000, tolerance=1.0)
        eng.step(args.profile_learned)
        torch.cuda.synchronize()
        print(json.dumps({"profile_learned_steps": args.profile_learned, "timings": eng.timings()}), flush=True)
        return 0
    if args.pair_shape >= 0:
        eng.set_pair_shape(args.pair_shape)
    if args.profile:
        # profiling mode: set-up plus `profile` plain steps, nothing else (for ncu)
        eng.step(args.profile)
        torch.cuda.synchronize()
        print(json.dumps({"profile_steps": args.profile, "timings": eng.timings()}), flush=True)
        return 0
    shape = eng.autotune(2) if args.pair_shape < 0 else args.pair_shape
    eng.step(max(args.warmup, 3))

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    sampler = NvmlSampler(local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    # ---- device-timed steps: each timed iteration is one pair-list period
    # (rebuild + PERIOD steps, energies on the last), eager launches, L2
    # flushed before every iteration
    n_iter = max(1, (args.steps + PERIOD - 1) // PERIOD)
    n_timed = n_iter * PERIOD
    barrier()
    sampler.start()
    eng.reset_timings()
    t_wall0 = time.perf_counter()
    dev_ms = 0.0
    launches = 0
    for k in range(n_iter):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        eng.step(PERIOD)
        t = eng.timings()
        dev_ms += t["step"] * t["steps"] / 1000.0
        launches += t["kernel_launches"]
        eng.reset_timings()
    t_wall = time.perf_counter() - t_wall0
    barrier()
    clocks = sampler.stop()
    step_s = dev_ms / 1000.0 / n_timed
    if dist is not None:
        tt = torch.tensor([step_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        step_s = float(tt.item())
    value = world * ns_per_day(step_s)

    # ---- per-phase device times (events around each phase, phases serialised),
    # the same mix of steps as the timed region: periods of PERIOD steps, one
    # energy step per period, L2 flushed before each period
    n_phase = max(1, min(n_iter, 10)) * PERIOD
    eng.phase_timing(True)
    eng.reset_timings()
    for k in range(n_phase // PERIOD):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        eng.step(PERIOD)
    ph = eng.timings()
    # phase timings accumulate per step call; step() resets nothing, so average over n_phase
    eng.phase_timing(False)
    pairs = len(eng.pairlist())
    nb_s = ph["nonbonded"] * ph["steps"] / n_phase / 1e6 if n_phase else float("nan")
    peaks = load_peaks()
    sm_max = float(peaks.get("sm_max_mhz", 1965.0))
    fp32_peak = 148 * 128 * 2 * sm_max * 1e6 / 1e12      # TFLOP/s, FMA = 2
    achieved = pairs * FLOPS_PER_PAIR / nb_s / 1e12 if nb_s > 0 else None
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    plstats = eng.pairlist_stats()
    stages = stage_rooflines({k: ph[k] for k in ("integrate", "bonded", "pme", "nblist")}, s,
                             plstats["rows_built"], hbm)
    traffic = None
    prof = os.path.join(ROOT, "profiles", "nonbonded_water100k.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        except Exception:
            traffic = None

    # ---- end to end through the C-ABI with host buffers: set_state -> step -> get_state
    n_e2e = min(args.steps, 50)
    # pinned host buffers: the caller's state goes in and comes back through them
    pos_h = torch.from_numpy(s.pos.astype(np.float64)).pin_memory().numpy()
    vel_h = torch.from_numpy(s.vel.astype(np.float32)).pin_memory().numpy()
    eng.state(pos_h, vel_h)
    barrier()
    t0 = time.perf_counter()
    for k in range(n_e2e):
        eng.set_state(pos_h, vel_h)
        eng.step(1)
        eng.state(pos_h, vel_h)
        en = eng.energies()
    barrier()
    e2e_s = (time.perf_counter() - t0) / n_e2e
    if dist is not None:
        tt = torch.tensor([e2e_s], device=f"cuda:{local}", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_s = float(tt.item())
    h2d = s.n * (3 * 8 + 3 * 4)
    d2h = s.n * (3 * 8 + 3 * 4) + 15 * 8

    # ---- the same headline workload with each pair-list period replayed as a CUDA graph
    eng_g = Engine(cutoff=CUTOFF, electrostatics=E.ES_EWALD, ewald_tol=1e-5, nstlist=10, dt=DT_NS, device=local,
                   use_graphs=1)
    eng_g.load(s, pme_grid=GRID)
    eng_g.autotune(2)
    eng_g.step(21)
    graph_step_s = _timed_steps(eng_g, max(args.steps, 21))[0][0]
    eng_g.close()

    others = other_configs(args, local) if (rank == 0 and not args.no_other_configs) else None
    if others is not None and not args.skip_learned:
        others["c3_learned_pme_coarse32"] = learned_config(args, local)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        n_cpu = 2
        t_cpu = cpu_step_time(s, n_cpu, threads)
        cpu = {"value": ns_per_day(t_cpu), "unit": "ns/day", "cores": threads, "kind": "port",
               "sample": f"{n_cpu} full MD steps of the same {s.n}-atom box on the host (oracle port: FP32 pair "
                         f"loop with {threads} threads, FP64 SPME 96^3 and bonded terms), median"}

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {
        "metric": "ns_per_day", "value": value, "unit": "ns/day", "n_gpus": world, "steps": n_timed,
        "warmup": max(args.warmup, 3), "ms_per_step": step_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "fp32", "data": "synthetic",
        "config": headline_config(s.n, world),
        "pair_launch_shape": shape,
        "pairs_per_s": world * pairs / step_s,
        "pairs_per_step": pairs,
        "pairlist": plstats,
        "wall_ms_per_step": t_wall / args.steps * 1e3,
        "phase_us": {k: ph[k] for k in ("nonbonded", "bonded", "pme", "integrate", "nblist")},
        "pme_grid_points_per_s": stages.get("pme", {}).get("grid_points_per_s"),
        "stages": stages,
        "roofline": {"kernel": "k_nonbonded (pair kernel)", "bound": "fp32", "achieved": achieved,
                     "peak": fp32_peak, "unit": "TFLOP/s",
                     "frac": achieved / fp32_peak if achieved else None, "traffic": traffic,
                     "peak_source": "nominal FP32 FMA rate at the measured max SM clock (148 SM x 128 lanes x 2 x "
                                    f"{sm_max:.0f} MHz); MEASURED_PEAKS.json holds no FP32 figure",
                     "work": f"{FLOPS_PER_PAIR} flops per in-cutoff pair x {pairs} pairs per launch"},
        "e2e": {"value": world * ns_per_day(e2e_s), "unit": "ns/day", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "path": "lima_set_state(host) -> lima_step(1) -> lima_get_state(host) + lima_get_energies"},
        "gpu_launches": launches,
        "clocks": clocks,
        "cpu_baseline": cpu,
        "graph_mode": {"ns_per_day": world * ns_per_day(graph_step_s), "ms_per_step": graph_step_s * 1e3,
                       "l2": "not flushed: each pair-list period (rebuild + 10 steps) replays as one CUDA graph"},
        "other_configs": others,
        "accuracy": accuracy_summary(),
    }
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="lima", choices=["lima", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile", type=int, default=0, help="only set up and run this many steps (ncu)")
    ap.add_argument("--pair-shape", type=int, default=-1,
                    help="launch shape of the pair kernel (0-11) instead of the autotuner's choice")
    ap.add_argument("--profile-learned", type=int, default=0,
                    help="only set up the learned correction and run this many steps with it (ncu)")
    ap.add_argument("--profile-large", type=int, default=0,
                    help="only set up a 2 M-atom water box with chains and run this many steps (ncu)")
    ap.add_argument("--no-other-configs", action="store_true")
    ap.add_argument("--skip-batch", action="store_true")
    ap.add_argument("--other-steps", type=int, default=100)
    ap.add_argument("--skip-learned", action="store_true")
    ap.add_argument("--c3-frames", type=int, default=64)
    ap.add_argument("--c3-epochs", type=int, default=20)
    ap.add_argument("--workload", default="c2", choices=["c2", "c4"],
                    help="c2: the 100k-atom water box (headline, replicas over ranks); c4: the 256-system batch "
                         "partitioned over ranks")
    ap.add_argument("--c4-systems", type=int, default=256)
    ap.add_argument("--no-cpu-other", dest="cpu_other", action="store_false",
                    help="skip the CPU baselines of the secondary workloads")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_lima(args)


if __name__ == "__main__":
    sys.exit(main())
