"""Per-configuration accuracy of the CUDA path against the FP64 oracle.

For each benchmark configuration this runs the engine (through the C-ABI),
takes seeded frames along its trajectory and compares the engine's forces and
energy terms on each frame with the FP64 oracle's on the same positions:
max and RMS force error, relative RMS, and the relative error of every energy
term.  A separate constant-energy run with the reference's velocity-Verlet
integrator measures the total-energy drift per ns and the reference's own
stability statistics (variance coefficient and energy gradient of its
analyser, code/LIMA_MD/src/Analyzer.cu:216-345, restated in
lima_b200.trajectory).

Needs a GPU (test tooling; the oracle is the checker):

    python tests/accuracy_report.py OUT_DIR [--c2-frames 100] [--quick]

writes OUT_DIR/accuracy_configs.json and OUT_DIR/accuracy_configs.md.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from lima_b200 import Engine, systems, trajectory  # noqa: E402
from lima_b200 import engine as E  # noqa: E402
from oracle import oracle as O  # noqa: E402
from tests._ref import kappa_from_tol, oracle_total  # noqa: E402

DT = 1e-6


def fft_friendly(n):
    """The smallest m >= max(n, 4) whose only prime factors are 2, 3 and 5."""
    m = max(n, 4)
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


def frame_errors(eng, s, rc, es_mode, kappa, grid):
    """Engine vs oracle on the engine's current positions."""
    eng.compute_forces(energy=True)
    f = eng.forces()
    en = eng.energies()
    pos, _ = eng.state()
    sf = dataclasses.replace(s, pos=pos)
    fr, er = oracle_total(O, sf, rc, es_mode, kappa, grid)
    df = np.linalg.norm(f - fr, axis=1)
    rms_ref = float(np.sqrt((fr ** 2).sum(1).mean()))
    out = {"max_abs_err": float(df.max()), "rms_err": float(np.sqrt((df ** 2).mean())), "rms_force": rms_ref}
    out["rel_rms"] = out["rms_err"] / rms_ref
    out["max_err_over_rms_force"] = out["max_abs_err"] / rms_ref
    if es_mode == 1:
        # plain cutoff Coulomb: a pair within 1e-5 nm of the cutoff is in or out
        # by the rounding of r^2 (FP32 here, FP64 in the oracle) and moves its
        # atoms' forces by a whole k q q / rc^2; the error over the other atoms.
        # Band pairs lie on both sides of the cutoff, so they are taken from the
        # oracle's pair set within rc + band.
        band = 1e-5
        near, _, _ = O.pairset(sf.pos, sf.box, sf.exclusions(), rc + band)
        d = sf.pos[near[:, 0]] - sf.pos[near[:, 1]]
        d -= sf.box * np.round(d / sf.box)
        in_band = np.abs(np.linalg.norm(d, axis=1) - rc) < band
        touched = np.zeros(sf.n, bool)
        touched[near[in_band].ravel()] = True
        keep = ~touched
        out["band_atoms"] = int(touched.sum())
        out["rel_rms_outside_band"] = float(np.sqrt((df[keep] ** 2).mean()) /
                                            np.sqrt((fr[keep] ** 2).sum(1).mean()))
    terms = {}
    # a term that vanishes (a bond energy of waters at their template geometry)
    # is measured against 1e-7 of the summed magnitude of all terms
    floor = 1e-7 * sum(abs(v) for v in er.values())
    for k, b in er.items():
        a = en[k]
        rel = 0.0 if a == b else abs(a - b) / max(abs(b), floor)
        terms[k] = {"engine": a, "oracle": b, "rel": rel}
    pot_ref = sum(er.values())
    pot_eng = sum(en[k] for k in er)
    terms["potential"] = {"engine": pot_eng, "oracle": pot_ref, "rel": abs(pot_eng - pot_ref) / abs(pot_ref)}
    out["energy"] = terms
    return out


def summarise(frames):
    keys = ["max_abs_err", "rms_err", "rms_force", "rel_rms", "max_err_over_rms_force"]
    keys += [k for k in ("band_atoms", "rel_rms_outside_band") if k in frames[0]]
    s = {k: {"max": float(max(f[k] for f in frames)), "mean": float(np.mean([f[k] for f in frames]))}
         for k in keys}
    terms = frames[0]["energy"].keys()
    s["energy_rel"] = {t: {"max": float(max(f["energy"][t]["rel"] for f in frames)),
                           "mean": float(np.mean([f["energy"][t]["rel"] for f in frames]))} for t in terms}
    s["frames"] = len(frames)
    return s


def equilibrate(make_engine, s, grid, em_steps, md_steps):
    """The reference's energy minimisation, fresh Maxwell-Boltzmann velocities at
    300 K, then md_steps of MD with the reference's thermostat measuring and
    rescaling every step (clamp 1 -+ 0.001 per measurement) towards 300 K."""
    eng = make_engine(apply_thermostat=1, thermostat_interval=1, target_temperature=300.0)
    eng.load(s, pme_grid=grid)
    if em_steps:
        eng.minimize(force_tol=1e4, max_steps=em_steps)
    p, _ = eng.state()
    rng = np.random.default_rng(11)
    v = systems.maxwell_boltzmann(rng, s.mass, 300.0)
    eng.set_state(p, v)
    eng.step(md_steps)
    p, v = eng.state()
    temp = eng.thermostat()["temperature"]
    eng.close()
    return dataclasses.replace(s, pos=p, vel=v), temp


def drift(make_engine, s, grid, steps, dt, every=10, relax=200):
    """Constant-energy run with the reference's velocity Verlet from an
    equilibrated state: `relax` steps, then the total energy every `every`
    steps over `steps` steps: least-squares slope per ns, the analyser's
    statistics, and the status bits the run raised."""
    eng = make_engine(integrator=1, dt=dt)    # LIMA_INTEGRATOR_VV
    eng.load(s, pme_grid=grid)
    eng.step(relax)
    status = eng.status()
    pot, kin, t = [], [], []
    for k in range(steps // every):
        eng.step(every)
        status |= eng.status()
        en = eng.energies()
        pot.append(en["potential"])
        kin.append(en["kinetic"])
        t.append((k + 1) * every * dt)
    eng.close()
    pot, kin, t = np.array(pot), np.array(kin), np.array(t)
    tot = pot + kin
    slope = float(np.polyfit(t, tot, 1)[0])              # J/mol per ns
    an = trajectory.analyze_energy(pot, kin)
    return {"steps": steps, "dt_fs": dt * 1e6, "samples": len(tot), "mean_total_j_mol": float(tot.mean()),
            "mean_kinetic_j_mol": float(kin.mean()),
            "temperature_k": float(2.0 * kin.mean() / (3.0 * s.n - 3.0) / systems.KB_J_MOL_K),
            "drift_j_mol_per_ns": slope, "drift_kj_mol_per_ns_per_atom": slope / 1e3 / s.n,
            "drift_rel_per_ns": slope / abs(float(tot.mean())),
            "drift_per_ns_over_kinetic": slope / float(kin.mean()),
            "total_std_j_mol": float(tot.std()),
            "variance_coefficient": float(an.variance_coefficient),
            "energy_gradient": float(an.energy_gradient),
            "status_bits": int(status)}


def run_config(name, s, rc, es_mode, kappa, grid, frames, every, drift_steps, prep_min=0, kw=None, eq_steps=2000):
    kw = dict(kw or {})

    def make_engine(**extra):
        args = dict(cutoff=rc, electrostatics=es_mode, nstlist=10, dt=DT)
        args.update(kw)
        args.update(extra)
        if es_mode == E.ES_EWALD:
            args["ewald_kappa"] = kappa
        return Engine(**args)

    t0 = time.time()
    s, t_eq = equilibrate(make_engine, s, grid, prep_min, eq_steps)
    eng = make_engine()
    eng.load(s, pme_grid=grid)
    out_frames = []
    status = 0
    for k in range(frames):
        if k:
            eng.step(every)
            status |= eng.status()
        out_frames.append(frame_errors(eng, s, rc, es_mode if es_mode != E.ES_EWALD else 2, kappa, grid))
    eng.close()
    res = {"config": name, "atoms": s.n, "cutoff_nm": rc, "pme_grid": list(grid) if grid else None,
           "kappa": kappa, "frame_interval_steps": every,
           "prep": {"em_steps": prep_min, "thermostat_md_steps": eq_steps, "temperature_k": t_eq},
           "frames_status_bits": int(status), "summary": summarise(out_frames)}
    if drift_steps:
        res["drift"] = [drift(make_engine, s, grid, drift_steps, DT),
                        drift(make_engine, s, grid, 2 * drift_steps, 0.5 * DT)]
    res["seconds"] = time.time() - t0
    return res


def markdown(results, cmd):
    lines = ["# Accuracy against the FP64 oracle, per configuration", "",
             "Command (one B200):", "", "    " + cmd, "",
             "Forces: per frame, |F_engine - F_oracle| per atom; `max` over atoms, `rms` over atoms, relative RMS = "
             "rms error / rms force.  Energies: |E_engine - E_oracle| / |E_oracle| per term.  Drift: least-squares "
             "slope of the total energy of a constant-energy velocity-Verlet run (no thermostat), and the "
             "reference analyser's variance coefficient and energy gradient over the same samples.", "",
             "| config | atoms | frames | max force err [J/mol/nm] | RMS force err | rel RMS (max over frames) | "
             "max err / RMS force | worst energy term (rel) | potential (rel) |",
             "|---|---:|---:|---:|---:|---:|---:|---|---:|"]
    for r in results:
        sm = r["summary"]
        worst = max(((k, v["max"]) for k, v in sm["energy_rel"].items() if k != "potential"), key=lambda x: x[1])
        lines.append(f"| {r['config']} | {r['atoms']} | {sm['frames']} | {sm['max_abs_err']['max']:.3e} | "
                     f"{sm['rms_err']['max']:.3e} | {sm['rel_rms']['max']:.2e} | "
                     f"{sm['max_err_over_rms_force']['max']:.2e} | {worst[0]} {worst[1]:.2e} | "
                     f"{sm['energy_rel']['potential']['max']:.2e} |")
    lines += ["", "Every configuration is first prepared: the reference's energy minimisation, fresh velocities at "
              "300 K and MD with the reference's thermostat (rescaling every step); the frames then follow the "
              "constant-energy trajectory from there.", "",
              "| config | EM steps | thermostatted MD steps | T after preparation [K] | status bits over the frames |",
              "|---|---:|---:|---:|---:|"]
    for r in results:
        pr = r["prep"]
        lines.append(f"| {r['config']} | {pr['em_steps']} | {pr['thermostat_md_steps']} | {pr['temperature_k']:.0f} | "
                     f"{r['frames_status_bits']:#x} |")
    lines += ["", "| config | energy term | rel err (max over frames) | rel err (mean) |", "|---|---|---:|---:|"]
    for r in results:
        for k, v in r["summary"]["energy_rel"].items():
            lines.append(f"| {r['config']} | {k} | {v['max']:.2e} | {v['mean']:.2e} |")
    lines += ["", "| config | dt [fs] | NVE steps | T [K] | drift [J/mol/ns] | drift [kJ/mol/ns/atom] | "
              "drift per ns / kinetic | variance coeff. | energy gradient | status bits |",
              "|---|---:|---:|---:|---:|---:|---:|---:|---:|---:|"]
    for r in results:
        for d in r.get("drift") or []:
            lines.append(f"| {r['config']} | {d['dt_fs']:g} | {d['steps']} | {d['temperature_k']:.0f} | "
                         f"{d['drift_j_mol_per_ns']:.4g} | {d['drift_kj_mol_per_ns_per_atom']:.3g} | "
                         f"{d['drift_per_ns_over_kinetic']:.3g} | {d['variance_coefficient']:.3g} | "
                         f"{d['energy_gradient']:.3g} | {d['status_bits']:#x} |")
    for r in results:
        sm = r["summary"]
        if "rel_rms_outside_band" in sm:
            lines += ["", f"{r['config']}: relative RMS force error over the atoms without a pair within 1e-5 nm of "
                          f"the cutoff: {sm['rel_rms_outside_band']['max']:.2e} (max over frames); "
                          f"{sm['band_atoms']['max']:.0f} atoms at most touched such a pair in a frame."]
    return "\n".join(lines) + "\n"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--c2-frames", type=int, default=100)
    ap.add_argument("--quick", action="store_true", help="few frames and short drift runs")
    ap.add_argument("--only", default="", help="comma-separated config name prefixes to keep in the report")
    a = ap.parse_args()
    q = a.quick
    res = []
    keep = tuple(a.only.split(",")) if a.only else ("",)

    def add(name, *args, **kw):
        if name.startswith(keep):
            res.append(run_config(name, *args, **kw))

    kap1 = kappa_from_tol(1.2, 1e-5)
    kap2 = kappa_from_tol(1.0, 1e-5)
    add("C0 water1k cutoff 1.2", systems.config0(), 1.2, E.ES_CUTOFF, 0.0, None,
        3 if q else 10, 100, 500 if q else 4000, prep_min=300)
    # plain truncated Coulomb: a pair the list missed (an atom that moved more
    # than half the buffer since the build) would cost the whole force jump
    # q_i q_j k_e / rc^2 at the cutoff, so C0 also runs with a buffer that no
    # atom outruns in ten steps; its errors match the 0.1 nm run's
    add("C0 water1k cutoff 1.2, skin 0.25", systems.config0(), 1.2, E.ES_CUTOFF, 0.0, None,
        3 if q else 10, 100, 500 if q else 4000, prep_min=300, kw={"skin": 0.25})
    add("C1 chains+water PME 48x48x80", systems.config1(), 1.2, E.ES_EWALD, kap1, (48, 48, 80),
        2 if q else 10, 100, 500 if q else 4000, prep_min=300)
    add("C2 water100k PME 96^3", systems.config2(), 1.0, E.ES_EWALD, kap2, (96, 96, 96),
        3 if q else a.c2_frames, 20, 500 if q else 4000, prep_min=300)
    batch = systems.batch_systems(4 if q else 8, seed=20241203)
    for i, sb in enumerate(batch):
        # the grid the engine derives from a 0.12 nm spacing (api.cu fft_friendly)
        g = tuple(fft_friendly(int(np.ceil(L / 0.12))) for L in sb.box)
        add(f"C4 system {i} ({sb.n} atoms, PME {g[0]}x{g[1]}x{g[2]})", sb, 1.0, E.ES_EWALD,
            kap2, g, 1, 20, 0, prep_min=100, eq_steps=500)
    os.makedirs(a.out, exist_ok=True)
    with open(os.path.join(a.out, "accuracy_configs.json"), "w") as f:
        json.dump(res, f, indent=1)
    cmd = "python tests/accuracy_report.py profiles" + (" --quick" if q else f" --c2-frames {a.c2_frames}")
    with open(os.path.join(a.out, "accuracy_configs.md"), "w") as f:
        f.write(markdown(res, cmd))
    print(markdown(res, cmd))


if __name__ == "__main__":
    main()
