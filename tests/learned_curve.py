"""Held-out error of the learned coarse-grid PME correction against the number
of training frames (one B200; not collected by pytest).

    python tests/learned_curve.py profiles [--frames 16,64,256,1000,2000]

For each frame count F a fresh engine continues one trajectory of the
100,200-atom water box (cutoff 1.0 nm, full grid 96^3, coarse grid 32^3):
F frames 20 steps apart, each labelled by the full grid; the network is trained
on the GPU (Adam, lr 1e-3, 65,536-row batches, max(3, 1280/F) epochs), the
engine steps 100 further steps and the relative RMSE of the reciprocal force
against the full grid is measured there, for the coarse grid alone and with
the network.  Writes learned_pme_curve.json and .md into the output folder.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from lima_b200 import Engine, systems  # noqa: E402
from lima_b200 import engine as E  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("out")
    ap.add_argument("--frames", default="16,64,256,1000,2000")
    a = ap.parse_args()
    counts = [int(v) for v in a.frames.split(",")]
    s = systems.config2()
    rows = []
    for F in counts:
        eng = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5, nstlist=10, dt=1e-6)
        eng.load(s, pme_grid=(96, 96, 96))
        lp = E.LearnedPME(eng, coarse_grid=(32, 32, 32), max_frames=F)
        eng.step(20)
        t0 = time.perf_counter()
        for _ in range(F):
            eng.step(20)
            lp.collect()
        t_collect = time.perf_counter() - t0
        epochs = max(3, math.ceil(1280 / F))
        t0 = time.perf_counter()
        loss = lp.train(epochs=epochs, batch=65536, lr=1e-3, seed=1)
        t_train = time.perf_counter() - t0
        eng.step(100)
        coarse, learned = lp.eval()
        pos, vel = eng.state()
        s = dataclasses.replace(s, pos=pos, vel=vel)     # the next count continues the trajectory
        eng.close()
        r = {"frames": F, "epochs": epochs, "rows_seen": F * s.n * epochs, "final_train_loss": loss,
             "collect_s": t_collect, "train_s": t_train, "heldout_rel_rmse_coarse": coarse,
             "heldout_rel_rmse_learned": learned, "gain": coarse / learned if learned > 0 else None}
        print(json.dumps(r), flush=True)
        rows.append(r)
    os.makedirs(a.out, exist_ok=True)
    with open(os.path.join(a.out, "learned_pme_curve.json"), "w") as f:
        json.dump(rows, f, indent=1)
    md = ["# Learned coarse-grid PME: held-out error against training frames", "",
          "Command (one B200):", "", f"    python tests/learned_curve.py profiles --frames {a.frames}", "",
          "100,200-atom water box, full grid 96^3, coarse grid 32^3; frames 20 steps apart along one trajectory; "
          "error measured 100 steps after the last frame (relative RMSE of the reciprocal force against the full "
          "grid).  The bound for using the correction in stepping is 1e-3.", "",
          "| frames | epochs | rows seen | train loss | collect [s] | train [s] | coarse grid alone | with network | gain |",
          "|---:|---:|---:|---:|---:|---:|---:|---:|---:|"]
    for r in rows:
        md.append(f"| {r['frames']} | {r['epochs']} | {r['rows_seen']:.3g} | {r['final_train_loss']:.4g} | "
                  f"{r['collect_s']:.1f} | {r['train_s']:.1f} | {r['heldout_rel_rmse_coarse']:.4f} | "
                  f"{r['heldout_rel_rmse_learned']:.4f} | {r['gain']:.2f}x |")
    with open(os.path.join(a.out, "learned_pme_curve.md"), "w") as f:
        f.write("\n".join(md) + "\n")
    print("\n".join(md))


if __name__ == "__main__":
    main()
