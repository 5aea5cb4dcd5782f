"""Generates tests/golden/ref_terms.npz: golden vectors of the reference's own
per-term device functions.

Runs oracle/_ref/ref_terms (built by `make -C oracle ref` from the reference
tree, with the reference's flags) on seeded inputs and stores inputs and
outputs.  It needs a GPU, since the reference's functions are device code:

    python tests/golden/make_ref_golden.py [out.npz]

The fixture is committed; tests/test_oracle_ref_golden.py checks the CPU
oracle against it without a GPU.  Each kind names the reference function it
evaluates (see oracle/ref_harness.cu).
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
BIN = os.path.join(ROOT, "oracle", "_ref", "ref_terms")
E_KCMOL = 96.48533212331002          # kC/mol per elementary charge (Constants.h:58)

IN_W = {"lj": 5, "lj_em": 5, "coulomb": 5, "bond": 8, "bond_em": 8, "angle": 13, "dihedral": 15,
        "improper": 14, "bspline": 1, "vvs": 11, "activate": 4, "adam": 10, "interact": 16}
OUT_W = {"lj": 4, "lj_em": 3, "coulomb": 4, "bond": 7, "bond_em": 7, "angle": 10, "dihedral": 13,
         "improper": 13, "bspline": 4, "vvs": 6, "activate": 3, "adam": 9, "interact": 1}


def run(kind, x, *params):
    x = np.ascontiguousarray(x, dtype=np.float32)
    n = x.shape[0]
    assert x.shape[1] == IN_W[kind]
    with tempfile.TemporaryDirectory() as d:
        fi, fo = os.path.join(d, "in.f32"), os.path.join(d, "out.f32")
        x.tofile(fi)
        subprocess.run([BIN, kind, str(n), fi, fo] + [str(p) for p in params], check=True)
        return np.fromfile(fo, dtype=np.float32).reshape(n, OUT_W[kind])


def unit(rng, n):
    v = rng.normal(size=(n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def chain(rng, n, lengths, angle_deg):
    """n chains of len(lengths)+1 points: consecutive bonds with the given lengths
    and bond angles drawn from angle_deg = (lo, hi)."""
    pts = [rng.uniform(0.0, 3.0, (n, 3))]
    d = unit(rng, n)
    pts.append(pts[0] + d * lengths[0])
    for L in lengths[1:]:
        # new direction at a bond angle theta to the previous bond, random azimuth
        th = np.radians(rng.uniform(*angle_deg, n))
        ref = unit(rng, n)
        perp = ref - (ref * d).sum(1, keepdims=True) * d
        perp /= np.linalg.norm(perp, axis=1, keepdims=True)
        nd = -d * np.cos(th)[:, None] + perp * np.sin(th)[:, None]
        pts.append(pts[-1] + nd * L)
        d = nd
    return np.stack(pts, 1)


def main(out_path):
    rng = np.random.default_rng(20241203)
    out = {}

    n = 2000                                                     # LJ::calcLJForceOptim
    r = rng.uniform(0.2, 1.2, n)
    x = np.concatenate([unit(rng, n) * r[:, None], rng.uniform(0.25, 0.45, (n, 1)),
                        rng.uniform(50.0, 2000.0, (n, 1))], 1)
    out["lj_in"], out["lj_out"] = x.astype(np.float32), run("lj", x)

    n = 500                                                      # EM variant: clamp + activation
    r = rng.uniform(0.105, 1.0, n)
    x = np.concatenate([unit(rng, n) * r[:, None], rng.uniform(0.25, 0.4, (n, 1)),
                        rng.uniform(100.0, 1000.0, (n, 1))], 1)
    out["lj_em_in"], out["lj_em_out"] = x.astype(np.float32), run("lj_em", x)

    for tag, kappa in (("coulomb_plain", 0.0), ("coulomb_ewald", 2.5)):   # kappa = 3/rc at rc 1.2
        n = 2000
        r = rng.uniform(0.105, 1.2, n)
        x = np.concatenate([rng.uniform(-1.0, 1.0, (n, 2)) * E_KCMOL, unit(rng, n) * r[:, None]], 1)
        out[tag + "_in"], out[tag + "_out"] = x.astype(np.float32), run("coulomb", x, kappa, 1.2, 10)
        out[tag + "_kappa"] = np.float64(kappa)

    for kind, nn in (("bond", 500), ("bond_em", 200)):           # calcSinglebondForces
        p = chain(rng, nn, [1.0], (0, 1))
        p[:, 1] = p[:, 0] + (p[:, 1] - p[:, 0]) * rng.uniform(0.08, 0.6 if kind == "bond_em" else 0.2, (nn, 1))
        x = np.concatenate([p.reshape(nn, 6), rng.uniform(0.09, 0.16, (nn, 1)),
                            rng.uniform(1e5, 4e5, (nn, 1))], 1)
        out[kind + "_in"], out[kind + "_out"] = x.astype(np.float32), run(kind, x)

    n = 1000                                                     # calcAnglebondForces (+ Urey-Bradley)
    p = chain(rng, n, rng.uniform(0.09, 0.16, 2), (40.0, 175.0))
    ub = rng.random(n) < 0.5
    x = np.concatenate([p.reshape(n, 9), np.radians(rng.uniform(95.0, 125.0, (n, 1))),
                        rng.uniform(200.0, 800.0, (n, 1)) * 1e3,
                        np.where(ub, rng.uniform(0.2, 0.26, n), 0.0)[:, None],
                        np.where(ub, rng.uniform(1e4, 5e4, n), 0.0)[:, None] * 1e3], 1)
    out["angle_in"], out["angle_out"] = x.astype(np.float32), run("angle", x)

    n = 2000                                                     # calcDihedralbondForces
    p = chain(rng, n, [0.153, 0.153, 0.153], (100.0, 125.0))
    # a quarter near the cis/trans planes, where |sin phi| < 0.1 picks the other gradient branch
    k = n // 4
    flat = chain(rng, k, [0.153, 0.153, 0.153], (100.0, 125.0))
    b2 = flat[:, 2] - flat[:, 1]
    b2 /= np.linalg.norm(b2, axis=1, keepdims=True)
    # rotate the last atom about the middle bond into the plane of the first three (+ small jitter)
    b1 = flat[:, 1] - flat[:, 0]
    nrm = np.cross(b1, b2)
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    v = flat[:, 3] - flat[:, 2]
    comp = (v * nrm).sum(1, keepdims=True)
    flat[:, 3] = flat[:, 3] - comp * nrm * rng.uniform(0.9, 1.1, (k, 1))
    p[:k] = flat
    x = np.concatenate([p.reshape(n, 12), np.radians(rng.choice([0.0, 180.0, 60.0], (n, 1))),
                        rng.uniform(0.3, 3.0, (n, 1)) * 1e3, rng.choice([1.0, 2.0, 3.0], (n, 1))], 1)
    out["dihedral_in"], out["dihedral_out"] = x.astype(np.float32), run("dihedral", x)

    n = 1000                                                     # calcImproperdihedralbondForces
    c = rng.uniform(0.0, 3.0, (n, 3))
    pts = [c]
    for _ in range(3):
        pts.append(c + unit(rng, n) * rng.uniform(0.1, 0.15, (n, 1)))
    p = np.stack([pts[1], pts[0], pts[2], pts[3]], 1)            # i out of plane of (j, k, l) as in the reference
    x = np.concatenate([p.reshape(n, 12), np.radians(rng.uniform(-20.0, 20.0, (n, 1))),
                        rng.uniform(100.0, 800.0, (n, 1)) * 1e3], 1)
    out["improper_in"], out["improper_out"] = x.astype(np.float32), run("improper", x)

    x = rng.uniform(0.0, 1.0, (200, 1))                          # LAL::CalcBspline
    x[:4, 0] = [0.0, 0.25, 0.5, 0.999]
    out["bspline_in"], out["bspline_out"] = x.astype(np.float32), run("bspline", x)

    n = 500                                                      # integratePositionVVS / integrateVelocityVVS
    m = rng.choice([0.001008, 0.015999, 0.012011], (n, 1))
    x = np.concatenate([rng.normal(0.0, 500.0, (n, 3)), rng.normal(0.0, 3e5, (n, 6)), m,
                        np.full((n, 1), 1e-6)], 1)
    o = run("vvs", x)
    out["vvs_in"], out["vvs_out"] = x.astype(np.float32), o
    out["vvs_step_int"] = o[:, :3].view(np.int32).copy()

    n = 500                                                      # ForceActivationFunction
    f = unit(rng, n) * (10.0 ** rng.uniform(2.0, 10.0, (n, 1)))
    x = np.concatenate([f, rng.choice([1.0, 100.0], (n, 1))], 1)
    out["activate_in"], out["activate_out"] = x.astype(np.float32), run("activate", x)

    n = 500                                                      # IntegratePositionADAM
    f = unit(rng, n) * (10.0 ** rng.uniform(0.0, 7.0, (n, 1)))
    m1 = rng.normal(0.0, 1e-3, (n, 3))
    m2 = rng.uniform(0.0, 1e-6, (n, 3))
    x = np.concatenate([f, m1, m2, rng.integers(1, 200, (n, 1))], 1)
    o = run("adam", x)
    out["adam_in"], out["adam_out"] = x.astype(np.float32), o
    out["adam_step_int"] = o[:, :3].view(np.int32).copy()

    n = 4000                                                     # canCompoundsInteract (box 10 nm, rc 1.0)
    L = 10.0
    kl = rng.uniform(0.0, L, (n, 6))
    kr = (kl + rng.normal(0.0, 1.6, (n, 6))) % L
    x = np.concatenate([kl, kr, rng.uniform(0.0, 0.6, (n, 4))], 1)
    o = run("interact", x, 0.0, 1.0, 10)
    out["interact_in"], out["interact_out"] = x.astype(np.float32), o
    out["interact_box"], out["interact_cutoff"] = np.float64(L), np.float64(1.0)

    for tag, K, Lb, kap in (("green10", 10, 1.0, 2.5), ("green30", 30, 3.0, 3.0 / 1.2)):   # Green function
        with tempfile.TemporaryDirectory() as d:
            fo = os.path.join(d, "g.f32")
            subprocess.run([BIN, "green", str(K), "-", fo, str(Lb), str(kap)], check=True)
            out[tag] = np.fromfile(fo, dtype=np.float32)
        out[tag + "_params"] = np.array([K, Lb, kap], np.float64)

    np.savez_compressed(out_path, **out)
    print("wrote", out_path, sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                             "ref_terms.npz"))
