"""The CPU oracle against golden vectors of the reference's own device functions.

tests/golden/ref_terms.npz holds inputs and outputs of the reference's per-term
functions, compiled from the reference tree with its own flags (fast-math FP32)
and run on a GPU by tests/golden/make_ref_golden.py.  Each test evaluates the
same inputs through the oracle's per-term entry points, which run the very
functions the oracle's system-level calls use, and bounds the difference.

Tolerances: the reference computes in FP32 with -use_fast_math (approximate
reciprocal, square root and transcendental functions), the oracle in FP64, so
the bars are relative RMS differences of a few 1e-6 (the measured differences are
1e-7 to 1.5e-6: FP32 rounding of the reference's side) and state which reference
quirk they absorb where one matters.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_terms.npz")
pytestmark = pytest.mark.skipif(not os.path.exists(GOLD), reason="golden vectors not generated")


@pytest.fixture(scope="module")
def g():
    return dict(np.load(GOLD))


def rel_rms(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def rel_max(a, b, floor):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def test_lj_pair(g):
    """LJ::calcLJForceOptim (LennardJonesInteractions.cuh:74-108), x24 as its callers apply."""
    x, ref = g["lj_in"].astype(np.float64), g["lj_out"].astype(np.float64)
    f, elj, _ = O.pair_terms(x[:, :3], x[:, 3], x[:, 4], np.zeros(len(x)), 0)
    # the oracle returns the force on i for diff = r_j - r_i, as the reference does
    assert rel_rms(f, ref[:, :3]) < 1e-6
    assert rel_max(f, ref[:, :3], 1e-3 * np.abs(ref[:, :3]).max()) < 1e-4
    # the reference stores half the pair energy per atom (its 0.5 split)
    assert rel_rms(0.5 * elj, ref[:, 3]) < 1e-6


def test_lj_pair_energy_minimisation_variant(g):
    """The EM variant: scalar clamp at +-1e20 and ForceActivationFunction(., 100)."""
    x, ref = g["lj_em_in"].astype(np.float64), g["lj_em_out"].astype(np.float64)
    f, _, _ = O.pair_terms(x[:, :3], x[:, 3], x[:, 4], np.zeros(len(x)), 0, em=True)
    assert rel_rms(f, ref) < 5e-6
    assert rel_max(f, ref, 1e-3 * np.abs(ref).max()) < 1e-4
    # the saturated pairs sit at the activation's bound, 24 x 1e8 J/mol/nm
    sat = np.linalg.norm(ref, axis=1) > 0.99 * 2.4e9
    assert sat.sum() > 10


@pytest.mark.parametrize("tag", ["coulomb_plain", "coulomb_ewald"])
def test_coulomb_pair(g, tag):
    """CalcCoulumbForce_optim / CalcCoulumbPotential_optim (DeviceAlgorithmsPrivate.cuh:38-95).
    The reference leaves k_e to its callers (LennardJonesInteractions.cuh:195-203);
    its erfc term is always on, kappa = 0 making it plain Coulomb."""
    x, ref = g[tag + "_in"].astype(np.float64), g[tag + "_out"].astype(np.float64)
    kappa = float(g[tag + "_kappa"])
    ke = O.coulomb_constant()
    qq = (x[:, 0].astype(np.float32) * x[:, 1].astype(np.float32)).astype(np.float64)
    # reference: force on self = qq (r_self - r_other)/r^3 scalar, called with -diff
    diff = x[:, 2:5]                       # here r_other - r_self = -(argument)
    f, _, ec = O.pair_terms(-diff, np.ones(len(x)), np.zeros(len(x)), qq, 2, kappa)
    assert rel_rms(f / ke, ref[:, :3]) < 1e-6
    assert rel_rms(ec / ke, ref[:, 3]) < 1e-6


@pytest.mark.parametrize("kind", ["bond", "bond_em"])
def test_bond(g, kind):
    """calcSinglebondForces (ForceComputations.cuh:17-51).  The EM variant caps the
    force at the bond stretched to 2 b0 beyond rest (the energy is not capped)."""
    x, ref = g[kind + "_in"].astype(np.float64), g[kind + "_out"].astype(np.float64)
    f, e = O.bonded_terms("bond", x[:, :6], x[:, 6:8])
    f = f.reshape(len(x), 6)
    if kind == "bond_em":
        d = np.linalg.norm(x[:, :3] - x[:, 3:6], axis=1)
        capped = (d - x[:, 6]) > 2 * x[:, 6]
        assert capped.sum() > 5
        u = (x[:, :3] - x[:, 3:6]) / d[:, None]
        fc = -x[:, 7:8] * 2 * x[:, 6:7] * u
        f[capped] = np.concatenate([fc, -fc], 1)[capped]
    assert rel_rms(f, ref[:, :6]) < 1e-6
    assert rel_rms(e, ref[:, 6]) < 1e-6


def test_angle_urey_bradley(g):
    """calcAnglebondForces (ForceComputations.cuh:53-115)."""
    x, ref = g["angle_in"].astype(np.float64), g["angle_out"].astype(np.float64)
    f, e = O.bonded_terms("angle", x[:, :9], x[:, 9:13])
    assert rel_rms(f.reshape(len(x), 9), ref[:, :9]) < 2e-6
    assert rel_rms(e, ref[:, 9]) < 2e-6


def test_dihedral_both_gradient_branches(g):
    """calcDihedralbondForces (ForceComputations.cuh:119-210), including the
    |sin phi| <= 0.1 branch."""
    x, ref = g["dihedral_in"].astype(np.float64), g["dihedral_out"].astype(np.float64)
    f, e = O.bonded_terms("dihedral", x[:, :12], x[:, 12:15])
    f = f.reshape(len(x), 12)
    p = x[:, :12].reshape(-1, 4, 3)
    b1, b2, b3 = p[:, 1] - p[:, 0], p[:, 2] - p[:, 1], p[:, 3] - p[:, 2]
    A, B = np.cross(b1, b2), np.cross(b2, b3)
    C = np.cross(b2, A)
    sphi = (C * B).sum(1) / np.linalg.norm(C, axis=1) / np.linalg.norm(B, axis=1)
    small = np.abs(sphi) <= 0.1
    assert small.sum() > 100 and (~small).sum() > 100
    # per-sample relative error of the force vector (quadruple of atoms)
    err = np.linalg.norm(f - ref[:, :12], axis=1) / np.maximum(np.linalg.norm(ref[:, :12], axis=1), 1e-3)
    assert np.median(err[~small]) < 1e-5 and np.median(err[small]) < 1e-4
    assert rel_rms(f[~small], ref[~small, :12]) < 3e-6
    assert rel_rms(f[small], ref[small, :12]) < 3e-6
    assert rel_rms(e, ref[:, 12]) < 2e-6


def test_improper(g):
    """calcImproperdihedralbondForces (ForceComputations.cuh:214-264)."""
    x, ref = g["improper_in"].astype(np.float64), g["improper_out"].astype(np.float64)
    f, e = O.bonded_terms("improper", x[:, :12], x[:, 12:14])
    assert rel_rms(f.reshape(len(x), 12), ref[:, :12]) < 4e-6
    assert rel_rms(e, ref[:, 12]) < 6e-6


def test_bspline_weights(g):
    """LAL::CalcBspline (DeviceAlgorithmsPrivate.cuh:7-30)."""
    w = O.bspline4(g["bspline_in"].astype(np.float64)[:, 0])
    assert np.abs(w - g["bspline_out"]).max() < 1e-6


def test_velocity_verlet_step(g):
    """integratePositionVVS / integrateVelocityVVS (EngineUtils.cuh:31-41): the
    position step is truncated to the reference's 1e-8 nm integer coordinate."""
    x = g["vvs_in"].astype(np.float64)
    step_ref = g["vvs_step_int"].astype(np.float64) * 1e-8
    v_ref = g["vvs_out"][:, 3:6].astype(np.float64)
    n = len(x)
    pos = np.zeros((n, 3))
    vel = x[:, 0:3].copy()
    fprev = x[:, 3:6].copy()
    O.integrate(pos, vel, fprev, x[:, 6:9], x[:, 9], float(x[0, 10]), 1)
    # one 1e-8 nm unit of truncation, plus FP32 rounding of the step
    assert np.abs(step_ref - pos).max() < 1.01e-8 + 1e-6 * np.abs(pos).max()
    assert rel_rms(vel, v_ref) < 1e-6


def test_force_activation(g):
    """ForceActivationFunction (EngineUtils.cuh:112-140)."""
    x = g["activate_in"].astype(np.float64)
    out = np.stack([O.force_activation(x[i, :3], x[i, 3])[0] for i in range(len(x))])
    assert rel_max(out, g["activate_out"], 1e-3 * np.abs(g["activate_out"]).max()) < 1e-5


def test_adam_move(g):
    """IntegratePositionADAM (EngineUtils.cuh:44-72)."""
    x = g["adam_in"].astype(np.float64)
    d, m1, m2 = O.adam(x[:, :3], x[:, 3:6], x[:, 6:9], x[:, 9].astype(np.int32))
    out = g["adam_out"].astype(np.float64)
    assert rel_rms(m1, out[:, 3:6]) < 1e-6
    assert rel_rms(m2, out[:, 6:9]) < 1e-5
    step_ref = g["adam_step_int"].astype(np.float64) * 1e-8
    assert np.abs(d - step_ref).max() < 1.01e-8 + 1e-5 * np.abs(d).max()


def test_compound_neighbour_rule(g):
    """canCompoundsInteract (Neighborlists.cuh:64-79): every decision identical."""
    x = g["interact_in"].astype(np.float64)
    got = O.compounds_interact(x[:, 0:6], x[:, 6:12], x[:, 12:14], x[:, 14:16], float(g["interact_box"]),
                               float(g["interact_cutoff"]))
    ref = g["interact_out"][:, 0] > 0.5
    assert 0.2 < ref.mean() < 0.8
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("tag", ["green10", "green30"])
def test_reference_influence_function(g, tag):
    """PrecomputeGreensFunctionKernel (PME.cuh:434-495): FP64 arithmetic stored as FP32."""
    K, L, kappa = g[tag + "_params"]
    got = O.ref_green(int(K), L, kappa)
    ref = g[tag].astype(np.float64)
    assert rel_max(got, ref, 1e-6 * np.abs(ref).max()) < 1e-6
