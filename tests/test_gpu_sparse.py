"""Sparse, tiny and inhomogeneous systems through the C-ABI against the FP64 CPU oracle.

A few ions in a 3 nm box (the reference's electrostatics tests use such
systems, ElectrostaticsTests.h:300-396): the column grid has one column and all
atoms share one 8-atom cluster, so a pair that meets across the periodic
boundary is a pair of the cluster with its own periodic image.  Pair sets,
forces and energies must match the oracle as for dense systems.
"""
import numpy as np
import pytest

from lima_b200 import Engine, systems
from lima_b200 import engine as E
from tests._ref import kappa_from_tol, oracle_total, rel_rms

pytestmark = pytest.mark.gpu

L = 3.0
RC = 1.0
GRID = (30, 30, 30)

CASES = {
    # one ion: Ewald self energy and the lone ion's reciprocal energy, no pairs
    "one_ion": ([(1.5, 1.5, 1.5)], [1.0]),
    # two ions 0.35 nm apart inside the box (where the pair kernel's erfc
    # approximation, 1.5e-7 absolute, is also within 1e-6 relative)
    "two_ions": ([(1.30, 1.5, 1.5), (1.65, 1.5, 1.5)], [1.0, -1.0]),
    # three pairs that meet only across the boundary: through x, through y and z,
    # and through a corner (x and y)
    "boundary_pairs": ([(0.10, 1.50, 1.50), (2.80, 1.50, 1.50),
                        (1.50, 0.20, 0.30), (1.50, 2.90, 2.85),
                        (2.95, 2.95, 1.00), (0.05, 0.10, 1.20)],
                       [1.0, -1.0, 1.0, -1.0, 0.5, -0.5]),
}


def ions(pos, q_e):
    n = len(pos)
    return systems.System(box=np.array([L, L, L]), pos=np.array(pos, dtype=np.float64),
                          vel=np.zeros((n, 3), np.float32),
                          charge=(np.asarray(q_e) * systems.E_TO_KCMOL).astype(np.float32),
                          mass=np.full(n, 39.948, np.float32), sigma=np.full(n, 0.30, np.float32),
                          epsilon=np.full(n, 500.0, np.float32), name="ions")


def min_image(s, i, j):
    d = s.pos[i] - s.pos[j]
    return np.linalg.norm(d - s.box * np.round(d / s.box))


@pytest.mark.parametrize("case", sorted(CASES))
def test_sparse_system_matches_oracle(oracle, case):
    s = ions(*CASES[case])
    kappa = kappa_from_tol(RC, 1e-5)
    e = Engine(cutoff=RC, electrostatics=E.ES_EWALD, ewald_kappa=kappa)
    e.load(s, pme_grid=GRID)
    e.compute_forces(energy=True)

    # pair set: every pair within the cutoff, through whichever image, exactly once
    got = e.pairlist()
    ref, flags, nband = oracle.pairset(s.pos, s.box, s.exclusions(), RC, band=1e-5)
    assert len(got) == len(set(map(tuple, got.tolist())))
    assert set(map(tuple, got.tolist())) == set(map(tuple, ref.tolist()))
    if case == "boundary_pairs":
        assert {(0, 1), (2, 3), (4, 5)} <= set(map(tuple, got.tolist()))
        for i, j in ((0, 1), (2, 3), (4, 5)):
            assert min_image(s, i, j) < RC < np.linalg.norm(s.pos[i] - s.pos[j])

    f = e.forces()
    fr, er = oracle_total(oracle, s, RC, 2, kappa, GRID)
    if s.n > 1:
        assert rel_rms(f, fr) < 1e-4, rel_rms(f, fr)
    else:
        # a lone ion feels only the grid's own small self force
        scale = 1e-4 * 138935.458 / 0.3 ** 2   # 1e-4 of k_e e^2 / (0.3 nm)^2 [J/mol/nm]
        assert np.abs(f - fr).max() < scale, (f, fr)
    en = e.energies()
    for k, b in er.items():
        assert abs(en[k] - b) <= 1e-5 * max(abs(b), 1e-3 * abs(en["potential"]), 1e-6), (k, en[k], b)


def droplet(radius=1.4, box=6.0):
    """Waters of a 3 nm box within `radius` of its centre, whole molecules, in the
    middle of an empty `box` nm cube: the central columns of the pair-search grid
    hold several times the average column count."""
    w = systems.water_box(900, 3.0, seed=11)
    c = w.box / 2
    d = w.pos[0::3] - c
    d -= w.box * np.round(d / w.box)
    keep = np.nonzero(np.linalg.norm(d, axis=1) < radius)[0]
    atoms = (3 * keep[:, None] + np.arange(3)).ravel()
    p = (w.pos[atoms] - c).reshape(-1, 3, 3)
    p[:, 0] -= w.box * np.round(p[:, 0] / w.box)
    h = p[:, 1:] - p[:, :1]
    p[:, 1:] = p[:, :1] + (h - w.box * np.round(h / w.box))
    p = p.reshape(-1, 3) + box / 2
    remap = -np.ones(w.n, np.int64)
    remap[atoms] = np.arange(len(atoms))
    kb = np.all(np.isin(w.bonds, atoms), axis=1)
    ka = np.all(np.isin(w.angles, atoms), axis=1)
    return systems.System(box=np.array([box] * 3), pos=p, vel=w.vel[atoms], charge=w.charge[atoms],
                          mass=w.mass[atoms], sigma=w.sigma[atoms], epsilon=w.epsilon[atoms],
                          bonds=remap[w.bonds[kb]].astype(np.int32), bond_par=w.bond_par[kb],
                          angles=remap[w.angles[ka]].astype(np.int32), angle_par=w.angle_par[ka],
                          name="droplet")


def test_droplet_in_vacuum(oracle):
    """An inhomogeneous system: column and pair-list capacities follow the
    densest columns, not the average density; forces and energies match the
    oracle before and after 20 steps (two list rebuilds)."""
    s = droplet()
    kappa = kappa_from_tol(RC, 1e-5)
    grid = (60, 60, 60)
    e = Engine(cutoff=RC, electrostatics=E.ES_EWALD, ewald_kappa=kappa, nstlist=10, dt=1e-6)
    e.load(s, pme_grid=grid)
    for n_steps in (0, 20):
        if n_steps:
            e.step(n_steps)
        e.compute_forces(energy=True)
        pos, _ = e.state()
        s2 = systems.System(**{**s.__dict__, "pos": pos})
        fr, er = oracle_total(oracle, s2, RC, 2, kappa, grid)
        f = e.forces()
        assert rel_rms(f, fr) < 1e-4, (n_steps, rel_rms(f, fr))
        en = e.energies()
        for k, b in er.items():
            assert abs(en[k] - b) <= 1e-5 * max(abs(b), 1e-3 * abs(en["potential"]), 1e-6), (n_steps, k, en[k], b)


def dilute_slab(n=240, lxy=14.0, lz=2.4, seed=3, min_dist=0.35):
    """A dilute gas of +/-0.5 e ions in a thin slab box: columns of the pair
    search hold about 10 atoms spread over the whole 2.4 nm height, so a cluster
    meets its own periodic image along z while the column window stays narrower
    than the grid in x and y (the search's fixed x-y shift branch)."""
    rng = np.random.default_rng(seed)
    box = np.array([lxy, lxy, lz])
    pts = []
    while len(pts) < n:
        p = rng.random(3) * box
        if pts:
            d = np.asarray(pts) - p
            d -= box * np.round(d / box)
            if (np.linalg.norm(d, axis=1) < min_dist).any():
                continue
        pts.append(p)
    q = np.where(np.arange(n) % 2 == 0, 0.5, -0.5)
    s = ions(pts, q)
    s.box = box
    return s


def test_dilute_slab_own_z_images(oracle):
    s = dilute_slab()
    kappa = kappa_from_tol(RC, 1e-5)
    grid = (144, 144, 24)
    e = Engine(cutoff=RC, electrostatics=E.ES_EWALD, ewald_kappa=kappa)
    e.load(s, pme_grid=grid)
    e.compute_forces(energy=True)
    got = e.pairlist()
    ref, flags, nband = oracle.pairset(s.pos, s.box, s.exclusions(), RC, band=1e-5)
    assert len(got) == len(set(map(tuple, got.tolist())))
    assert set(map(tuple, got.tolist())) == set(map(tuple, ref.tolist()))
    # pairs that meet only across the z boundary (direct distance beyond the cutoff)
    across = [(i, j) for i, j in ref.tolist() if np.linalg.norm(s.pos[i] - s.pos[j]) > RC]
    assert len(across) > 5
    f = e.forces()
    fr, er = oracle_total(oracle, s, RC, 2, kappa, grid)
    assert rel_rms(f, fr) < 1e-4, rel_rms(f, fr)
    en = e.energies()
    for k, b in er.items():
        assert abs(en[k] - b) <= 1e-5 * max(abs(b), 1e-3 * abs(en["potential"]), 1e-6), (k, en[k], b)
