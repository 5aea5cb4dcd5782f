"""No boundary condition (the reference's BoundaryConditionSelect::NoBC,
Simulation.cuh:13, BoundaryCondition.cuh:5-15) through the C-ABI against the
FP64 oracle without a box: a water droplet straddling the nominal box's edge,
cutoff Coulomb, before and after 20 steps (two list rebuilds, no wrapping)."""
import numpy as np
import pytest

from lima_b200 import Engine, LimaError, systems
from lima_b200 import engine as E
from tests._ref import rel_rms
from tests.test_gpu_sparse import droplet

pytestmark = pytest.mark.gpu

RC = 1.2


def oracle_open(oracle, s, pos):
    """Forces and energy terms with plain differences (no images)."""
    fn, en, _ = oracle.nonbonded(pos, None, s.charge, s.sigma, s.epsilon, s.exclusions(), RC, 1)
    fb, eb = oracle.bonded(pos, None, s.bonds, s.bond_par, s.angles, s.angle_par)
    return fn + fb, {"lj": en["lj"], "coulomb_real": en["coulomb"], **eb}


def test_droplet_without_boundary(oracle):
    s = droplet()
    s.pos = s.pos - np.array([3.0, 0.0, 0.0])       # half the droplet lies at x < 0, outside the box
    assert (s.pos[:, 0] < 0).mean() > 0.3
    e = Engine(cutoff=RC, electrostatics=E.ES_CUTOFF, periodic=0, nstlist=10, dt=1e-6)
    e.load(s)
    for n_steps in (0, 20):
        if n_steps:
            e.step(n_steps)
        e.compute_forces(energy=True)
        pos, _ = e.state()
        assert (pos[:, 0] < 0).mean() > 0.3            # nothing is wrapped into the box
        fr, er = oracle_open(oracle, s, pos)
        f = e.forces()
        assert rel_rms(f, fr) < 1e-4, (n_steps, rel_rms(f, fr))
        en = e.energies()
        for k, b in er.items():
            assert abs(en[k] - b) <= 1e-5 * max(abs(b), 1e-3 * abs(en["potential"]), 1e-6), (n_steps, k, en[k], b)


def test_no_boundary_refuses_ewald():
    with pytest.raises(LimaError):
        Engine(cutoff=RC, electrostatics=E.ES_EWALD, periodic=0)


def test_system_entirely_outside_box(oracle):
    """Without a boundary the box only lays out the column grid: a droplet lying
    wholly at x < 0 is binned in the grid's first column row (each of those
    columns then holds atoms spread over 2.8 nm in x) and must still give the
    oracle's forces, before and after 20 steps."""
    s = droplet()
    s.pos = s.pos - np.array([6.0, 0.0, 0.0])
    assert (s.pos[:, 0] < 0).all()
    e = Engine(cutoff=RC, electrostatics=E.ES_CUTOFF, periodic=0, nstlist=10, dt=1e-6)
    e.load(s)
    for n_steps in (0, 20):
        if n_steps:
            e.step(n_steps)
        e.compute_forces(energy=True)
        pos, _ = e.state()
        assert (pos[:, 0] < 0).all()
        fr, _ = oracle_open(oracle, s, pos)
        assert rel_rms(e.forces(), fr) < 1e-4, (n_steps, rel_rms(e.forces(), fr))
    assert e.status() & 0x3 == 0      # no pair-list or column overflow
