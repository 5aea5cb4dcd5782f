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
