"""Per-particle logging (positions, potential energies, forces, speeds in a
device ring offloaded to the host) and the thermostat, through the C-ABI."""
import numpy as np
import pytest

from lima_b200 import Engine, systems
from lima_b200 import engine as E
from tests._ref import kappa_from_tol, oracle_total, rel_rms

pytestmark = pytest.mark.gpu

KB_NA = 1.380649e-23 * 6.02214076e23


def water(n=1500, box=3.6, seed=11):
    return systems.water_box(n, box, seed=seed, name="water_log")


def test_logged_energies_and_forces_match_oracle(oracle):
    s = water()
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (36, 36, 36)
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa, log_interval=1)
    e.load(s, pme_grid=grid)
    e.step(1)
    steps, pe, fs = e.log()
    assert list(steps) == [0]
    # the frame holds the state the step started from and its forces
    assert np.allclose(pe[0, :, :3], s.pos, atol=1e-5)
    fr, _ = oracle_total(oracle, s, 1.0, 2, kappa, grid=grid)
    assert rel_rms(fs[0, :, :3].astype(np.float64), fr) < 1e-4
    assert np.allclose(fs[0, :, 3], np.linalg.norm(s.vel, axis=1), rtol=1e-5)
    ae = oracle.atom_energies(s, 1.0, kappa, grid)
    got = pe[0, :, 3].astype(np.float64)
    assert rel_rms(got, ae) < 1e-4, rel_rms(got, ae)
    # the shares add up to the step's potential energy
    pot = e.energies()["potential"]
    assert abs(got.sum() - pot) < 1e-5 * abs(pot) + 1.0


def test_log_ring_offloads_every_frame():
    s = water(600, 3.0)
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5, log_interval=2, log_ring=3, use_graphs=1)
    e.load(s, pme_grid=(30, 30, 30))
    e.step(20)
    steps, pe, fs = e.log()
    assert list(steps) == list(range(0, 20, 2))
    assert np.all(np.isfinite(pe)) and np.all(np.isfinite(fs))
    # frames move with the trajectory and the last one precedes the final state
    assert not np.allclose(pe[0, :, :3], pe[-1, :, :3])
    pos, _ = e.state()
    assert np.abs(pe[-1, :, :3] - pos).max() < 0.05
    e.clear_log()
    assert len(e.log()[0]) == 0


@pytest.mark.parametrize("apply", [0, 1])
def test_thermostat_measures_and_scales(apply):
    s = water(600, 3.0)
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5, apply_thermostat=apply,
               thermostat_interval=10, target_temperature=310.0)
    e.load(s, pme_grid=(30, 30, 30))
    e.step(20)
    th = e.thermostat()
    assert th["step"] == 20
    _, v = e.state()
    ke = 0.5 * (s.mass.astype(np.float64) * (v.astype(np.float64) ** 2).sum(axis=1)).sum()
    T = 2.0 * ke / ((3 * s.n - 3) * KB_NA)
    assert abs(th["temperature"] - T) < 1e-6 * T
    # code/LIMA_ENGINE/src/Thermostat.cuh:55-67: clamp(310/T, 1 -+ 0.001/interval)
    expect = min(max(310.0 / T, 1.0 - 1e-4), 1.0 + 1e-4) if apply else 1.0
    assert abs(th["scale"] - expect) < 1e-7
