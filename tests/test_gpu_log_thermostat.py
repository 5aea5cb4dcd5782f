"""Per-particle logging (positions, potential energies, forces, speeds in a
device ring offloaded to the host) and the thermostat, through the C-ABI."""
import numpy as np
import pytest

from lima_b200 import Engine, systems
from lima_b200 import trajectory as T
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
    # the frame holds the updated state and the forces and energies of the
    # step's evaluation at the starting positions
    pos, vel = e.state()
    assert np.array_equal(pe[0, :, :3], pos.astype(np.float32))
    fr, _ = oracle_total(oracle, s, 1.0, 2, kappa, grid=grid)
    assert rel_rms(fs[0, :, :3].astype(np.float64), fr) < 1e-4
    assert np.allclose(fs[0, :, 3], np.linalg.norm(vel, axis=1), rtol=1e-5)
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


def test_trajectory_file_and_energy_analysis(tmp_path):
    """Logged frames go to a .trr file and through the reference's post-run
    energy analysis (variance coefficient, energy gradient)."""
    s = water(600, 3.0)
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5, log_interval=5,
               integrator=E.VELOCITY_VERLET)
    e.load(s, pme_grid=(30, 30, 30))
    e.step(100)                      # leave the lattice start behind
    e.clear_log()
    e.step(200)
    path = str(tmp_path / "trajectory.trr")
    assert T.write_log_trr(path, e, with_forces=True) == 40
    steps, pe, fs = e.log()
    assert list(steps) == list(range(100, 300, 5))
    frames = T.read_trr(path)
    assert [f.step for f in frames] == list(steps)
    for i in (0, 17, 39):
        assert np.array_equal(frames[i].x, pe[i, :, :3].astype(np.float64))
        assert np.allclose(frames[i].f, fs[i, :, :3] / 1000.0, rtol=1e-6)
        assert np.array_equal(frames[i].box, np.diag(s.box))
    a = T.analyze_log(e)
    pot, kin = T.log_energies(pe, fs, s.mass)
    tot = (pot + kin)[1:-1]
    assert len(a.total_energy) == 38 and np.allclose(a.total_energy, tot.astype(np.float32))
    assert abs(a.variance_coefficient - tot.std() / abs(tot.mean())) < 1e-4 * a.variance_coefficient
    slope = np.polyfit(np.arange(len(tot)), tot, 1)[0] / tot.mean()
    assert abs(a.energy_gradient - slope) < 1e-3 * abs(slope) + 1e-9
    # velocity Verlet: the logged speed is synchronous with the logged energy, so
    # the total only carries the integrator's O(dt^2) wobble (logging the speed a
    # step behind, as before the update, gave a variance coefficient of 2.6e-2)
    assert tot.std() < 1e-3 * a.kin_energy.mean(), (tot.std(), a.kin_energy.mean())
    assert a.variance_coefficient < 5e-3 and abs(a.energy_gradient) < 1e-4
