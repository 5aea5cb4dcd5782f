"""The reference's dynamics known-answer tests through the C-ABI: a uniform
external electric field, and a single bond's oscillation frequency.

The reference's known-answer test (ForceCorrectness.h:621-669,
VerletintegrationTesting::TestIntegration): one charged particle in a field of
0.5 V/nm along x for 1,000 steps reaches the kinetic energy of constant
acceleration, qE t / m, within 1 %.  The field force is q E on every atom and
carries no potential energy (EngineKernels.cuh:321-343, Bodies.cuh:363-385).
"""
import numpy as np
import pytest

from lima_b200 import Engine, systems
from lima_b200 import engine as E
from tests._ref import kappa_from_tol

pytestmark = pytest.mark.gpu


def lone_ion(box=3.0):
    return systems.System(box=np.array([box] * 3), pos=np.array([[1.0, 1.5, 1.5]]),
                          vel=np.zeros((1, 3), np.float32),
                          charge=np.array([systems.E_TO_KCMOL], np.float32),
                          mass=np.array([0.039948], np.float32), sigma=np.zeros(1, np.float32),
                          epsilon=np.zeros(1, np.float32), name="ion")


@pytest.mark.parametrize("electrostatics", ["cutoff", "pme"])
def test_constant_field_kinetic_energy(electrostatics):
    s = lone_ion()
    n_steps, dt, field = 1000, 1e-6, 0.5          # steps, ns, V/nm
    if electrostatics == "pme":
        e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa_from_tol(1.0, 1e-5), dt=dt)
        e.load(s, pme_grid=(30, 30, 30))
    else:
        e = Engine(cutoff=1.0, electrostatics=E.ES_CUTOFF, dt=dt)
        e.load(s)
    e.set_electric_field((field, 0.0, 0.0))
    e.step(n_steps)
    force = float(s.charge[0]) * 1000.0 * field     # J/mol/nm
    v = force / float(s.mass[0]) * n_steps * dt     # nm/ns (= m/s)
    ke = 0.5 * float(s.mass[0]) * v * v             # J/mol
    ke_got = e.energies()["kinetic"]
    assert abs(ke_got - ke) / ke < 0.01, (ke_got, ke)          # the reference's bar
    if electrostatics == "cutoff":
        # nothing but the field acts: leapfrog velocities are exact to FP32 rounding
        _, vel = e.state()
        assert abs(vel[0, 0] - v) / v < 1e-4 and vel[0, 1] == 0.0 and vel[0, 2] == 0.0, (vel, v)
        assert abs(ke_got - ke) / ke < 3e-3, (ke_got, ke)


def test_field_adds_qE_and_no_energy():
    s = systems.water_box(600, 3.0, seed=4)
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5)
    e.load(s, pme_grid=(30, 30, 30))
    e.compute_forces(energy=True)
    f0, en0 = e.forces(), e.energies()
    field = np.array([0.3, -0.2, 0.1])
    e.set_electric_field(field)
    e.compute_forces(energy=True)
    f1, en1 = e.forces(), e.energies()
    expected = s.charge.astype(np.float64)[:, None] * 1000.0 * field[None, :]
    assert np.abs((f1 - f0) - expected).max() <= 1e-6 * np.abs(expected).max()
    assert en1["potential"] == en0["potential"]
    e.set_electric_field((0.0, 0.0, 0.0))
    e.compute_forces(energy=True)
    assert np.array_equal(e.forces(), f0)


@pytest.mark.parametrize("integrator", [E.LEAPFROG, E.VELOCITY_VERLET])
def test_bond_oscillation_frequency(integrator):
    """The reference's known-answer test ForceCorrectness.h:169-230 through the
    engine: a stretched bond between masses 12 and 16 g/mol oscillates at
    sqrt(k / mu) within 1 %."""
    import math
    m = np.array([12e-3, 16e-3], np.float32)
    kb, b0 = 2.5e8, 0.12
    mu = float(m[0]) * float(m[1]) / float(m.sum())
    period = 2 * math.pi * math.sqrt(mu / kb)      # [ns]
    dt = period / 400
    s = systems.System(box=np.array([3.0] * 3), pos=np.array([[1.0, 1.0, 1.0], [1.0 + b0 + 0.004, 1.0, 1.0]]),
                       vel=np.zeros((2, 3), np.float32), charge=np.zeros(2, np.float32), mass=m,
                       sigma=np.zeros(2, np.float32), epsilon=np.zeros(2, np.float32),
                       bonds=np.array([[0, 1]], np.int32), bond_par=np.array([[b0, kb]], np.float32), name="bond")
    e = Engine(cutoff=1.0, electrostatics=E.ES_NONE, dt=dt, integrator=integrator)
    e.load(s)
    xs = []
    for _ in range(3000):
        e.step(1)
        p, _ = e.state()
        xs.append(np.linalg.norm(p[1] - p[0]) - b0)
    xs = np.array(xs)
    crossings = np.where((xs[:-1] > 0) & (xs[1:] <= 0))[0]
    measured = np.mean(np.diff(crossings)) * dt
    assert len(crossings) >= 5
    assert abs(measured - period) / period < 0.01, (measured, period)
