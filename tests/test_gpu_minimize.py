"""Energy minimisation through the C-ABI against the CPU oracle.

The reference's minimiser (LennardJonesInteractions.cuh:85-101,
EngineUtils.cuh:44-72 and :112-140) bounds every LJ pair force with a tanh
activation and takes ADAM steps on the per-atom force after a second tanh
bound.  A gas with one strongly overlapping pair makes the pair bound matter;
one lima_minimize step must give the oracle's forces and the oracle's step.
"""
import numpy as np
import pytest

from lima_b200 import Engine, systems
from lima_b200 import engine as E
from tests._ref import rel_rms

pytestmark = pytest.mark.gpu

RC = 1.0


def overlap_gas(n=150, box=3.5, seed=5, r_close=0.145):
    """LJ atoms (sigma 0.3 nm, epsilon 500 J/mol), a third of them +-0.3 e, at
    least 0.3 nm apart, except atoms 0 and 1, r_close apart: their LJ pair force
    (about 1e9 J/mol/nm) is where the tanh bound (2.4e9) takes off about 5 %."""
    rng = np.random.default_rng(seed)
    L = np.array([box] * 3)
    pts = [np.array([1.5, 1.5, 1.5]), np.array([1.5 + r_close, 1.5, 1.5])]
    while len(pts) < n:
        p = rng.random(3) * L
        d = np.asarray(pts) - p
        d -= L * np.round(d / L)
        if (np.linalg.norm(d, axis=1) < 0.3).any():
            continue
        pts.append(p)
    q = np.zeros(n)
    q[2:2 + n // 3] = np.where(np.arange(n // 3) % 2 == 0, 0.3, -0.3)
    return systems.System(box=L, pos=np.asarray(pts), vel=np.zeros((n, 3), np.float32),
                          charge=(q * systems.E_TO_KCMOL).astype(np.float32), mass=np.full(n, 39.948, np.float32),
                          sigma=np.full(n, 0.3, np.float32), epsilon=np.full(n, 500.0, np.float32), name="gas")


def test_minimize_step_matches_oracle(oracle):
    s = overlap_gas()
    e = Engine(cutoff=RC, electrostatics=E.ES_CUTOFF)
    e.load(s)
    steps, _ = e.minimize(force_tol=0.0, max_steps=1)
    assert steps == 1
    f = e.forces()                    # the forces the step used (initial positions)
    args = (s.pos, s.box, s.charge, s.sigma, s.epsilon, s.exclusions(), RC, 1)
    f_em, _, _ = oracle.nonbonded(*args, em=True)
    f_plain, _, _ = oracle.nonbonded(*args)
    assert rel_rms(f, f_em) < 1e-4, rel_rms(f, f_em)
    # the pair bound changes the overlapping pair's forces by several per cent
    change = np.linalg.norm(f_em[0] - f_plain[0]) / np.linalg.norm(f_plain[0])
    assert 0.03 < change < 0.1, change
    # one ADAM step on the tanh-bounded per-atom forces
    pos = s.pos.copy()
    oracle.em_step(pos, f_em, np.zeros(6 * s.n), 1)
    p1, _ = e.state()
    d = p1 - pos
    d -= s.box * np.round(d / s.box)
    # a component's first step is 8e-5 nm x g / (|g| + 1e-8), g = 1e-8 x its bounded
    # force: where |F| > 100 J/mol/nm that is 8e-5 nm with the force's sign; near
    # zero it is 8e-5 nm x F, so FP32 force noise (~0.01 J/mol/nm) shows there
    big = np.abs(f_em) > 100.0
    assert big.sum() > 0.9 * big.size
    assert np.abs(d[big]).max() < 1e-9, np.abs(d[big]).max()
    assert np.abs(d).max() < 2e-6, np.abs(d).max()
    assert np.abs(pos - s.pos).max() > 7e-5          # the step moved atoms by up to 8e-5 nm
