"""Seeded synthetic inputs: sizes, neutrality, clean starting geometry."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from lima_b200 import systems


def _close_pairs(s, d=0.17):
    tr = cKDTree(s.pos, boxsize=s.box)
    p = np.sort(tr.query_pairs(d, output_type="ndarray"), 1)
    ex = set(map(tuple, s.exclusions()))
    return [t for t in map(tuple, p) if t not in ex]


@pytest.mark.parametrize("make,n_atoms", [(systems.config0, 3000), (systems.config1, 16828)])
def test_config_sizes_and_geometry(make, n_atoms):
    s = make()
    assert s.n == n_atoms
    assert abs(s.charge.sum()) < 1e-2
    assert (s.pos >= 0).all() and (s.pos < s.box).all()
    assert not _close_pairs(s)
    # deterministic from the seed
    s2 = make()
    assert np.array_equal(s.pos, s2.pos) and np.array_equal(s.vel, s2.vel)


def test_config1_topology():
    s = systems.config1()
    assert len(s.dihedrals) == 64 * 51 and len(s.bonds) == 64 * 51 + 9000
    heads = s.charge[: 64 * 52].reshape(64, 52)[:, :8]
    assert np.abs(heads.sum(1)).max() < 1e-3


def test_maxwell_boltzmann_temperature():
    s = systems.config0()
    ke = 0.5 * (s.mass[:, None] * s.vel.astype(np.float64) ** 2).sum()
    T = 2 * ke / ((3 * s.n - 3) * systems.KB_J_MOL_K)
    assert abs(T - 300.0) < 15.0
    assert np.abs((s.mass[:, None] * s.vel).sum(0)).max() < 1e-3


def test_fft_friendly_and_kappa():
    assert systems.fft_friendly(97) == 100 and systems.fft_friendly(96) == 96
    k = systems.ewald_kappa(1.0, 1e-5)
    import math
    assert abs(math.erfc(k * 1.0) - 1e-5) < 1e-9
