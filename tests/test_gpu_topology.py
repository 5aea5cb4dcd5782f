"""A system that went through the topology files (.top/.gro written, then read
back) runs on the CUDA path through the C-ABI and matches the oracle on the
same parsed system, including the pairs the file's [ exclusions ] adds."""
import numpy as np
import pytest

from lima_b200 import Engine, systems, topology
from lima_b200 import engine as E
from tests._ref import kappa_from_tol, oracle_total, rel_rms

pytestmark = pytest.mark.gpu


def test_topology_files_through_engine(oracle, tmp_path):
    s = systems.water_with_chains(3000, 2, seed=11)
    chain = np.arange(40)                                # first chain (chains precede the water)
    s.extra_exclusions = np.stack([chain[:-5], chain[5:]], 1).astype(np.int32)
    tp, gp = str(tmp_path / "s.top"), str(tmp_path / "s.gro")
    topology.write_top(tp, s)
    topology.write_gro_system(gp, s)
    r = topology.load(gp, tp)
    assert np.array_equal(r.extra_exclusions, s.extra_exclusions)
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (32, 32, 32)
    eng = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa)
    eng.load(r, pme_grid=grid)
    eng.compute_forces(energy=True)
    fr, er = oracle_total(oracle, r, 1.0, 2, kappa, grid=grid)
    assert rel_rms(eng.forces(), fr) < 1e-4
    en = eng.energies()
    for k in ("lj", "coulomb_real", "pme_recip", "pme_excl", "bond", "angle", "dihedral"):
        if k in er:
            scale = max(abs(er[k]), 1e-3 * abs(en["potential"]), 1e-6)
            assert abs(en[k] - er[k]) <= 1e-5 * scale, (k, en[k], er[k])
    eng.step(20)
    assert np.isfinite(eng.energies()["total"])
