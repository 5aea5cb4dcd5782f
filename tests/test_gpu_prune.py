"""Dynamic pruning of the pair list (lima_params.prune_interval) through the
C-ABI: the inner list the pair kernel walks between prunes must hold every pair
inside the cutoff (the same pair set as the oracle outside the 1e-5 nm band) at
every list age, forces and energies must match the FP64 oracle, and handing in
moved positions must re-prune before the next forces.  Explicit intervals, so
that the small boxes here prune although the automatic rule leaves them alone."""
import numpy as np
import pytest

from lima_b200 import Engine, systems
from lima_b200 import engine as E
from tests._ref import kappa_from_tol, oracle_total, rel_rms

pytestmark = pytest.mark.gpu

RC = 1.0


def make(s, prune, **kw):
    e = Engine(cutoff=RC, electrostatics=E.ES_EWALD, ewald_kappa=kappa_from_tol(RC, 1e-5), nstlist=10,
               dt=1e-6, prune_interval=prune, **kw)
    e.load(s, pme_grid=(36, 36, 36))
    return e


def pair_keys(p, n):
    p = np.asarray(p, np.int64)
    return np.unique(p[:, 0] * n + p[:, 1])


def check_pairs(oracle, s, pos, got):
    band = 1e-5
    near, _, _ = oracle.pairset(pos, s.box, s.exclusions(), RC + band)
    d = pos[near[:, 0]] - pos[near[:, 1]]
    d -= s.box * np.round(d / s.box)
    r = np.linalg.norm(d, axis=1)
    ref = pair_keys(near[r <= RC], s.n)
    in_band = pair_keys(near[np.abs(r - RC) < band], s.n)
    gk = pair_keys(got, s.n)
    assert len(gk) == len(got)
    assert len(np.setdiff1d(np.setdiff1d(ref, gk), in_band)) == 0
    assert len(np.setdiff1d(np.setdiff1d(gk, ref), in_band)) == 0


@pytest.mark.parametrize("prune", [2, 3, 5])
def test_pruned_list_holds_every_pair_at_every_age(oracle, prune):
    """Steps 1..12 from a build (ages 1..9, a rebuild, ages 0..2): after each
    step the walked (inner) list gives the oracle's pair set and the forces
    match the oracle; fewer rows are walked than built."""
    s = systems.water_box(1500, 3.6, seed=21, name="w")
    e = make(s, prune)
    walked = []
    for k in range(12):
        e.step(1)
        e.compute_forces(energy=k == 11)
        pos, _ = e.state()
        check_pairs(oracle, s, pos, e.pairlist())
        st = e.pairlist_stats()
        walked.append(st["rows_walked"] < st["rows_built"])
        if k in (4, 11):
            s2 = systems.System(**{**s.__dict__, "pos": pos})
            fr, er = oracle_total(oracle, s2, RC, 2, kappa_from_tol(RC, 1e-5), grid=(36, 36, 36))
            assert rel_rms(e.forces(), fr) < 1e-4
    assert all(walked)
    en = e.energies()
    for k, b in er.items():
        assert abs(en[k] - b) <= 1e-5 * max(abs(b), 1e-3 * abs(en["potential"]), 1e-6), (k, en[k], b)


def test_pruned_and_unpruned_trajectories_agree(oracle):
    """Pruning changes only which zero contributions are skipped and the FP32
    summation order: 40 steps with and without it stay within 1e-4 relative RMS
    in forces of each other and of the oracle at the end."""
    s = systems.water_box(1500, 3.6, seed=22, name="w")
    a, b = make(s, 0), make(s, 2)
    a.step(40)
    b.step(40)
    pa, _ = a.state()
    pb, _ = b.state()
    assert np.abs(pa - pb).max() < 1e-4
    b.compute_forces()
    s2 = systems.System(**{**s.__dict__, "pos": pb})
    fr, _ = oracle_total(oracle, s2, RC, 2, kappa_from_tol(RC, 1e-5), grid=(36, 36, 36))
    assert rel_rms(b.forces(), fr) < 1e-4


def test_moved_hand_in_prunes_again(oracle):
    """Positions handed in mid-period (moved less than half the buffer, so the
    outer list stays) are pruned again before the next forces: the walked list
    then holds every pair of the new positions."""
    s = systems.water_box(1500, 3.6, seed=23, name="w")
    e = make(s, 5)
    e.step(3)                                  # age 3: the inner list from the prune at age 0
    p, v = e.state()
    rng = np.random.default_rng(5)
    q = p + rng.uniform(-0.015, 0.015, p.shape)  # well within half the 0.1 nm buffer
    e.reset_timings()
    e.set_state(q, v)
    e.compute_forces()
    assert e.timings()["rebuilds"] == 0
    pos, _ = e.state()
    check_pairs(oracle, s, pos, e.pairlist())
    s2 = systems.System(**{**s.__dict__, "pos": pos})
    fr, _ = oracle_total(oracle, s2, RC, 2, kappa_from_tol(RC, 1e-5), grid=(36, 36, 36))
    assert rel_rms(e.forces(), fr) < 1e-4


def test_automatic_rule():
    """prune_interval < 0 prunes a single system of >= 1,024 clusters only."""
    small = make(systems.water_box(1500, 3.6, seed=24, name="w"), -1)
    small.compute_forces()
    st = small.pairlist_stats()
    assert st["rows_walked"] == st["rows_built"]
    big = Engine(cutoff=RC, electrostatics=E.ES_EWALD, ewald_tol=1e-5, nstlist=10, dt=1e-6)
    big.load(systems.water_box(4500, 5.2, seed=25, name="w"), pme_grid=(48, 48, 48))
    big.compute_forces()
    st = big.pairlist_stats()
    assert st["rows_walked"] < st["rows_built"]
