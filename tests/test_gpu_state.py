"""lima_set_state on a built engine: atoms keep their slots and the pair list is
kept while no atom moved more than half the Verlet buffer since the list was
built; larger moves rebuild it.  Results must not depend on which path ran."""
import numpy as np
import pytest

from lima_b200 import Engine, LimaError, systems
from lima_b200 import engine as E
from tests._ref import kappa_from_tol, oracle_total, rel_rms

pytestmark = pytest.mark.gpu


def make(s, **kw):
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa_from_tol(1.0, 1e-5), **kw)
    e.load(s, pme_grid=(36, 36, 36))
    return e


def test_state_round_trip_keeps_trajectory_bitwise():
    s = systems.water_box(1500, 3.6, seed=3, name="w")
    a, b = make(s), make(s)
    # one step after the list build at step 10: no atom is near half the buffer
    a.step(11)
    b.step(11)
    p, v = b.state()
    b.reset_timings()
    b.set_state(p, v)            # same state back: same slots, the list is kept
    b.compute_forces()
    assert b.timings()["rebuilds"] == 0
    a.compute_forces()
    a.step(12)
    b.step(12)
    pa, va = a.state()
    pb, vb = b.state()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert a.energies()["potential"] == b.energies()["potential"]


def test_unchanged_hand_back_every_step_keeps_cadence():
    """Handing the engine's own state back before every step (the end-to-end
    pattern) keeps the pair list on its nstlist cadence: the same rebuilds and the
    same trajectory bits as stepping alone."""
    s = systems.water_box(1500, 3.6, seed=8, name="w")
    a, b = make(s), make(s)
    a.step(1)
    b.step(1)
    a.reset_timings()
    b.reset_timings()
    a.step(30)
    for _ in range(30):
        p, v = b.state()
        b.set_state(p, v)
        b.step(1)
    assert b.timings()["rebuilds"] == a.timings()["rebuilds"] == 3
    pa, va = a.state()
    pb, vb = b.state()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)


def test_large_moves_and_rewrapped_positions_rebuild(oracle):
    s = systems.water_box(1500, 3.6, seed=4, name="w")
    e = make(s)
    e.step(5)
    p, v = e.state()
    q = p + np.array([0.3, -0.2, 0.1])   # a rigid move far beyond half the buffer
    q[100] += s.box                      # the same point one image away
    e.reset_timings()
    e.set_state(q, v)
    e.compute_forces(energy=True)
    s2 = systems.System(**{**s.__dict__, "pos": q.astype(np.float64)})
    fr, _ = oracle_total(oracle, s2, 1.0, 2, kappa_from_tol(1.0, 1e-5), grid=(36, 36, 36))
    assert rel_rms(e.forces(), fr) < 1e-4
    assert e.timings()["rebuilds"] == 1


def test_topology_change_keeps_current_positions():
    s = systems.water_box(600, 3.0, seed=5, name="w")
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5)
    e.load(s, pme_grid=(30, 30, 30))
    e.step(10)
    p, v = e.state()
    e.set_box(s.box)             # forces a new set-up
    p2, v2 = e.state()
    assert np.array_equal(p, p2) and np.array_equal(v, v2)


def test_autotune_shapes_give_identical_trajectories():
    """The autotuner switches the pair kernel's launch shape between periods; every
    shape must give the same bits, so a tuned run equals an untuned one."""
    s = systems.water_box(1500, 3.6, seed=6, name="w")
    a, b = make(s), make(s)
    shape = a.autotune(1)                      # 12 + 3 x 12 periods of 10 steps, energies at each period's end
    assert 0 <= shape <= 11 and a.timings()["pair_shape"] == shape
    for _ in range(48):
        b.step(10)
    a.step(10)
    b.step(10)
    pa, va = a.state()
    pb, vb = b.state()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)
    assert a.energies()["potential"] == b.energies()["potential"]


@pytest.mark.parametrize("prune", [-1, 2])
@pytest.mark.parametrize("split", [1, -1])
@pytest.mark.parametrize("es", [E.ES_CUTOFF, E.ES_EWALD])
def test_every_pair_kernel_shape_gives_the_same_bits(es, split, prune):
    """The eight shapes of the plain pair kernel and the four of the staged,
    persistent one: forces (a step with a rebuild and the next one) and the
    energies of an energy step are bitwise identical — with whole clusters per
    warp, and with this small box's automatic row split (where the staged
    shapes run the plain kernel), on the built list and on a pruned one.  The
    plain kernel leaves the LJ arithmetic out for the LJ-free (hydrogen)
    i-pairs; the staged one evaluates LJ for every pair, so equal bits show
    that leaving it out changes nothing."""
    s = systems.water_box(1500, 3.6, seed=8, name="w")
    ref = None
    for shape in [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11]:
        e = Engine(cutoff=1.0, electrostatics=es, ewald_tol=1e-5, nstlist=10, pair_split=split,
                   prune_interval=prune)
        e.load(s, pme_grid=(30, 30, 30) if es == E.ES_EWALD else None)
        e.set_pair_shape(shape)
        e.compute_forces(energy=False)
        f0 = e.forces()
        e.step(3)
        e.compute_forces(energy=True)
        got = (f0, e.forces(), e.energies()["lj"], e.energies()["coulomb_real"], e.energies()["virial"])
        e.close()
        if ref is None:
            ref = got
            continue
        for a, b in zip(got, ref):
            assert np.array_equal(a, b), shape
    with pytest.raises(LimaError):
        Engine(cutoff=1.0).set_pair_shape(12)


def test_nonfinite_state_refused_on_built_engine():
    """On a built engine the handed-in state is checked on the device before it
    replaces the slot state: a non-finite position is refused with
    LIMA_ERR_NOT_FINITE and leaves the engine exactly as it was."""
    s = systems.water_box(600, 3.0, seed=4)
    e = Engine(cutoff=1.0, electrostatics=E.ES_EWALD, ewald_tol=1e-5)
    e.load(s, pme_grid=(30, 30, 30))
    e.step(3)
    p0, v0 = e.state()
    bad = p0.copy()
    bad[17, 2] = np.inf
    with pytest.raises(LimaError) as ex:
        e.set_state(bad, v0)
    assert ex.value.code == 7
    p1, v1 = e.state()
    assert np.array_equal(p0, p1) and np.array_equal(v0, v1)
    e.set_state(p0, v0)
    e.step(2)
    assert np.isfinite(e.energies()["total"])
