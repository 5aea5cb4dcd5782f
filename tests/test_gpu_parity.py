"""Parity of the CUDA path (through the C-ABI) with the FP64 CPU oracle.

Bars, from the path's specification: pair sets bit-exact outside a band of
|r - rc| < 1e-5 nm; forces within 1e-4 relative RMS; energy terms within 1e-5
relative (FP32 pair arithmetic, FP64 totals); results bit-reproducible run to run.
"""
import numpy as np
import pytest

from lima_b200 import Engine, LimaError, systems
from lima_b200 import engine as E
from tests._ref import kappa_from_tol, oracle_total, rel_rms

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-4
ENERGY_TOL = 1e-5


def small_water(n_waters=3000, box=4.6, seed=5):
    return systems.water_box(n_waters, box, seed=seed, name="water_small")


def make(s, grid=None, **kw):
    e = Engine(**kw)
    e.load(s, pme_grid=grid)
    return e


def check_energies(eng, ref, tol=ENERGY_TOL, keys=None):
    keys = keys or ref.keys()
    for k in keys:
        a, b = eng[k], ref[k]
        scale = max(abs(b), 1e-3 * abs(eng["potential"]) if eng.get("potential") else 0.0, 1e-6)
        assert abs(a - b) <= tol * scale, (k, a, b)


# ------------------------------------------------------------- (a) pair sets
@pytest.mark.parametrize("rc", [1.2, 0.9])
def test_pairset_bit_exact(oracle, rc):
    s = systems.config0()
    e = make(s, cutoff=rc, electrostatics=E.ES_CUTOFF)
    e.compute_forces()
    got = e.pairlist()
    band = 1e-5
    ref, flags, nband = oracle.pairset(s.pos, s.box, s.exclusions(), rc, band=band)
    gs = set(map(tuple, got.tolist()))
    rs = set(map(tuple, ref.tolist()))
    in_band = set(map(tuple, ref[flags == 1].tolist()))
    only_gpu = gs - rs
    only_ref = rs - gs
    assert only_ref <= in_band, len(only_ref - in_band)
    # a pair the GPU keeps but the oracle drops must sit just outside rc
    for i, j in only_gpu:
        d = s.pos[i] - s.pos[j]
        d -= s.box * np.round(d / s.box)
        assert abs(np.linalg.norm(d) - rc) < band
    assert len(got) == len(gs)        # no duplicates
    assert len(rs) > 100000 if rc == 1.2 else True


def _pair_keys(pairs, n):
    p = np.asarray(pairs, np.int64)
    return np.unique(p[:, 0] * n + p[:, 1])


@pytest.mark.parametrize("cfg", ["config1", "config2"])
def test_pairset_bit_exact_large(oracle, cfg):
    """The pair sets of the chain slab (C1, rc 1.2 nm) and the 100k-atom water box
    (C2, rc 1.0 nm) against the oracle: identical outside the 1e-5 nm band and
    no pair listed twice."""
    s = getattr(systems, cfg)()
    rc = 1.2 if cfg == "config1" else 1.0
    e = make(s, cutoff=rc, electrostatics=E.ES_CUTOFF)
    e.compute_forces()
    got = e.pairlist()
    gk = _pair_keys(got, s.n)
    assert len(gk) == len(got)                       # no duplicates
    band = 1e-5
    near, _, _ = oracle.pairset(s.pos, s.box, s.exclusions(), rc + band)
    d = s.pos[near[:, 0]] - s.pos[near[:, 1]]
    d -= s.box * np.round(d / s.box)
    r = np.linalg.norm(d, axis=1)
    ref_in = _pair_keys(near[r <= rc], s.n)
    in_band = _pair_keys(near[np.abs(r - rc) < band], s.n)
    only_ref = np.setdiff1d(np.setdiff1d(ref_in, gk), in_band)
    only_gpu = np.setdiff1d(np.setdiff1d(gk, ref_in), in_band)
    assert len(only_ref) == 0 and len(only_gpu) == 0, (len(only_ref), len(only_gpu))
    assert len(ref_in) > (3_000_000 if cfg == "config1" else 20_000_000)


# Energy bars per term against the FP64 oracle.  The engine's positions are FP32
# absolute coordinates (a 10 nm box resolves 1e-6 nm), which bounds the LJ term,
# whose r^-12 wall amplifies the coordinate rounding, near 1e-6; the
# reciprocal-space term sums an FP32 grid through two FP32 FFTs.
TERM_BARS = {"lj": 3e-6, "pme_recip": 2e-6}
TERM_BAR = 1e-6


def check_energy_bars(eng, ref):
    # a term below 1e-4 of the summed magnitudes (bonds at their rest length in a
    # freshly built system: ~1 J/mol beside 1e9) is measured against that floor
    floor = 1e-4 * sum(abs(v) for v in ref.values())
    for k, b in ref.items():
        a = eng[k]
        assert abs(a - b) <= TERM_BARS.get(k, TERM_BAR) * max(abs(b), floor), (k, a, b, abs(a - b) / max(abs(b), floor))
    pot = sum(ref.values())
    assert abs(sum(eng[k] for k in ref) - pot) <= TERM_BAR * abs(pot)


# ------------------------------------------------- (b)+(c) forces and energies
def test_cutoff_coulomb_config0(oracle):
    """Config 0: LJ + plain cutoff Coulomb at 1.2 nm, flexible water bonds/angles."""
    s = systems.config0()
    e = make(s, cutoff=1.2, electrostatics=E.ES_CUTOFF)
    e.compute_forces(energy=True)
    f = e.forces()
    fr, er = oracle_total(oracle, s, 1.2, 1)
    assert rel_rms(f, fr) < FORCE_TOL, rel_rms(f, fr)
    check_energies(e.energies(), er)


def test_ewald_pme_accurate(oracle):
    s = small_water()
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (48, 48, 48)
    e = make(s, grid=grid, cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa)
    e.compute_forces(energy=True)
    f = e.forces()
    fr, er = oracle_total(oracle, s, 1.0, 2, kappa, grid)
    assert rel_rms(f, fr) < FORCE_TOL, rel_rms(f, fr)
    check_energies(e.energies(), er)


def lj_pattern(s, pattern, seed=3):
    """The water box with other atoms LJ-free (epsilon = 0): all of them, only
    the oxygens (the hydrogens given a small LJ site), or a random half of the
    atoms (hydrogens with LJ too), so clusters carry every count of LJ atoms."""
    sig, eps = s.sigma.copy(), s.epsilon.copy()
    hyd = eps == 0.0
    if pattern == "none":
        eps[:] = 0.0
    else:
        sig[hyd], eps[hyd] = 0.1, 100.0
        if pattern == "oxygens_free":
            eps[~hyd] = 0.0
        else:
            eps[np.random.default_rng(seed).random(s.n) < 0.5] = 0.0
    return systems.System(**{**s.__dict__, "sigma": sig.astype(np.float32), "epsilon": eps.astype(np.float32)})


@pytest.mark.parametrize("pattern", ["none", "oxygens_free", "random_half"])
def test_lj_free_atoms(oracle, pattern):
    """The pair kernel leaves the LJ arithmetic out for a cluster's trailing
    i-atom pairs without LJ (each cluster's LJ atoms take its first slots).
    Whatever atoms are LJ-free, forces of force-only and energy steps and the
    energy terms match the oracle, and the staged kernel, which evaluates LJ for
    every pair, gives the same bits as the plain one."""
    s = lj_pattern(small_water(), pattern)
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (48, 48, 48)
    fr, er = oracle_total(oracle, s, 1.0, 2, kappa, grid)
    got = []
    for shape in (0, 8):
        e = make(s, grid=grid, cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa, pair_split=1)
        e.set_pair_shape(shape)
        e.compute_forces(energy=False)
        f0 = e.forces()
        e.compute_forces(energy=True)
        got.append((f0, e.forces(), e.energies()))
        e.close()
    for f0, f1, en in got:
        assert rel_rms(f0, fr) < FORCE_TOL, rel_rms(f0, fr)
        assert rel_rms(f1, fr) < FORCE_TOL, rel_rms(f1, fr)
        check_energies(en, er)
    assert np.array_equal(got[0][0], got[1][0]) and np.array_equal(got[0][1], got[1][1])
    assert all(got[0][2][k] == got[1][2][k] for k in ("lj", "coulomb_real", "virial"))


def test_ewald_pme_reference_conventions(oracle):
    """ref_compat: kappa = 3/rc, sinc^8 influence, central-difference gather, no
    exclusion correction, the reference's per-atom self-energy bookkeeping."""
    s = small_water(box=4.5)
    grid = (45, 45, 45)          # the reference's 10 points per nm
    e = make(s, grid=grid, cutoff=1.2, electrostatics=E.ES_EWALD, ref_compat=1)
    e.compute_forces(energy=True)
    f = e.forces()
    fr, er = oracle_total(oracle, s, 1.2, 2, 3.0 / 1.2, grid, ref_compat=True)
    assert rel_rms(f, fr) < FORCE_TOL, rel_rms(f, fr)
    en = e.energies()
    assert en["pme_excl"] == 0.0
    check_energies(en, er)


def test_reference_immediate_pairs_without_cutoff(oracle):
    """ref_compat with the reference builder's compounds (config 1's chains split
    into 32 + 20 atom compounds, one water per compound): pairs inside a
    compound and across bonded compounds are evaluated with no cutoff
    (EngineKernels.cuh:150-317), all others through the cutoff list; against
    the oracle's restatement of the same rule."""
    s = systems.config1().with_compounds()
    rc = 1.2
    grid = (50, 50, 80)                 # the reference's 10 points per nm
    ex = s.exclusions()
    imm = oracle.immediate_pairs(s.compound, s.bonded_compounds, ex)
    d = s.pos[imm[:, 1]] - s.pos[imm[:, 0]]
    d -= s.box * np.round(d / s.box)
    beyond = int((np.linalg.norm(d, axis=1) > rc).sum())
    assert len(imm) > 70000 and beyond > 1000     # pairs the cutoff alone would drop
    e = make(s, grid=grid, cutoff=rc, electrostatics=E.ES_EWALD, ref_compat=1)
    e.compute_forces(energy=True)
    f = e.forces()
    fr, er = oracle_total(oracle, s, rc, 2, 3.0 / rc, grid, ref_compat=True)
    assert rel_rms(f, fr) < FORCE_TOL, rel_rms(f, fr)
    check_energies(e.energies(), er)
    # Without compounds the same engine drops exactly the immediate pairs beyond
    # the cutoff.  On this unrelaxed box their share is small next to the
    # total (about 6 kJ/mol of LJ; ~10 J/mol/nm per chain atom, below the
    # rounding of the 1e7 J/mol/nm near-neighbour forces the two runs evaluate
    # in different kernels), so the LJ energy difference is checked against the
    # oracle's value for those pairs.
    e2 = make(systems.config1(), grid=grid, cutoff=rc, electrostatics=E.ES_EWALD, ref_compat=1)
    e2.compute_forces(energy=True)
    far = imm[np.linalg.norm(d, axis=1) > rc]
    _, elj_far, _ = oracle.immediate_forces(s.pos, s.box, s.charge, s.sigma, s.epsilon, far, 2, 3.0 / rc)
    d_lj = e.energies()["lj"] - e2.energies()["lj"]
    assert abs(d_lj - elj_far) <= 0.02 * abs(elj_far) + 2e-6 * abs(er["lj"]), (d_lj, elj_far)


def test_full_config1(oracle):
    """Config 1: chains + water, LJ per atom, Ewald + PME 48x48x80, bonds/angles/dihedrals."""
    s = systems.config1()
    kappa = kappa_from_tol(1.2, 1e-5)
    grid = (48, 48, 80)
    e = make(s, grid=grid, cutoff=1.2, electrostatics=E.ES_EWALD, ewald_kappa=kappa)
    e.compute_forces(energy=True)
    f = e.forces()
    fr, er = oracle_total(oracle, s, 1.2, 2, kappa, grid)
    assert rel_rms(f, fr) < FORCE_TOL, rel_rms(f, fr)
    check_energies(e.energies(), er)


def test_bonded_all_terms(oracle):
    """Bonds, angles with Urey-Bradley, dihedrals (both gradient branches),
    impropers and pair bonds; non-bonded switched off."""
    s = systems.config1()
    rng = np.random.default_rng(3)
    heads = np.arange(64) * 52
    # around head atom 6, the branch point of the head and tail A: angles between
    # the two planes of 75-108 degrees (an improper near 0 or 180 degrees puts
    # acos at its ill-conditioned ends in either precision)
    s.impropers = np.stack([heads + 5, heads + 6, heads + 7, heads + 8], 1).astype(np.int32)
    s.improper_par = np.stack([rng.uniform(-0.3, 0.3, 64), rng.uniform(1e4, 5e4, 64)], 1).astype(np.float32)
    s.pairbonds = np.stack([heads + 8, heads + 11], 1).astype(np.int32)
    s.pair_par = np.tile([0.34, 700.0], (64, 1)).astype(np.float32)
    s.angle_par = s.angle_par.copy()
    s.angle_par[:100, 2] = 0.25
    s.angle_par[:100, 3] = 1e5
    s.epsilon = np.zeros_like(s.epsilon)
    e = make(s, cutoff=1.2, electrostatics=E.ES_NONE)
    e.compute_forces(energy=True)
    f = e.forces()
    fr, er = oracle_total(oracle, s, 1.2, 0, nb=False)
    assert rel_rms(f, fr) < FORCE_TOL, rel_rms(f, fr)
    check_energies(e.energies(), er, keys=["bond", "angle", "dihedral", "improper", "pairbond"])


def test_config2_full_size(oracle):
    """100,200-atom water box, PME 96^3, cutoff 1.0 nm."""
    s = systems.config2()
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (96, 96, 96)
    e = make(s, grid=grid, cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa)
    e.compute_forces(energy=True)
    f = e.forces()
    fr, er = oracle_total(oracle, s, 1.0, 2, kappa, grid)
    assert rel_rms(f, fr) < FORCE_TOL, rel_rms(f, fr)
    check_energies(e.energies(), er)


@pytest.mark.parametrize("cfg", ["config1", "config2"])
def test_energy_bars_prepared(oracle, cfg):
    """The 1e-6 energy bars on a prepared state (energy minimisation, then
    thermostatted MD at 300 K: no lattice clashes left), the state the
    configurations are run from; forces at 1e-4 relative RMS as everywhere."""
    from tests.accuracy_report import equilibrate
    s = getattr(systems, cfg)()
    rc = 1.2 if cfg == "config1" else 1.0
    grid = (48, 48, 80) if cfg == "config1" else (96, 96, 96)
    kappa = kappa_from_tol(rc, 1e-5)

    def make_engine(**extra):
        return Engine(cutoff=rc, electrostatics=E.ES_EWALD, ewald_kappa=kappa, nstlist=10, dt=1e-6, **extra)

    s, _ = equilibrate(make_engine, s, grid, 300, 500)
    e = make_engine()
    e.load(s, pme_grid=grid)
    e.compute_forces(energy=True)
    fr, er = oracle_total(oracle, s, rc, 2, kappa, grid)
    assert rel_rms(e.forces(), fr) < FORCE_TOL
    check_energy_bars(e.energies(), er)


@pytest.mark.parametrize("split", [1, 2, 8])
def test_pair_split_matches_oracle(oracle, split):
    """The pair kernel's rows split over 1, 2 or 8 warps per i-cluster: forces
    and energies against the oracle, and the split results agree with the
    unsplit ones to FP32 summation order."""
    s = small_water()
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (48, 48, 48)
    e = make(s, grid=grid, cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa, pair_split=split)
    e.compute_forces(energy=True)
    fr, er = oracle_total(oracle, s, 1.0, 2, kappa, grid)
    assert rel_rms(e.forces(), fr) < FORCE_TOL
    check_energies(e.energies(), er)
    u = make(s, grid=grid, cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa, pair_split=1)
    u.compute_forces(energy=True)
    assert rel_rms(e.forces(), u.forces()) < 1e-6


# ------------------------------------------------------------- reproducibility
def test_bit_reproducible():
    s = small_water()
    a = make(s, grid=(48, 48, 48), cutoff=1.0)
    a.compute_forces(energy=True)
    fa, ea = a.forces(), a.energies()
    a.compute_forces(energy=True)
    fa2 = a.forces()
    b = make(s, grid=(48, 48, 48), cutoff=1.0)
    b.compute_forces(energy=True)
    fb, eb = b.forces(), b.energies()
    assert np.array_equal(fa, fa2) and np.array_equal(fa, fb)
    assert ea == eb
    a.step(25)
    b.step(25)
    pa, va = a.state()
    pb, vb = b.state()
    assert np.array_equal(pa, pb) and np.array_equal(va, vb)


# ------------------------------------------------------------------- (e) integration
@pytest.mark.parametrize("integrator", [E.LEAPFROG, E.VELOCITY_VERLET])
def test_integrator_matches_oracle(oracle, integrator):
    """20 steps against the oracle's integrator.  Erfc-screened real-space Coulomb
    (no reciprocal part) keeps the force continuous at the cutoff, so the two
    trajectories stay together to FP32 force precision (plain cutoff Coulomb
    jumps by ~3e4 J/mol/nm when a pair crosses rc and they part legitimately)."""
    s = systems.config0()
    n_steps, dt = 20, 1e-6
    kappa = kappa_from_tol(1.2, 1e-5)
    e = make(s, cutoff=1.2, electrostatics=E.ES_EWALD, ewald_kappa=kappa, integrator=integrator, dt=dt,
             nstlist=10)
    e.step(n_steps)
    pg, vg = e.state()
    p = s.pos.copy()
    v = s.vel.astype(np.float64).copy()
    fprev = np.zeros_like(p)
    m = s.mass.astype(np.float64)
    import dataclasses
    for k in range(n_steps):
        cur = dataclasses.replace(s, pos=p)
        f, _ = oracle_total(oracle, cur, 1.2, 2, kappa)
        oracle.integrate(p, v, fprev, f, m, dt, integrator)
    d = pg - p
    d -= s.box * np.round(d / s.box)
    assert np.abs(d).max() < 1e-6, np.abs(d).max()
    assert rel_rms(vg.astype(np.float64), v) < 1e-4


def test_energy_conservation():
    """NVE leapfrog, 1 fs, PME water: total energy drift stays small over 2,000 steps."""
    s = small_water(n_waters=1500, box=3.6)
    e = make(s, grid=(40, 40, 40), cutoff=1.0, nstlist=10)
    e.step(1)
    e0 = e.energies()["total"]
    totals = []
    for _ in range(20):
        e.step(100)
        totals.append(e.energies()["total"])
    kin = e.energies()["kinetic"]
    drift = abs(totals[-1] - e0)
    assert drift < 0.02 * kin, (drift, kin, totals)


def test_minimize_reduces_max_force():
    s = systems.config1()
    e = make(s, grid=(48, 48, 80), cutoff=1.2)
    e.compute_forces()
    f0 = np.linalg.norm(e.forces(), axis=1).max()
    steps, fmax = e.minimize(force_tol=1.0, max_steps=300)
    assert steps > 0 and fmax < f0


# --------------------------------------------------------------------- batching
@pytest.mark.parametrize("split", [1, 8])
def test_batch_matches_single(split):
    """Each system of a batch gives the same bits as the system alone, with the
    pair kernel's rows unsplit (a batch's default) or split over 8 warps per
    i-cluster (batch warps mapped to systems by their warp offsets)."""
    sys_list = [systems.water_box(n, L, seed=11 + n, name="b") for n, L in ((600, 2.8), (1500, 3.6), (900, 3.1))]
    grids = [(32, 32, 32), (40, 40, 40), (36, 36, 36)]
    batch = Engine(n_systems=3, cutoff=1.0, pair_split=split)
    for k, (s, g) in enumerate(zip(sys_list, grids)):
        batch.select(k)
        batch.load(s, pme_grid=g)
    batch.compute_forces(energy=True)
    for k, (s, g) in enumerate(zip(sys_list, grids)):
        single = make(s, grid=g, cutoff=1.0, pair_split=split)
        single.compute_forces(energy=True)
        batch.select(k)
        assert np.array_equal(batch.forces(), single.forces())
        eb, es = batch.energies(), single.energies()
        for key in ("lj", "coulomb_real", "pme_recip", "bond", "angle"):
            assert eb[key] == es[key], key


def test_nonfinite_positions_rejected():
    s = systems.config0()
    e = Engine(cutoff=1.2)
    e.load(s)
    p = s.pos.copy()
    p[5, 1] = np.nan
    with pytest.raises(LimaError) as ex:
        e.set_state(p)
    assert ex.value.code == 7


def test_graph_replay_equals_eager():
    """Pair-list periods replayed as CUDA graphs, one or two periods per graph,
    give the same trajectory bits as eager launches."""
    s = small_water(n_waters=1500, box=3.6)
    out = []
    for graphs in (0, 1, 2):
        e = make(s, grid=(40, 40, 40), cutoff=1.0, nstlist=10, use_graphs=graphs)
        e.step(1)
        e.step(45)
        p, v = e.state()
        out.append((p, v, e.energies()["total"], e.timings()))
    for o in out[1:]:
        assert np.array_equal(out[0][0], o[0]) and np.array_equal(out[0][1], o[1])
        assert out[0][2] == o[2]
    assert out[2][3]["rebuilds"] == out[1][3]["rebuilds"] == out[0][3]["rebuilds"]


def test_batch_with_chains_matches_single():
    """Config-4 style systems (water + inserted chains, per-system PME grids from
    0.12 nm spacing) batched in one engine equal the same systems run alone."""
    sys_list = [systems.water_with_chains(n, c, seed=40 + n) for n, c in ((2200, 1), (5000, 3), (1600, 0))]
    batch = Engine(n_systems=3, cutoff=1.0, pme_spacing=0.12)
    for k, s in enumerate(sys_list):
        batch.select(k)
        batch.load(s)
    batch.step(12)
    for k, s in enumerate(sys_list):
        single = Engine(cutoff=1.0, pme_spacing=0.12, pair_split=1)   # a batch does not split
        single.load(s)
        single.step(12)
        batch.select(k)
        pb, vb = batch.state()
        ps, vs = single.state()
        assert np.array_equal(pb, ps) and np.array_equal(vb, vs), k


# ------------------------------------------------------- single-site solvent
def test_single_site_solvent_mixture(oracle):
    """One-site LJ solvent atoms mixed into water (the reference's separate
    solvent-block path) go through the general atom path: forces and energies
    against the oracle with PME, then stable stepping."""
    s = systems.water_with_single_sites(1500, 3.6, 300, seed=9)
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (36, 36, 36)
    e = make(s, grid=grid, cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa)
    e.compute_forces(energy=True)
    fr, er = oracle_total(oracle, s, 1.0, 2, kappa, grid=grid)
    assert rel_rms(e.forces(), fr) < FORCE_TOL
    check_energies(e.energies(), er, keys=["lj", "coulomb_real", "pme_recip", "bond", "angle"])
    e.step(50)
    assert np.isfinite(e.energies()["total"])


# ------------------------------------------------------------ charge spreading
def test_spread_after_drift_fine_grid(oracle):
    """Charges are spread by blocks of pair-search columns into shared-memory
    boxes; atoms that drifted since the list build may fall outside their
    block's box and go to the grid directly.  A fine grid (0.025 nm: boxes of
    42 x 42 nodes in chunks of 14 z nodes) after nine steps without a rebuild
    exercises both routes; forces and the reciprocal energy against the oracle
    at the current positions."""
    s = small_water(n_waters=900, box=3.0)
    kappa = kappa_from_tol(1.0, 1e-5)
    grid = (120, 120, 120)
    e = make(s, grid=grid, cutoff=1.0, electrostatics=E.ES_EWALD, ewald_kappa=kappa, nstlist=10)
    e.step(9)
    pos, vel = e.state()
    e.compute_forces(energy=True)
    s2 = systems.System(**{**s.__dict__, "pos": pos, "vel": vel})
    fr, er = oracle_total(oracle, s2, 1.0, 2, kappa, grid=grid)
    assert rel_rms(e.forces(), fr) < FORCE_TOL
    check_energies(e.energies(), er, keys=["pme_recip", "coulomb_real", "lj"])
