"""Compound grouping and the reference's compound neighbour rule, on the CPU.

The reference evaluates atom pairs inside a compound and across bonded
compounds without a cutoff, and all other pairs only between compounds its
neighbour list names (Neighborlists.cuh:64-79: any of the 2 x 2 key-particle
distances below cutoff + radius_left + radius_right).  These tests check the
grouping against the reference's rules on the benchmark systems and that every
atom pair within the cutoff lies in a compound pair the rule lists, so that
the reference's evaluated pair set at a list build equals the set of pairs
within the cutoff that this engine evaluates.
"""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from lima_b200 import compounds, systems
from oracle import oracle as O


def test_water_is_one_compound_per_molecule():
    s = systems.water_box(300, 2.5, seed=3).with_compounds()
    assert s.compound.max() + 1 == 300
    assert np.array_equal(np.bincount(s.compound), np.full(300, 3))
    assert len(s.bonded_compounds) == 0
    # every intra-compound pair of a water shares a bond or the angle: no immediate pair
    assert len(O.immediate_pairs(s.compound, s.bonded_compounds, s.exclusions())) == 0


def test_tinymols_belong_to_no_compound():
    s = systems.water_box(50, 2.0, seed=3)
    c, b = compounds.build_compounds(s, tinymol_max_atoms=3)
    assert (c == -1).all() and len(b) == 0


def test_chain_splits_into_two_bonded_compounds():
    """A 52-atom chain exceeds the 32-atom compound: two compounds (32 + 20), one
    bonded pair; config 1 then has 4,500 + 128 compounds."""
    s = systems.config1().with_compounds()
    n_chain = 64 * systems.CHAIN_ATOMS
    cc = s.compound[:n_chain]
    sizes = np.bincount(cc)
    assert len(sizes) == 128 and set(sizes[0::2]) == {32} and set(sizes[1::2]) == {20}
    assert s.compound.max() + 1 == 4628
    assert len(s.bonded_compounds) == 64
    assert (s.bonded_compounds[:, 1] - s.bonded_compounds[:, 0] == 1).all()
    # each compound's atoms form a connected piece of the chain's bond graph
    bonds = s.bonds[: 64 * 51]
    for c in range(2):
        atoms = set(np.nonzero(cc == c)[0])
        adj = {a: [] for a in atoms}
        for a, b in bonds:
            if a in atoms and b in atoms:
                adj[a].append(b)
                adj[b].append(a)
        seen, st = set(), [min(atoms)]
        while st:
            x = st.pop()
            if x not in seen:
                seen.add(x)
                st.extend(adj[x])
        assert seen == atoms
    imm = O.immediate_pairs(s.compound, s.bonded_compounds, s.exclusions())
    # 52 atoms: C(52,2) = 1326 pairs per chain minus its excluded pairs
    ex_chain = s.exclusions()
    ex_chain = ex_chain[ex_chain[:, 1] < n_chain]
    assert len(imm) == 64 * 1326 - len(ex_chain)


def _check_neighbour_rule(s, rc):
    s = s.with_compounds()
    L = float(s.box[0])
    assert np.allclose(s.box, L), "the reference's box is cubic"
    keys, radii = compounds.interaction_boundaries(s, s.compound)
    tree = cKDTree(np.mod(s.pos, s.box), boxsize=s.box)
    pairs = tree.query_pairs(rc, output_type="ndarray")
    ci, cj = s.compound[pairs[:, 0]], s.compound[pairs[:, 1]]
    cp = np.unique(np.sort(np.stack([ci, cj], 1), 1), axis=0)
    cp = cp[cp[:, 0] != cp[:, 1]]
    bonded = {tuple(b) for b in np.sort(s.bonded_compounds, 1)}
    cp = np.array([p for p in cp if tuple(p) not in bonded])
    pos = np.mod(s.pos, s.box)
    kl = pos[keys[cp[:, 0]]].reshape(-1, 6)
    kr = pos[keys[cp[:, 1]]].reshape(-1, 6)
    listed = O.compounds_interact(kl, kr, radii[cp[:, 0]], radii[cp[:, 1]], L, rc)
    return len(pairs), len(cp), int((~listed).sum())


@pytest.mark.parametrize("name,make,rc", [("C0", lambda: systems.water_box(1000, 3.0, seed=5), 1.2),
                                          ("C1", lambda: systems.lipid_slab(box=(8.0, 8.0, 8.0)), 1.2),
                                          ("C2", systems.config2, 1.0)])
def test_every_pair_within_cutoff_lies_in_a_listed_compound_pair(name, make, rc):
    """Reference-representable boxes (integer cubes): C0 in 3 nm, C1's molecules in an
    8 nm cube, C2 as specified."""
    n_pairs, n_cpairs, missing = _check_neighbour_rule(make(), rc)
    assert n_pairs > 0 and n_cpairs > 0
    assert missing == 0, f"{name}: {missing} of {n_cpairs} compound pairs holding in-cutoff atom pairs not listed"
