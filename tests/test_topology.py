"""Topology ingestion (.gro / .top / .itp) on the CPU: round trips of the
engine's own systems, type-table resolution with the reference's unit
conventions, and (when the reference tree is present) its example inputs."""
import math
import os

import numpy as np
import pytest

from lima_b200 import systems, topology

# the reference source tree, when a copy is at hand (its example inputs are read)
REF = os.environ.get("LIMA_REFERENCE_DIR", "")


def test_gro_round_trip(tmp_path):
    s = systems.water_box(200, 2.5, seed=2)
    p = str(tmp_path / "w.gro")
    topology.write_gro_system(p, s)
    g = topology.read_gro(p)
    assert np.allclose(g.pos, s.pos, atol=6e-4)
    assert np.allclose(g.vel * 1000.0, s.vel, atol=0.06)
    assert np.allclose(g.box, s.box)


def test_top_round_trip_chains(tmp_path):
    s = systems.water_with_chains(3000, 2, seed=3)
    tp, gp = str(tmp_path / "s.top"), str(tmp_path / "s.gro")
    topology.write_top(tp, s)
    topology.write_gro_system(gp, s)
    r = topology.load(gp, tp)
    assert r.n == s.n
    assert np.allclose(r.charge, s.charge, rtol=1e-6, atol=1e-6)
    assert np.allclose(r.mass, s.mass, rtol=1e-6)
    assert np.allclose(r.sigma, s.sigma, atol=1e-6) and np.allclose(r.epsilon, s.epsilon, rtol=1e-6)
    for a, b in ((r.bonds, s.bonds), (r.angles, s.angles), (r.dihedrals, s.dihedrals),
                 (r.impropers, s.impropers), (r.pairbonds, s.pairbonds)):
        assert np.array_equal(a, b)
    for a, b in ((r.bond_par, s.bond_par), (r.angle_par, s.angle_par), (r.dihedral_par, s.dihedral_par),
                 (r.improper_par, s.improper_par), (r.pair_par, s.pair_par)):
        assert np.allclose(a, b, rtol=1e-5, atol=1e-6)


FF = """
[ defaults ]
1 2 yes 0.5 0.8333
[ atomtypes ]
CA  6 12.011 0.0 A 0.34 0.36
HA  1 1.008  0.0 A 0.25 0.12
OX  8 15.999 0.0 A 0.30 0.50
[ bondtypes ]
CA CA 1 0.150 2.0e5
CA HA 1 0.109 3.0e5
[ angletypes ]
HA CA CA 5 110.0 300.0 0.21 15000.0
CA CA CA 1 112.0 450.0
[ dihedraltypes ]
X  CA CA X  9 0.0 1.2 3
HA CA CA HA 9 180.0 0.5 2
HA CA CA HA 9 0.0 0.3 3
CA X  X  OX 2 0.0 400.0
[ pairtypes ]
HA HA 1 0.22 0.05
"""

MOL = """
#include "ff.itp"
#define FLEX
[ moleculetype ]
MOL 3
[ atoms ]
1 HA 1 MOL H1 1  0.10
2 CA 1 MOL C1 1 -0.20
3 CA 1 MOL C2 1  0.15
4 HA 1 MOL H2 1 -0.05 1.5
5 OX 1 MOL O1 1  0.00
[ bonds ]
1 2 1
2 3 1
3 4 1
#ifdef FLEX
2 5 1 0.14 1.0e5
#else
2 5 1 0.99 9.9e9
#endif
[ pairs ]
1 4 1
[ angles ]
1 2 3 5
2 3 4 5
[ dihedrals ]
1 2 3 4 9
2 3 4 5 2
[ exclusions ]
1 5
[ system ]
test
[ molecules ]
MOL 2
"""


def test_type_tables_and_units(tmp_path):
    (tmp_path / "ff.itp").write_text(FF)
    (tmp_path / "m.top").write_text(MOL)
    n = 10
    g = topology.GroFile("t", [1] * n, ["MOL"] * n, ["X"] * n, np.random.default_rng(0).uniform(0, 2, (n, 3)),
                         None, np.array([3.0, 3.0, 3.0]))
    s = topology.build_system(topology.read_top(str(tmp_path / "m.top")), g)
    assert s.n == 10 and len(s.bonds) == 8 and len(s.angles) == 4
    kj = 1000.0
    assert np.allclose(s.bond_par[0], [0.109, 3.0e5 * kj])          # HA-CA reversed lookup
    assert np.allclose(s.bond_par[3], [0.14, 1.0e5 * kj])           # explicit, #ifdef branch taken
    th = s.angle_par[0]
    assert np.allclose(th, [110.0 * math.pi / 180, 300.0 * kj, 0.21, 15000.0 * kj])
    # HA-CA-CA-HA: the two exact lines win over the wildcard; constants halved on load
    d = s.dihedral_par[:2]
    assert len(s.dihedrals) == 4
    assert np.allclose(sorted(d[:, 1]), sorted([0.5 * kj / 2, 0.3 * kj / 2]))
    assert np.allclose(s.improper_par[0], [0.0, 400.0 * kj])
    assert np.allclose(s.pair_par[0], [0.22, 0.05 * kj])            # from [ pairtypes ]
    assert np.allclose(s.mass[:5], [1.008e-3, 12.011e-3, 12.011e-3, 1.5e-3, 15.999e-3])
    assert np.allclose(s.charge[:5] / systems.E_TO_KCMOL, [0.10, -0.20, 0.15, -0.05, 0.0], atol=1e-7)
    assert np.array_equal(s.extra_exclusions, [[0, 4], [5, 9]])
    assert np.allclose(s.epsilon[0], 0.12 * kj) and np.allclose(s.sigma[1], 0.34)


def test_unknown_atom_type_is_an_error(tmp_path):
    (tmp_path / "ff.itp").write_text(FF)
    (tmp_path / "m.top").write_text(MOL.replace("5 OX 1 MOL O1 1  0.00", "5 QQ 1 MOL O1 1  0.00"))
    g = topology.GroFile("t", [1] * 10, ["MOL"] * 10, ["X"] * 10, np.zeros((10, 3)), None, np.array([3.0, 3.0, 3.0]))
    with pytest.raises(KeyError, match="QQ"):
        topology.build_system(topology.read_top(str(tmp_path / "m.top")), g)


@pytest.mark.skipif(not (REF and os.path.isdir(REF)), reason="LIMA_REFERENCE_DIR not set to the reference tree")
def test_reference_example_inputs():
    top_path = os.path.join(REF, "tests/userinterfacetests/test.top")
    gro_path = os.path.join(REF, "tests/userinterfacetests/test.gro")
    ffdir = os.path.join(REF, "resources/forcefields")
    s = topology.load(gro_path, top_path, include_dirs=[ffdir])
    g = topology.read_gro(gro_path)
    assert s.n == len(g.pos) > 0
    assert len(s.bonds) > 0 and len(s.angles) > 0 and len(s.dihedrals) > 0
    assert np.all(s.mass > 0) and np.all(np.isfinite(s.bond_par)) and np.all(np.isfinite(s.dihedral_par))
    # the molecule is neutral or carries an integer charge
    qe = s.charge.sum() / systems.E_TO_KCMOL
    assert abs(qe - round(qe)) < 1e-3
