"""Seeded synthetic systems for the force/integration path.

The reference's benchmark inputs live in an external data directory that is
not distributed, so every workload here is generated from a seed with the
shapes, sizes and parameter distributions of the named configurations.

Units are LIMA's own (code/LIMA_BASE/include/Constants.h:43-60): nm, ns,
kg/mol, kC/mol, J/mol.  Exclusions follow the reference rule that every atom
pair sharing a bonded term is excluded from LJ and Coulomb
(code/LIMA_TOOLS/src/CompoundBuilder.cpp:40-60).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

E_TO_KCMOL = 1.602176634e-19 * 6.02214076e23 / 1000.0   # Constants.h:60
KB_J_MOL_K = 1.380649e-23 * 6.02214076e23               # J/mol/K
KJ = 1000.0                                              # kJ -> J (Forcefield.cpp:341-347)
DEG = math.pi / 180.0

# flexible 3-site water (all sizes in LIMA units)
WATER = dict(r_oh=0.09572, theta=104.52 * DEG, kb=345000.0 * KJ, kth=383.0 * KJ,
             q_o=-0.834 * E_TO_KCMOL, q_h=0.417 * E_TO_KCMOL,
             sig_o=0.3151, eps_o=0.6364 * KJ, m_o=15.9994e-3, m_h=1.008e-3)


@dataclass
class System:
    """Flat description of one system, in the reference's units."""
    box: np.ndarray                       # (3,) nm
    pos: np.ndarray                       # (n,3) float64 nm
    vel: np.ndarray                       # (n,3) float32 nm/ns
    charge: np.ndarray                    # (n,) float32 kC/mol
    mass: np.ndarray                      # (n,) float32 kg/mol
    sigma: np.ndarray                     # (n,) float32 nm
    epsilon: np.ndarray                   # (n,) float32 J/mol
    bonds: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    bond_par: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.float32))
    angles: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))
    angle_par: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.float32))
    dihedrals: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    dihedral_par: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.float32))
    impropers: np.ndarray = field(default_factory=lambda: np.zeros((0, 4), np.int32))
    improper_par: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.float32))
    pairbonds: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    pair_par: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.float32))
    name: str = ""
    # pairs excluded beyond those sharing a bonded term (e.g. a topology's [ exclusions ])
    extra_exclusions: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.int32))
    # compound of each atom (-1: none) and bonded compound pairs (lima_b200.compounds);
    # None: not set
    compound: np.ndarray | None = None
    bonded_compounds: np.ndarray | None = None

    def with_compounds(self, tinymol_max_atoms: int = 0) -> "System":
        """This system with the reference builder's compound grouping attached."""
        from dataclasses import replace

        from .compounds import build_compounds
        c, b = build_compounds(self, tinymol_max_atoms)
        return replace(self, compound=c, bonded_compounds=b)

    @property
    def n(self) -> int:
        return len(self.pos)

    def exclusions(self) -> np.ndarray:
        """Unique (i<j) atom pairs sharing any bond, angle, dihedral or improper."""
        pairs = []
        for terms in (self.bonds, self.angles, self.dihedrals, self.impropers, self.extra_exclusions):
            t = np.asarray(terms)
            if len(t) == 0:
                continue
            t = t.reshape(len(t), -1)
            k = t.shape[1]
            for a in range(k):
                for b in range(a + 1, k):
                    pairs.append(np.stack([t[:, a], t[:, b]], 1))
        if not pairs:
            return np.zeros((0, 2), np.int32)
        p = np.concatenate(pairs).astype(np.int64)
        p = np.sort(p, axis=1)
        p = p[p[:, 0] != p[:, 1]]
        p = np.unique(p, axis=0)
        return p.astype(np.int32)


def _random_rotations(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform random rotation matrices from uniform unit quaternions."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], 1)


def maxwell_boltzmann(rng: np.random.Generator, mass: np.ndarray, temperature: float) -> np.ndarray:
    """Velocities [nm/ns == m/s] at temperature [K] with the centre-of-mass motion removed."""
    sd = np.sqrt(KB_J_MOL_K * temperature / mass.astype(np.float64))
    v = rng.normal(size=(len(mass), 3)) * sd[:, None]
    com = (v * mass[:, None]).sum(0) / mass.sum()
    return (v - com).astype(np.float32)


def _water_template() -> np.ndarray:
    r, th = WATER["r_oh"], WATER["theta"]
    h = th / 2
    return np.array([[0.0, 0.0, 0.0],
                     [r * math.sin(h), 0.0, r * math.cos(h)],
                     [-r * math.sin(h), 0.0, r * math.cos(h)]])


def _orient_waters(rng, centres: np.ndarray, fixed: np.ndarray | None, box: np.ndarray,
                   min_dist: float = 0.17, rounds: int = 40, tries: int = 16) -> np.ndarray:
    """Random orientations; a water with an atom closer than min_dist to an atom
    of another molecule (H atoms carry no LJ, so such contacts would blow up the
    first steps) draws `tries` candidate orientations per round and keeps the
    first one that is clear of the current positions of everything else."""
    from scipy.spatial import cKDTree

    nw = len(centres)
    tmpl = _water_template()
    rot = _random_rotations(rng, nw)
    nfix = 0 if fixed is None else len(fixed)
    mol = np.concatenate([-1 - np.arange(nfix), np.repeat(np.arange(nw), 3)])
    wpos = np.einsum("nij,aj->nai", rot, tmpl) + centres[:, None, :]          # (nw, 3, 3)

    def all_pos():
        p = wpos.reshape(-1, 3)
        return np.mod(p if nfix == 0 else np.concatenate([fixed, p]), box)

    tree = cKDTree(all_pos(), boxsize=box)
    pairs = tree.query_pairs(min_dist, output_type="ndarray")
    if len(pairs):
        pairs = pairs[mol[pairs[:, 0]] != mol[pairs[:, 1]]]
    bad = np.unique(mol[pairs.ravel()]) if len(pairs) else np.zeros(0, np.int64)
    bad = bad[bad >= 0]
    for _ in range(rounds):
        if len(bad) == 0:
            break
        cand = _random_rotations(rng, len(bad) * tries).reshape(len(bad), tries, 3, 3)
        pts = np.einsum("btij,aj->btai", cand, tmpl) + centres[bad][:, None, None, :]
        d, idx = tree.query(np.mod(pts.reshape(-1, 3), box), k=4)
        own = mol[idx] == np.repeat(bad, tries * 3)[:, None]
        d = np.where(own, np.inf, d).min(1).reshape(len(bad), tries, 3).min(2)
        ok = d >= min_dist
        pick = np.where(ok.any(1), ok.argmax(1), 0)
        rot[bad] = cand[np.arange(len(bad)), pick]
        wpos[bad] = pts[np.arange(len(bad)), pick]
        # re-check only the waters that moved, against everything at its new place
        tree = cKDTree(all_pos(), boxsize=box)
        moved = np.mod(wpos[bad].reshape(-1, 3), box)
        hits = tree.query_ball_point(moved, min_dist)
        still = np.zeros(len(bad), bool)
        for k, h in enumerate(hits):
            w = bad[k // 3]
            if any(mol[j] != w for j in h):
                still[k // 3] = True
        # neighbours hit by a moved water are re-drawn too
        bad = bad[still]
    return rot


def _append_waters(rng, centres: np.ndarray, first_atom: int, box=None, fixed=None):
    """Atoms, bonds and angles for waters whose oxygens sit at centres."""
    nw = len(centres)
    if box is None:
        rot = _random_rotations(rng, nw)
    else:
        rot = _orient_waters(rng, centres, fixed, np.asarray(box, dtype=np.float64))
    tmpl = _water_template()
    pos = (np.einsum("nij,aj->nai", rot, tmpl) + centres[:, None, :]).reshape(-1, 3)
    base = first_atom + 3 * np.arange(nw)
    bonds = np.concatenate([np.stack([base, base + 1], 1), np.stack([base, base + 2], 1)])
    bonds = bonds.reshape(2, nw, 2).transpose(1, 0, 2).reshape(-1, 2)
    angles = np.stack([base + 1, base, base + 2], 1)
    q = np.tile([WATER["q_o"], WATER["q_h"], WATER["q_h"]], nw)
    m = np.tile([WATER["m_o"], WATER["m_h"], WATER["m_h"]], nw)
    s = np.tile([WATER["sig_o"], 0.0, 0.0], nw)
    e = np.tile([WATER["eps_o"], 0.0, 0.0], nw)
    bpar = np.tile([WATER["r_oh"], WATER["kb"]], (len(bonds), 1))
    apar = np.tile([WATER["theta"], WATER["kth"], 0.0, 0.0], (nw, 1))
    return pos, q, m, s, e, bonds, bpar, angles, apar


def solvate_sites(rng, box: np.ndarray, occupied: np.ndarray, n_waters: int, clearance: float = 0.3,
                  jitter: float = 0.02) -> np.ndarray:
    """n_waters oxygen sites on a jittered cubic lattice that keep `clearance`
    from occupied atoms; the lattice is refined until enough sites are free."""
    from scipy.spatial import cKDTree

    tree = cKDTree(np.mod(occupied, box), boxsize=box)
    free_vol = float(np.prod(box)) * 0.6
    spacing = (free_vol / n_waters) ** (1.0 / 3.0)
    for _ in range(60):
        n = np.maximum(1, np.floor(box / spacing)).astype(int)
        g = [(np.arange(n[d]) + 0.5) * box[d] / n[d] for d in range(3)]
        sites = np.stack(np.meshgrid(*g, indexing="ij"), -1).reshape(-1, 3)
        d, _ = tree.query(sites, k=1)
        sites = sites[d > clearance]
        if len(sites) >= n_waters:
            sites = sites[np.sort(rng.choice(len(sites), n_waters, replace=False))]
            return sites + rng.uniform(-jitter, jitter, size=sites.shape)
        spacing *= 0.985
    raise RuntimeError("cannot place the requested number of waters")


def _lattice_sites(n_per_dim, box, jitter, rng):
    g = (np.arange(n_per_dim) + 0.5) / n_per_dim
    pts = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) * box
    return pts + rng.uniform(-jitter, jitter, size=pts.shape)


def water_box(n_waters: int, box_nm: float, seed: int = 20241203, jitter: float = 0.02,
              temperature: float = 300.0, name: str = "water") -> System:
    """Flexible 3-site waters on a jittered cubic lattice (config 0 and 2)."""
    rng = np.random.default_rng(seed)
    box = np.array([box_nm] * 3, dtype=np.float64)
    per = int(math.ceil(n_waters ** (1.0 / 3.0) - 1e-9))
    sites = _lattice_sites(per, box, jitter, rng)
    if len(sites) > n_waters:
        sites = sites[np.sort(rng.choice(len(sites), n_waters, replace=False))]
    pos, q, m, s, e, bonds, bpar, angles, apar = _append_waters(rng, sites, 0, box=box)
    pos = np.mod(pos, box)
    vel = maxwell_boltzmann(rng, m, temperature)
    return System(box=box, pos=pos, vel=vel, charge=q.astype(np.float32), mass=m.astype(np.float32),
                  sigma=s.astype(np.float32), epsilon=e.astype(np.float32),
                  bonds=bonds.astype(np.int32), bond_par=bpar.astype(np.float32),
                  angles=angles.astype(np.int32), angle_par=apar.astype(np.float32), name=name)


def water_with_single_sites(n_waters: int, box_nm: float, n_sites: int, seed: int = 20241203,
                            temperature: float = 300.0) -> System:
    """Flexible water in which n_sites molecules are replaced by single-site,
    LJ-only solvent atoms (argon-like: sigma 0.3405 nm, eps 0.996 kJ/mol, no
    charge) at their oxygen positions.  The reference treats such one-site
    molecules on a separate solvent-block path; here they are ordinary atoms
    without bonded terms."""
    rng = np.random.default_rng(seed + 17)
    w = water_box(n_waters, box_nm, seed=seed, temperature=temperature)
    nw = w.n // 3
    swap = np.sort(rng.choice(nw, n_sites, replace=False))
    keep_mol = np.ones(nw, bool)
    keep_mol[swap] = False
    keep_atoms = np.repeat(keep_mol, 3)
    new_index = -np.ones(w.n, np.int64)
    new_index[keep_atoms] = np.arange(int(keep_atoms.sum()))
    bmask = keep_atoms[w.bonds[:, 0]]
    amask = keep_atoms[w.angles[:, 0]]
    site_pos = w.pos[3 * swap]
    mass = np.float32(39.948e-3)
    site_vel = maxwell_boltzmann(rng, np.full(n_sites, mass, np.float32), temperature).astype(np.float32)
    return System(box=w.box, pos=np.concatenate([w.pos[keep_atoms], site_pos]),
                  vel=np.concatenate([w.vel[keep_atoms], site_vel]),
                  charge=np.concatenate([w.charge[keep_atoms], np.zeros(n_sites, np.float32)]),
                  mass=np.concatenate([w.mass[keep_atoms], np.full(n_sites, mass, np.float32)]),
                  sigma=np.concatenate([w.sigma[keep_atoms], np.full(n_sites, 0.3405, np.float32)]),
                  epsilon=np.concatenate([w.epsilon[keep_atoms], np.full(n_sites, 0.996 * KJ, np.float32)]),
                  bonds=new_index[w.bonds[bmask]].astype(np.int32), bond_par=w.bond_par[bmask],
                  angles=new_index[w.angles[amask]].astype(np.int32), angle_par=w.angle_par[amask],
                  name="water_single_sites")


# ------------------------------------------------------------ lipid-like chains
CHAIN_HEAD = 8
CHAIN_TAIL = 22
CHAIN_ATOMS = CHAIN_HEAD + 2 * CHAIN_TAIL   # 52
CHAIN = dict(b0=0.153, kb=2.2e5 * KJ, theta0=111.0 * DEG, kth=460.0 * KJ, kphi=0.6 * KJ, mult=3.0,
             phi0=0.0, mass=12.011e-3)


def chain_topology():
    """Bond graph of one 52-atom chain: an 8-atom linear head (0..7), tail A
    (8..29) attached to head atom 6 and tail B (30..51) to head atom 7; every
    angle and proper dihedral along the bond paths."""
    bonds = [(i, i + 1) for i in range(CHAIN_HEAD - 1)]
    a0, b0 = CHAIN_HEAD, CHAIN_HEAD + CHAIN_TAIL
    bonds.append((6, a0))
    bonds += [(a0 + i, a0 + i + 1) for i in range(CHAIN_TAIL - 1)]
    bonds.append((7, b0))
    bonds += [(b0 + i, b0 + i + 1) for i in range(CHAIN_TAIL - 1)]
    nb = [[] for _ in range(CHAIN_ATOMS)]
    for i, j in bonds:
        nb[i].append(j)
        nb[j].append(i)
    angles = []
    for j in range(CHAIN_ATOMS):
        for x in range(len(nb[j])):
            for y in range(x + 1, len(nb[j])):
                angles.append((nb[j][x], j, nb[j][y]))
    dihedrals = []
    for j, k in bonds:
        for i in nb[j]:
            if i == k:
                continue
            for l in nb[k]:
                if l == j or l == i:
                    continue
                dihedrals.append((i, j, k, l))
    return (np.array(bonds, np.int32), np.array(angles, np.int32), np.array(dihedrals, np.int32))


def _zigzag(p0, axis, zig, n):
    """n atoms of an all-trans strand after p0: bonds of b0, bond angles theta0,
    advancing along `axis` and zig-zagging along `zig` (both unit, orthogonal)."""
    b = CHAIN["b0"]
    hang = CHAIN["theta0"] / 2
    dz, zz = b * math.sin(hang), 0.5 * b * math.cos(hang)
    return np.array([p0 + m * dz * axis + ((-1) ** m - 1) * zz * zig for m in range(1, n + 1)])


def _chain_geometry(up: bool, half: float) -> np.ndarray:
    """One chain around the origin with every bond at b0.  Each tail is a
    hairpin: an all-trans strand of 10 atoms, a 2-atom turn, a second strand
    of 10; tail A's strands sit at x = +half, y = +-half, tail B's at
    x = -half.  Head atoms 6 and 7 sit a bond from the first atoms of tails A
    and B, at the bond angle to the tails' first bonds, and a bond apart;
    atoms 5..0 continue from atom 6 outwards, every bond angle at theta0."""
    b = CHAIN["b0"]
    hang = CHAIN["theta0"] / 2
    dz = b * math.sin(hang)           # axial advance per bond of an all-trans strand
    zz = 0.5 * b * math.cos(hang)     # lateral zig-zag amplitude
    sgn = -1.0 if up else 1.0         # tails grow away from the head
    strand = (CHAIN_TAIL - 2) // 2    # 10 atoms per strand, 2 in the turn
    pos = np.zeros((CHAIN_ATOMS, 3))
    # turn atoms at y = +-b/2 on the strands' x line, offset along the tail so
    # that their bonds to the strand ends are b: zz^2 + (half - b/2)^2 + e^2 = b^2
    e_turn = math.sqrt(max(b * b - zz * zz - (half - 0.5 * b) ** 2, 1e-4))
    z_end = sgn * dz * (strand - 1)
    for start, x0, side in ((CHAIN_HEAD, half, 1.0), (CHAIN_HEAD + CHAIN_TAIL, -half, -1.0)):
        for k in range(CHAIN_TAIL):
            if k < strand or k >= CHAIN_TAIL - strand:
                kk = k if k < strand else (CHAIN_TAIL - 1 - k)
                y0 = half if k < strand else -half
                # the zig-zag starts towards the chain's centre line on both tails
                pos[start + k] = [x0 + side * (zz if kk % 2 else -zz), y0, sgn * dz * kk]
            else:
                yt = 0.5 * b if k == strand else -0.5 * b
                pos[start + k] = [x0, yt, z_end + sgn * e_turn]
    # head atoms 6 and 7, a bond apart, each a bond from its tail's first atom
    # at the bond angle theta0 to the tail's first bond: on the cone of such
    # points, the one at x = +-b/2 on the outer (+y) side
    def attach(first, second, x_target):
        w = (second - first) / b
        e1 = np.cross(w, [0.0, 1.0, 0.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(w, e1)
        phis = np.linspace(-math.pi, math.pi, 20001)
        c, s_ = math.cos(CHAIN["theta0"]), math.sin(CHAIN["theta0"])
        pts = first + b * (c * w[None, :] + s_ * (np.cos(phis)[:, None] * e1 + np.sin(phis)[:, None] * e2))
        ok = pts[:, 1] > first[1]
        k = np.argmin(np.where(ok, np.abs(pts[:, 0] - x_target), np.inf))
        return pts[k]
    ta, tb = pos[CHAIN_HEAD], pos[CHAIN_HEAD + CHAIN_TAIL]
    p6 = attach(ta, pos[CHAIN_HEAD + 1], 0.5 * b)
    p7 = attach(tb, pos[CHAIN_HEAD + CHAIN_TAIL + 1], -0.5 * b)
    pos[6], pos[7] = p6, p7
    u = (p6 - p7) / np.linalg.norm(p6 - p7)
    # atoms 5..0: each a bond from the previous at the bond angle theta0 to the
    # previous bond, at the azimuth (of 72 tried) that advances furthest along
    # the leaflet's outward normal among those at least 0.3 nm from every atom
    # placed so far (a deterministic walk away from the tails)
    out = np.array([0.0, 0.0, -sgn])
    placed = [i for i in range(6, CHAIN_ATOMS)]
    prev, cur = ta, p6
    c, s_ = math.cos(CHAIN["theta0"]), math.sin(CHAIN["theta0"])
    for m in range(5, -1, -1):
        w = (prev - cur) / np.linalg.norm(prev - cur)
        e1 = np.cross(w, out if abs(np.dot(w, out)) < 0.9 else [1.0, 0.0, 0.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(w, e1)
        best, best_score = None, -1e9
        for phi in np.linspace(0.0, 2 * math.pi, 72, endpoint=False):
            cand = cur + b * (c * w + s_ * (math.cos(phi) * e1 + math.sin(phi) * e2))
            dmin = np.linalg.norm(pos[placed] - cand, axis=1).min()
            score = np.dot(cand - cur, out) - (10.0 if dmin < 0.3 else 0.0)
            if score > best_score:
                best, best_score = cand, score
        pos[m] = best
        placed.append(m)
        prev, cur = cur, best
    return pos


def lipid_slab(n_chains: int = 64, n_waters: int = 4500, box=(5.0, 5.0, 8.0),
               seed: int = 20241203, temperature: float = 300.0) -> System:
    """Config 1: two leaflets of lipid-like chains solvated by flexible water.

    Sizes, charges and force-field parameters follow the named configuration.
    The two leaflets interdigitate (the lower leaflet's strands sit in the
    gaps of the upper one's) so that 3,328 chain atoms and 4,500 waters fit
    the 5 x 5 x 8 nm box near normal density."""
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=np.float64)
    cb, ca, cd = chain_topology()
    per_leaflet = n_chains // 2
    nx = int(math.ceil(math.sqrt(per_leaflet)))
    d = box[0] / nx                   # chain spacing
    half = d / 4                      # strands on a uniform d/2 lattice
    sites = [(ix, iy) for ix in range(nx) for iy in range(nx)][:per_leaflet]
    # depth of a tail below its chain's top (strand plus turn), and 0.35 nm of
    # clearance between one leaflet's tail turns and the other's head atoms
    g0 = _chain_geometry(True, half)
    strand_len = float(-g0[CHAIN_HEAD:, 2].min()) + 0.35
    zc = box[2] / 2
    z_top = zc + 0.5 * strand_len     # upper tails hang down from here
    z_bot = zc - 0.5 * strand_len     # lower tails rise from here
    pos_l, q_l, s_l, e_l = [], [], [], []
    bonds, angles, dihedrals = [], [], []
    for leaflet in range(2):
        up = leaflet == 0
        geo = _chain_geometry(up, half)
        off_xy = 0.0 if up else d / 4
        for ix, iy in sites:
            off = len(pos_l) * CHAIN_ATOMS
            shift = np.array([(ix + 0.5) * d + off_xy, (iy + 0.5) * box[1] / nx + off_xy,
                              z_top if up else z_bot])
            pos_l.append(geo + shift)
            hq = rng.normal(0.0, 0.4, CHAIN_HEAD)
            hq -= hq.mean()
            q = np.zeros(CHAIN_ATOMS)
            q[:CHAIN_HEAD] = hq * E_TO_KCMOL
            q_l.append(q)
            s_l.append(rng.uniform(0.30, 0.39, CHAIN_ATOMS))
            e_l.append(rng.uniform(0.2, 0.9, CHAIN_ATOMS) * KJ)
            bonds.append(cb + off)
            angles.append(ca + off)
            dihedrals.append(cd + off)
    lip_pos = np.concatenate(pos_l)
    n_lip = len(lip_pos)
    # water fills the space the chains leave free
    cand = solvate_sites(rng, box, lip_pos, n_waters)
    wpos, wq, wm, ws, we, wb, wbp, wa, wap = _append_waters(rng, cand, n_lip, box=box, fixed=lip_pos)
    n_b = sum(len(b) for b in bonds)
    n_a = sum(len(a) for a in angles)
    n_d = sum(len(d) for d in dihedrals)
    pos = np.mod(np.concatenate([lip_pos, wpos]), box)
    charge = np.concatenate([np.concatenate(q_l), wq])
    mass = np.concatenate([np.full(n_lip, CHAIN["mass"]), wm])
    sigma = np.concatenate([np.concatenate(s_l), ws])
    eps = np.concatenate([np.concatenate(e_l), we])
    bond_par = np.concatenate([np.tile([CHAIN["b0"], CHAIN["kb"]], (n_b, 1)), wbp])
    angle_par = np.concatenate([np.tile([CHAIN["theta0"], CHAIN["kth"], 0.0, 0.0], (n_a, 1)), wap])
    dih_par = np.tile([CHAIN["phi0"], CHAIN["kphi"], CHAIN["mult"]], (n_d, 1))
    vel = maxwell_boltzmann(rng, mass, temperature)
    return System(box=box, pos=pos, vel=vel, charge=charge.astype(np.float32),
                  mass=mass.astype(np.float32), sigma=sigma.astype(np.float32),
                  epsilon=eps.astype(np.float32),
                  bonds=np.concatenate(bonds + [wb]).astype(np.int32), bond_par=bond_par.astype(np.float32),
                  angles=np.concatenate(angles + [wa]).astype(np.int32), angle_par=angle_par.astype(np.float32),
                  dihedrals=np.concatenate(dihedrals).astype(np.int32), dihedral_par=dih_par.astype(np.float32),
                  name="lipid_slab")


def ewald_kappa(cutoff: float, tol: float) -> float:
    """kappa with erfc(kappa*rc) = tol (bisection)."""
    lo, hi = 0.0, 20.0 / cutoff
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if math.erfc(mid * cutoff) > tol:
            lo = mid
        else:
            hi = mid
    return 0.5 * (lo + hi)


def fft_friendly(n: int) -> int:
    """Smallest m >= n whose prime factors are 2, 3 and 5."""
    m = max(n, 4)
    while True:
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        if k == 1:
            return m
        m += 1


# --------------------------------------------------------------- named configs
def config0(seed=20241203):
    """1,000 flexible waters, 3.1 nm cube, LJ + cutoff Coulomb at 1.2 nm."""
    return water_box(1000, 3.1, seed=seed, name="water1k_3.1nm")


def config1(seed=20241203):
    """64 lipid-like chains x 52 atoms + 4,500 waters, 5x5x8 nm, PME 48x48x80."""
    return lipid_slab(seed=seed)


def config2(seed=20241203):
    """33,400 waters (100,200 atoms), 10 nm cube, PME 96^3, cutoff 1.0 nm."""
    return water_box(33400, 10.0, seed=seed, name="water100k_10nm")


def _merge(a: System, b: System) -> System:
    """Concatenates two systems sharing a box (b's indices shifted)."""
    off = a.n
    cat = lambda x, y: np.concatenate([x, y]) if len(x) or len(y) else x
    sh = lambda t: (t + off).astype(np.int32) if len(t) else t
    return System(box=a.box, pos=np.concatenate([a.pos, b.pos]), vel=np.concatenate([a.vel, b.vel]),
                  charge=cat(a.charge, b.charge), mass=cat(a.mass, b.mass), sigma=cat(a.sigma, b.sigma),
                  epsilon=cat(a.epsilon, b.epsilon),
                  bonds=cat(a.bonds, sh(b.bonds)), bond_par=cat(a.bond_par, b.bond_par),
                  angles=cat(a.angles, sh(b.angles)), angle_par=cat(a.angle_par, b.angle_par),
                  dihedrals=cat(a.dihedrals, sh(b.dihedrals)), dihedral_par=cat(a.dihedral_par, b.dihedral_par),
                  impropers=cat(a.impropers, sh(b.impropers)), improper_par=cat(a.improper_par, b.improper_par),
                  pairbonds=cat(a.pairbonds, sh(b.pairbonds)), pair_par=cat(a.pair_par, b.pair_par), name=a.name)


def _chains(rng, n_chains: int, box: np.ndarray, temperature: float) -> System:
    """n_chains lipid-like chains (config-1 topology and parameters) at random
    positions and orientations."""
    from scipy.spatial import cKDTree

    cb, ca, cd = chain_topology()
    geo = _chain_geometry(True, 0.21)
    geo -= geo.mean(0)
    pos, q, s, e, bonds, angles, dihedrals = [], [], [], [], [], [], []
    for c in range(n_chains):
        # a random placement clear of the chains placed before (no atom pair
        # closer than 0.4 nm across chains); the last try is kept if none is
        for _ in range(200):
            cand = np.mod(geo @ _random_rotations(rng, 1)[0].T + rng.uniform(0, 1, 3) * box, box)
            if not pos:
                break
            d, _ = cKDTree(np.concatenate(pos), boxsize=box).query(cand, k=1)
            if d.min() >= 0.4:
                break
        pos.append(cand)
        hq = rng.normal(0.0, 0.4, CHAIN_HEAD)
        hq -= hq.mean()
        qq = np.zeros(CHAIN_ATOMS)
        qq[:CHAIN_HEAD] = hq * E_TO_KCMOL
        q.append(qq)
        s.append(rng.uniform(0.30, 0.39, CHAIN_ATOMS))
        e.append(rng.uniform(0.2, 0.9, CHAIN_ATOMS) * KJ)
        off = c * CHAIN_ATOMS
        bonds.append(cb + off)
        angles.append(ca + off)
        dihedrals.append(cd + off)
    n = n_chains * CHAIN_ATOMS
    mass = np.full(n, CHAIN["mass"], np.float32)
    return System(box=box, pos=np.mod(np.concatenate(pos), box), vel=maxwell_boltzmann(rng, mass, temperature),
                  charge=np.concatenate(q).astype(np.float32), mass=mass,
                  sigma=np.concatenate(s).astype(np.float32), epsilon=np.concatenate(e).astype(np.float32),
                  bonds=np.concatenate(bonds).astype(np.int32),
                  bond_par=np.tile([CHAIN["b0"], CHAIN["kb"]], (len(cb) * n_chains, 1)).astype(np.float32),
                  angles=np.concatenate(angles).astype(np.int32),
                  angle_par=np.tile([CHAIN["theta0"], CHAIN["kth"], 0, 0], (len(ca) * n_chains, 1)).astype(np.float32),
                  dihedrals=np.concatenate(dihedrals).astype(np.int32),
                  dihedral_par=np.tile([CHAIN["phi0"], CHAIN["kphi"], CHAIN["mult"]],
                                       (len(cd) * n_chains, 1)).astype(np.float32), name="chains")


def water_with_chains(n_atoms: int, n_chains: int, density: float = 33.4, seed: int = 1,
                      temperature: float = 300.0, name: str = "sys") -> System:
    """A config-0-style water box of about n_atoms atoms (density waters/nm^3)
    with n_chains config-1 chains inserted at random positions; waters with an
    atom within 0.3 nm of a chain atom are removed."""
    from scipy.spatial import cKDTree

    rng = np.random.default_rng(seed)
    n_w = max(8, n_atoms // 3)
    L = (n_w / density) ** (1.0 / 3.0)
    box = np.array([L, L, L])
    w = water_box(n_w, L, seed=seed, temperature=temperature, name=name)
    if n_chains == 0:
        return w
    ch = _chains(rng, n_chains, box, temperature)
    d, _ = cKDTree(ch.pos, boxsize=box).query(np.mod(w.pos, box), k=1)
    bad = np.unique(np.nonzero(d < 0.3)[0] // 3)
    keep = np.setdiff1d(np.arange(w.n // 3), bad)
    atoms = (3 * keep[:, None] + np.arange(3)).ravel()
    remap = -np.ones(w.n, np.int64)
    remap[atoms] = np.arange(len(atoms))
    kb = np.all(np.isin(w.bonds, atoms), axis=1)
    ka = np.all(np.isin(w.angles, atoms), axis=1)
    w2 = System(box=box, pos=w.pos[atoms], vel=w.vel[atoms], charge=w.charge[atoms], mass=w.mass[atoms],
                sigma=w.sigma[atoms], epsilon=w.epsilon[atoms],
                bonds=remap[w.bonds[kb]].astype(np.int32), bond_par=w.bond_par[kb],
                angles=remap[w.angles[ka]].astype(np.int32), angle_par=w.angle_par[ka], name=name)
    return _merge(ch, w2)


def batch_specs(n_systems=256, seed=20241203, lo=1500, hi=30000, density=33.4):
    """Config 4's systems as (index, atom count, chain count, seed, edge [nm]):
    atom counts log-uniform in [lo, hi] from a seed, 0-4 chains each.  Cheap, so
    that every rank of a multi-GPU run can partition the whole batch and then
    generate only its own systems (each system has its own seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_systems):
        n_atoms = int(math.exp(rng.uniform(math.log(lo), math.log(hi))))
        n_chains = int(rng.integers(0, 5))
        n_w = max(8, n_atoms // 3)
        out.append((s, n_atoms, n_chains, seed + 1 + s, (n_w / density) ** (1.0 / 3.0)))
    return out


def batch_system(spec, density=33.4) -> System:
    """One config-4 system from its batch_specs entry."""
    s, n_atoms, n_chains, sseed, _ = spec
    return water_with_chains(n_atoms, n_chains, density, seed=sseed, name=f"batch{s}")


def batch_systems(n_systems=256, seed=20241203, lo=1500, hi=30000, density=33.4):
    """Config 4: atom counts log-uniform in [lo, hi] from a seed; each a water box
    at the given density with 0-4 chains inserted at random positions."""
    return [batch_system(sp, density) for sp in batch_specs(n_systems, seed, lo, hi, density)]
