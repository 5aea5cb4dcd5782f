"""Topology and coordinate ingestion: GROMACS-format .gro / .top / .itp files,
as LIMA reads them, turned into a ``systems.System`` for the engine.

Follows the reference's readers and parameter conventions:
  * .gro fixed columns (code/LIMA_BASE/src/MDFiles.cpp:13-56): residue number
    (5), residue name (5), atom name (5), atom number (5), x y z (8 each, nm),
    optional vx vy vz (8 each, nm/ps); last line: box edges (nm);
  * .top / .itp sections and #include (code/LIMA_BASE/src/Topologyfile.cpp):
    [ atomtypes ] [ bondtypes ] [ pairtypes ] [ angletypes ] [ dihedraltypes ]
    [ moleculetype ] [ atoms ] [ bonds ] [ pairs ] [ angles ] [ dihedrals ]
    [ exclusions ] [ system ] [ molecules ]; ';' comments; #define / #ifdef /
    #ifndef / #else / #endif; parameters on a term's own line take precedence
    over the type tables;
  * unit conversion on load (code/LIMA_BASE/src/Bodies.cpp:9-45): kJ -> J
    (x1000), degrees -> radians, and the proper-dihedral force constant halved
    (DihedralBond::Parameters::CreateFromCharmm), charges e -> kC/mol, masses
    g/mol -> kg/mol, velocities nm/ps -> nm/ns.
Bonded functions: bonds 1 (harmonic), angles 1 (harmonic) and 5 (Urey-Bradley),
dihedrals 1/4/9 (periodic; several matching type lines give several terms) and
2 (harmonic improper), pairs 1 (LJ from [ pairtypes ], else the atom types).
Dihedral type lines match in either direction, exact type names before 'X'
wildcards.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

from .systems import DEG, E_TO_KCMOL as E_KCMOL, KJ, System


# ---------------------------------------------------------------------- .gro
@dataclass
class GroFile:
    title: str
    resid: list
    resname: list
    name: list
    pos: np.ndarray            # (n,3) nm
    vel: np.ndarray | None     # (n,3) nm/ps, or None
    box: np.ndarray            # (3,) nm


def read_gro(path: str) -> GroFile:
    with open(path) as f:
        lines = f.read().splitlines()
    title = lines[0]
    n = int(lines[1].strip())
    resid, resname, name = [], [], []
    pos = np.zeros((n, 3))
    vel = np.zeros((n, 3))
    has_vel = True
    for i in range(n):
        ln = lines[2 + i]
        resid.append(int(ln[0:5]))
        resname.append(ln[5:10].strip())
        name.append(ln[10:15].strip())
        pos[i] = [float(ln[20:28]), float(ln[28:36]), float(ln[36:44])]
        if len(ln) >= 68:
            vel[i] = [float(ln[44:52]), float(ln[52:60]), float(ln[60:68])]
        else:
            has_vel = False
    box = np.array([float(v) for v in lines[2 + n].split()[:3]])
    return GroFile(title, resid, resname, name, pos, vel if has_vel else None, box)


def write_gro(path: str, g: GroFile):
    with open(path, "w") as f:
        f.write(g.title + "\n")
        f.write(f"{len(g.pos):5d}\n")
        for i, p in enumerate(g.pos):
            line = (f"{g.resid[i] % 100000:5d}{g.resname[i]:<5.5s}{g.name[i]:>5.5s}{(i + 1) % 100000:5d}"
                    f"{p[0]:8.3f}{p[1]:8.3f}{p[2]:8.3f}")
            if g.vel is not None:
                v = g.vel[i]
                line += f"{v[0]:8.4f}{v[1]:8.4f}{v[2]:8.4f}"
            f.write(line + "\n")
        f.write(f"{g.box[0]:10.5f}{g.box[1]:10.5f}{g.box[2]:10.5f}\n")


# ---------------------------------------------------------------------- .top
@dataclass
class MoleculeType:
    name: str
    nrexcl: int
    atoms: list = field(default_factory=list)      # (type, charge e, mass g/mol or None, name)
    bonds: list = field(default_factory=list)      # (i, j, func, params[])  0-based
    pairs: list = field(default_factory=list)
    angles: list = field(default_factory=list)
    dihedrals: list = field(default_factory=list)
    exclusions: list = field(default_factory=list)


@dataclass
class Topology:
    atomtypes: dict = field(default_factory=dict)      # name -> (mass, sigma nm, eps kJ/mol)
    bondtypes: dict = field(default_factory=dict)      # (t1, t2, func) -> params
    pairtypes: dict = field(default_factory=dict)      # (t1, t2) -> (sigma, eps)
    angletypes: dict = field(default_factory=dict)     # (t1, t2, t3, func) -> params
    dihedraltypes: list = field(default_factory=list)  # (types4, func, params)
    moleculetypes: dict = field(default_factory=dict)
    molecules: list = field(default_factory=list)      # (name, count)
    fudge_lj: float = 1.0
    system_name: str = ""


def _numbers(tokens):
    out = []
    for t in tokens:
        try:
            out.append(float(t))
        except ValueError:
            break
    return out


def read_top(path: str, include_dirs=(), defines=()) -> Topology:
    """Parses a topology with its #include files (searched next to the including
    file, then in include_dirs)."""
    top = Topology()
    state = {"section": None, "mol": None}
    defs = set(defines)

    def parse_file(p):
        base = os.path.dirname(os.path.abspath(p))
        skip = []          # stack of booleans: inside a false #ifdef branch
        with open(p, encoding="utf-8", errors="replace") as f:
            for raw in f:
                line = raw.split(";", 1)[0].strip()
                if not line:
                    continue
                if line.startswith("#"):
                    words = line.split()
                    d = words[0]
                    if d == "#ifdef":
                        skip.append(words[1] not in defs)
                    elif d == "#ifndef":
                        skip.append(words[1] in defs)
                    elif d == "#else":
                        skip[-1] = not skip[-1]
                    elif d == "#endif":
                        skip.pop()
                    elif any(skip):
                        continue
                    elif d == "#define":
                        defs.add(words[1])
                    elif d == "#include":
                        name = line.split(None, 1)[1].strip().strip('"<>')
                        for cand in [os.path.join(base, name)] + [os.path.join(dd, name) for dd in include_dirs]:
                            if os.path.exists(cand):
                                parse_file(cand)
                                break
                        else:
                            raise FileNotFoundError(f"#include {name} not found from {p}")
                    continue
                if any(skip):
                    continue
                if line.startswith("["):
                    state["section"] = line.strip("[] ").lower()
                    continue
                handle(state["section"], line.split())

    def handle(sec, w):
        mol = state["mol"]
        if sec == "defaults":
            nums = _numbers(w[3:])
            if nums:
                top.fudge_lj = nums[0]
        elif sec == "atomtypes":
            # name [at.num] mass charge ptype sigma epsilon: the ptype letter anchors the columns
            k = next(i for i, t in enumerate(w) if t in ("A", "D", "S", "V"))
            top.atomtypes[w[0]] = (float(w[k - 2]), float(w[k + 1]), float(w[k + 2]))
        elif sec == "bondtypes":
            top.bondtypes[(w[0], w[1], int(w[2]))] = _numbers(w[3:])
        elif sec == "pairtypes":
            top.pairtypes[(w[0], w[1])] = tuple(_numbers(w[3:])[:2])
        elif sec == "angletypes":
            top.angletypes[(w[0], w[1], w[2], int(w[3]))] = _numbers(w[4:])
        elif sec == "dihedraltypes":
            # 4-type form; 2-type forms (older files) name the central pair
            if len(w) >= 5 and not _is_number(w[2]) and not _is_number(w[3]):
                top.dihedraltypes.append(((w[0], w[1], w[2], w[3]), int(w[4]), _numbers(w[5:])))
            else:
                top.dihedraltypes.append((("X", w[0], w[1], "X"), int(w[2]), _numbers(w[3:])))
        elif sec == "moleculetype":
            m = MoleculeType(w[0], int(w[1]) if len(w) > 1 else 3)
            top.moleculetypes[m.name] = m
            state["mol"] = m
        elif sec == "atoms":
            charge = float(w[6]) if len(w) > 6 else 0.0
            mass = float(w[7]) if len(w) > 7 and _is_number(w[7]) else None
            mol.atoms.append((w[1], charge, mass, w[4]))
        elif sec in ("bonds", "pairs"):
            term = (int(w[0]) - 1, int(w[1]) - 1, int(w[2]) if len(w) > 2 else 1, _numbers(w[3:]))
            (mol.bonds if sec == "bonds" else mol.pairs).append(term)
        elif sec == "angles":
            mol.angles.append((int(w[0]) - 1, int(w[1]) - 1, int(w[2]) - 1, int(w[3]) if len(w) > 3 else 1,
                               _numbers(w[4:])))
        elif sec == "dihedrals":
            mol.dihedrals.append(tuple(int(x) - 1 for x in w[:4]) + (int(w[4]) if len(w) > 4 else 1,
                                                                     _numbers(w[5:])))
        elif sec == "exclusions":
            i = int(w[0]) - 1
            for j in w[1:]:
                mol.exclusions.append((i, int(j) - 1))
        elif sec == "system":
            top.system_name = " ".join(w)
        elif sec == "molecules":
            top.molecules.append((w[0], int(w[1])))

    parse_file(path)
    return top


def _is_number(t) -> bool:
    try:
        float(t)
        return True
    except ValueError:
        return False


def _match_dihedral(top: Topology, types, funcs):
    """Every type line for this dihedral: exact names (either direction) first,
    else the best wildcard match."""
    best, best_wild = [], 5
    for pat, func, par in top.dihedraltypes:
        if func not in funcs:
            continue
        for seq in (types, types[::-1]):
            ok = all(p == "X" or p == t for p, t in zip(pat, seq))
            if ok:
                wild = sum(p == "X" for p in pat)
                if wild < best_wild:
                    best, best_wild = [par], wild
                elif wild == best_wild and par not in best:
                    best.append(par)
                break
    return best


def build_system(top: Topology, gro: GroFile, name: str = "") -> System:
    """Flattens [ molecules ] into atoms and bonded terms in the engine's units."""
    pos = gro.pos.astype(np.float64)
    n = len(pos)
    q, m, sig, eps = [], [], [], []
    bonds, bpar, angles, apar, dihs, dpar, imps, ipar, pairs, ppar, excl = ([] for _ in range(11))
    off = 0
    molecules = top.molecules or [(name, 1) for name in top.moleculetypes]   # a bare .itp: each type once
    for molname, count in molecules:
        mt = top.moleculetypes[molname]
        types = [a[0] for a in mt.atoms]
        for _ in range(count):
            for (t, charge, mass, _nm) in mt.atoms:
                if t not in top.atomtypes:
                    raise KeyError(f"atom type {t!r} of molecule {molname!r} is not in [ atomtypes ]")
                at = top.atomtypes[t]
                q.append(charge * E_KCMOL)
                m.append((mass if mass is not None else at[0]) * 1e-3)
                sig.append(at[1])
                eps.append(at[2] * KJ)
            for i, j, func, par in mt.bonds:
                if not par:
                    par = top.bondtypes.get((types[i], types[j], func)) or top.bondtypes.get((types[j], types[i], func))
                if par is None:
                    raise KeyError(f"no bondtype for {types[i]}-{types[j]}")
                bonds.append((off + i, off + j))
                bpar.append((par[0], par[1] * KJ))
            for i, j, k, func, par in mt.angles:
                if not par:
                    key = (types[i], types[j], types[k], func)
                    par = top.angletypes.get(key) or top.angletypes.get((types[k], types[j], types[i], func))
                if par is None:
                    raise KeyError(f"no angletype for {types[i]}-{types[j]}-{types[k]}")
                ub0, kub = (par[2], par[3] * KJ) if func == 5 and len(par) >= 4 else (0.0, 0.0)
                angles.append((off + i, off + j, off + k))
                apar.append((par[0] * DEG, par[1] * KJ, ub0, kub))
            for i, j, k, l, func, par in mt.dihedrals:
                quad = (types[i], types[j], types[k], types[l])
                if func == 2:
                    plist = [par] if par else _match_dihedral(top, quad, (2,))
                    for pp in plist:
                        imps.append((off + i, off + j, off + k, off + l))
                        ipar.append((pp[0] * DEG, pp[1] * KJ))
                else:
                    plist = [par] if par else _match_dihedral(top, quad, (1, 4, 9))
                    if any(len(pp) < 3 for pp in plist):
                        raise ValueError(f"dihedral {quad} (func {func}) needs phi0, k and multiplicity")
                    for pp in plist:
                        # the reference halves the force constant on load (Bodies.cpp:36-38)
                        dihs.append((off + i, off + j, off + k, off + l))
                        dpar.append((pp[0] * DEG, pp[1] * KJ / 2.0, pp[2]))
                if not plist:
                    raise KeyError(f"no dihedraltype for {quad} (func {func})")
            for i, j, func, par in mt.pairs:
                if par:
                    s14, e14 = par[0], par[1]
                else:
                    pt = top.pairtypes.get((types[i], types[j])) or top.pairtypes.get((types[j], types[i]))
                    if pt is not None:
                        s14, e14 = pt
                    else:
                        ai, aj = top.atomtypes[types[i]], top.atomtypes[types[j]]
                        s14, e14 = 0.5 * (ai[1] + aj[1]), top.fudge_lj * math.sqrt(ai[2] * aj[2])
                pairs.append((off + i, off + j))
                ppar.append((s14, e14 * KJ))
            for i, j in mt.exclusions:
                excl.append((off + i, off + j))
            off += len(mt.atoms)
    if off != n:
        raise ValueError(f"topology has {off} atoms, coordinates {n}")
    vel = (gro.vel * 1000.0).astype(np.float32) if gro.vel is not None else np.zeros((n, 3), np.float32)

    def arr(x, k, dt):
        return np.asarray(x, dt).reshape(-1, k)

    return System(box=gro.box.astype(np.float64), pos=pos, vel=vel, charge=np.asarray(q, np.float32),
                  mass=np.asarray(m, np.float32), sigma=np.asarray(sig, np.float32),
                  epsilon=np.asarray(eps, np.float32),
                  bonds=arr(bonds, 2, np.int32), bond_par=arr(bpar, 2, np.float32),
                  angles=arr(angles, 3, np.int32), angle_par=arr(apar, 4, np.float32),
                  dihedrals=arr(dihs, 4, np.int32), dihedral_par=arr(dpar, 3, np.float32),
                  impropers=arr(imps, 4, np.int32), improper_par=arr(ipar, 2, np.float32),
                  pairbonds=arr(pairs, 2, np.int32), pair_par=arr(ppar, 2, np.float32),
                  name=name or top.system_name, extra_exclusions=arr(excl, 2, np.int32))


def load(gro_path: str, top_path: str, include_dirs=(), defines=(), name: str = "") -> System:
    """A System from a coordinate file and its topology."""
    return build_system(read_top(top_path, include_dirs, defines), read_gro(gro_path), name=name)


# -------------------------------------------------------------- writing .top
def write_top(path: str, s: System, molname: str = "SYS"):
    """The whole System as one molecule type with explicit per-term parameters
    (so reading it back needs no type tables); units converted back to the
    file conventions (kJ, degrees, e, g/mol, unhalved dihedral constants)."""
    with open(path, "w") as f:
        f.write("; written by lima_b200.topology\n[ defaults ]\n1 2 yes 1.0 1.0\n\n[ atomtypes ]\n")
        for i in range(s.n):
            f.write(f"T{i} 0 {s.mass[i] * 1e3:.6f} 0.0 A {s.sigma[i]:.6f} {s.epsilon[i] / KJ:.8f}\n")
        f.write(f"\n[ moleculetype ]\n{molname} 3\n\n[ atoms ]\n")
        for i in range(s.n):
            f.write(f"{i + 1} T{i} 1 RES A{i} {i + 1} {s.charge[i] / E_KCMOL:.8f} {s.mass[i] * 1e3:.6f}\n")
        f.write("\n[ bonds ]\n")
        for (a, b), (b0, kb) in zip(s.bonds, s.bond_par):
            f.write(f"{a + 1} {b + 1} 1 {b0:.6f} {kb / KJ:.6f}\n")
        f.write("\n[ pairs ]\n")
        for (a, b), (sg, ep) in zip(s.pairbonds, s.pair_par):
            f.write(f"{a + 1} {b + 1} 1 {sg:.6f} {ep / KJ:.8f}\n")
        f.write("\n[ angles ]\n")
        for (a, b, c), (th, kth, ub, kub) in zip(s.angles, s.angle_par):
            f.write(f"{a + 1} {b + 1} {c + 1} 5 {th / DEG:.6f} {kth / KJ:.6f} {ub:.6f} {kub / KJ:.6f}\n")
        f.write("\n[ dihedrals ]\n")
        for (a, b, c, d), (p0, kp, mult) in zip(s.dihedrals, s.dihedral_par):
            f.write(f"{a + 1} {b + 1} {c + 1} {d + 1} 9 {p0 / DEG:.6f} {2.0 * kp / KJ:.6f} {int(round(mult))}\n")
        for (a, b, c, d), (p0, kp) in zip(s.impropers, s.improper_par):
            f.write(f"{a + 1} {b + 1} {c + 1} {d + 1} 2 {p0 / DEG:.6f} {kp / KJ:.6f}\n")
        if len(s.extra_exclusions):
            f.write("\n[ exclusions ]\n")
            for a, b in s.extra_exclusions:
                f.write(f"{a + 1} {b + 1}\n")
        f.write(f"\n[ system ]\n{s.name or molname}\n\n[ molecules ]\n{molname} 1\n")


def write_gro_system(path: str, s: System, title: str = ""):
    write_gro(path, GroFile(title or s.name or "lima_b200", [1] * s.n, ["RES"] * s.n,
                            [f"A{i}"[:5] for i in range(s.n)], s.pos, s.vel.astype(np.float64) / 1000.0, s.box))
