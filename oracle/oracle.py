"""ctypes wrapper of the CPU oracle (oracle/lima_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` as the checker.  The product library never
imports it.  Each function documents the reference formula it restates in
``oracle/lima_oracle.h``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_d = ctypes.POINTER(ctypes.c_double)
_i = ctypes.POINTER(ctypes.c_int)
_i32 = ctypes.POINTER(ctypes.c_int32)
_u8 = ctypes.POINTER(ctypes.c_uint8)
_i64 = ctypes.POINTER(ctypes.c_int64)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (g++ -O3 -fopenmp); make rebuilds it
    when its sources are newer than the library."""
    subprocess.run(["make", "-s", "-C", _HERE] + (["-B"] if force else []), check=True)
    return _LIB_PATH


def build_reference_harness(ref_dir: str | None = None) -> str | None:
    """Compile oracle/_ref/ref_terms (the reference's own per-term device
    functions, built from the reference tree; see ref_harness.cu) when that tree
    is at hand: LIMA_REFERENCE_DIR, or the given directory.  Returns the binary's
    path, or None when there is no reference tree."""
    ref_dir = ref_dir or os.environ.get("LIMA_REFERENCE_DIR", "")
    if not ref_dir or not os.path.isdir(os.path.join(ref_dir, "code", "LIMA_ENGINE")):
        return None
    subprocess.run(["make", "-s", "-C", _HERE, "ref", f"REF_DIR={ref_dir}"], check=True)
    return os.path.join(_HERE, "_ref", "ref_terms")


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.orc_coulomb_constant.restype = ctypes.c_double
        L.orc_e_to_kcmol.restype = ctypes.c_double
        L.orc_nonbonded.restype = ctypes.c_int64
        L.orc_nonbonded.argtypes = [ctypes.c_int, _d, _d, _d, _d, _d, _i, _i, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, _d, _d]
        L.orc_nonbonded_em.restype = ctypes.c_int64
        L.orc_nonbonded_em.argtypes = [ctypes.c_int, _d, _d, _d, _d, _d, _i, _i, ctypes.c_double,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_int, _d, _d]
        L.orc_pairset.restype = ctypes.c_int64
        L.orc_pairset.argtypes = [ctypes.c_int, _d, _d, _i, _i, ctypes.c_double, ctypes.c_double,
                                  ctypes.c_int64, _i32, _u8, _i64]
        L.orc_bonded.restype = None
        L.orc_bonded.argtypes = [ctypes.c_int, _d, _d] + [ctypes.c_int, _i, _d] * 5 + [_d, _d]
        L.orc_pme.restype = None
        L.orc_pme.argtypes = [ctypes.c_int, _d, _d, _d, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.c_double, ctypes.c_int, ctypes.c_int, _d, _d, _d]
        L.orc_ewald_recip.restype = None
        L.orc_ewald_recip.argtypes = [ctypes.c_int, _d, _d, _d, ctypes.c_double, ctypes.c_int, _d, _d]
        L.orc_exclusion_correction.restype = None
        L.orc_exclusion_correction.argtypes = [ctypes.c_int, _d, _d, _d, ctypes.c_int, _i,
                                               ctypes.c_double, _d, _d]
        L.orc_integrate.restype = None
        L.orc_integrate.argtypes = [ctypes.c_int, _d, _d, _d, _d, _d, ctypes.c_double, ctypes.c_int,
                                    ctypes.c_double]
        L.orc_em_step.restype = None
        L.orc_em_step.argtypes = [ctypes.c_int, _d, _d, _d, ctypes.c_int]
        L.orc_fft3d.restype = None
        L.orc_fft3d.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _d, ctypes.c_int]
        L.orc_nonbonded_atoms.restype = ctypes.c_int64
        L.orc_nonbonded_atoms.argtypes = [ctypes.c_int, _d, _d, _d, _d, _d, _i, _i, ctypes.c_double,
                                          ctypes.c_int, ctypes.c_double, ctypes.c_int, _d, _d, _d]
        L.orc_bonded_atoms.restype = None
        L.orc_bonded_atoms.argtypes = [ctypes.c_int, _d, _d] + [ctypes.c_int, _i, _d] * 5 + [_d, _d, _d]
        L.orc_exclusion_correction_atoms.restype = None
        L.orc_exclusion_correction_atoms.argtypes = [ctypes.c_int, _d, _d, _d, ctypes.c_int, _i,
                                                     ctypes.c_double, _d, _d, _d]
        L.orc_mlp_forward.restype = None
        L.orc_mlp_forward.argtypes = [ctypes.c_int, _d, _d, _d]
        L.orc_mlp_grads.restype = ctypes.c_double
        L.orc_mlp_grads.argtypes = [ctypes.c_int, _d, _d, _d, _d]
        L.orc_pair_terms.restype = None
        L.orc_pair_terms.argtypes = [ctypes.c_int, _d, _d, _d, _d, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                     ctypes.c_int, _d, _d]
        L.orc_bonded_terms.restype = None
        L.orc_bonded_terms.argtypes = [ctypes.c_int, ctypes.c_int, _d, _d, _d, _d]
        L.orc_bspline4.restype = None
        L.orc_bspline4.argtypes = [ctypes.c_int, _d, _d]
        L.orc_ref_green.restype = None
        L.orc_ref_green.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, _d]
        L.orc_force_activation.restype = None
        L.orc_force_activation.argtypes = [ctypes.c_int, _d, ctypes.c_double, _d]
        L.orc_adam.restype = None
        L.orc_adam.argtypes = [ctypes.c_int, _d, _d, _d, _i, _d]
        L.orc_compounds_interact.restype = ctypes.c_int
        L.orc_compounds_interact.argtypes = [ctypes.c_int, _d, _d, _d, _d, ctypes.c_double, ctypes.c_double, _u8]
        _lib = L
    return _lib


def _dp(a):
    return None if a is None else a.ctypes.data_as(_d)


def _ip(a):
    return None if a is None else a.ctypes.data_as(_i)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def coulomb_constant() -> float:
    return lib().orc_coulomb_constant()


def e_to_kcmol() -> float:
    return lib().orc_e_to_kcmol()


def exclusion_csr(n: int, pairs) -> tuple[np.ndarray, np.ndarray]:
    """CSR (both directions) of excluded atom pairs given as an (m,2) array."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    if len(pairs) == 0:
        return np.zeros(n + 1, np.int32), np.zeros(1, np.int32)
    a = np.concatenate([pairs[:, 0], pairs[:, 1]])
    b = np.concatenate([pairs[:, 1], pairs[:, 0]])
    order = np.lexsort((b, a))
    a, b = a[order], b[order]
    off = np.zeros(n + 1, np.int64)
    np.add.at(off, a + 1, 1)
    off = np.cumsum(off)
    return off.astype(np.int32), b.astype(np.int32)


def nonbonded(pos, box, q, sigma, eps, excl_pairs, rc, es_mode, kappa=0.0, precision=64,
              nthreads=0, em=False):
    """Returns (forces (n,3), {'lj','coulomb','virial'}, n_pairs).  em: the
    energy-minimisation variant of the LJ pair force (FP64 only)."""
    pos = _f64(pos).reshape(-1, 3)
    n = len(pos)
    off, idx = exclusion_csr(n, excl_pairs)
    f = np.zeros((n, 3))
    e = np.zeros(3)
    box = _f64(box)
    if em:
        npairs = lib().orc_nonbonded_em(n, _dp(pos), _dp(box), _dp(_f64(q)), _dp(_f64(sigma)),
                                        _dp(_f64(eps)), _ip(off), _ip(idx), rc, es_mode, kappa, nthreads,
                                        _dp(f), _dp(e))
        return f, {"lj": e[0], "coulomb": e[1], "virial": e[2]}, int(npairs)
    npairs = lib().orc_nonbonded(n, _dp(pos), _dp(box), _dp(_f64(q)), _dp(_f64(sigma)), _dp(_f64(eps)),
                                 _ip(off), _ip(idx), rc, es_mode, kappa, precision, nthreads, _dp(f), _dp(e))
    return f, {"lj": e[0], "coulomb": e[1], "virial": e[2]}, int(npairs)


def pairset(pos, box, excl_pairs, rc, band=0.0, cap=None):
    """Sorted (i<j) pairs within rc; returns (pairs (m,2), band_flags (m,), n_band)."""
    pos = _f64(pos).reshape(-1, 3)
    n = len(pos)
    off, idx = exclusion_csr(n, excl_pairs)
    box = _f64(box)
    if cap is None:
        cap = 0
        total = lib().orc_pairset(n, _dp(pos), _dp(box), _ip(off), _ip(idx), rc, band, 0,
                                  None, None, None)
        cap = total
    out = np.zeros((max(cap, 1), 2), np.int32)
    flags = np.zeros(max(cap, 1), np.uint8)
    nb = ctypes.c_int64(0)
    total = lib().orc_pairset(n, _dp(pos), _dp(box), _ip(off), _ip(idx), rc, band, cap,
                              out.ctypes.data_as(_i32), flags.ctypes.data_as(_u8), ctypes.byref(nb))
    return out[:total], flags[:total], int(nb.value)


def _terms(idx, par, k, p):
    if idx is None or len(idx) == 0:
        return 0, None, None
    idx = np.ascontiguousarray(idx, dtype=np.int32).reshape(-1, k)
    par = np.ascontiguousarray(par, dtype=np.float64).reshape(-1, p)
    return len(idx), idx, par


def bonded(pos, box, bonds=None, bond_par=None, angles=None, angle_par=None, dihedrals=None,
           dihedral_par=None, impropers=None, improper_par=None, pairbonds=None, pair_par=None):
    """Returns (forces (n,3), {'bond','angle','dihedral','improper','pairbond'})."""
    pos = _f64(pos).reshape(-1, 3)
    n = len(pos)
    f = np.zeros((n, 3))
    e = np.zeros(5)
    call = []
    keep = []  # holds the converted arrays alive during the call
    for idx, par, k, p in ((bonds, bond_par, 2, 2), (angles, angle_par, 3, 4),
                           (dihedrals, dihedral_par, 4, 3), (impropers, improper_par, 4, 2),
                           (pairbonds, pair_par, 2, 2)):
        m, ii, pp = _terms(idx, par, k, p)
        keep.append((ii, pp))
        call += [m, None if ii is None else ii.ctypes.data_as(_i), _dp(pp)]
    box = _f64(box)
    lib().orc_bonded(n, _dp(pos), _dp(box), *call, _dp(f), _dp(e))
    return f, dict(zip(["bond", "angle", "dihedral", "improper", "pairbond"], e.tolist()))


def pme(pos, q, box, grid, kappa, influence=0, gather=0, want_potential=False):
    """Returns (forces (n,3), e_recip, e_self[, phi])."""
    pos = _f64(pos).reshape(-1, 3)
    n = len(pos)
    f = np.zeros((n, 3))
    e = np.zeros(2)
    phi = np.zeros(n) if want_potential else None
    lib().orc_pme(n, _dp(pos), _dp(_f64(q)), _dp(_f64(box)), int(grid[0]), int(grid[1]), int(grid[2]),
                  kappa, influence, gather, _dp(f), _dp(e), _dp(phi))
    if want_potential:
        return f, e[0], e[1], phi
    return f, e[0], e[1]


def ewald_recip(pos, q, box, kappa, mmax):
    pos = _f64(pos).reshape(-1, 3)
    n = len(pos)
    f = np.zeros((n, 3))
    e = ctypes.c_double(0.0)
    lib().orc_ewald_recip(n, _dp(pos), _dp(_f64(q)), _dp(_f64(box)), kappa, mmax, _dp(f), ctypes.byref(e))
    return f, e.value


def exclusion_correction(pos, q, box, pairs, kappa):
    pos = _f64(pos).reshape(-1, 3)
    n = len(pos)
    pairs = np.ascontiguousarray(pairs, dtype=np.int32).reshape(-1, 2)
    f = np.zeros((n, 3))
    e = ctypes.c_double(0.0)
    lib().orc_exclusion_correction(n, _dp(pos), _dp(_f64(q)), _dp(_f64(box)), len(pairs),
                                   pairs.ctypes.data_as(_i), kappa, _dp(f), ctypes.byref(e))
    return f, e.value


def integrate(pos, vel, fprev, forces, mass, dt, integrator, scale=1.0):
    """In place on float64 arrays (pos, vel, fprev)."""
    n = len(mass)
    lib().orc_integrate(n, _dp(pos), _dp(vel), _dp(fprev), _dp(_f64(forces)), _dp(_f64(mass)), dt,
                        integrator, scale)


def em_step(pos, forces, adam, step):
    lib().orc_em_step(len(pos), _dp(pos), _dp(_f64(forces)), _dp(adam), step)


def fft3d(data: np.ndarray, sign: int) -> np.ndarray:
    """data complex128 array of shape (kz, ky, kx); returns transformed copy."""
    a = np.ascontiguousarray(data, dtype=np.complex128).copy()
    kz, ky, kx = a.shape
    lib().orc_fft3d(kx, ky, kz, a.view(np.float64).ctypes.data_as(_d), sign)
    return a


MLP_NPARAM = 80 * 128 + 128 + 2 * (128 * 128 + 128) + 128 * 8 + 8


def mlp_grads(x, t, params):
    """FP64 loss and parameter gradients of the learned-PME network.

    x (rows, 68), t (rows, 3), params (MLP_NPARAM,) in the engine's layout."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 68)
    t = np.ascontiguousarray(t, dtype=np.float64).reshape(-1, 3)
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
    assert params.size == MLP_NPARAM and len(t) == len(x)
    g = np.zeros(MLP_NPARAM)
    loss = lib().orc_mlp_grads(len(x), _dp(x), _dp(t), _dp(params), _dp(g))
    return loss, g


def atom_energies(s, rc, kappa, grid):
    """Per-atom potential energies in FP64 for the accurate Ewald/PME setup: half
    of each pair energy, equal shares of bonded terms, 1/2 q phi + the self term
    -kappa/sqrt(pi) k_e q^2, and half of each exclusion-correction pair."""
    pos = _f64(s.pos).reshape(-1, 3)
    n = len(pos)
    box = _f64(s.box)
    ex = s.exclusions()
    off, idx = exclusion_csr(n, ex)
    ae = np.zeros(n)
    f = np.zeros((n, 3))
    e = np.zeros(3)
    lib().orc_nonbonded_atoms(n, _dp(pos), _dp(box), _dp(_f64(s.charge)), _dp(_f64(s.sigma)),
                              _dp(_f64(s.epsilon)), _ip(off), _ip(idx), rc, 2, kappa, 0, _dp(f), _dp(e), _dp(ae))
    call, keep = [], []
    for ii, pp, k, pn in ((s.bonds, s.bond_par, 2, 2), (s.angles, s.angle_par, 3, 4),
                          (s.dihedrals, s.dihedral_par, 4, 3), (s.impropers, s.improper_par, 4, 2),
                          (s.pairbonds, s.pair_par, 2, 2)):
        m, a, b = _terms(ii, pp, k, pn)
        keep.append((a, b))
        call += [m, None if a is None else a.ctypes.data_as(_i), _dp(b)]
    eb = np.zeros(5)
    lib().orc_bonded_atoms(n, _dp(pos), _dp(box), *call, _dp(f), _dp(eb), _dp(ae))
    q = _f64(s.charge)
    _, _, _, phi = pme(pos, q, box, grid, kappa, influence=0, gather=0, want_potential=True)
    ae += 0.5 * q * phi - kappa / np.sqrt(np.pi) * coulomb_constant() * q * q
    xp = ex[(q[ex[:, 0]] != 0) & (q[ex[:, 1]] != 0)] if len(ex) else ex
    xp = np.ascontiguousarray(xp, dtype=np.int32).reshape(-1, 2)
    ee = ctypes.c_double(0.0)
    lib().orc_exclusion_correction_atoms(n, _dp(pos), _dp(q), _dp(box), len(xp), xp.ctypes.data_as(_i), kappa,
                                         _dp(f), ctypes.byref(ee), _dp(ae))
    return ae


def mlp_forward(x, params):
    """FP64 network output (rows, 3) for normalised inputs x (rows, 68)."""
    x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1, 68)
    params = np.ascontiguousarray(params, dtype=np.float64).reshape(-1)
    y = np.zeros((len(x), 3))
    lib().orc_mlp_forward(len(x), _dp(x), _dp(params), _dp(y))
    return y


# ------------------------------------------------ per-term entry points
def pair_terms(diff, sig, eps, qq, es_mode, kappa=0.0, precision=64, em=False):
    """Per-sample pair term: (force on i (n,3), LJ energy (n,), Coulomb energy (n,))."""
    diff = _f64(diff).reshape(-1, 3)
    n = len(diff)
    f = np.zeros((n, 3))
    e = np.zeros((n, 2))
    lib().orc_pair_terms(n, _dp(diff), _dp(_f64(sig)), _dp(_f64(eps)), _dp(_f64(qq)), int(es_mode), float(kappa),
                         int(precision), 1 if em else 0, _dp(f), _dp(e))
    return f, e[:, 0], e[:, 1]


BONDED_KINDS = {"bond": (0, 2, 2), "angle": (1, 3, 4), "dihedral": (2, 4, 3), "improper": (3, 4, 2),
                "pairbond": (4, 2, 2)}


def bonded_terms(kind, pos, par):
    """Per-sample bonded term: (forces (n, natoms, 3), energy (n,))."""
    k, na, npar = BONDED_KINDS[kind]
    pos = _f64(pos).reshape(-1, na, 3)
    par = _f64(par).reshape(-1, npar)
    n = len(pos)
    f = np.zeros((n, na, 3))
    e = np.zeros(n)
    lib().orc_bonded_terms(k, n, _dp(pos), _dp(par), _dp(f), _dp(e))
    return f, e


def bspline4(f):
    f = _f64(f).ravel()
    w = np.zeros((len(f), 4))
    lib().orc_bspline4(len(f), _dp(f), _dp(w))
    return w


def ref_green(K, L, kappa):
    out = np.zeros((K // 2 + 1) * K * K)
    lib().orc_ref_green(int(K), float(L), float(kappa), _dp(out))
    return out


def force_activation(f, scalar):
    f = _f64(f).reshape(-1, 3)
    out = np.zeros_like(f)
    lib().orc_force_activation(len(f), _dp(f), float(scalar), _dp(out))
    return out


def adam(f, m1, m2, step):
    f = _f64(f).reshape(-1, 3)
    m1 = _f64(m1).reshape(-1, 3).copy()
    m2 = _f64(m2).reshape(-1, 3).copy()
    st = np.ascontiguousarray(step, dtype=np.int32).ravel()
    d = np.zeros_like(f)
    lib().orc_adam(len(f), _dp(f), _dp(m1), _dp(m2), _ip(st), _dp(d))
    return d, m1, m2


def compounds_interact(keys_left, keys_right, radii_left, radii_right, box_nm, cutoff):
    kl = _f64(keys_left).reshape(-1, 6)
    n = len(kl)
    out = np.zeros(n, np.uint8)
    lib().orc_compounds_interact(n, _dp(kl), _dp(_f64(keys_right).reshape(-1, 6)), _dp(_f64(radii_left)),
                                 _dp(_f64(radii_right)), float(box_nm), float(cutoff),
                                 out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
    return out.astype(bool)


def immediate_pairs(compound, bonded, excl_pairs):
    """The reference's immediate-neighbour pair set (EngineKernels.cuh:150-317):
    every (i<j) pair inside one compound or across two bonded compounds that is
    not excluded (the BondedParticlesLUT, CompoundBuilder.cpp:40-60)."""
    compound = np.asarray(compound)
    members = {}
    for i, c in enumerate(compound):
        if c >= 0:
            members.setdefault(int(c), []).append(i)
    ex = {(int(min(a, b)), int(max(a, b))) for a, b in np.asarray(excl_pairs).reshape(-1, 2)}
    out = set()
    def add(a, b):
        p = (min(a, b), max(a, b))
        if a != b and p not in ex:
            out.add(p)
    for m in members.values():
        for x in range(len(m)):
            for y in range(x + 1, len(m)):
                add(m[x], m[y])
    for c0, c1 in np.asarray(bonded if bonded is not None else np.zeros((0, 2)), dtype=np.int64).reshape(-1, 2):
        for a in members.get(int(c0), ()):
            for b in members.get(int(c1), ()):
                add(a, b)
    return np.array(sorted(out), np.int32).reshape(-1, 2)


def immediate_forces(pos, box, q, sigma, eps, pairs, es_mode, kappa, precision=64):
    """Forces and (LJ, Coulomb) energies of the immediate pairs, no cutoff,
    minimum image; the same pair function as the cutoff loop."""
    pos = _f64(pos).reshape(-1, 3)
    f = np.zeros_like(pos)
    pairs = np.asarray(pairs, np.int64).reshape(-1, 2)
    if len(pairs) == 0:
        return f, 0.0, 0.0
    i, j = pairs[:, 0], pairs[:, 1]
    d = pos[j] - pos[i]
    if box is not None:
        b = _f64(box)
        d -= b * np.rint(d / b)
    sig = 0.5 * (_f64(sigma)[i] + _f64(sigma)[j])
    ep = np.sqrt(_f64(eps)[i] * _f64(eps)[j])
    qq = _f64(q)[i] * _f64(q)[j]
    fi, elj, ec = pair_terms(d, sig, ep, qq, es_mode, kappa, precision=precision)
    np.add.at(f, i, fi)
    np.add.at(f, j, -fi)
    return f, float(elj.sum()), float(ec.sum())
