"""Oracle-side evaluation of a whole system (test helper; the oracle is the checker)."""
import math

import numpy as np


def kappa_from_tol(rc, tol):
    lo, hi = 0.0, 20.0 / rc
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if math.erfc(mid * rc) > tol else (lo, mid)
    return 0.5 * (lo + hi)


def oracle_total(O, s, rc, es_mode, kappa=0.0, grid=None, ref_compat=False, nb=True, bonded=True,
                 precision=64):
    """Forces (n,3) and the energy terms the engine reports, from the CPU oracle.
    With ref_compat and compounds on the system, pairs inside a compound and
    across bonded compounds are evaluated without a cutoff and left out of the
    cutoff loop, as in the reference."""
    ex = s.exclusions()
    f = np.zeros((s.n, 3))
    e = {}
    imm = None
    if ref_compat and getattr(s, "compound", None) is not None:
        imm = O.immediate_pairs(s.compound, s.bonded_compounds, ex)
    if nb:
        ex_nb = np.concatenate([ex, imm]) if imm is not None and len(imm) else ex
        fn, en, npairs = O.nonbonded(s.pos, s.box, s.charge, s.sigma, s.epsilon, ex_nb, rc, es_mode, kappa,
                                     precision=precision)
        f += fn
        e["lj"] = en["lj"]
        e["coulomb_real"] = en["coulomb"]
        if imm is not None:
            fi, elj, ec = O.immediate_forces(s.pos, s.box, s.charge, s.sigma, s.epsilon, imm, es_mode, kappa)
            f += fi
            e["lj"] += elj
            e["coulomb_real"] += ec
    if grid is not None:
        if ref_compat:
            fl, er, es = O.pme(s.pos, s.charge, s.box, grid, kappa, influence=1, gather=1)
            nq = int((s.charge != 0).sum())
            pi_ref = 3.14159
            q2 = float((s.charge.astype(np.float64) ** 2).sum())
            self_total = -kappa / math.sqrt(pi_ref) * q2 * O.coulomb_constant()
            e["pme_self"] = 0.5 * nq * self_total
        else:
            fl, er, es = O.pme(s.pos, s.charge, s.box, grid, kappa, influence=0, gather=0)
            e["pme_self"] = es
            q = s.charge
            xp = ex[(q[ex[:, 0]] != 0) & (q[ex[:, 1]] != 0)] if len(ex) else ex
            fx, exc = O.exclusion_correction(s.pos, s.charge, s.box, xp, kappa)
            f += fx
            e["pme_excl"] = exc
        f += fl
        e["pme_recip"] = er
    if bonded:
        fb, eb = O.bonded(s.pos, s.box, s.bonds, s.bond_par, s.angles, s.angle_par, s.dihedrals, s.dihedral_par,
                          s.impropers, s.improper_par, s.pairbonds, s.pair_par)
        f += fb
        e.update(eb)
    return f, e


def rel_rms(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
