"""Python binding of the C-ABI in include/lima_b200.h.

``Engine`` mirrors the lifecycle of LIMA_ENGINE's ``class Engine``
(code/LIMA_ENGINE/include/Engine.cuh:78-170): construct it from parameters,
load a box and topology, then ``step``/``run``/``minimize`` and read back
forces, energies and state.  Every call goes through liblima_b200.so; there is
no Python or CPU fallback, and a missing library raises at import of the
binding.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "liblima_b200.so")

LIMA_OK = 0
ERRORS = {1: "INVALID_ARG", 2: "CUDA", 3: "STATE", 4: "OVERFLOW", 5: "TIMEOUT", 6: "NO_DEVICE",
          7: "NOT_FINITE", 8: "UNSUPPORTED"}
ES_NONE, ES_CUTOFF, ES_EWALD = 0, 1, 2
LEAPFROG, VELOCITY_VERLET = 0, 1
CALC_ENERGY = 0x1
STATUS_BITS = {0x1: "PAIRLIST_OVERFLOW", 0x2: "COLUMN_OVERFLOW", 0x4: "NONFINITE",
               0x8: "FORCE_SATURATED", 0x10: "MOVED_TOO_FAR", 0x20: "MLP_FALLBACK"}

# every symbol the header declares (checked by tests/test_abi.py)
EXPORTED = [
    "lima_default_params", "lima_error_string", "lima_last_error", "lima_version", "lima_create",
    "lima_create_batch", "lima_destroy", "lima_select_system", "lima_num_systems", "lima_set_box",
    "lima_set_atoms", "lima_set_bonds", "lima_set_angles", "lima_set_dihedrals", "lima_set_impropers",
    "lima_set_pairbonds", "lima_set_exclusions", "lima_set_compounds", "lima_set_pme_grid", "lima_set_electric_field",
    "lima_set_state",
    "lima_get_state", "lima_compute_forces", "lima_step", "lima_minimize", "lima_get_forces",
    "lima_get_energies", "lima_get_pairlist", "lima_get_pairlist_stats", "lima_get_status", "lima_clear_status",
    "lima_get_timings", "lima_reset_timings", "lima_enable_phase_timing", "lima_pme_recip_noalloc",
    "lima_learned_pme_setup", "lima_learned_pme_collect", "lima_learned_pme_train", "lima_learned_pme_enable",
    "lima_learned_pme_eval", "lima_learned_pme_status", "lima_learned_pme_weights",
    "lima_learned_pme_gradients", "lima_learned_pme_predict", "lima_autotune", "lima_set_pair_shape",
    "lima_get_thermostat", "lima_get_log", "lima_clear_log",
]
MLP_NPARAM = 80 * 128 + 128 + 2 * (128 * 128 + 128) + 128 * 8 + 8   # network parameters
MLP_NSTATE = MLP_NPARAM + 2 * 68 + 1                               # + normalisation and output scale


class LimaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"LIMA_ERR_{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("dt", ctypes.c_double), ("cutoff", ctypes.c_double),
                ("skin", ctypes.c_double), ("nstlist", ctypes.c_int), ("electrostatics", ctypes.c_int),
                ("pme_grid", ctypes.c_int * 3), ("pme_spacing", ctypes.c_double),
                ("ewald_kappa", ctypes.c_double), ("ewald_tol", ctypes.c_double),
                ("ref_compat", ctypes.c_int), ("integrator", ctypes.c_int),
                ("thermostat_scalar", ctypes.c_double), ("exclude_bonded", ctypes.c_int),
                ("use_graphs", ctypes.c_int), ("apply_thermostat", ctypes.c_int),
                ("thermostat_interval", ctypes.c_int), ("target_temperature", ctypes.c_double),
                ("log_interval", ctypes.c_int), ("log_ring", ctypes.c_int), ("periodic", ctypes.c_int),
                ("prune_interval", ctypes.c_int), ("pair_split", ctypes.c_int)]


class Energies(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in
                ("lj", "coulomb_real", "pme_recip", "pme_self", "pme_excl", "bond", "angle", "dihedral",
                 "improper", "pairbond", "kinetic", "potential", "total", "virial", "temperature")] + \
               [("step", ctypes.c_int64)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class PairlistStats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int64) for k in ("rows_built", "rows_walked", "pairs_evaluated", "pairs_in_cutoff")] + \
               [("reserved", ctypes.c_int64 * 4)]


class Timings(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("nblist", "nonbonded", "bonded", "pme", "integrate", "step")] + \
               [("steps", ctypes.c_int64), ("rebuilds", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("pair_shape", ctypes.c_int32), ("reserved", ctypes.c_int32)]


_lib = None


def load_library(path: str = LIB_PATH):
    """Loads liblima_b200.so; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m lima_b200.build`")
    L = ctypes.CDLL(path)
    P = ctypes.POINTER
    h = ctypes.c_void_p
    i32p, f32p, f64p = P(ctypes.c_int32), P(ctypes.c_float), P(ctypes.c_double)
    sig = {
        "lima_default_params": (None, [P(Params)]),
        "lima_error_string": (ctypes.c_char_p, [ctypes.c_int]),
        "lima_last_error": (ctypes.c_char_p, [h]),
        "lima_version": (ctypes.c_int, []),
        "lima_create": (ctypes.c_int, [P(Params), P(h)]),
        "lima_create_batch": (ctypes.c_int, [P(Params), ctypes.c_int, P(h)]),
        "lima_destroy": (ctypes.c_int, [h]),
        "lima_select_system": (ctypes.c_int, [h, ctypes.c_int]),
        "lima_num_systems": (ctypes.c_int, [h, P(ctypes.c_int)]),
        "lima_set_box": (ctypes.c_int, [h, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
        "lima_set_atoms": (ctypes.c_int, [h, ctypes.c_int, f32p, f32p, f32p, f32p]),
        "lima_set_bonds": (ctypes.c_int, [h, ctypes.c_int, i32p, f32p]),
        "lima_set_angles": (ctypes.c_int, [h, ctypes.c_int, i32p, f32p]),
        "lima_set_dihedrals": (ctypes.c_int, [h, ctypes.c_int, i32p, f32p]),
        "lima_set_impropers": (ctypes.c_int, [h, ctypes.c_int, i32p, f32p]),
        "lima_set_pairbonds": (ctypes.c_int, [h, ctypes.c_int, i32p, f32p]),
        "lima_set_exclusions": (ctypes.c_int, [h, ctypes.c_int, i32p]),
        "lima_set_compounds": (ctypes.c_int, [h, ctypes.c_int, i32p, ctypes.c_int, i32p]),
        "lima_set_pme_grid": (ctypes.c_int, [h, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "lima_set_electric_field": (ctypes.c_int, [h, ctypes.c_double, ctypes.c_double, ctypes.c_double]),
        "lima_set_state": (ctypes.c_int, [h, f64p, f32p]),
        "lima_get_state": (ctypes.c_int, [h, f64p, f32p]),
        "lima_compute_forces": (ctypes.c_int, [h, ctypes.c_int]),
        "lima_step": (ctypes.c_int, [h, ctypes.c_int]),
        "lima_minimize": (ctypes.c_int, [h, ctypes.c_double, ctypes.c_int, P(ctypes.c_int), f64p]),
        "lima_get_forces": (ctypes.c_int, [h, f64p]),
        "lima_get_energies": (ctypes.c_int, [h, P(Energies)]),
        "lima_get_pairlist": (ctypes.c_int, [h, ctypes.c_int64, i32p, P(ctypes.c_int64)]),
        "lima_get_pairlist_stats": (ctypes.c_int, [h, P(PairlistStats)]),
        "lima_get_status": (ctypes.c_int, [h, P(ctypes.c_uint32)]),
        "lima_clear_status": (ctypes.c_int, [h]),
        "lima_get_timings": (ctypes.c_int, [h, P(Timings)]),
        "lima_reset_timings": (ctypes.c_int, [h]),
        "lima_enable_phase_timing": (ctypes.c_int, [h, ctypes.c_int]),
        "lima_pme_recip_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                                  ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                  ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p,
                                                  ctypes.c_void_p]),
        "lima_learned_pme_predict": (ctypes.c_int, [h, ctypes.c_int, f32p, f32p, ctypes.c_int]),
        "lima_autotune": (ctypes.c_int, [h, ctypes.c_int, P(ctypes.c_int)]),
        "lima_set_pair_shape": (ctypes.c_int, [h, ctypes.c_int]),
        "lima_get_thermostat": (ctypes.c_int, [h, f64p, f64p, P(ctypes.c_int64)]),
        "lima_get_log": (ctypes.c_int, [h, ctypes.c_int64, ctypes.c_int64, P(ctypes.c_int64), f32p, f32p,
                                        P(ctypes.c_int64)]),
        "lima_clear_log": (ctypes.c_int, [h]),
        "lima_learned_pme_setup": (ctypes.c_int, [h, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
        "lima_learned_pme_collect": (ctypes.c_int, [h]),
        "lima_learned_pme_train": (ctypes.c_int, [h, ctypes.c_int, ctypes.c_int, ctypes.c_float, ctypes.c_uint64,
                                                  f64p]),
        "lima_learned_pme_enable": (ctypes.c_int, [h, ctypes.c_int, ctypes.c_int, ctypes.c_double]),
        "lima_learned_pme_eval": (ctypes.c_int, [h, f64p, f64p]),
        "lima_learned_pme_status": (ctypes.c_int, [h, P(ctypes.c_int), P(ctypes.c_int), f64p]),
        "lima_learned_pme_weights": (ctypes.c_int, [h, ctypes.c_int, f32p, ctypes.c_int64, P(ctypes.c_int64)]),
        "lima_learned_pme_gradients": (ctypes.c_int, [h, ctypes.c_int, f32p, f32p, f32p, f64p]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def default_params(**kw) -> Params:
    p = Params()
    load_library().lima_default_params(ctypes.byref(p))
    for k, v in kw.items():
        if k == "pme_grid":
            for d in range(3):
                p.pme_grid[d] = int(v[d])
        else:
            setattr(p, k, v)
    return p


def _i32(a, k):
    a = np.ascontiguousarray(a, dtype=np.int32).reshape(-1, k)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _f32(a, k=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if k:
        a = a.reshape(-1, k)
    return a, a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


class Engine:
    """One engine handle over ``n_systems`` independent systems."""

    def __init__(self, params: Params | None = None, n_systems: int = 1, **kw):
        self.lib = load_library()
        self.params = params if params is not None else default_params(**kw)
        self.h = ctypes.c_void_p()
        self._check(self.lib.lima_create_batch(ctypes.byref(self.params), n_systems, ctypes.byref(self.h)))
        self.n_systems = n_systems
        self.natoms = [0] * n_systems
        self._boxes = [np.zeros(3)] * n_systems
        self._masses = [np.zeros(0, np.float32)] * n_systems
        self._sel = 0

    # ------------------------------------------------------------- plumbing
    def _check(self, rc: int):
        if rc != LIMA_OK:
            msg = self.lib.lima_last_error(self.h).decode() if self.h else ""
            raise LimaError(rc, msg or self.lib.lima_error_string(rc).decode())

    def close(self):
        if self.h:
            self.lib.lima_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def select(self, system: int):
        self._check(self.lib.lima_select_system(self.h, system))
        self._sel = system
        return self

    # ------------------------------------------------------------- loading
    def set_box(self, box):
        b = np.broadcast_to(np.asarray(box, dtype=np.float64), (3,))
        self._check(self.lib.lima_set_box(self.h, float(b[0]), float(b[1]), float(b[2])))
        self._boxes[self._sel] = np.array(b, np.float64)

    def box(self) -> np.ndarray:
        """Edge lengths [nm] of the selected system (as last set)."""
        return self._boxes[self._sel].copy()

    def masses(self) -> np.ndarray:
        """Atom masses [kg/mol] of the selected system (as last set)."""
        return self._masses[self._sel].copy()

    def set_atoms(self, charge, mass, sigma, epsilon):
        q, qp = _f32(charge)
        m, mp = _f32(mass)
        s, sp = _f32(sigma)
        e, ep = _f32(epsilon)
        self._check(self.lib.lima_set_atoms(self.h, len(q), qp, mp, sp, ep))
        self.natoms[self._sel] = len(q)
        self._masses[self._sel] = m.copy()

    def _terms(self, fn, idx, par, k, np_):
        if idx is None or len(idx) == 0:
            self._check(fn(self.h, 0, None, None))
            return
        ia, ip = _i32(idx, k)
        if np_:
            pa, pp = _f32(par, np_)
            self._check(fn(self.h, len(ia), ip, pp))
        else:
            self._check(fn(self.h, len(ia), ip))

    def set_bonds(self, idx, par):
        self._terms(self.lib.lima_set_bonds, idx, par, 2, 2)

    def set_angles(self, idx, par):
        self._terms(self.lib.lima_set_angles, idx, par, 3, 4)

    def set_dihedrals(self, idx, par):
        self._terms(self.lib.lima_set_dihedrals, idx, par, 4, 3)

    def set_impropers(self, idx, par):
        self._terms(self.lib.lima_set_impropers, idx, par, 4, 2)

    def set_pairbonds(self, idx, par):
        self._terms(self.lib.lima_set_pairbonds, idx, par, 2, 2)

    def set_exclusions(self, idx):
        if idx is None or len(idx) == 0:
            self._check(self.lib.lima_set_exclusions(self.h, 0, None))
            return
        ia, ip = _i32(idx, 2)
        self._check(self.lib.lima_set_exclusions(self.h, len(ia), ip))

    def set_compounds(self, compound, bonded=None):
        """Compound of each atom (-1: none) and bonded compound pairs; with
        ref_compat the engine evaluates pairs inside a compound and across bonded
        compounds without a cutoff, as the reference does."""
        c = np.ascontiguousarray(compound, dtype=np.int32).ravel()
        b = np.ascontiguousarray(np.zeros((0, 2)) if bonded is None else bonded, dtype=np.int32).reshape(-1, 2)
        i32 = ctypes.POINTER(ctypes.c_int32)
        self._check(self.lib.lima_set_compounds(self.h, len(c), c.ctypes.data_as(i32), len(b),
                                                b.ctypes.data_as(i32) if len(b) else None))

    def set_pme_grid(self, grid):
        self._check(self.lib.lima_set_pme_grid(self.h, int(grid[0]), int(grid[1]), int(grid[2])))

    def set_electric_field(self, field):
        """Uniform external electric field [V/nm] on the selected system."""
        self._check(self.lib.lima_set_electric_field(self.h, float(field[0]), float(field[1]), float(field[2])))

    def set_state(self, pos, vel=None):
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        if vel is None:
            self._check(self.lib.lima_set_state(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None))
        else:
            v = np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
            self._check(self.lib.lima_set_state(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                v.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))

    def load(self, system, pme_grid=None):
        """Loads a lima_b200.systems.System into the selected system slot."""
        self.set_box(system.box)
        self.set_atoms(system.charge, system.mass, system.sigma, system.epsilon)
        self.set_bonds(system.bonds, system.bond_par)
        self.set_angles(system.angles, system.angle_par)
        self.set_dihedrals(system.dihedrals, system.dihedral_par)
        self.set_impropers(system.impropers, system.improper_par)
        self.set_pairbonds(system.pairbonds, system.pair_par)
        extra = getattr(system, "extra_exclusions", None)
        if extra is not None and len(extra):
            self.set_exclusions(extra)
        comp = getattr(system, "compound", None)
        if comp is not None and len(comp):
            self.set_compounds(comp, getattr(system, "bonded_compounds", None))
        if pme_grid is not None:
            self.set_pme_grid(pme_grid)
        self.set_state(system.pos, system.vel)

    # ------------------------------------------------------------- running
    def compute_forces(self, energy: bool = True):
        self._check(self.lib.lima_compute_forces(self.h, CALC_ENERGY if energy else 0))

    def step(self, n: int = 1):
        self._check(self.lib.lima_step(self.h, int(n)))

    run = step

    def minimize(self, force_tol: float, max_steps: int):
        k = ctypes.c_int(0)
        f = ctypes.c_double(0.0)
        self._check(self.lib.lima_minimize(self.h, force_tol, max_steps, ctypes.byref(k), ctypes.byref(f)))
        return k.value, f.value

    # ------------------------------------------------------------- readback
    def forces(self) -> np.ndarray:
        f = np.zeros((self.natoms[self._sel], 3))
        self._check(self.lib.lima_get_forces(self.h, f.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return f

    def energies(self) -> dict:
        e = Energies()
        self._check(self.lib.lima_get_energies(self.h, ctypes.byref(e)))
        return e.as_dict()

    def state(self, pos_out=None, vel_out=None):
        """Positions (n,3) float64 and velocities (n,3) float32 of the selected
        system, written into pos_out / vel_out when given (e.g. pinned buffers)."""
        n = self.natoms[self._sel]
        p = np.zeros((n, 3)) if pos_out is None else pos_out
        v = np.zeros((n, 3), np.float32) if vel_out is None else vel_out
        assert p.dtype == np.float64 and p.flags.c_contiguous and p.size == 3 * n
        assert v.dtype == np.float32 and v.flags.c_contiguous and v.size == 3 * n
        self._check(self.lib.lima_get_state(self.h, p.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                            v.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return p, v

    def pairlist(self) -> np.ndarray:
        n = ctypes.c_int64(0)
        self._check(self.lib.lima_get_pairlist(self.h, 0, None, ctypes.byref(n)))
        out = np.zeros((max(n.value, 1), 2), np.int32)
        self._check(self.lib.lima_get_pairlist(self.h, n.value, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                               ctypes.byref(n)))
        return out[: n.value]

    def pairlist_stats(self) -> dict:
        """Rows built / walked, pairs evaluated and pairs within the cutoff (all systems)."""
        st = PairlistStats()
        self._check(self.lib.lima_get_pairlist_stats(self.h, ctypes.byref(st)))
        return {k: getattr(st, k) for k in ("rows_built", "rows_walked", "pairs_evaluated", "pairs_in_cutoff")}

    def status(self) -> int:
        s = ctypes.c_uint32(0)
        self._check(self.lib.lima_get_status(self.h, ctypes.byref(s)))
        return s.value

    def timings(self) -> dict:
        t = Timings()
        self._check(self.lib.lima_get_timings(self.h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def reset_timings(self):
        self._check(self.lib.lima_reset_timings(self.h))

    def phase_timing(self, enable: bool):
        self._check(self.lib.lima_enable_phase_timing(self.h, 1 if enable else 0))

    def set_pair_shape(self, shape: int):
        """Launch shape of the pair kernel (0-11, see lima_autotune)."""
        self._check(self.lib.lima_set_pair_shape(self.h, int(shape)))

    def autotune(self, periods: int = 1) -> int:
        """Picks the fastest launch shape of the pair kernel on this system (advances
        the simulation by 12 + 36 x periods pair-list periods); returns the shape."""
        shape = ctypes.c_int(0)
        self._check(self.lib.lima_autotune(self.h, int(periods), ctypes.byref(shape)))
        return shape.value

    def thermostat(self) -> dict:
        """Last temperature measurement of the selected system."""
        t, sc, st = ctypes.c_double(0.0), ctypes.c_double(0.0), ctypes.c_int64(0)
        self._check(self.lib.lima_get_thermostat(self.h, ctypes.byref(t), ctypes.byref(sc), ctypes.byref(st)))
        return {"temperature": t.value, "scale": sc.value, "step": st.value}

    def log(self, first: int = 0, max_frames: int | None = None):
        """Logged frames of the selected system: (steps, pos_epot (f,n,4), force_speed (f,n,4))."""
        total = ctypes.c_int64(0)
        self._check(self.lib.lima_get_log(self.h, 0, 0, None, None, None, ctypes.byref(total)))
        nf = max(0, total.value - first)
        if max_frames is not None:
            nf = min(nf, max_frames)
        n = self.natoms[self._sel]
        steps = np.zeros(max(nf, 1), np.int64)
        pe = np.zeros((max(nf, 1), n, 4), np.float32)
        fs = np.zeros((max(nf, 1), n, 4), np.float32)
        self._check(self.lib.lima_get_log(self.h, first, nf, steps.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                          _f32(pe)[1], _f32(fs)[1], ctypes.byref(total)))
        return steps[:nf], pe[:nf], fs[:nf]

    def clear_log(self):
        self._check(self.lib.lima_clear_log(self.h))


class LearnedPME:
    """The learned coarse-grid PME correction of one engine (no reference
    counterpart): collect frames from the engine's own states, train the
    network on the GPU, then let stepping use coarse PME + network with a
    full-grid check every ``check_interval`` steps."""

    def __init__(self, engine: Engine, coarse_grid=(32, 32, 32), max_frames: int = 16):
        self.engine = engine
        self.lib = engine.lib
        g = [int(v) for v in coarse_grid]
        engine._check(self.lib.lima_learned_pme_setup(engine.h, g[0], g[1], g[2], int(max_frames)))

    def collect(self):
        """Labels the engine's current state (one training frame)."""
        self.engine._check(self.lib.lima_learned_pme_collect(self.engine.h))

    def train(self, epochs: int, batch: int = 65536, lr: float = 1e-3, seed: int = 1) -> float:
        loss = ctypes.c_double(0.0)
        self.engine._check(self.lib.lima_learned_pme_train(self.engine.h, int(epochs), int(batch), float(lr),
                                                           int(seed), ctypes.byref(loss)))
        return loss.value

    def enable(self, on: bool = True, check_interval: int = 50, tolerance: float = 1e-3):
        self.engine._check(self.lib.lima_learned_pme_enable(self.engine.h, 1 if on else 0, int(check_interval),
                                                            float(tolerance)))

    def eval(self) -> tuple[float, float]:
        """(coarse, corrected) relative RMSE of the reciprocal force vs the full grid."""
        c, l = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self.engine._check(self.lib.lima_learned_pme_eval(self.engine.h, ctypes.byref(c), ctypes.byref(l)))
        return c.value, l.value

    def status(self) -> dict:
        a, f, r = ctypes.c_int(0), ctypes.c_int(0), ctypes.c_double(0.0)
        self.engine._check(self.lib.lima_learned_pme_status(self.engine.h, ctypes.byref(a), ctypes.byref(f),
                                                            ctypes.byref(r)))
        return {"active": bool(a.value), "fell_back": bool(f.value), "last_rel": r.value}

    def weights(self) -> np.ndarray:
        buf = np.zeros(MLP_NSTATE, np.float32)
        need = ctypes.c_int64(0)
        self.engine._check(self.lib.lima_learned_pme_weights(self.engine.h, 1, _f32(buf)[1], buf.size,
                                                             ctypes.byref(need)))
        return buf

    def set_weights(self, state):
        buf, ptr = _f32(np.asarray(state, np.float32).reshape(-1))
        self.engine._check(self.lib.lima_learned_pme_weights(self.engine.h, 0, ptr, buf.size, None))

    def predict(self, features, impl: int = 0) -> np.ndarray:
        """Network output (rows, 3) for raw feature rows (rows, 68); impl 0 = tcgen05
        tensor-core kernel, 1 = warp-level mma.sync kernel, 2 = the tcgen05 kernel's
        bounded-wait self-test (raises LimaError LIMA_ERR_TIMEOUT)."""
        x, xp = _f32(features, 68)
        y = np.zeros((len(x), 3), np.float32)
        self.engine._check(self.lib.lima_learned_pme_predict(self.engine.h, len(x), xp, _f32(y)[1], int(impl)))
        return y

    def gradients(self, x, t) -> tuple[float, np.ndarray]:
        """Loss and parameter gradients of one pass over caller rows (no update)."""
        x, xp = _f32(x, 68)
        t, tp = _f32(t, 3)
        g = np.zeros(MLP_NPARAM, np.float32)
        loss = ctypes.c_double(0.0)
        self.engine._check(self.lib.lima_learned_pme_gradients(self.engine.h, len(x), xp, tp, _f32(g)[1],
                                                               ctypes.byref(loss)))
        return loss.value, g
