"""Trajectory files and energy analysis of logged runs.

TRR: the GROMACS trajectory format the reference writes
(code/LIMA_BASE/src/TrrFileInterface.cpp:107-196): per frame the magic 1993,
the version string "GMX_trn_file" (length with terminator, then as an XDR
opaque: length, bytes, zero fill to 4), thirteen int32 block sizes and counts
(ir, e, box, vir, pres, top, sym, x, v, f, natoms, step, nre), time and lambda
in the frame's precision, then the 3x3 box and the x / v / f blocks present.
The reference writes a box and positions only, in single precision; this writer
also takes velocities and forces.  Files are written in XDR (big-endian) byte
order as GROMACS reads them.  The reference's writer does not swap bytes, so on
x86 its files are little-endian; the reader takes either order from the magic
number and the precision from the block sizes.

The reference fills TrrFile from its logging ring (code/LIMA_BASE/src/
Simulation.cpp:191-215) and dumps it after a run (code/LIMA_MD/src/
Environment.cpp:292-293); here the engine's log (lima_get_log) gives the frames.

Energy analysis (code/LIMA_MD/src/Analyzer.cu:216-365): per logged entry the
potential energy summed over atoms, the kinetic energy 0.5 m |v|^2 summed over
atoms (code/LIMA_BASE/include/PhysicsUtils.cuh:11-13) and their sum; the first
and last entries are dropped; then the mean, the variance coefficient
(population standard deviation over |mean|, code/LIMA_MD/src/Analyzer.cu:289-296
with code/LIMA_BASE/src/Statistics.cpp:106-124) and the energy gradient (FP32
least-squares slope over entry index divided by the mean, code/LIMA_MD/src/
Analyzer.cu:316-335).  ``evaluate`` is the pass rule of the reference's
stability tests (code/LIMA_TESTS/src/TestUtils.h:120-182).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

TRR_MAGIC = 1993
TRR_VERSION = b"GMX_trn_file"
_HEADER_INTS = ("ir_size", "e_size", "box_size", "vir_size", "pres_size", "top_size", "sym_size",
                "x_size", "v_size", "f_size", "natoms", "step", "nre")


@dataclass
class TrrFrame:
    step: int
    time: float
    lam: float
    box: np.ndarray                      # (3, 3) [nm], rows are box vectors
    x: np.ndarray | None = None          # (n, 3) [nm]
    v: np.ndarray | None = None          # (n, 3) [nm/ps]
    f: np.ndarray | None = None          # (n, 3) [kJ/mol/nm]
    double: bool = False


def box_matrix(box) -> np.ndarray:
    """3x3 box from edge lengths (the reference's rectangular cell, get_cell)."""
    b = np.asarray(box, np.float64)
    return np.diag(b) if b.shape == (3,) else b.reshape(3, 3)


class TrrWriter:
    """Appends frames to a .trr file (XDR byte order unless byteorder='<')."""

    def __init__(self, path: str, byteorder: str = ">"):
        if not str(path).endswith(".trr"):
            raise ValueError(f"expected extension .trr, got '{path}'")
        if byteorder not in "<>":
            raise ValueError("byteorder must be '<' or '>'")
        self.bo = byteorder
        self.f = open(path, "wb")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def close(self):
        if not self.f.closed:
            self.f.close()

    def write_frame(self, step: int, box, x=None, v=None, f=None, time: float = 0.0, lam: float = 0.0,
                    double: bool = False):
        arrays = [None if a is None else np.asarray(a, np.float64).reshape(-1, 3) for a in (x, v, f)]
        present = [a for a in arrays if a is not None]
        natoms = len(present[0]) if present else 0
        if any(len(a) != natoms for a in present):
            raise ValueError("x, v and f must have the same number of atoms")
        real = "d" if double else "f"
        rs = 8 if double else 4
        bo = self.bo
        sizes = dict.fromkeys(_HEADER_INTS, 0)
        sizes["box_size"] = 9 * rs
        for key, a in zip(("x_size", "v_size", "f_size"), arrays):
            sizes[key] = 0 if a is None else 3 * natoms * rs
        sizes["natoms"], sizes["step"] = natoms, int(step)
        pad = (-len(TRR_VERSION)) % 4
        out = [struct.pack(bo + "iii", TRR_MAGIC, len(TRR_VERSION) + 1, len(TRR_VERSION)), TRR_VERSION,
               b"\0" * pad, struct.pack(bo + "13i", *(sizes[k] for k in _HEADER_INTS)),
               struct.pack(bo + 2 * real, time, lam),
               box_matrix(box).astype(bo + real).tobytes()]
        out += [a.astype(bo + real).tobytes() for a in arrays if a is not None]
        self.f.write(b"".join(out))


def write_trr(path: str, positions, box, steps=None, velocities=None, forces=None, times=None,
              byteorder: str = ">"):
    """One frame per entry of positions (f, n, 3); the step of frame i is
    steps[i] (default i, as the reference's TrrFile::Dump)."""
    positions = np.asarray(positions)
    with TrrWriter(path, byteorder) as w:
        for i in range(len(positions)):
            w.write_frame(int(steps[i]) if steps is not None else i, box, positions[i],
                          None if velocities is None else velocities[i], None if forces is None else forces[i],
                          time=0.0 if times is None else float(times[i]))


def read_trr(path: str) -> list[TrrFrame]:
    data = open(path, "rb").read()
    frames, off = [], 0
    while off < len(data):
        if len(data) - off < 12:
            raise ValueError(f"truncated frame header at byte {off}")
        magic_be = struct.unpack_from(">i", data, off)[0]
        magic_le = struct.unpack_from("<i", data, off)[0]
        if magic_be == TRR_MAGIC:
            bo = ">"
        elif magic_le == TRR_MAGIC:
            bo = "<"
        else:
            raise ValueError(f"bad TRR magic at byte {off}")
        _, slen, olen = struct.unpack_from(bo + "iii", data, off)
        if olen != slen - 1 or olen < 0:
            raise ValueError(f"bad TRR version string at byte {off}")
        off += 12 + olen + (-olen) % 4
        vals = dict(zip(_HEADER_INTS, struct.unpack_from(bo + "13i", data, off)))
        off += 52
        natoms = vals["natoms"]
        if vals["box_size"]:
            rs = vals["box_size"] // 9
        elif natoms:
            rs = max(vals["x_size"], vals["v_size"], vals["f_size"]) // (3 * natoms)
        else:
            rs = 4
        if rs not in (4, 8):
            raise ValueError(f"cannot infer TRR precision at byte {off}")
        real = "d" if rs == 8 else "f"
        time, lam = struct.unpack_from(bo + 2 * real, data, off)
        off += 2 * rs
        # blocks the reference never writes (ir, e, vir, pres, top, sym) are skipped by size
        off += vals["ir_size"] + vals["e_size"]
        box = np.zeros((3, 3))
        if vals["box_size"]:
            box = np.frombuffer(data, bo + real, 9, off).astype(np.float64).reshape(3, 3)
            off += vals["box_size"]
        off += vals["vir_size"] + vals["pres_size"] + vals["top_size"] + vals["sym_size"]
        blocks = {}
        for key in ("x", "v", "f"):
            size = vals[key + "_size"]
            if size:
                if size != 3 * natoms * rs or off + size > len(data):
                    raise ValueError(f"bad {key} block at byte {off}")
                blocks[key] = np.frombuffer(data, bo + real, 3 * natoms, off).astype(np.float64).reshape(natoms, 3)
                off += size
        frames.append(TrrFrame(vals["step"], float(time), float(lam), box, blocks.get("x"), blocks.get("v"),
                               blocks.get("f"), rs == 8))
    return frames


def write_log_trr(path: str, engine, box=None, first: int = 0, max_frames: int | None = None,
                  with_forces: bool = False, byteorder: str = ">"):
    """The engine's logged frames of its selected system as a .trr file:
    positions, and forces (converted to kJ/mol/nm) when with_forces."""
    steps, pos_epot, force_speed = engine.log(first, max_frames)
    if box is None:
        box = engine.box()
    with TrrWriter(path, byteorder) as w:
        for i, st in enumerate(steps):
            w.write_frame(int(st), box, pos_epot[i, :, :3],
                          f=force_speed[i, :, :3] / 1000.0 if with_forces else None)
    return len(steps)


# ------------------------------------------------------------------ analysis
def variance_coefficient(vec) -> float:
    """Population standard deviation over |mean| (FP64 sums, FP32 result);
    0 when both are 0."""
    v = np.asarray(vec, np.float32)
    if len(v) == 0:
        return 0.0
    mean = np.float32(v.astype(np.float64).sum() / len(v))
    sd = np.float32(np.sqrt(((v.astype(np.float64) - np.float64(mean)) ** 2).sum() / len(v)))
    if sd == 0 and mean == 0:
        return 0.0
    return float(np.float32(sd / np.float32(abs(mean))))


def energy_gradient(vec, mean: float) -> float:
    """Least-squares slope of vec over its index, divided by mean, with the
    sums accumulated in order in FP32."""
    y = np.asarray(vec, np.float32)
    n = len(y)
    if n == 0:
        return float("nan")
    i = np.arange(n, dtype=np.float32)
    sx = np.cumsum(i, dtype=np.float32)[-1]
    sy = np.cumsum(y, dtype=np.float32)[-1]
    sxy = np.cumsum(i * y, dtype=np.float32)[-1]
    sxx = np.cumsum(i * i, dtype=np.float32)[-1]
    nf = np.float32(n)
    with np.errstate(divide="ignore", invalid="ignore"):
        slope = (nf * sxy - sx * sy) / (nf * sxx - sx * sx)
        return float(np.float32(slope / np.float32(mean)))


@dataclass
class AnalyzedPackage:
    pot_energy: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    kin_energy: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    total_energy: np.ndarray = field(default_factory=lambda: np.zeros(0, np.float32))
    temperature: np.ndarray = field(default_factory=lambda: np.zeros(0))
    mean_energy: float = 0.0
    energy_gradient: float = 0.0
    variance_coefficient: float = 0.0

    def table(self) -> str:
        """min, max, standard deviation and relative change first->last per series."""
        rows = ["%-8s %14s %14s %14s %14s" % ("", "min", "max", "Std. deviation", "Change 0->n")]
        for name, v in (("potE", self.pot_energy), ("kinE", self.kin_energy), ("totalE", self.total_energy)):
            if len(v):
                sd = np.sqrt(((v.astype(np.float64) - v.astype(np.float64).mean()) ** 2).mean())
                rows.append("%-8s %14.6e %14.6e %14.6e %14.6e" % (name, v.min(), v.max(), sd,
                                                                  (v[-1] - v[0]) / v[0] if v[0] else float("nan")))
        return "\n".join(rows)


def analyze_energy(pot, kin, temperature=None) -> AnalyzedPackage:
    """Per-entry potential and kinetic energy [J/mol] of consecutive logged
    entries; entries 0 and n-1 are left out, as the reference does."""
    pot = np.asarray(pot, np.float64)
    kin = np.asarray(kin, np.float64)
    if len(pot) < 2:
        return AnalyzedPackage()
    p = pot[1:-1].astype(np.float32)
    k = kin[1:-1].astype(np.float32)
    t = (pot[1:-1] + kin[1:-1]).astype(np.float32)
    mean = float(np.float32(t.astype(np.float64).sum() / len(t))) if len(t) else 0.0
    return AnalyzedPackage(p, k, t, np.asarray(temperature if temperature is not None else []),
                           mean, energy_gradient(t, mean) if len(t) else 0.0, variance_coefficient(t))


def log_energies(pos_epot, force_speed, mass):
    """Potential and kinetic energy per logged frame from the engine's log:
    sum of per-atom potential energies, sum of 0.5 m |v|^2 (FP64 sums)."""
    pe = np.asarray(pos_epot)[..., 3].astype(np.float64).sum(axis=1)
    sp = np.asarray(force_speed)[..., 3].astype(np.float64)
    ke = 0.5 * (np.asarray(mass, np.float64)[None, :] * sp * sp).sum(axis=1)
    return pe, ke


def analyze_log(engine, first: int = 0) -> AnalyzedPackage:
    """The reference's post-run energy analysis over the engine's log of its
    selected system."""
    _, pe, fs = engine.log(first)
    pot, kin = log_energies(pe, fs, engine.masses())
    return analyze_energy(pot, kin)


def evaluate(vcs, target_vc: float, gradients, max_gradient: float) -> tuple[bool, str]:
    """Stability-test verdict: with one variance coefficient it must lie within
    10 % of target_vc, with several none may exceed it; every gradient must be
    finite and at most max_gradient in magnitude."""
    vcs = [float(v) for v in np.atleast_1d(vcs)]
    for vc in vcs:
        bad = vc > target_vc if len(vcs) > 1 else (np.isnan(vc) or abs(vc - target_vc) / target_vc > 0.1)
        if bad:
            return False, f"Variance Coefficient of {vc:.3e} was too far from the target {target_vc:.3e}"
    for g in np.atleast_1d(gradients):
        if np.isnan(g) or abs(g) > max_gradient:
            return False, f"Energygradient of {g:.3e} superceeded the max of {max_gradient:.3e}"
    return True, f"VC {max(vcs):.3e} / {target_vc:.3e}"
