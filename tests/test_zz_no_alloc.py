"""The allocation-free PME entry point against the engine's own PME stage and
against the FP64 oracle.

lima_pme_recip_noalloc serves callers that may not allocate device memory
(plug-ins inside an application that owns every device allocation through its
own pool, real-time loops that must not allocate after start-up).  It must
return the same reciprocal-space forces and energy as the engine, call after
call, using only its static scratch array.  The system is a lattice of ions
farther apart than the cutoff, with LJ off and no bonds, so the engine's forces
are the PME reciprocal forces alone.  Beyond the cubic case, mixed-radix
non-cubic grids, an odd grid and grids at the scratch array's limits (64^3
points in total; K0 = 8, whose half-complex grid is the largest fraction of the
real one) are checked against the oracle's FP64 smooth PME.
"""
import ctypes

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

FORCE_TOL = 1e-4     # relative RMS, as in the other parity tests
ENERGY_TOL = 1e-5


def ion_lattice(per=6, spacing=0.8, seed=4):
    rng = np.random.default_rng(seed)
    g = (np.arange(per) + 0.5) * spacing
    pos = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3)
    pos += rng.uniform(-0.05, 0.05, pos.shape)
    q = np.where((np.indices((per,) * 3).sum(0).ravel() % 2) == 0, 1.0, -1.0) * 96.4853321233100184
    return pos, q.astype(np.float32), np.array([per * spacing] * 3)


def random_ions(n, box, seed):
    """n ions (net charge zero) at uniform positions in a rectangular box."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 1.0, (n, 3)) * np.asarray(box)
    q = np.where(np.arange(n) % 2 == 0, 1.0, -1.0) * 96.4853321233100184
    return pos, q.astype(np.float32), np.asarray(box, dtype=np.float64)


def call_noalloc(lib, pos, q, box, grid, kappa, forces=None, energy=None):
    import torch
    dev = torch.device("cuda:0")
    n = len(pos)
    xyzq = torch.tensor(np.concatenate([pos.astype(np.float32), q[:, None]], 1), device=dev).contiguous()
    if forces is None:
        forces = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    if energy is None:
        energy = torch.zeros(1, dtype=torch.float64, device=dev)
    forces.fill_(123.0)
    energy.fill_(-1.0)
    rc = lib.lima_pme_recip_noalloc(ctypes.c_void_p(xyzq.data_ptr()), n, float(box[0]), float(box[1]),
                                    float(box[2]), int(grid[0]), int(grid[1]), int(grid[2]), float(kappa),
                                    ctypes.c_void_p(forces.data_ptr()), ctypes.c_void_p(energy.data_ptr()), None)
    torch.cuda.synchronize()
    return rc, forces.cpu().numpy(), float(energy.cpu().item())


def test_noalloc_matches_engine_pme():
    import torch
    from lima_b200 import Engine
    from lima_b200 import engine as E

    pos, q, box = ion_lattice()
    n = len(pos)
    grid = (40, 40, 40)
    kappa = 3.0
    eng = Engine(cutoff=0.5, electrostatics=E.ES_EWALD, ewald_kappa=kappa, exclude_bonded=1)
    eng.set_box(box)
    eng.set_atoms(q, np.full(n, 0.02, np.float32), np.zeros(n, np.float32), np.zeros(n, np.float32))
    eng.set_pme_grid(grid)
    eng.set_state(pos)
    eng.compute_forces(energy=True)
    f_eng = eng.forces()
    e_eng = eng.energies()
    assert e_eng["lj"] == 0.0 and e_eng["coulomb_real"] == 0.0   # no pair inside the cutoff

    lib = E.load_library()
    dev = torch.device("cuda:0")
    xyzq = torch.tensor(np.concatenate([pos.astype(np.float32), q[:, None]], 1), device=dev).contiguous()
    forces = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    energy = torch.zeros(1, dtype=torch.float64, device=dev)
    for call in range(2):
        forces.fill_(123.0)
        energy.fill_(-1.0)
        rc = lib.lima_pme_recip_noalloc(ctypes.c_void_p(xyzq.data_ptr()), n, float(box[0]), float(box[1]),
                                        float(box[2]), grid[0], grid[1], grid[2], kappa,
                                        ctypes.c_void_p(forces.data_ptr()), ctypes.c_void_p(energy.data_ptr()),
                                        None)
        assert rc == 0, (call, rc)
        torch.cuda.synchronize()
        f = forces.cpu().numpy()
        rel = np.sqrt(((f - f_eng) ** 2).sum() / (f_eng ** 2).sum())
        assert rel < FORCE_TOL, (call, rel)
        e = float(energy.cpu().item())
        assert abs(e - e_eng["pme_recip"]) <= ENERGY_TOL * abs(e_eng["pme_recip"]), (call, e, e_eng["pme_recip"])


def test_noalloc_rejects_oversize_grid():
    import torch
    from lima_b200 import engine as E

    lib = E.load_library()
    dev = torch.device("cuda:0")
    xyzq = torch.zeros((4, 4), dtype=torch.float32, device=dev)
    forces = torch.zeros((4, 3), dtype=torch.float64, device=dev)
    energy = torch.zeros(1, dtype=torch.float64, device=dev)
    rc = lib.lima_pme_recip_noalloc(ctypes.c_void_p(xyzq.data_ptr()), 4, 5.0, 5.0, 5.0, 96, 96, 96, 3.0,
                                    ctypes.c_void_p(forces.data_ptr()), ctypes.c_void_p(energy.data_ptr()), None)
    assert rc == 4   # LIMA_ERR_OVERFLOW: beyond the 64^3-point static scratch


# (grid, box): mixed radix 2-3-5 and non-cubic; odd K = 45 = 3^2 5; exactly
# 64^3 points with 16 along z; K0 = 8, the smallest first dimension, whose
# half-complex grid (K0/2 + 1) K1 K2 is the largest share of the scratch
NOALLOC_GRIDS = [
    ((36, 40, 60), (3.0, 3.4, 5.0)),
    ((45, 45, 45), (4.0, 4.0, 4.0)),
    ((128, 128, 16), (9.0, 9.0, 1.2)),
    ((8, 128, 128), (0.7, 9.0, 9.0)),
]


@pytest.mark.parametrize("grid,box", NOALLOC_GRIDS, ids=lambda v: "x".join(map(str, v)))
def test_noalloc_matches_fp64_oracle(grid, box):
    """Two calls in a row against the oracle's FP64 smooth PME (same B-spline
    moduli and analytic gather) on the same ions."""
    from lima_b200 import engine as E

    pos, q, box = random_ions(300, box, seed=sum(grid))
    kappa = 3.2
    f_ref, e_ref, _ = O.pme(pos, q.astype(np.float64), box, grid, kappa)
    lib = E.load_library()
    for call in range(2):
        rc, f, e = call_noalloc(lib, pos, q, box, grid, kappa)
        assert rc == 0, (grid, call, rc)
        rel = np.sqrt(((f - f_ref) ** 2).sum() / (f_ref ** 2).sum())
        assert rel < FORCE_TOL, (grid, call, rel)
        assert abs(e - e_ref) <= ENERGY_TOL * abs(e_ref), (grid, call, e, e_ref)
