"""TRR trajectory files and the post-run energy analysis, on the CPU."""
import struct

import numpy as np
import pytest

from lima_b200 import trajectory as T


def frames(nf=4, n=37, seed=1):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, 3, (nf, n, 3)), np.array([3.0, 3.1, 3.2])


def test_trr_round_trip_positions(tmp_path):
    pos, box = frames()
    p = str(tmp_path / "t.trr")
    T.write_trr(p, pos, box, steps=[0, 10, 20, 30])
    r = T.read_trr(p)
    assert [f.step for f in r] == [0, 10, 20, 30]
    for i, f in enumerate(r):
        assert np.array_equal(f.x, pos[i].astype(np.float32)) and f.v is None and f.f is None
        assert np.array_equal(f.box, np.diag(box).astype(np.float32)) and not f.double


def test_trr_xdr_layout(tmp_path):
    """Big-endian XDR: magic 1993, string length 13, opaque length 12, the
    version, 13 int32, time and lambda, 9 box reals, then 3n positions."""
    pos, box = frames(1, 5)
    p = str(tmp_path / "t.trr")
    T.write_trr(p, pos, box, steps=[7])
    b = open(p, "rb").read()
    assert len(b) == 84 + 36 + 12 * 5
    assert struct.unpack(">iii", b[:12]) == (1993, 13, 12) and b[12:24] == b"GMX_trn_file"
    ints = struct.unpack(">13i", b[24:76])
    assert ints == (0, 0, 36, 0, 0, 0, 0, 60, 0, 0, 5, 7, 0)
    assert np.array_equal(np.frombuffer(b, ">f4", 15, 120), pos[0].ravel().astype(np.float32))


def test_trr_double_with_velocities_and_forces(tmp_path):
    pos, box = frames(2, 11)
    rng = np.random.default_rng(2)
    v, f = rng.normal(size=pos.shape), rng.normal(size=pos.shape) * 100
    p = str(tmp_path / "t.trr")
    with T.TrrWriter(p) as w:
        for i in range(2):
            w.write_frame(i * 5, box, pos[i], v[i], f[i], time=i * 0.005, lam=0.25, double=True)
    r = T.read_trr(p)
    assert all(fr.double for fr in r)
    assert np.array_equal(r[1].x, pos[1]) and np.array_equal(r[1].v, v[1]) and np.array_equal(r[1].f, f[1])
    assert r[1].time == 0.005 and r[1].lam == 0.25


def test_reads_native_little_endian_files(tmp_path):
    """The reference's writer emits host byte order (little-endian on x86):
    build such a frame by hand and read it back."""
    pos, box = frames(1, 4)
    hdr = struct.pack("<iii", 1993, 13, 12) + b"GMX_trn_file"
    hdr += struct.pack("<13i", 0, 0, 36, 0, 0, 0, 0, 48, 0, 0, 4, 3, 0) + struct.pack("<ff", 0.0, 0.0)
    body = np.diag(box).astype("<f4").tobytes() + pos[0].astype("<f4").tobytes()
    p = tmp_path / "ref.trr"
    p.write_bytes(hdr + body)
    r = T.read_trr(str(p))
    assert len(r) == 1 and r[0].step == 3 and np.array_equal(r[0].x, pos[0].astype(np.float32))


def test_trr_rejects_bad_input(tmp_path):
    with pytest.raises(ValueError):
        T.TrrWriter(str(tmp_path / "x.xtc"))
    p = tmp_path / "bad.trr"
    p.write_bytes(b"\0" * 100)
    with pytest.raises(ValueError):
        T.read_trr(str(p))
    pos, box = frames(1, 4)
    good = tmp_path / "g.trr"
    T.write_trr(str(good), pos, box)
    (tmp_path / "cut.trr").write_bytes(good.read_bytes()[:-5])
    with pytest.raises(ValueError):
        T.read_trr(str(tmp_path / "cut.trr"))


def test_variance_coefficient_and_gradient():
    rng = np.random.default_rng(3)
    y = (-5.0e4 + rng.normal(0, 3.0, 200)).astype(np.float32)
    vc = T.variance_coefficient(y)
    assert abs(vc - np.std(y.astype(np.float64)) / abs(np.mean(y.astype(np.float64)))) < 1e-6 * vc
    assert T.variance_coefficient([]) == 0.0 and T.variance_coefficient([0, 0]) == 0.0
    lin = (-1000.0 + 0.5 * np.arange(50)).astype(np.float32)
    m = float(lin.mean())
    assert abs(T.energy_gradient(lin, m) - 0.5 / m) < 1e-5 * abs(0.5 / m)   # FP32 sums


def test_analyze_drops_first_and_last_entry():
    pot = np.array([99.0, -10.0, -11.0, -12.0, 77.0])
    kin = np.array([1.0, 2.0, 2.5, 3.0, 1.0])
    a = T.analyze_energy(pot, kin)
    assert np.allclose(a.total_energy, [-8.0, -8.5, -9.0])
    assert np.allclose(a.pot_energy, [-10, -11, -12]) and np.allclose(a.kin_energy, [2, 2.5, 3])
    assert abs(a.mean_energy + 8.5) < 1e-6
    assert abs(a.energy_gradient - (-0.5 / -8.5)) < 1e-6
    assert T.analyze_energy([1.0], [1.0]).variance_coefficient == 0.0
    assert "totalE" in a.table()


def test_log_energies_sum_atoms():
    pe = np.zeros((2, 3, 4), np.float32)
    fs = np.zeros((2, 3, 4), np.float32)
    pe[..., 3] = [[1, 2, 3], [4, 5, 6]]
    fs[..., 3] = [[1, 0, 2], [0, 1, 1]]
    pot, kin = T.log_energies(pe, fs, np.array([2.0, 4.0, 1.0]))
    assert np.allclose(pot, [6, 15]) and np.allclose(kin, [0.5 * (2 + 4), 0.5 * (4 + 1)])


def test_evaluate_rules():
    assert T.evaluate([1.05e-3], 1e-3, [1e-8], 1e-7)[0]
    assert not T.evaluate([1.2e-3], 1e-3, [1e-8], 1e-7)[0]       # one VC: within 10 % of the target
    assert T.evaluate([1e-5, 9e-4], 1e-3, [0.0], 1e-7)[0]         # several: none above the target
    assert not T.evaluate([1e-5, 2e-3], 1e-3, [0.0], 1e-7)[0]
    assert not T.evaluate([1e-3], 1e-3, [float("nan")], 1e-7)[0]
    assert not T.evaluate([1e-3], 1e-3, [2e-7], 1e-7)[0]
