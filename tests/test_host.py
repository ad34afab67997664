"""Host-side logic: file formats of the reference, the alpha sweep, the
system generators and the method table.  CPU only."""
import os

import numpy as np
import pytest

import p3mg

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_method_table_matches_reference_ids():
    assert sorted(p3mg.METHODS) == [0, 1, 2, 3, 6, 7]
    assert p3mg.METHODS[7][1] == "p3m-ad-r"
    assert p3mg.Method(1).flags & p3mg.FLAG_INTERLACED
    assert p3mg.Method(2).flags & p3mg.FLAG_SELF_FORCE
    assert not p3mg.Method(3).flags & p3mg.FLAG_SELF_FORCE  # ad-i has no self-force correction
    with pytest.raises(Exception):
        p3mg.Method(5)


def test_alpha_sweep_reproduces_reference_accumulation():
    a = p3mg.alpha_sweep(0.1, 2.5, 0.05)
    assert len(a) == 49 and a[-1] == 2.4999999999999991
    assert p3mg.alpha_sweep(0.9, 0.9, 0.1) == [0.9]


def test_position_file_roundtrip(tmp_path):
    x, y, z, q = p3mg.generate_system(0, 17, 7.5, seed=2)
    path = tmp_path / "pos.dat"
    p3mg.write_system(str(path), x, y, z, q, 7.5)
    x2, y2, z2, q2, L = p3mg.read_system(str(path))
    assert L == 7.5 and len(x2) == 17
    assert np.max(np.abs(x2 - x)) <= 5e-7 and np.array_equal(q2, q)


def test_position_file_with_extra_header_and_errors(tmp_path):
    p = tmp_path / "k.dat"
    p.write_text("# Teilchenzahl: 2\n# Len: 3.0\n# Mesh: 8\n0.1 0.2 0.3 1.0\n1 2 2.5 -1\n")
    x, y, z, q, L = p3mg.read_system(str(p))
    assert list(q) == [1.0, -1.0] and L == 3.0
    bad = tmp_path / "bad.dat"
    bad.write_text("# Teilchenzahl: 3\n# Len: 3.0\n0 0 0 1\n")
    with pytest.raises(ValueError):
        p3mg.read_system(str(bad))


def test_forces_file_formats(tmp_path):
    f = np.arange(12.0).reshape(3, 4) / 7.0
    p = tmp_path / "f.dat"
    p3mg.write_exact_forces(str(p), f, 2 * f)
    g = p3mg.read_exact_forces(str(p), 4)   # 7-column layout, total force columns
    assert np.max(np.abs(g - f)) <= 5e-7
    p4 = tmp_path / "f4.dat"
    p4.write_text("".join("%d\t%r\t%r\t%r\n" % (i, float(f[0, i]), float(f[1, i]), float(f[2, i])) for i in range(4)))
    assert np.array_equal(p3mg.read_exact_forces(str(p4), 4), f)


def test_tests_wall_fixture_reads_like_the_reference():
    w = np.load(os.path.join(GOLD, "wall.npz"))
    assert w["x"].shape == (300,) and float(w["L"]) == 10.0
    assert abs(np.sum(w["q"])) < 1e-12


@pytest.mark.parametrize("t", range(6))
def test_generators(t):
    x, y, z, q = p3mg.generate_system(t, 1000, 20.0, seed=5)
    n = len(x)
    for a in (x, y, z):
        assert np.all(a >= 0.0) and np.all(a < 20.0)
    assert abs(np.sum(q)) <= 1e-9  # neutral
    if t == p3mg.SYSTEM_SLAB:
        assert np.all(x >= 5.0) and np.all(x < 15.0)
    if t == p3mg.SYSTEM_SEPARATED_DIPOLE:
        d = np.stack([x[1::2] - x[0::2], y[1::2] - y[0::2], z[1::2] - z[0::2]])
        d -= 20.0 * np.round(d / 20.0)
        assert np.allclose(np.sqrt((d ** 2).sum(0)), 1.0)
    if t == p3mg.SYSTEM_MADELUNG:
        assert n == 1000
    # same seed -> same system
    x2, *_ = p3mg.generate_system(t, 1000, 20.0, seed=5)
    assert np.array_equal(x, x2)


def test_rms_error_definition():
    f = np.zeros((3, 4))
    ref = np.ones((3, 4))
    assert p3mg.rms_error(f, ref) == pytest.approx(np.sqrt(3.0))
