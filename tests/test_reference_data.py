"""The reference's own data sets (Data/ReferenceDataVincent, committed as
raw text in tests/golden/vincent.npz): the readers for their file layouts
(konfig_N snapshots, Konfig_NN.dat with its parameter header, .exact
force files) in the Python package and in the p3m_gpu program, and the
oracle's FP64 Ewald forces against the data sets' exact forces.

The .exact forces were made by the data's authors with their own Ewald
code; they agree with a converged Ewald sum to about 1e-6 absolute RMS
(the oracle's own sum is converged to 5e-8 here), which bounds every
comparison with them."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import p3mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
V = np.load(os.path.join(ROOT, "tests", "golden", "vincent.npz"))
EXE = os.path.join(ROOT, "p3m-standalone_b200", "p3m_gpu")
# absolute RMS force difference allowed against each data set's .exact forces
EXACT_TOL = {"nacl300": 2e-6, "melt": 3e-7, "water": 1e-6}


def put(tmp_path, key, name=None):
    p = tmp_path / (name or key)
    p.write_bytes(V[key].tobytes())
    return str(p)


def test_konfig_and_dat_layouts_hold_the_same_system(tmp_path):
    for a, b in (("nacl300_konfig", "nacl300"), ("melt_konfig", "melt")):
        x1, y1, z1, q1, L1 = p3mg.read_system(put(tmp_path, a + "_pos"))
        x2, y2, z2, q2, L2 = p3mg.read_system(put(tmp_path, b + "_pos"))
        # the .dat header prints L to 6 decimals
        assert len(x1) == len(x2) == 512 and abs(L1 - L2) <= 1e-6 * L1
        # konfig coordinates are unwrapped and come back folded into [0, L);
        # the melt's .dat coordinates are unwrapped too, folded here with its L
        for v in (x1, y1, z1):
            assert np.all((v >= 0) & (v < L1))
        for u, v in ((x1, x2), (y1, y2), (z1, z2)):
            assert np.max(np.abs(u - np.mod(v, L2))) <= 4 * abs(L1 - L2) + 1e-12
        assert np.array_equal(q1, q2) and abs(q1.sum()) == 0.0


def test_dat_header_parameters(tmp_path):
    h = p3mg.read_system_header(put(tmp_path, "nacl300_pos"))
    assert h["Teilchenzahl"] == 512 and h["Len"] == 22.728
    assert h["Mesh"] == 8 and h["kmax"] == 20 and h["ip"] == 6 and h["rcut"] == 9.0
    assert h["alpha"] == 0.861531 and h["Bjerrum"] == 1.0


def test_exact_files_read_with_energy(tmp_path):
    f, e = p3mg.read_exact_forces(put(tmp_path, "nacl300_exact"), 512, with_energy=True)
    assert f.shape == (3, 512) and e == pytest.approx(-157.6430689727608, rel=1e-15)
    assert f[0, 0] == pytest.approx(0.0076408150296421, rel=1e-15)
    # the reference layout has no energy column
    (tmp_path / "four.txt").write_text("".join("%d\t1.0\t2.0\t3.0\n" % i for i in range(4)))
    f4, e4 = p3mg.read_exact_forces(str(tmp_path / "four.txt"), 4, with_energy=True)
    assert e4 is None and np.all(f4[2] == 3.0)


@pytest.mark.parametrize("key", ["nacl300", "melt", "water"])
def test_oracle_ewald_matches_exact_forces(tmp_path, key):
    x, y, z, q, L = p3mg.read_system(put(tmp_path, key + "_pos"))
    ref = p3mg.read_exact_forces(put(tmp_path, key + "_exact"), len(x))
    fold = [np.mod(v, L) for v in (x, y, z)]
    r = O.ewald(*fold, q, L, 16)
    assert O.abs_rms(r["f"], ref) <= EXACT_TOL[key]


@pytest.mark.skipif(not os.access(EXE, os.X_OK), reason="p3m_gpu not built")
def test_program_reads_every_layout(tmp_path):
    # konfig snapshot -> system_out: the folded positions in the reference layout
    put(tmp_path, "nacl300_konfig_pos", "konfig_0")
    common = "mesh 8 cao 3 rcut 2 method 1 alpha 1 no_reference_force"
    subprocess.run([EXE, "positions", "konfig_0"] + common.split() + ["system_out", "k.txt"], cwd=tmp_path,
                   capture_output=True, timeout=120)
    xk, yk, zk, qk, Lk = p3mg.read_system(str(tmp_path / "k.txt"))
    x, y, z, q, L = p3mg.read_system(str(tmp_path / "konfig_0"))
    assert len(xk) == 512 and abs(Lk - L) <= 1e-6
    assert np.max(np.abs(np.concatenate([xk - x, yk - y, zk - z]))) <= 1e-6 and np.array_equal(qk, q)
    # Konfig_NN.dat with its full header, and its .exact forces
    put(tmp_path, "nacl300_pos", "Konfig_01.dat")
    put(tmp_path, "nacl300_exact", "Konfig_01.exact")
    r = subprocess.run([EXE, "positions", "Konfig_01.dat", "forces", "Konfig_01.exact"] +
                       "mesh 8 cao 7 rcut 9 method 2 alpha 0.861531 system_out d.txt".split(), cwd=tmp_path,
                       capture_output=True, text=True, timeout=120)
    out = r.stdout + r.stderr
    assert "Reading reference forces" in out and "Error while reading" not in out, out
    xd, _, _, qd, Ld = p3mg.read_system(str(tmp_path / "d.txt"))
    assert len(xd) == 512 and Ld == pytest.approx(22.728)
    # a 7-field line whose first field is not an integer is malformed
    (tmp_path / "bad.exact").write_text("1.5 1 2 3 4 5 6\n" * 512)
    r = subprocess.run([EXE, "positions", "Konfig_01.dat", "forces", "bad.exact"] +
                       "mesh 8 cao 7 rcut 9 method 2 alpha 0.8".split(), cwd=tmp_path, capture_output=True,
                       text=True, timeout=120)
    assert r.returncode == 255 and "Error while reading" in r.stdout + r.stderr
