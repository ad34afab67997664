"""The drop-in command-line program p3m_gpu (host/*.c): parameter handling,
exit codes, file formats and generated systems, all before any GPU work.
The program writes system_out before it creates a GPU context, so without
a GPU it is expected to stop at "Init" with a CUDA error (exit 1)."""
import os
import subprocess

import numpy as np
import pytest

import p3mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "p3m-standalone_b200")
REF_EXE = os.path.join(ROOT, "oracle", "_ref", "p3m")


@pytest.fixture(scope="session")
def exe():
    import importlib.util
    spec = importlib.util.spec_from_file_location("p3mg_build", os.path.join(PKG, "build.py"))
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build(host=True)
    path = os.path.join(PKG, "p3m_gpu")
    assert os.access(path, os.X_OK)
    return path


def run(exe, args, cwd):
    return subprocess.run([exe] + args.split(), cwd=cwd, capture_output=True, text=True, timeout=120)


@pytest.mark.parametrize("args,code,msg", [
    ("mesh 8 cao 3 rcut 2 method 1 alpha 1 bogus", 23, "Unknown parameter 'bogus'"),
    ("mesh 8 cao 3 method 1 alpha 1 particles 10 box 5", 255, "Required parameter 'rcut' missing."),
    ("mesh 8 cao 3 rcut 2 method 1 particles 10 box 5", 1, "Need to provide either alpha-range"),
    ("mesh 8 cao 3 rcut 2 method 1 alpha 1", 1, "Need to provide either 'positions'"),
    ("mesh 8 cao 3 rcut 2 method 5 alpha 1 particles 10 box 5 no_reference_force", 126, "Method 5 not know."),
    ("mesh 8 cao 3 rcut 2 method 1 alpha 1 positions /nonexistent/file", 127, "Could not open"),
])
def test_exit_codes_and_messages(exe, tmp_path, args, code, msg):
    r = run(exe, args, tmp_path)
    assert r.returncode == code, (r.stdout, r.stderr)
    assert msg in r.stdout + r.stderr


@pytest.mark.parametrize("system_type", [0, 1, 2, 3, 4, 5])
def test_generated_systems_match_reference_program(exe, tmp_path, system_type):
    if not os.access(REF_EXE, os.X_OK):
        pytest.skip("oracle/_ref/p3m not built")
    common = "particles 80 box 6 mesh 8 cao 3 rcut 2 method 7 alphamin 1 alphamax 1 alphastep 1 " \
             "no_reference_force no_calculation no_estimate system_type %d" % system_type
    subprocess.run([REF_EXE] + (common + " system_out ref.txt outfile o.dat").split(), cwd=tmp_path,
                   capture_output=True, check=True, timeout=120)
    run(exe, common + " system_out our.txt outfile o2.dat", tmp_path)
    assert (tmp_path / "ref.txt").read_bytes() == (tmp_path / "our.txt").read_bytes()


def test_read_system_skips_extra_comment_lines(exe, tmp_path):
    x, y, z, q = p3mg.generate_system(0, 20, 5.0, seed=3)
    lines = ["# Teilchenzahl: 20", "# Len: 5.000000", "# Mesh: 32"]
    lines += ["%lf\t%lf\t%lf\t%lf" % t for t in zip(x, y, z, q)]
    (tmp_path / "in.txt").write_text("\n".join(lines) + "\n")
    run(exe, "positions in.txt mesh 8 cao 3 rcut 2 method 1 alpha 1 no_reference_force system_out out.txt",
        tmp_path)
    out = (tmp_path / "out.txt").read_text().splitlines()
    assert out[:2] == lines[:2] and out[2:] == lines[3:]


def test_malformed_positions_file(exe, tmp_path):
    (tmp_path / "bad.txt").write_text("# Teilchenzahl: 3\n# Len: 5.0\n1 2 3 1\n1 2\n")
    r = run(exe, "positions bad.txt mesh 8 cao 3 rcut 2 method 1 alpha 1", tmp_path)
    assert r.returncode == 255 and "Error while reading file" in r.stderr


def test_forces_file_four_and_seven_columns(exe, tmp_path):
    # both layouts are accepted; a short file is an error (-1)
    x, y, z, q = p3mg.generate_system(0, 6, 5.0, seed=4)
    p3mg.write_system(str(tmp_path / "s.txt"), x, y, z, q, 5.0)
    four = "".join("%d\t%lf\t%lf\t%lf\n" % (i, 0.1 * i, 0.2, -0.3) for i in range(6))
    seven = "".join("%d\t%lf\t%lf\t%lf\t%lf\t%lf\t%lf\n" % (i, 0.1 * i, 0.2, -0.3, 1, 2, 3) for i in range(6))
    for name, text, code in [("f4.txt", four, None), ("f7.txt", seven, None), ("short.txt", four[:40], 255)]:
        (tmp_path / name).write_text(text)
        r = run(exe, "positions s.txt forces %s mesh 8 cao 3 rcut 2 method 1 alpha 1" % name, tmp_path)
        out = r.stdout + r.stderr
        if code is None:
            assert "Reading reference forces" in out and "Error while reading" not in out, out
        else:
            assert r.returncode == code and "Error while reading" in out
