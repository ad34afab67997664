"""Tile autotuner (p3mg_autotune, p3mg_set_tiles) and the reference's
parameter tuner on the GPU (p3mg_tune): choices are valid, forces do not
change beyond summation order, and the tuned parameters meet the target
against the Ewald reference."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("method,mesh,cao", [(1, 32, 5), (0, 128, 7), (1, 128, 7), (7, 128, 7)])
def test_pencil_fft_matches_stockham_fft(gpu, method, mesh, cao):
    # FP32 meshes of 32, 64 (the tiles test) and 128 points take the
    # register-tiled pencil FFT by default (ik, one mesh or interlaced: with
    # the convolution folded into the first backward pass and the packing
    # into the last; ad: plain passes); the Stockham kernel (a tile width)
    # gives the same forces up to FP32 rounding
    x, y, z, q = p3mg.generate_system(0, 4000, 14.0, seed=83)
    with p3mg.Context(method, mesh, cao, 1, p3mg.FP32_MIXED) as ctx, p3mg.Context(method, mesh, cao, 1) as c64:
        for c in (ctx, c64):
            c.set_system(x, y, z, q, 14.0)
            c.influence(1.0)
        fk64 = c64.calculate_forces(0.0)["f_k"]
        fk = ctx.calculate_forces(0.0)["f_k"]
        ctx.set_tiles(8 if mesh >= 64 else 4, 16)
        fs = ctx.calculate_forces(0.0)["f_k"]
        assert O.rel_rms(fk.ravel(), fs.ravel()) <= 2e-6
        # both within FP32 rounding of the FP64 k-space forces
        assert O.rel_rms(fk.ravel(), fk64.ravel()) <= 5e-6
        assert O.rel_rms(fs.ravel(), fk64.ravel()) <= 5e-6


@pytest.mark.parametrize("precision", [p3mg.FP64, p3mg.FP32_MIXED])
def test_tiles_do_not_change_forces(gpu, precision):
    x, y, z, q = p3mg.generate_system(0, 3000, 14.0, seed=81)
    with p3mg.Context(1, 64, 7, 1, precision) as ctx:
        ctx.set_system(x, y, z, q, 14.0)
        ctx.influence(1.0)
        f0 = ctx.calculate_forces(3.0)["f"]
        tol = 1e-13 if precision == p3mg.FP64 else 1e-6
        for brick, w in [(4, 4), (4, 16), (8, 8), (8, 0)]:
            ctx.set_tiles(brick, w)
            f = ctx.calculate_forces(3.0)["f"]
            assert O.rel_rms(f.ravel(), f0.ravel()) <= tol, (brick, w)
        best = ctx.autotune(3.0)
        assert best["brick"] in (4, 8) and best["fft_w"] in (0, 4, 8, 16) and best["ms"] > 0
        f = ctx.calculate_forces(3.0)["f"]
        assert O.rel_rms(f.ravel(), f0.ravel()) <= tol
        with pytest.raises(p3mg.P3MGError):
            ctx.set_tiles(5, 0)


def test_tune_meets_target(gpu):
    L = 12.0
    x, y, z, q = p3mg.generate_system(0, 1728, L, seed=82)
    target = 1e-3
    t = p3mg.tune(1, x, y, z, q, L, 3.0, target)
    assert t["estimate"] <= target and t["mesh"] % 2 == 0 and 1 <= t["cao"] <= 7 and t["ms"] > 0
    ew = O.ewald(x, y, z, q, L, 16)
    with p3mg.Context(1, t["mesh"], t["cao"], 1) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(t["alpha"])
        f = ctx.calculate_forces(3.0)["f"]
    rms = np.sqrt(np.sum((f - ew["f"]) ** 2) / len(x))
    assert rms <= 2.0 * target, (t, rms)
    # a fixed cao is kept
    t5 = p3mg.tune(1, x, y, z, q, L, 3.0, target, cao=5)
    assert t5["cao"] == 5 and t5["estimate"] <= target


def test_cli_tune(gpu, tmp_path):
    exe = os.path.join(ROOT, "p3m-standalone_b200", "p3m_gpu")
    r = subprocess.run([exe] + "particles 1000 box 10 mesh 0 cao 0 rcut 3.0 method 7 tune prec 1e-3 "
                       "outfile out.dat".split(), cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Tuned for precision" in r.stdout
    row = open(tmp_path / "out.dat").read().split()
    assert float(row[1]) <= 2e-3  # RMS error against the Ewald reference
