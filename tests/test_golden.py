"""The oracle against the committed golden fixtures, which hold outputs of
the reference itself (tests/golden/make_golden.py) and the reference's own
fixture tests-wall.pos / tests-wall.for.  CPU only."""
import os

import numpy as np
import pytest

import oracle as O
import p3mg

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def wall():
    return dict(np.load(os.path.join(GOLD, "wall.npz")))


@pytest.fixture(scope="module")
def sweep():
    return dict(np.load(os.path.join(GOLD, "sweep.npz")))


@pytest.mark.parametrize("k", range(6))
def test_oracle_p3m_matches_reference_golden(wall, k):
    m, mesh, cao, mc, alpha, rcut = wall["cases"][k]
    m, mesh, cao, mc = int(m), int(mesh), int(cao), int(mc)
    args = (wall["x"], wall["y"], wall["z"], wall["q"], float(wall["L"]))
    r = O.forces(m, mesh, cao, mc, alpha, rcut, *args, cells=False)
    assert O.rel_rms(r["f_k"], wall["fk_%d" % k]) <= 1e-12
    assert O.rel_rms(r["f_r"], wall["fr_%d" % k]) <= 1e-12
    assert O.rel_rms(r["f"], wall["f_%d" % k]) <= 1e-12
    assert abs(r["energy"] - float(wall["energy_%d" % k])) <= 1e-12 * abs(float(wall["energy_%d" % k]))
    G = O.influence(m, mesh, cao, mc, alpha, float(wall["L"]))
    assert O.rel_rms(G, wall["G_%d" % k]) <= 1e-13
    if m in (2, 7):
        b = O.self_force_coeffs(mesh, cao, float(wall["L"]), G)
        assert O.rel_rms(b, wall["self_%d" % k]) <= 1e-12


def test_oracle_ewald_matches_tests_wall_for(wall):
    # tests-wall.for columns 2-4 are total Ewald forces written by the
    # reference's Write_exact_forces with 22 digits; the Ewald oracle must
    # reproduce them to the reference precision (1e-8, common.c:40).
    e = O.ewald(wall["x"], wall["y"], wall["z"], wall["q"], float(wall["L"]), 16)
    assert O.abs_rms(e["f"], wall["for_total"]) <= 1e-6
    assert O.rel_rms(e["f"], wall["for_total"]) <= 1e-6


def test_sweep_values_match_reference_loop(sweep):
    a = p3mg.alpha_sweep(0.1, 2.5, 0.05)
    assert len(a) == int(sweep["n_alphas"]) == 49
    assert a[-1] == 2.4999999999999991
    assert a[24] == float(sweep["alphas"][1])


@pytest.mark.parametrize("k", [0, 2])
def test_oracle_sweep_golden(sweep, k):
    args = (sweep["x"], sweep["y"], sweep["z"], sweep["q"], float(sweep["L"]))
    r = O.forces(7, 16, 7, 2, float(sweep["alphas"][k]), 3.0, *args)
    assert O.rel_rms(r["f"], sweep["f_%d" % k]) <= 1e-12
    assert O.rel_rms(r["f_k"], sweep["fk_%d" % k]) <= 1e-12


def test_oracle_ewald_golden(sweep):
    args = (sweep["x"], sweep["y"], sweep["z"], sweep["q"], float(sweep["L"]))
    e = O.ewald(*args, 16, targets=np.arange(0, 1000, 37))
    assert e["kmax"] == int(sweep["ewald_kmax"])
    assert e["alpha"] == float(sweep["ewald_alpha"])
    assert O.rel_rms(e["f"], sweep["ewald_f"][:, ::37]) <= 1e-12
