"""GPU path against the committed golden fixtures (outputs of the reference
itself, tests/golden/make_golden.py), plus edge cases and properties."""
import os

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_FP64 = 1e-10


@pytest.fixture(scope="module")
def wall():
    return dict(np.load(os.path.join(GOLD, "wall.npz")))


@pytest.fixture(scope="module")
def sweep():
    return dict(np.load(os.path.join(GOLD, "sweep.npz")))


@pytest.mark.parametrize("k", range(6))
def test_wall_golden(gpu, wall, k):
    m, mesh, cao, mc, alpha, rcut = wall["cases"][k]
    with p3mg.Context(int(m), int(mesh), int(cao), int(mc)) as ctx:
        ctx.set_system(wall["x"], wall["y"], wall["z"], wall["q"], float(wall["L"]))
        ctx.influence(alpha)
        out = ctx.calculate_forces(rcut)
        G, b = ctx.get_influence()
    assert O.rel_rms(out["f"], wall["f_%d" % k]) <= TOL_FP64
    assert O.rel_rms(out["f_k"], wall["fk_%d" % k]) <= TOL_FP64
    assert O.rel_rms(out["f_r"], wall["fr_%d" % k]) <= TOL_FP64
    assert abs(out["energy"] - float(wall["energy_%d" % k])) <= 1e-10 * abs(float(wall["energy_%d" % k]))
    assert O.rel_rms(G, wall["G_%d" % k]) <= 1e-13
    if int(m) in (2, 7):
        assert O.rel_rms(b, wall["self_%d" % k]) <= 1e-12


def test_sweep_golden_all_alphas_one_context(gpu, sweep):
    """Config-1 sweep: one context, influence per alpha (main.c:375-386)."""
    args = (sweep["x"], sweep["y"], sweep["z"], sweep["q"], float(sweep["L"]))
    with p3mg.Context(7, 16, 7, 2) as ctx:
        ctx.set_system(*args)
        for k, a in enumerate(sweep["alphas"]):
            ctx.influence(float(a))
            out = ctx.calculate_forces(3.0)
            assert O.rel_rms(out["f"], sweep["f_%d" % k]) <= TOL_FP64
            assert O.rel_rms(out["f_k"], sweep["fk_%d" % k]) <= TOL_FP64


def test_empty_and_single_particle(gpu):
    with p3mg.Context(1, 16, 7, 1) as ctx:
        ctx.set_system(np.zeros(0), np.zeros(0), np.zeros(0), np.zeros(0), 10.0)
        ctx.influence(1.0)
        out = ctx.calculate_forces(3.0)
        assert out["f"].shape == (3, 0) and out["energy"] == 0.0
    x, y, z, q = np.array([1.3]), np.array([2.2]), np.array([9.9]), np.array([1.0])
    for method in (0, 1, 2, 3, 6, 7):
        with p3mg.Context(method, 8, 4, 1) as ctx:
            ctx.set_system(x, y, z, q, 10.0)
            ctx.influence(1.0)
            out = ctx.calculate_forces(3.0)
        ref = O.forces(method, 8, 4, 1, 1.0, 3.0, x, y, z, q, 10.0)
        assert np.max(np.abs(out["f"] - ref["f"])) <= 1e-12 + 1e-10 * np.max(np.abs(ref["f"]))


def test_mesh_equal_to_cao_and_edges(gpu):
    L = 8.0
    pts = np.array([[0.0, 0.0, 0.0], [L - 1e-12, 0.5, 7.999999], [4.0, 4.0, 4.0], [1.0, 2.0, 3.0],
                    [0.25, 7.75, 0.5], [2.5, 2.5, 2.5]])
    q = np.array([1.0, -1.0, 1.0, -1.0, 2.0, -2.0])
    for method, mesh, cao in [(0, 7, 7), (1, 8, 7), (2, 8, 3), (3, 5, 5), (6, 8, 3), (7, 6, 6)]:
        with p3mg.Context(method, mesh, cao, 1) as ctx:
            ctx.set_system(pts[:, 0], pts[:, 1], pts[:, 2], q, L)
            ctx.influence(1.0)
            out = ctx.calculate_forces(2.0)
        ref = O.forces(method, mesh, cao, 1, 1.0, 2.0, pts[:, 0], pts[:, 1], pts[:, 2], q, L)
        assert O.rel_rms(out["f"], ref["f"]) <= TOL_FP64


@pytest.mark.parametrize("system_type", [1, 3, 4, 5])
def test_nonuniform_systems(gpu, system_type):
    x, y, z, q = p3mg.generate_system(system_type, 3000, 16.0, seed=9)
    for method in (1, 2):
        with p3mg.Context(method, 24, 5, 1) as ctx:
            ctx.set_system(x, y, z, q, 16.0)
            ctx.influence(0.9)
            out = ctx.calculate_forces(3.0)
        ref = O.forces(method, 24, 5, 1, 0.9, 3.0, x, y, z, q, 16.0)
        assert O.rel_rms(out["f"], ref["f"]) <= TOL_FP64


def test_kspace_forces_accumulate_like_reference(gpu):
    """Kspace_force adds into f_k and subtracts the ad self-force from f."""
    x, y, z, q = p3mg.generate_system(0, 200, 9.0, seed=1)
    fk_ref, ft_ref = O.kspace(7, 12, 5, 1, 1.0, x, y, z, q, 9.0)
    with p3mg.Context(7, 12, 5, 1) as ctx:
        ctx.set_system(x, y, z, q, 9.0)
        ctx.influence(1.0)
        fk = np.full((3, 200), 0.5)
        ft = np.full((3, 200), -0.25)
        ctx.kspace_forces(fk, ft)
    assert O.rel_rms(fk - 0.5, fk_ref) <= TOL_FP64
    assert O.rel_rms(ft + 0.25, ft_ref) <= 1e-9


def test_deterministic_to_rounding(gpu):
    x, y, z, q = p3mg.generate_system(0, 20000, 27.0, seed=4)
    with p3mg.Context(1, 32, 7, 1) as ctx:
        ctx.set_system(x, y, z, q, 27.0)
        ctx.influence(0.9)
        a = ctx.calculate_forces(3.5)
        b = ctx.calculate_forces(3.5)
    assert O.rel_rms(a["f"], b["f"]) <= 1e-13


def test_graph_replay_matches_eager(gpu):
    x, y, z, q = p3mg.generate_system(0, 5000, 17.0, seed=8)
    with p3mg.Context(3, 24, 6, 1) as ctx:
        ctx.set_system(x, y, z, q, 17.0)
        ctx.influence(1.0)
        eager = ctx.calculate_forces(3.0)
        ctx.set_graph(True)
        outs = []
        for _ in range(4):
            ctx.compute(3.0)
            outs.append(ctx.get_forces())
        n0 = ctx.launch_count()
        ctx.compute(3.0)
        ctx.get_forces()
        per_replay = ctx.launch_count() - n0
    for o in outs:
        assert O.rel_rms(o["f"], eager["f"]) <= 1e-13
    assert per_replay > 5


def test_newton_third_law_real_space(gpu):
    x, y, z, q = p3mg.generate_system(0, 50000, 36.8, seed=2)
    for prec, tol in ((p3mg.FP64, 1e-12), (p3mg.FP32_MIXED, 1e-5)):
        with p3mg.Context(1, 32, 3, 1, prec) as ctx:
            ctx.set_system(x, y, z, q, 36.8)
            fr, e = ctx.real_forces(3.5, 0.9)
        assert np.max(np.abs(fr.sum(axis=1))) <= tol * np.sqrt(np.sum(fr ** 2))


def test_fp32_error_against_ewald_within_1p1_of_fp64(gpu):
    """FP32-mixed bar: its RMS error vs the FP64 Ewald forces is within 1.1x
    of the FP64 path's at the same (mesh, cao, rcut, alpha).  The cases sit
    in the 1e-4..1e-2 absolute RMS error regime the FP32 path targets (the
    headline configuration estimates 4.7e-3); FP32 rounding of the closest
    random pairs sets a floor near 1e-5, so far more accurate parameter sets
    are the FP64 path's domain."""
    n, L = 2000, 12.6
    x, y, z, q = p3mg.generate_system(0, n, L, seed=11)
    ew = O.ewald(x, y, z, q, L, 32)
    for method, mesh, cao, alpha in [(1, 20, 5, 0.9), (3, 20, 5, 0.9), (7, 24, 5, 0.9), (0, 24, 4, 0.85),
                                     (2, 20, 4, 0.85), (6, 24, 6, 0.95)]:
        errs = {}
        for prec in (p3mg.FP64, p3mg.FP32_MIXED):
            with p3mg.Context(method, mesh, cao, 1, prec) as ctx:
                ctx.set_system(x, y, z, q, L)
                ctx.influence(alpha)
                errs[prec] = p3mg.rms_error(ctx.calculate_forces(3.5)["f"], ew["f"])
        assert errs[p3mg.FP64] >= 1e-4, (method, errs)  # stay in the regime described above
        assert errs[p3mg.FP32_MIXED] <= 1.1 * errs[p3mg.FP64], (method, errs)


def test_headline_size_fp32_vs_fp64(gpu):
    """At the full headline size (1M particles, mesh 128, cao 7, ik-i) the
    FP32-mixed forces agree with the FP64 path far below the P3M error (the
    reference's own estimate there is 4.7e-3 absolute RMS, i.e. a relative
    RMS of order 1e-3), and the total force sums to ~0 (neutral system;
    ik differentiation and pair forces conserve momentum)."""
    x, y, z, q = p3mg.generate_system(0, 1_000_000, 100.0, seed=12345)
    outs = {}
    for prec in (p3mg.FP64, p3mg.FP32_MIXED):
        with p3mg.Context(1, 128, 7, 1, prec) as ctx:
            ctx.set_system(x, y, z, q, 100.0)
            ctx.influence(0.9)
            outs[prec] = ctx.calculate_forces(3.5)
    d = O.rel_rms(outs[p3mg.FP32_MIXED]["f"], outs[p3mg.FP64]["f"])
    assert d <= 1e-4, d
    f = outs[p3mg.FP64]["f"]
    assert np.max(np.abs(f.sum(axis=1))) <= 1e-6 * np.sqrt(np.sum(f ** 2))
