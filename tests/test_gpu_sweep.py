"""Batched alpha sweep (p3mg_sweep) against single-alpha evaluations, the
reference's own sweep forces (golden sweep.npz: method 7, 1000 particles,
mesh 16, cao 7, mc 2, rcut 3, alphas of 0.1..2.5 step 0.05) and its RMS
errors against the reference's Ewald forces."""
import os

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_alpha_range_matches_reference_loop():
    a = p3mg.alpha_range(0.1, 2.5, 0.05)
    assert len(a) == 49 and a[-1] == 2.4999999999999991
    ref = []
    x = 0.1
    while x <= 2.5:
        ref.append(x)
        x += 0.05
    assert np.array_equal(a, np.array(ref))


@pytest.mark.parametrize("method", [0, 1, 2, 3, 6, 7])
@pytest.mark.parametrize("precision", [p3mg.FP64, p3mg.FP32_MIXED])
def test_sweep_equals_single_alpha_steps(gpu, method, precision):
    x, y, z, q = p3mg.generate_system(0, 400, 9.0, seed=51)
    alphas = np.array([0.6, 0.85, 1.1, 1.35, 1.6])
    with p3mg.Context(method, 16, 5, 1, precision) as ctx:
        ctx.set_system(x, y, z, q, 9.0)
        singles = []
        for a in alphas:
            ctx.influence(a)
            singles.append(ctx.calculate_forces(2.8)["f"].copy())
        for mb in (0, 2):  # one pass, and passes of two alphas
            sw = ctx.sweep(2.8, alphas, want_forces=True, max_batch=mb)["forces"]
            for k in range(len(alphas)):
                tol = 1e-13 if precision == p3mg.FP64 else 1e-6
                assert O.rel_rms(sw[k].ravel(), singles[k].ravel()) <= tol, (mb, k)


@pytest.mark.parametrize("system_type,n,L,na", [
    (0, 600, 10.0, 9),    # 16 lanes per pair, two pairs per step
    (0, 600, 10.0, 12),
    (0, 600, 10.0, 20),   # one alpha per lane
    (0, 600, 10.0, 40),   # two per lane
    (4, 4000, 20.0, 70),  # two groups (64 + 6: 8 lanes per pair); the Gaussian centre overflows the staging array
])
def test_fp32_many_alpha_sweep_equals_single_alpha_steps(gpu, system_type, n, L, na):
    # 9 or more alphas in one pass: FP32 real space with the lanes on the
    # alphas (one candidate search for up to 64 alphas)
    x, y, z, q = p3mg.generate_system(system_type, n, L, seed=61)
    alphas = np.linspace(0.7, 1.6, na)
    with p3mg.Context(1, 16, 5, 1, p3mg.FP32_MIXED) as ctx:
        ctx.set_system(x, y, z, q, L)
        sw = ctx.sweep(2.8, alphas, want_forces=True, max_batch=na)["forces"]
        for k in sorted({0, 31, 32, 33, na // 2, 63, 64, na - 1} & set(range(na))):
            ctx.influence(alphas[k])
            one = ctx.calculate_forces(2.8)["f"]
            assert O.rel_rms(sw[k].ravel(), one.ravel()) <= 1e-6, k


def test_sweep_golden_method7_config(gpu):
    g = np.load(os.path.join(GOLD, "sweep.npz"))
    x, y, z, q, L = g["x"], g["y"], g["z"], g["q"], float(g["L"])
    alphas = p3mg.alpha_range(0.1, 2.5, 0.05)
    assert len(alphas) == int(g["n_alphas"])
    ref = np.asarray(g["ewald_f"]).reshape(3, len(x))
    with p3mg.Context(7, 16, 7, 2) as ctx:
        ctx.set_system(x, y, z, q, L)
        r = ctx.sweep(3.0, alphas, ref=ref, want_forces=True)
    for j, k in enumerate((0, 24, 48)):
        assert alphas[k] == g["alphas"][j]
        assert O.rel_rms(r["forces"][k].ravel(), np.asarray(g["f_%d" % j]).ravel()) <= 1e-10
    # RMS error column of the reference's out.dat: sqrt(sum |f - f_ewald|^2) / sqrt(N)
    for k in range(len(alphas)):
        want = np.sqrt(np.sum((r["forces"][k] - ref) ** 2)) / np.sqrt(len(x))
        assert abs(r["rms"][k] - want) <= 1e-12 * want


def test_graph_replay_follows_alpha_changes(gpu):
    # a captured step reads alpha from the device, so recomputing G for a new
    # alpha between replays gives that alpha's real-space forces too
    x, y, z, q = p3mg.generate_system(0, 500, 10.0, seed=52)
    with p3mg.Context(1, 16, 5, 1) as ref_ctx, p3mg.Context(1, 16, 5, 1) as ctx:
        ref_ctx.set_system(x, y, z, q, 10.0)
        ctx.set_system(x, y, z, q, 10.0)
        ctx.set_graph(True)
        for a in (0.7, 0.9, 1.1, 1.3):
            ctx.influence(a)
            got = ctx.calculate_forces(3.0)
            ref_ctx.influence(a)
            want = ref_ctx.calculate_forces(3.0)
            assert O.rel_rms(got["f"].ravel(), want["f"].ravel()) <= 1e-14
            assert O.rel_rms(got["f_r"].ravel(), want["f_r"].ravel()) <= 1e-14


def test_graph_replay_follows_box_changes(gpu):
    # a new box length with the same particle count re-captures the step
    x, y, z, q = p3mg.generate_system(0, 600, 10.0, seed=53)
    with p3mg.Context(7, 16, 5, 1) as ctx, p3mg.Context(7, 16, 5, 1) as ref:
        ctx.set_graph(True)
        for L in (10.0, 10.0, 10.0, 11.5, 11.5, 12.25):
            s = L / 10.0
            for c in (ctx, ref):
                c.set_system(x * s, y * s, z * s, q, L)
                c.influence(1.0)
            got = ctx.calculate_forces(3.0)["f"]
            want = ref.calculate_forces(3.0)["f"]
            assert O.rel_rms(got.ravel(), want.ravel()) <= 1e-14, L


@pytest.mark.parametrize("method", [1, 7])
@pytest.mark.parametrize("precision,lo,hi,na,nodes,tol", [
    (p3mg.FP32_MIXED, 0.7, 1.4, 32, 10, 2e-6),   # interpolated: FP32 noise level
    (p3mg.FP64, 0.8, 1.2, 48, 16, 1e-12),        # interpolated: checked to 1e-12
    (p3mg.FP64, 0.7, 1.4, 48, 0, 1e-13),         # check ~1e-9 > 1e-12: every alpha evaluated
])
def test_interpolated_sweep_matches_single_alpha_steps(gpu, method, precision, lo, hi, na, nodes, tol):
    # many alphas over a narrow range: forces interpolated in 1/alpha^2 from
    # exact evaluations at Chebyshev nodes when two check alphas confirm it;
    # every alpha's forces must still match its own single-alpha step
    x, y, z, q = p3mg.generate_system(0, 3000, 14.4, seed=54)
    alphas = np.linspace(lo, hi, na)
    ref = np.zeros((3, len(x)))
    with p3mg.Context(method, 32, 7, 1, precision) as ctx:
        ctx.set_system(x, y, z, q, 14.4)
        r = ctx.sweep(3.0, alphas, ref=ref, want_forces=True)
        assert r["nodes"] == nodes, r["check"]
        assert r["check"] >= 0.0  # the interpolation was tried
        if nodes == 0:
            assert r["check"] > 1e-12
        ex = ctx.sweep(3.0, alphas[:5], want_forces=True, max_batch=32)
        assert ex["nodes"] == 0 and ex["check"] == -1.0  # a batch limit: every alpha evaluated
        for k in range(0, len(alphas), 5):
            ctx.influence(alphas[k])
            single = ctx.calculate_forces(3.0)["f"]
            assert O.rel_rms(r["forces"][k].ravel(), single.ravel()) <= tol, k
            # rms against the (zero) reference is the RMS force itself
            assert abs(r["rms"][k] - np.sqrt(np.sum(r["forces"][k] ** 2) / len(x))) <= 1e-12 * r["rms"][k]


@pytest.mark.parametrize("precision,nodes,rtol", [
    (p3mg.FP32_MIXED, 10, 2e-6),   # two sweeps: FP32 sums in atomic binning order differ at ~1e-7
    (p3mg.FP64, 16, 1e-9),
])
def test_rms_only_interpolated_sweep_matches_forces_sweep(gpu, precision, nodes, rtol):
    # without a force output the interpolation goes straight into the squared
    # errors (one kernel); the RMS must equal the one of the interpolated
    # forces against the same (host) reference rows
    x, y, z, q = p3mg.generate_system(0, 3000, 14.4, seed=56)
    alphas = np.linspace(0.8, 1.2, 40)
    with p3mg.Context(1, 32, 7, 1, precision) as ctx:
        ctx.set_system(x, y, z, q, 14.4)
        ctx.influence(1.0)
        f1 = ctx.calculate_forces(3.0)["f"]
        rng = np.random.default_rng(7)
        ref = f1 + 0.01 * np.sqrt(np.mean(f1 ** 2)) * rng.standard_normal(f1.shape)
        a = ctx.sweep(3.0, alphas, ref=ref)
        b = ctx.sweep(3.0, alphas, ref=ref, want_forces=True)
        assert a["nodes"] == b["nodes"] == nodes, (a["check"], b["check"])
        assert a["forces"] is None
        direct = np.sqrt(np.sum((b["forces"] - ref[None]) ** 2, axis=(1, 2)) / len(x))
        np.testing.assert_allclose(a["rms"], direct, rtol=rtol)
        np.testing.assert_allclose(b["rms"], direct, rtol=1e-9)


def test_wide_alpha_range_is_evaluated_alpha_by_alpha(gpu):
    x, y, z, q = p3mg.generate_system(0, 1000, 10.0, seed=55)
    with p3mg.Context(7, 16, 7, 2) as ctx:
        ctx.set_system(x, y, z, q, 10.0)
        r = ctx.sweep(3.0, p3mg.alpha_range(0.1, 2.5, 0.05))
        assert r["nodes"] == 0


@pytest.mark.parametrize("precision,tol", [(p3mg.FP64, 1e-12), (p3mg.FP32_MIXED, 1e-6)])
def test_sweep_grid_matches_sweeps(gpu, precision, tol):
    # p3mg_sweep_grid: several (mesh, cao) points of one system, real space
    # computed once and shared, k-space passes concurrent -- the same RMS
    # errors per alpha as each context's own exact sweep
    L = 12.0
    x, y, z, q = p3mg.generate_system(5, 1500, L, seed=29)
    al = np.linspace(0.5, 2.0, 12)
    with p3mg.Context(7, 16, 7, 1) as ec:
        ec.set_system(x, y, z, q, L)
        ref = ec.ewald_forces()["f"]
    frms = float(np.sqrt(np.sum(ref ** 2) / len(x)))
    pts = [(7, 16, 5), (7, 24, 7), (7, 32, 3), (2, 20, 4)]
    ctxs = [p3mg.Context(m, mesh, cao, 1, precision) for m, mesh, cao in pts]
    try:
        for c in ctxs:
            c.set_system(x, y, z, q, L)
        grid = p3mg.sweep_grid(ctxs, 3.0, al, ref)
        for i, c in enumerate(ctxs):
            own = c.sweep(3.0, al, ref=ref, max_batch=len(al))["rms"]
            # the mesh sums take floating-point atomics: runs agree to the
            # rounding of the forces, tol of the RMS force
            assert np.max(np.abs(grid[i] - own)) <= tol * frms
    finally:
        for c in ctxs:
            c.close()
