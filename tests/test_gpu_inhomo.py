"""Inhomogeneous k-space error estimate and error map on the GPU
(p3mg_inhomo_error, p3mg_error_map) against the reference's outputs in
tests/golden/inhomo.npz and the oracle (Generic_error_estimate_inhomo
p3m-common.c:437-719, Error_map p3m-common.c:402-435).

Tolerances: FP64 throughout; the alias-sum estimates to 1e-10 relative
(the GPU forms the factored alias sum and the DFTs in another order than
the reference), mesh columns to 1e-10 of their scale.  With mc = 0 the
reference's kernel U2 G_opt - Ghat vanishes up to rounding, so that
estimate is rounding noise on both sides and only its size is checked."""
import os

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
G = np.load(os.path.join(ROOT, "tests", "golden", "inhomo.npz"))


def ctx_with(x, y, z, q, L):
    c = p3mg.Context(0, 8, 3, 1)
    c.set_system(x, y, z, q, L)
    return c


def golden_ctx():
    return ctx_with(G["x"], G["y"], G["z"], G["q"], float(G["L"]))


@pytest.mark.parametrize("k", range(len(G["inhomo_cases"])))
def test_estimate_matches_reference_fixture(gpu, k):
    cm, cc, a, uni, m, c, mc = G["inhomo_cases"][k]
    ref = float(G["inhomo_estimates"][k])
    with golden_ctx() as ctx:
        ours = ctx.inhomo_error(a, mesh=int(m), cao=int(c), mc=int(mc), uniform=bool(uni), collect_mesh=int(cm),
                                collect_cao=int(cc))
    if mc == 0:
        assert ref < 1e-9 and 0.0 <= ours < 1e-8
    else:
        assert abs(ours - ref) <= 1e-10 * abs(ref), (ours, ref)


def test_mesh_columns_match_oracle_and_reference_file(gpu):
    cm, cc, a, uni, m, c, mc = (int(v) if i != 2 else v for i, v in enumerate(G["inhomo_cases"][1]))
    x, y, z, q, L = G["x"], G["y"], G["z"], G["q"], float(G["L"])
    with golden_ctx() as ctx:
        est, cols = ctx.inhomo_error(a, mesh=m, cao=c, mc=mc, uniform=bool(uni), collect_mesh=cm, collect_cao=cc,
                                     want_meshes=True)
    oest, ocols = O.inhomo_error(x, y, z, q, L, a, uni, m, c, mc, cm, cc, want_meshes=True)
    assert abs(est - oest) <= 1e-10 * oest
    real_of = [0, 1, 1, 3, 3]
    for col in range(5):
        scale = np.max(np.abs(ocols[:, real_of[col]]))
        assert np.max(np.abs(cols[:, col] - ocols[:, col])) <= 1e-10 * scale, col
    ref = G["inhomo_columns_1"]
    for col in (0, 1, 3):
        assert np.all(np.abs(cols[:, col] - ref[:, 3 + col]) <= 6e-7 * np.abs(ref[:, 3 + col]) + 1e-12), col


@pytest.mark.parametrize("n,L,mesh,cao,mc,cm,cc,uniform", [
    (20000, 20.0, 64, 5, 1, 24, 4, False),   # the reference CLI's default estimator mesh and cao
    (20000, 20.0, 32, 5, 2, 24, 4, False),
    (3000, 10.0, 30, 4, 1, 30, 4, True),     # 2*3*5 mesh, uniform rho^2
    (3000, 10.0, 16, 7, 1, 40, 3, False),    # collection mesh above twice the estimator's (indices wrap)
])
def test_estimate_matches_oracle(gpu, n, L, mesh, cao, mc, cm, cc, uniform):
    x, y, z, q = p3mg.generate_system(0, n, L, seed=3)
    with ctx_with(x, y, z, q, L) as ctx:
        ours = ctx.inhomo_error(1.1, mesh=mesh, cao=cao, mc=mc, uniform=uniform, collect_mesh=cm, collect_cao=cc)
    ref = O.inhomo_error(x, y, z, q, L, 1.1, int(uniform), mesh, cao, mc, cm, cc)
    assert abs(ours - ref) <= 1e-10 * abs(ref), (ours, ref)


def test_uniform_estimate_at_full_size(gpu):
    # rho^2 constant: the error density is the constant q2 * sum_r K2(r), so with
    # the estimator's own stencil (weights summing to 1) the estimate is
    # q2 * sqrt(DFT(K2)(0) / n), and it does not depend on the positions
    n, L = 1_000_000, 100.0
    x, y, z, q = p3mg.generate_system(0, n, L, seed=9)
    q2 = float(np.sum(q * q))
    with ctx_with(x, y, z, q, L) as ctx:
        est, cols = ctx.inhomo_error(0.3, mesh=64, cao=5, mc=1, uniform=True, want_meshes=True)
        ctx.set_system(np.roll(x, 17), y[::-1].copy(), np.roll(z, -5), q, L)
        est2 = ctx.inhomo_error(0.3, mesh=64, cao=5, mc=1, uniform=True)
    assert est > 0
    assert abs(est - q2 * np.sqrt(cols[0, 3] / n)) <= 1e-10 * est
    assert abs(est2 - est) <= 1e-10 * est
    assert np.allclose(cols[:, 0], q2 / 64 ** 3, rtol=1e-14, atol=0)


def test_rho2_mesh_holds_every_charge_square(gpu):
    # assigned rho^2 sums to sum q^2 (B-spline weights partition unity)
    n, L = 200_000, 40.0
    x, y, z, q = p3mg.generate_system(0, n, L, seed=4)
    q = q * np.linspace(0.5, 2.0, n)
    with ctx_with(x, y, z, q, L) as ctx:
        _, cols = ctx.inhomo_error(0.5, mesh=48, cao=6, mc=0, want_meshes=True)
    assert abs(cols[:, 0].sum() - np.sum(q * q)) <= 1e-10 * np.sum(q * q)


@pytest.mark.parametrize("k", range(len(G["map_cases"])))
def test_error_map_matches_reference_fixture(gpu, k):
    m, c = (int(v) for v in G["map_cases"][k])
    with golden_ctx() as ctx:
        ours, tot = ctx.error_map(G["fk"], G["fk_ref"], mesh=m, cao=c)
    ref = G["map_%d" % k]
    assert np.max(np.abs(ours - ref)) <= 1e-13 * np.max(np.abs(ref))
    total = np.sum((G["fk_ref"] - G["fk"]) ** 2)
    assert abs(tot[0] - total) <= 1e-13 * total
    assert abs(tot[1] - total) <= 1e-12 * total


def test_error_map_at_full_size(gpu):
    # 1M particles: the map holds every particle's squared error once, and a
    # small case of the same draw matches the oracle point by point
    n, L = 1_000_000, 100.0
    x, y, z, q = p3mg.generate_system(0, n, L, seed=8)
    rng = np.random.default_rng(2)
    fk = rng.normal(size=(3, n))
    fr = fk + 1e-2 * rng.normal(size=(3, n))
    with ctx_with(x, y, z, q, L) as ctx:
        ours, tot = ctx.error_map(fk, fr, mesh=64, cao=5)
    total = np.sum((fr - fk) ** 2)
    assert abs(tot[0] - total) <= 1e-11 * total
    assert abs(ours.sum() - total) <= 1e-11 * total
    k = 5000
    with ctx_with(x[:k], y[:k], z[:k], q[:k], L) as ctx:
        small, _ = ctx.error_map(fk[:, :k], fr[:, :k], mesh=20, cao=4)
    ref = O.error_map(x[:k], y[:k], z[:k], L, fk[:, :k], fr[:, :k], 20, 4)
    assert np.max(np.abs(small - ref)) <= 1e-13 * np.max(ref)


def test_bad_arguments(gpu):
    with golden_ctx() as ctx:
        for kw, code in [(dict(mesh=11), p3mg.ERR_MESH), (dict(mesh=3), p3mg.ERR_MESH), (dict(cao=8), p3mg.ERR_CAO),
                         (dict(collect_cao=0), p3mg.ERR_CAO), (dict(mc=11), p3mg.ERR_ARG),
                         (dict(collect_mesh=0), p3mg.ERR_ARG)]:
            with pytest.raises(p3mg.P3MGError) as e:
                ctx.inhomo_error(1.0, **kw)
            assert e.value.status == code, kw
        with pytest.raises(p3mg.P3MGError) as e:
            ctx.error_map(G["fk"], G["fk_ref"], mesh=8, cao=0)
        assert e.value.status == p3mg.ERR_CAO
    with p3mg.Context(0, 8, 3, 1) as ctx:
        with pytest.raises(p3mg.P3MGError) as e:
            ctx.inhomo_error(1.0, mesh=8)
        assert e.value.status == p3mg.ERR_NOSYS


def test_kernels_are_counted(gpu):
    with golden_ctx() as ctx:
        before = ctx.launch_count()
        ctx.inhomo_error(1.0, mesh=8, cao=3, mc=1)
        after = ctx.launch_count()
    # rho^2, kernel, 3 FFT axes per transform, alias sums and passes, collection, sums
    assert after - before >= 15
