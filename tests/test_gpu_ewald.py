"""FP64 Ewald reference forces on the GPU (p3mg_ewald_forces) against the
oracle's Ewald, the reference's own Ewald outputs (golden fixtures) and
the reference fixture tests-wall.for; the analytic error estimates
(p3mg_error_estimate) against the oracle's restatement of the reference's
estimate functions."""
import os

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_ewald_matches_oracle_all_targets(gpu):
    x, y, z, q = p3mg.generate_system(0, 300, 9.0, seed=31)
    ref = O.ewald(x, y, z, q, 9.0, 16)
    with p3mg.Context(1, 16, 5, 1) as ctx:
        ctx.set_system(x, y, z, q, 9.0)
        out = ctx.ewald_forces()
    assert (out["alpha"], out["kmax"]) == (ref["alpha"], ref["kmax"])
    assert O.rel_rms(out["f"], ref["f"]) <= 1e-10


def test_ewald_target_subset(gpu):
    x, y, z, q = p3mg.generate_system(4, 500, 11.0, seed=32)
    tg = np.array([3, 77, 12, 499, 250])
    ref = O.ewald(x, y, z, q, 11.0, 24, targets=tg)
    with p3mg.Context(3, 24, 5, 1) as ctx:
        ctx.set_system(x, y, z, q, 11.0)
        out = ctx.ewald_forces(tg)
    assert O.rel_rms(out["f"], ref["f"]) <= 1e-10


def test_ewald_matches_reference_golden(gpu):
    s = dict(np.load(os.path.join(GOLD, "sweep.npz")))
    with p3mg.Context(7, 16, 7, 2) as ctx:
        ctx.set_system(s["x"], s["y"], s["z"], s["q"], float(s["L"]))
        out = ctx.ewald_forces()
    assert out["kmax"] == int(s["ewald_kmax"]) and out["alpha"] == float(s["ewald_alpha"])
    assert O.rel_rms(out["f"], s["ewald_f"]) <= 1e-10


def test_ewald_matches_tests_wall_for(gpu):
    w = dict(np.load(os.path.join(GOLD, "wall.npz")))
    with p3mg.Context(0, 16, 7, 1) as ctx:
        ctx.set_system(w["x"], w["y"], w["z"], w["q"], float(w["L"]))
        out = ctx.ewald_forces()
    assert O.rel_rms(out["f"], w["for_total"]) <= 1e-6


def test_p3m_error_close_to_reference_estimate(gpu):
    """DeltaF of the GPU P3M against the GPU Ewald is of the size of the
    reference's analytic error estimate (main.c:428-434 prints both)."""
    n, L = 3000, 14.4
    x, y, z, q = p3mg.generate_system(0, n, L, seed=33)
    with p3mg.Context(2, 24, 5, 1) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(1.0)
        f = ctx.calculate_forces(3.5)["f"]
        ew = ctx.ewald_forces()["f"]
    err = p3mg.rms_error(f, ew)
    est = np.hypot(O.kspace_error(2, 24, 5, 1, 1.0, n, float(np.sum(q * q)), L),
                   O.realspace_error(n, float(np.sum(q * q)), L, 3.5, 1.0))
    assert 0.3 * est <= err <= 3.0 * est, (err, est)


@pytest.mark.parametrize("method", [0, 1, 2, 3, 6, 7])
def test_error_estimates_match_oracle(gpu, method):
    n, L = 400, 9.0
    x, y, z, q = p3mg.generate_system(0, n, L, seed=34)
    q2 = float(np.sum(q * q))
    # 16, 20, 12 take the reference's tabulated branch for ik/ik-i (alpha*L on
    # and off the table's grid); 34 and 38 are untabulated (and have no FFT
    # here, so they go through the context-free entry).
    for mesh, cao, mc, alpha, rcut in [(16, 5, 1, 1.1, 3.0), (20, 3, 2, 0.9, 2.5), (12, 7, 1, 1.4, 3.0),
                                       (16, 7, 2, 10.0 / 9.0, 3.0), (34, 3, 1, 1.1, 3.0), (38, 5, 2, 0.95, 3.0)]:
        est = p3mg.estimate_errors(method, mesh, cao, n, q2, L, alpha, rcut, mc)
        ek = O.kspace_error(method, mesh, cao, mc, alpha, n, q2, L)
        er = O.realspace_error(n, q2, L, rcut, alpha)
        # The k-space estimate is 2 q2 sqrt(he / n) / L^2 with he a difference
        # of O(1) mesh sums (the aliased numerator minus the optimal-G term);
        # the GPU adds them in another order, so he agrees to its roundoff
        # floor (~1e-15 absolute) rather than relative to a tiny he.
        he = lambda e: (e * L * L / (2.0 * q2)) ** 2 * n  # noqa: E731
        assert abs(he(est["kspace"]) - he(ek)) <= 1e-6 * he(ek) + 1e-15, (mesh, cao, est["kspace"], ek)
        assert abs(est["realspace"] - er) <= 1e-12 * er
        et = np.hypot(ek, er)
        assert abs(est["total"] - et) <= 1e-6 * et + abs(est["kspace"] - ek)


def test_ewald_reference_outputs_match_oracle(gpu):
    x, y, z, q = p3mg.generate_system(0, 300, 9.0, seed=36)
    ref = O.ewald(x, y, z, q, 9.0, 12)
    tg = np.arange(0, 300, 7)
    with p3mg.Context(2, 12, 4, 1) as ctx:
        ctx.set_system(x, y, z, q, 9.0)
        r = ctx.ewald_reference()
        rt = ctx.ewald_reference(tg)
    assert (r["alpha"], r["kmax"]) == (ref["alpha"], ref["kmax"])
    assert O.rel_rms(r["f"].ravel(), ref["f"].ravel()) <= 1e-10
    assert O.rel_rms(r["f_k"].ravel(), ref["f_k"].ravel()) <= 1e-10
    assert O.rel_rms(rt["f_k"].ravel(), ref["f_k"][:, tg].ravel()) <= 1e-10
    assert 0.0 < r["precision"] <= 1e-8


def test_ewald_kspace_forces_error_k_column(gpu):
    x, y, z, q = p3mg.generate_system(0, 250, 8.0, seed=37)
    with p3mg.Context(1, 10, 5, 1) as ctx:
        ctx.set_system(x, y, z, q, 8.0)
        for alpha, kmax in [(0.9, 9), (1.4, 5)]:
            fk = ctx.ewald_kspace_forces(alpha, kmax)
            o = O.ewald_kspace_plain(x, y, z, q, 8.0, alpha, kmax)
            assert O.rel_rms(fk.ravel(), o.ravel()) <= 1e-10
        with pytest.raises(p3mg.P3MGError):
            ctx.ewald_kspace_forces(0.0, 5)


def test_context_free_estimates_match_context(gpu):
    x, y, z, q = p3mg.generate_system(0, 500, 10.0, seed=38)
    q2 = float(np.sum(q * q))
    for method in (0, 1, 2, 3, 6, 7):
        with p3mg.Context(method, 16, 5, 1) as ctx:
            ctx.set_system(x, y, z, q, 10.0)
            a = ctx.error_estimate(0.83, 3.0, 1)
        b = p3mg.estimate_errors(method, 16, 5, 500, q2, 10.0, 0.83, 3.0, 1)
        for k in ("total", "kspace", "realspace"):
            assert abs(a[k] - b[k]) <= 1e-12 * abs(a[k])
