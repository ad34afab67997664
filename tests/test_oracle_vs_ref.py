"""Pin the oracle restatement against the reference compiled from its own
sources (oracle/_ref, built by oracle/build_ref.sh where the sources are
present).  Skipped where oracle/_ref was not built."""
import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built")


@pytest.mark.parametrize("method", [0, 1, 2, 3, 6, 7])
@pytest.mark.parametrize("mesh,cao,mc", [(16, 7, 2), (12, 3, 1), (8, 1, 1), (10, 4, 1), (15, 5, 1)])
def test_forces(method, mesh, cao, mc):
    if method in (6, 7) and mesh % 2:
        pytest.skip("r2c methods need an even mesh")
    x, y, z, q = p3mg.generate_system(0, 300, 10.0, seed=mesh * 10 + cao)
    r = O.ref_forces(method, mesh, cao, mc, 1.1, 3.0, x, y, z, q, 10.0, want_G=True)
    o = O.forces(method, mesh, cao, mc, 1.1, 3.0, x, y, z, q, 10.0)
    assert O.rel_rms(o["f_k"], r["f_k"]) <= 1e-12
    assert O.rel_rms(o["f"], r["f"]) <= 1e-12
    assert O.rel_rms(O.influence(method, mesh, cao, mc, 1.1, 10.0), r["G"]) <= 1e-13


@pytest.mark.parametrize("system_type", [1, 3, 4, 5])
def test_forces_nonuniform_systems(system_type):
    x, y, z, q = p3mg.generate_system(system_type, 400, 12.0, seed=4)
    for method in (1, 7):
        r = O.ref_forces(method, 16, 5, 1, 0.9, 3.5, x, y, z, q, 12.0)
        o = O.forces(method, 16, 5, 1, 0.9, 3.5, x, y, z, q, 12.0)
        assert O.rel_rms(o["f"], r["f"]) <= 1e-12


def test_edge_positions_on_mesh_points_and_box_edges():
    L = 8.0
    pts = np.array([[0.0, 0.0, 0.0], [L - 1e-12, 0.5, 7.999999], [4.0, 4.0, 4.0], [1.0, 2.0, 3.0],
                    [0.25, 7.75, 0.5], [2.5, 2.5, 2.5]])
    q = np.array([1.0, -1.0, 1.0, -1.0, 2.0, -2.0])
    for method in (0, 1, 2, 3, 6, 7):
        r = O.ref_forces(method, 8, 3, 1, 1.0, 2.0, pts[:, 0], pts[:, 1], pts[:, 2], q, L)
        o = O.forces(method, 8, 3, 1, 1.0, 2.0, pts[:, 0], pts[:, 1], pts[:, 2], q, L)
        assert O.rel_rms(o["f"], r["f"]) <= 1e-12


def test_self_force_coefficients():
    x, y, z, q = p3mg.generate_system(0, 50, 9.0, seed=1)
    for method in (2, 7):
        b = O.ref_self_force_coeffs(method, 12, 4, 1, 1.3, x, y, z, q, 9.0)
        G = O.influence(method, 12, 4, 1, 1.3, 9.0)
        assert O.rel_rms(O.self_force_coeffs(12, 4, 9.0, G), b) <= 1e-12


def test_realspace_and_ewald():
    x, y, z, q = p3mg.generate_system(0, 250, 9.0, seed=2)
    fr, e = O.ref_realteil(x, y, z, q, 9.0, 2.9, 1.1)
    fo, eo = O.realspace(x, y, z, q, 9.0, 2.9, 1.1, cells=True)
    assert O.rel_rms(fo, fr) <= 1e-13 and abs(eo - e) <= 1e-12 * abs(e)
    r = O.ref_ewald(x, y, z, q, 9.0, 16)
    o = O.ewald(x, y, z, q, 9.0, 16)
    assert (o["alpha"], o["kmax"]) == (r["alpha"], r["kmax"])
    assert O.rel_rms(o["f"], r["f"]) <= 1e-13


@pytest.mark.parametrize("method", [0, 1, 2, 3, 6, 7])
def test_error_estimates_untabulated(method):
    # meshes 34 and 38 are not tabulated in the reference's q tables -> analytic branch
    q = 1.0 - 2.0 * (np.arange(200) % 2)
    for mesh, cao, mc in [(34, 3, 1), (38, 5, 2)]:
        e = O.ref_error_estimates(method, mesh, cao, mc, 1.1, 3.0, q, 8.0)
        ok = O.kspace_error(method, mesh, cao, mc, 1.1, 200, 200.0, 8.0)
        assert abs(ok - e[1]) <= 1e-12 * abs(e[1])
        assert abs(O.realspace_error(200, 200.0, 8.0, 3.0, 1.1) - e[2]) <= 1e-15


def test_estimate_table_meshes_match_reference_lookup():
    # The table lookup answers -1 exactly for the meshes the reference has no table for.
    for mesh in range(1, 601):
        assert (O.ref_find_error(50.5, mesh, 3, 1) >= 0.0) == O.estimate_table_mesh(mesh), mesh


@pytest.mark.parametrize("method", [0, 1, 6])
def test_error_estimates_tabulated(method):
    # Tabulated (mesh, cao): the reference interpolates its precomputed tables; the
    # oracle evaluates the same mesh sum at the two bracketing alpha*L grid points.
    # The tables hold 7 significant digits; at alpha*L where the mesh sum falls
    # below ~1e-8 it is a cancellation of much larger terms and the table and
    # the sum only agree to a few digits, so the cases stay above that.
    n, L = 200, 8.0
    q = 1.0 - 2.0 * (np.arange(n) % 2)
    for mesh, cao, alpha in [(16, 7, 1.25), (16, 3, 0.8), (20, 5, 1.6), (12, 2, 2.0), (32, 4, 2.2), (16, 7, 12.6)]:
        e = O.ref_error_estimates(method, mesh, cao, 2, alpha, 3.0, q, L)
        ok = O.kspace_error(method, mesh, cao, 2, alpha, n, float(n), L)
        assert abs(ok - e[1]) <= 2e-6 * abs(e[1]), (mesh, cao, alpha, ok, e[1])
        assert abs(np.hypot(ok, O.realspace_error(n, float(n), L, 3.0, alpha)) - e[0]) <= 2e-6 * e[0]


def test_ewald_kspace_error_k_column_matches_reference():
    # main.c's error_k column: Ewald k-space forces with the P3M mesh as table size
    x, y, z, q = p3mg.generate_system(0, 120, 7.0, seed=5)
    for mesh, alpha in [(6, 1.2), (8, 0.7)]:
        r = O.ref_ewald_kspace_main(x, y, z, q, 7.0, mesh, alpha)
        o = O.ewald_kspace_plain(x, y, z, q, 7.0, alpha, mesh - 1)
        assert O.rel_rms(o.ravel(), r.ravel()) <= 1e-13
