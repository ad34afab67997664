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
