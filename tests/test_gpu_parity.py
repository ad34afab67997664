"""GPU parity: the p3mg C ABI (CUDA kernels) against the CPU oracle on the
same seeded inputs.  FP64 bar: relative RMS force difference <= 1e-10
(rel_rms = sqrt(sum |F_gpu - F_ref|^2) / sqrt(sum |F_ref|^2))."""
import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10

CASES = [
    # method, mesh, cao, mc, alpha, rcut, n, L
    (0, 16, 7, 2, 1.1, 3.0, 300, 10.0),
    (1, 16, 7, 1, 1.1, 3.0, 300, 10.0),
    (2, 16, 7, 2, 1.1, 3.0, 300, 10.0),
    (3, 16, 7, 1, 1.1, 3.0, 300, 10.0),
    (6, 16, 7, 1, 1.1, 3.0, 300, 10.0),
    (7, 16, 7, 2, 1.1, 3.0, 300, 10.0),
    (0, 12, 3, 1, 0.8, 2.5, 500, 9.0),
    (1, 20, 5, 1, 1.3, 2.0, 700, 11.0),
    (2, 10, 4, 1, 0.9, 3.0, 200, 8.0),
    (3, 24, 6, 1, 1.5, 2.4, 800, 12.0),
    (6, 18, 2, 1, 0.7, 3.0, 400, 10.0),
    (7, 14, 1, 1, 1.0, 3.0, 256, 9.5),
    (1, 15, 3, 1, 1.0, 3.0, 300, 10.0),   # odd mesh (c2c methods only)
    (2, 64, 5, 1, 1.0, 3.0, 4000, 20.0),  # brick edge 8 path
    (1, 72, 7, 1, 0.9, 3.5, 6000, 22.0),
]


def _gpu_forces(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, precision=p3mg.FP64):
    with p3mg.Context(method, mesh, cao, mc, precision) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        return ctx.calculate_forces(rcut)


@pytest.mark.parametrize("case", CASES, ids=lambda c: "m%d_mesh%d_cao%d_mc%d" % c[:4])
def test_fp64_forces_match_oracle(gpu, case):
    method, mesh, cao, mc, alpha, rcut, n, L = case
    x, y, z, q = p3mg.generate_system(0, n, L, seed=100 + mesh + cao)
    ref = O.forces(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L)
    out = _gpu_forces(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L)
    assert O.rel_rms(out["f_k"], ref["f_k"]) <= TOL_FP64
    assert O.rel_rms(out["f_r"], ref["f_r"]) <= TOL_FP64
    assert O.rel_rms(out["f"], ref["f"]) <= TOL_FP64
    assert abs(out["energy"] - ref["energy"]) <= 1e-10 * max(1.0, abs(ref["energy"]))


@pytest.mark.parametrize("method", [0, 1, 2, 3, 6, 7])
def test_influence_matches_oracle(gpu, method):
    mesh, cao, mc, alpha, L = 16, 5, 2, 1.2, 10.0
    x, y, z, q = p3mg.generate_system(0, 50, L, seed=7)
    with p3mg.Context(method, mesh, cao, mc) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        G, b = ctx.get_influence()
    Gref = O.influence(method, mesh, cao, mc, alpha, L)
    assert O.rel_rms(G, Gref) <= 1e-13
    if method in (2, 7):
        bref = O.self_force_coeffs(mesh, cao, L, Gref)
        assert O.rel_rms(b, bref) <= 1e-12
    else:
        assert not np.any(b)


def test_realspace_matches_oracle(gpu):
    L, rcut, alpha = 12.0, 3.9, 0.8
    x, y, z, q = p3mg.generate_system(0, 900, L, seed=3)
    fr_ref, e_ref = O.realspace(x, y, z, q, L, rcut, alpha, cells=False)
    with p3mg.Context(1, 16, 3, 1) as ctx:
        ctx.set_system(x, y, z, q, L)
        fr, e = ctx.real_forces(rcut, alpha)
    assert O.rel_rms(fr, fr_ref) <= TOL_FP64
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)


def test_realspace_bruteforce_branch(gpu):
    # fewer than 3 cells per side -> all-pairs kernel
    L, rcut, alpha = 10.0, 4.9, 0.7
    x, y, z, q = p3mg.generate_system(0, 500, L, seed=5)
    fr_ref, e_ref = O.realspace(x, y, z, q, L, rcut, alpha, cells=False)
    with p3mg.Context(0, 8, 3, 1) as ctx:
        ctx.set_system(x, y, z, q, L)
        fr, e = ctx.real_forces(rcut, alpha)
    assert O.rel_rms(fr, fr_ref) <= TOL_FP64
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref)


@pytest.mark.parametrize("precision", [p3mg.FP64, p3mg.FP32_MIXED])
def test_overlap_switch_keeps_forces(gpu, precision):
    # the pairs beside the k-space chain (default) or before it
    # (p3mg_set_overlap): the same forces, up to the order of the atomics;
    # the FP64 step still matches the oracle
    method, mesh, cao, mc, alpha, rcut, n, L = (1, 32, 7, 1, 0.9, 3.5, 20000, 20000 ** (1.0 / 3.0))
    x, y, z, q = p3mg.generate_system(0, n, L, seed=21)
    with p3mg.Context(method, mesh, cao, mc, precision) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        ctx.enable_timing(True)
        on = ctx.calculate_forces(rcut)
        ctx.set_overlap(False)
        off = ctx.calculate_forces(rcut)
        kt = ctx.kernel_times()
        ctx.set_overlap(True)
    assert O.rel_rms(off["f"], on["f"]) <= (1e-14 if precision == p3mg.FP64 else 1e-6)
    assert all(v > 0.0 for v in kt.values())
    if precision == p3mg.FP64:
        ref = O.forces(method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, cells=True)
        assert O.rel_rms(off["f"], ref["f"]) <= TOL_FP64
