"""GPU parity at the benchmarked configuration and at every mesh size of the
batched workloads, against the CPU oracle (not against this library's own
FP64 path).

The benchmarked step is method 1 (P3M_ik_i, p3m-ik-i.c:169-246, with the
influence function of p3m-ik-i.c:78-166) at mesh 128, cao 7, mc 1,
alpha 0.9, rcut 3.5 at density 1.  At a particle count the oracle finishes
in seconds (30,000) the same parameters run every kernel the 1M-particle
step runs: FP64 through the Stockham FFT, FP32-mixed through the
register-tiled pencil FFT with the ik convolution folded into its first
backward pass and the field packing into its last.  Meshes 32 and 64 (the
other pencil sizes) run for methods 0/1/3, 48 and 96 (the tuning grid's
other sizes, Stockham FFT) for methods 1 and 7, and 160 (the largest mesh of
the multi-system batch) for methods 1 and 3; the real-input methods 6 and
7 run from mesh 16 to 128.

Bars: FP64 relative RMS <= 1e-10 on f, f_k and f_r (rel_rms =
sqrt(sum |F_gpu - F_ref|^2) / sqrt(sum |F_ref|^2)) and 1e-10 relative on the
pair energy.  FP32-mixed: <= 5e-6 on the k-space force f_k (the mesh, the
FFTs, the convolution and the interpolation in FP32; measured 3e-7 .. 1.2e-6
on a B200) and <= 1.5e-5 on the real-space and total forces: the closest
pairs dominate the RMS force (1/r^2), and FP32 coordinates relative to a
cell origin carry about 1e-7 absolute rounding (measured 2e-6 .. 9e-6).  The
FP32 pair energy is a sum of terms of both signs that cancel to a few
percent of the largest ones, so its bar is 5e-4 relative.
"""
import functools

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_FP32_FK = 5e-6
TOL_FP32_F = 1.5e-5
TOL_FP32_E = 5e-4

ALPHA, RCUT, CAO, MC = 0.9, 3.5, 7, 1

# method, mesh, n (density 1: L = n^(1/3))
CASES = [
    (1, 128, 30000),  # the benchmarked configuration's parameters
    (0, 32, 20000),
    (1, 32, 20000),
    (3, 32, 20000),
    (0, 64, 20000),
    (1, 64, 20000),
    (3, 64, 20000),
    (1, 48, 20000),
    (7, 48, 20000),
    (1, 96, 20000),
    (7, 96, 20000),
    (1, 160, 20000),
    (3, 160, 20000),
    # the real-input methods (r2c forward, convolution over the half
    # spectrum, c2r backward: p3m-ik-real.c:72-76,108-138,
    # p3m-ad-real.c:62-64,90-104) from mesh 16 to 128
    (6, 16, 6000),
    (7, 16, 6000),
    (6, 24, 6000),
    (7, 40, 12000),
    (6, 32, 20000),
    (7, 32, 20000),
    (6, 64, 20000),
    (7, 64, 20000),
    (6, 128, 30000),
    (7, 128, 30000),
]


def _ids(c):
    return "m%d_mesh%d_n%d" % c


@functools.lru_cache(maxsize=None)
def _system(n, seed):
    L = float(n) ** (1.0 / 3.0)
    return p3mg.generate_system(0, n, L, seed=seed) + (L,)


@functools.lru_cache(maxsize=None)
def _oracle(method, mesh, n):
    x, y, z, q, L = _system(n, 1000 + mesh)
    return O.forces(method, mesh, CAO, MC, ALPHA, RCUT, x, y, z, q, L, cells=True)


def _gpu(method, mesh, n, precision, tiles=None):
    x, y, z, q, L = _system(n, 1000 + mesh)
    with p3mg.Context(method, mesh, CAO, MC, precision) as ctx:
        if tiles is not None:
            ctx.set_tiles(*tiles)
        ctx.set_system(x, y, z, q, L)
        ctx.influence(ALPHA)
        return ctx.calculate_forces(RCUT)


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_fp64_matches_oracle(gpu, case):
    ref = _oracle(*case)
    out = _gpu(*case, p3mg.FP64)
    assert O.rel_rms(out["f_k"], ref["f_k"]) <= TOL_FP64
    assert O.rel_rms(out["f_r"], ref["f_r"]) <= TOL_FP64
    assert O.rel_rms(out["f"], ref["f"]) <= TOL_FP64
    assert abs(out["energy"] - ref["energy"]) <= TOL_FP64 * abs(ref["energy"])


@pytest.mark.parametrize("case", CASES, ids=_ids)
def test_fp32_mixed_matches_oracle(gpu, case):
    ref = _oracle(*case)
    out = _gpu(*case, p3mg.FP32_MIXED)
    assert O.rel_rms(out["f_k"], ref["f_k"]) <= TOL_FP32_FK
    assert O.rel_rms(out["f_r"], ref["f_r"]) <= TOL_FP32_F
    assert O.rel_rms(out["f"], ref["f"]) <= TOL_FP32_F
    assert abs(out["energy"] - ref["energy"]) <= TOL_FP32_E * abs(ref["energy"])


@pytest.mark.parametrize("case", [c for c in CASES if c[1] in (32, 64, 128)], ids=_ids)
def test_fp32_stockham_fft_matches_oracle(gpu, case):
    # the same FP32 step with the Stockham FFT instead of the pencil FFT
    # (a tile width chosen): both FFTs are held to the oracle
    ref = _oracle(*case)
    out = _gpu(*case, p3mg.FP32_MIXED, tiles=(8 if case[1] >= 64 else 4, 16))
    assert O.rel_rms(out["f_k"], ref["f_k"]) <= TOL_FP32_FK
    assert O.rel_rms(out["f"], ref["f"]) <= TOL_FP32_F


def test_fp32_zero_charges_match_oracle(gpu):
    # particles without charge next to charged ones: the FP32 pair kernel's
    # Newton-3 partner accumulators take no units for them, and their forces
    # are exactly zero
    x, y, z, q, L = _system(20000, 77)
    q = q.copy()
    q[::7] = 0.0
    ref = O.forces(1, 32, CAO, MC, ALPHA, RCUT, x, y, z, q, L, cells=True)
    with p3mg.Context(1, 32, CAO, MC, p3mg.FP32_MIXED) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(ALPHA)
        out = ctx.calculate_forces(RCUT)
    assert O.rel_rms(out["f"], ref["f"]) <= TOL_FP32_F
    assert not np.any(out["f_r"][:, ::7])


@pytest.mark.parametrize("case", [(1, 128, 30000), (0, 32, 20000), (6, 64, 20000)], ids=_ids)
@pytest.mark.parametrize("precision", [p3mg.FP64, p3mg.FP32_MIXED])
def test_gather_variants_match_oracle(gpu, case, precision):
    # every ik back-interpolation kernel (lanes on the stencil's z offsets,
    # one thread per particle; FP32 also the shared-memory brick tiles,
    # TMA-staged and plain-loaded) against the oracle
    ref = _oracle(*case)
    method, mesh, n = case
    x, y, z, q, L = _system(n, 1000 + mesh)
    tol = TOL_FP64 if precision == p3mg.FP64 else TOL_FP32_FK
    modes = (1, 0) if precision == p3mg.FP64 else (1, 0, 2, 3)
    with p3mg.Context(method, mesh, CAO, MC, precision) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(ALPHA)
        if precision == p3mg.FP64:
            # the brick-tile kernels are FP32 only
            with pytest.raises(p3mg.P3MGError):
                ctx.set_gather(2)
        for mode in modes:
            ctx.set_gather(mode)
            fk = ctx.calculate_forces(0.0)["f_k"]
            assert O.rel_rms(fk, ref["f_k"]) <= tol, mode


@pytest.mark.parametrize("method", [0, 1, 6])
@pytest.mark.parametrize("cao,mesh,brick", [(3, 32, 4), (5, 32, 8), (7, 16, 4), (4, 20, 8), (7, 36, 8)])
def test_fp32_tile_gather_shapes(gpu, method, cao, mesh, brick):
    # the brick-tile gather at other orders, brick edges and meshes that
    # are not multiples of the brick (tiles wrapping around the periodic
    # mesh, TMA boxes reaching past its end) against the oracle
    if method == 6 and mesh % 2:
        pytest.skip("method 6 needs an even mesh")
    n = 3000
    L = float(n) ** (1.0 / 3.0)
    x, y, z, q = p3mg.generate_system(0, n, L, seed=cao * 100 + mesh)
    ref = O.forces(method, mesh, cao, MC, ALPHA, 0.0, x, y, z, q, L)
    with p3mg.Context(method, mesh, cao, MC, p3mg.FP32_MIXED) as ctx:
        ctx.set_tiles(brick, 0)
        ctx.set_system(x, y, z, q, L)
        ctx.influence(ALPHA)
        for mode in (2, 3):
            ctx.set_gather(mode)
            fk = ctx.calculate_forces(0.0)["f_k"]
            assert O.rel_rms(fk, ref["f_k"]) <= TOL_FP32_FK, mode


@pytest.mark.parametrize("system_type,n,L", [(4, 30000, 31.0), (0, 60000, 20.0)], ids=["gaussian", "density7"])
def test_fp32_dense_cells_match_oracle(gpu, system_type, n, L):
    # cells whose forward neighbourhood exceeds the pair kernel's staging
    # arrays (the centre of a Gaussian system with sigma L/6, 13.7 times the
    # mean density; a uniform system at density 7.5): the half-cell groups
    # stream their candidates through shared memory in chunks.  Closer pairs
    # than at density 1 raise the FP32 rounding of the closest ones.
    x, y, z, q = p3mg.generate_system(system_type, n, L, seed=91)
    fr_ref, e_ref = O.realspace(x, y, z, q, L, RCUT, ALPHA, cells=True)
    for prec, tol in ((p3mg.FP64, TOL_FP64), (p3mg.FP32_MIXED, 5e-5)):
        with p3mg.Context(1, 32, CAO, MC, prec) as ctx:
            ctx.set_system(x, y, z, q, L)
            fr, e = ctx.real_forces(RCUT, ALPHA)
        assert O.rel_rms(fr, fr_ref) <= tol
        assert abs(e - e_ref) <= (TOL_FP64 if prec == p3mg.FP64 else TOL_FP32_E) * abs(e_ref)
