"""The FP32-mixed path on inputs that stress its fixed-point accumulators:
the scatter's brick tiles (scale 2^30 / sum |q| of the brick) and the pair
kernel's Newton-3 partner forces (scale from the chunk's charge maxima, the
closest pairs sent to the global FP64 force).

- a clustered system whose densest bricks hold thousands of charges,
- charges spanning six decades,
- pairs at distance 1e-3 (forces ~1e6, far beyond the fixed-point range).

Bars as for every FP32 result: FP32 vs FP64 forces to 1e-4 relative RMS
and, where the P3M error dominates the FP32 rounding, within 1.1x of the
FP64 path's RMS error against the FP64 Ewald forces.  In the clustered
system the FP32 rounding of the close pairs of the dense blob (1.8e-5 of
the force, the same with float accumulators) exceeds the P3M error, so
there the k-space part -- where the scatter's fixed point acts -- is held
to 2e-6 of the FP64 path's (float accumulators: 4e-7).  With charges over
six decades the FP32 rounding of the largest pair forces (~1e6) dominates
as well (float accumulators reach 1.18x, these 1.2x of the FP64 error);
there the real-space part -- where the partner accumulators act -- is held
to 2e-6 of the FP64 path's (float accumulators: 9e-7, one scale shared by
all partners: 2.4e-6)."""
import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu


def ewald(x, y, z, q, L, targets):
    with p3mg.Context(1, 32, 5, 1) as ctx:
        ctx.set_system(x, y, z, q, L)
        return ctx.ewald_forces(targets)["f"]


def forces_all(method, mesh, cao, alpha, rcut, x, y, z, q, L, prec):
    with p3mg.Context(method, mesh, cao, 1, prec) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        return ctx.calculate_forces(rcut)


def check(x, y, z, q, L, method=1, mesh=64, cao=7, alpha=0.9, rcut=3.5, rel=1e-4, vs_ewald=True, rel_r=None):
    o32 = forces_all(method, mesh, cao, alpha, rcut, x, y, z, q, L, p3mg.FP32_MIXED)
    o64 = forces_all(method, mesh, cao, alpha, rcut, x, y, z, q, L, p3mg.FP64)
    f32, f64 = o32["f"], o64["f"]
    assert np.all(np.isfinite(f32))
    d = O.rel_rms(f32, f64)
    assert d <= rel, d
    dk = O.rel_rms(o32["f_k"], o64["f_k"])
    assert dk <= 2e-6, dk
    if rel_r is not None:
        dr = O.rel_rms(o32["f_r"], o64["f_r"])
        assert dr <= rel_r, dr
    if vs_ewald:
        tg = np.sort(np.random.default_rng(5).choice(len(x), min(2000, len(x)), replace=False))
        ew = ewald(x, y, z, q, L, tg)
        e32 = p3mg.rms_error(f32[:, tg], ew)
        e64 = p3mg.rms_error(f64[:, tg], ew)
        assert e32 <= 1.1 * e64, (e32, e64)
    return f32, f64


def test_clustered_bricks(gpu):
    # 80 % of 60k charges in a Gaussian blob of sigma L/10: the central bricks
    # hold thousands of charges, so their fixed-point scale is coarse
    rng = np.random.default_rng(11)
    n, L = 60_000, 39.1
    nb = int(0.8 * n)
    blob = rng.normal(0.5 * L, L / 10, size=(3, nb))
    rest = rng.uniform(0, L, size=(3, n - nb))
    pos = np.mod(np.concatenate([blob, rest], axis=1), L)
    q = 1.0 - 2.0 * (np.arange(n) % 2)
    check(pos[0].copy(), pos[1].copy(), pos[2].copy(), q, L, vs_ewald=False)


def test_charges_over_six_decades(gpu):
    rng = np.random.default_rng(12)
    n, L = 40_000, 34.2
    x, y, z = rng.uniform(0, L, size=(3, n))
    q = np.exp(rng.uniform(np.log(1e-3), np.log(1e3), n)) * np.where(rng.random(n) < 0.5, -1.0, 1.0)
    q[-1] -= q.sum()  # neutral
    check(x, y, z, q, L, vs_ewald=False, rel_r=2e-6)


def test_close_pairs_take_the_fallback(gpu):
    # 200 pairs 1e-3 apart inside a uniform system: their forces (~1e6) leave
    # the partner accumulators' range and go to the global FP64 force
    rng = np.random.default_rng(13)
    n0, L = 30_000, 31.1
    x, y, z = rng.uniform(0, L, size=(3, n0))
    q = 1.0 - 2.0 * (np.arange(n0) % 2)
    k = 200
    d = rng.normal(size=(3, k))
    d *= 1e-3 / np.linalg.norm(d, axis=0)
    x = np.concatenate([x, np.mod(x[:k] + d[0], L)])
    y = np.concatenate([y, np.mod(y[:k] + d[1], L)])
    z = np.concatenate([z, np.mod(z[:k] + d[2], L)])
    q = np.concatenate([q, -q[:k]])
    with p3mg.Context(1, 32, 7, 1, p3mg.FP32_MIXED) as c32, p3mg.Context(1, 32, 7, 1, p3mg.FP64) as c64:
        c32.set_system(x, y, z, q, L)
        c64.set_system(x, y, z, q, L)
        f32, _ = c32.real_forces(3.5, 0.9)
        f64, _ = c64.real_forces(3.5, 0.9)
    assert np.all(np.isfinite(f32))
    close = np.r_[0:k, n0:n0 + k]
    other = np.setdiff1d(np.arange(n0 + k), close)
    # the close pairs' forces: FP32 distances of 1e-3 carry ~1e-4 relative rounding
    assert O.rel_rms(f32[:, close], f64[:, close]) <= 1e-3
    assert O.rel_rms(f32[:, other], f64[:, other]) <= 1e-4
    # Newton's third law still holds to the FP32 rounding of the pair forces
    assert np.max(np.abs(f32.sum(axis=1))) <= 1e-5 * np.sqrt(np.sum(f32 ** 2))
