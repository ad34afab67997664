"""Batches of independent systems (p3mg_batch_*): uneven sizes, methods,
meshes and precisions in one CUDA graph give each context the forces of
its own p3mg_compute, on the eager run, the capture and the replays."""
import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu

SYSTEMS = [  # (system_type, n, box, method, mesh, cao, precision, rcut)
    (0, 500, 8.0, 1, 16, 7, p3mg.FP64, 2.5),
    (4, 3000, 14.4, 3, 32, 7, p3mg.FP32_MIXED, 3.5),
    (0, 20000, 27.1, 1, 36, 7, p3mg.FP32_MIXED, 3.5),
    (0, 1200, 10.6, 7, 20, 5, p3mg.FP64, 3.0),
    (3, 800, 9.3, 2, 16, 4, p3mg.FP64, 3.0),
]


def make(k, seed_shift=0):
    st, n, L, method, mesh, cao, prec, rcut = SYSTEMS[k]
    x, y, z, q = p3mg.generate_system(st, n, L, seed=90 + k + seed_shift)
    ctx = p3mg.Context(method, mesh, cao, 1, prec)
    ctx.set_system(x, y, z, q, L)
    ctx.influence(0.9)
    return ctx, (x, y, z, q, L), rcut


def test_batch_matches_single_contexts(gpu):
    made = [make(k) for k in range(len(SYSTEMS))]
    ctxs = [m[0] for m in made]
    rcuts = [m[2] for m in made]
    want = [c.calculate_forces(r)["f"].copy() for c, r in zip(ctxs, rcuts)]
    with p3mg.Batch(ctxs) as b:
        for run in range(4):  # eager, capture, replay, replay
            b.compute(rcuts)
            for k, c in enumerate(ctxs):
                got = c.get_forces()["f"]
                tol = 1e-14 if SYSTEMS[k][6] == p3mg.FP64 else 1e-6
                assert O.rel_rms(got.ravel(), want[k].ravel()) <= tol, (run, k)
        # a new system in one context re-captures the batch
        st, n, L = SYSTEMS[0][:3]
        x, y, z, q = p3mg.generate_system(st, n + 37, L, seed=123)
        ctxs[0].set_system(x, y, z, q, L)
        ctxs[0].influence(0.9)
        ref = p3mg.Context(SYSTEMS[0][3], SYSTEMS[0][4], SYSTEMS[0][5], 1, SYSTEMS[0][6])
        ref.set_system(x, y, z, q, L)
        ref.influence(0.9)
        w0 = ref.calculate_forces(rcuts[0])["f"]
        ref.close()
        for run in range(3):
            b.compute(rcuts)
            assert O.rel_rms(ctxs[0].get_forces()["f"].ravel(), w0.ravel()) <= 1e-14
            assert O.rel_rms(ctxs[2].get_forces()["f"].ravel(), want[2].ravel()) <= 1e-6
    for c in ctxs:
        c.close()


def test_batch_rejects_bad_arguments(gpu):
    ctx, _, _ = make(0)
    with pytest.raises(p3mg.P3MGError):
        p3mg.Batch([ctx, ctx])
    ctx.close()
