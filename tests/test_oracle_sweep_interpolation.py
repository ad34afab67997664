"""The numerical premise of the interpolated alpha sweep (p3mg_sweep with
many alphas over a narrow range), checked on the CPU with the oracle's FP64
P3M forces: forces evaluated at R Chebyshev nodes in t = 1/alpha^2 and
interpolated with Lagrange weights reproduce the forces at other alphas
within the tolerances the sweep checks them against (1e-6 of the RMS force
with 10 nodes in FP32, 1e-12 with 16 in FP64) over the ranges where the GPU
accepts the interpolation, and miss them over the wider ranges where it
falls back to evaluating every alpha.  The node placement restates
sweep_interpolated in p3mg_sweep.cu.

G_opt itself does not interpolate to that accuracy: its high-|k| modes are
exp(-k^2 t / 4) terms with large rates, but they reach the forces only
through the charge-assignment filter twice, which is why the sweep checks
forces, not G."""
import math

import numpy as np
import pytest

import oracle as O


def chebyshev_nodes_t(amin, amax, R):
    lo, hi = 1.0 / (amax * amax), 1.0 / (amin * amin)
    return np.array([0.5 * (lo + hi) + 0.5 * (hi - lo) * math.cos((2 * r + 1) * math.pi / (2.0 * R))
                     for r in range(R)])


def lagrange_weights(tn, t):
    w = np.ones(len(tn))
    for i in range(len(tn)):
        for j in range(len(tn)):
            if j != i:
                w[i] *= (t - tn[j]) / (tn[i] - tn[j])
    return w


@pytest.fixture(scope="module")
def system():
    return O.uniform_system(2000, 12.6, seed=5)


def _interp_error(system, lo, hi, R):
    x, y, z, q = system
    tn = chebyshev_nodes_t(lo, hi, R)
    force = lambda a: np.asarray(O.forces(1, 16, 7, 1, a, 3.0, x, y, z, q, 12.6)["f"])
    fn = [force(1.0 / math.sqrt(t)) for t in tn]
    err = 0.0
    for a in np.linspace(lo * 1.01, hi * 0.99, 5):
        w = lagrange_weights(tn, 1.0 / (a * a))
        fi = sum(wi * f for wi, f in zip(w, fn))
        err = max(err, O.rel_rms(fi.ravel(), force(a).ravel()))
    return err


@pytest.mark.parametrize("lo,hi,R,bound", [
    (0.6, 1.2, 10, 1e-6),   # FP32: 10 nodes over a 2x range (measured 6.5e-7)
    (0.8, 1.2, 16, 1e-12),  # FP64: 16 nodes over a 1.5x range (measured 1.6e-13)
])
def test_forces_interpolate_within_the_sweep_tolerance(system, lo, hi, R, bound):
    assert _interp_error(system, lo, hi, R) <= bound


@pytest.mark.parametrize("lo,hi,R,bound", [
    (0.4, 1.2, 10, 1e-6),   # FP32 over a 3x range (measured 2.6e-5): the sweep evaluates every alpha
    (0.7, 1.4, 16, 1e-12),  # FP64 over a 2x range (measured 1.1e-9): likewise
])
def test_wider_ranges_miss_the_tolerance(system, lo, hi, R, bound):
    assert _interp_error(system, lo, hi, R) > bound
