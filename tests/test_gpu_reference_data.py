"""The GPU path on the reference's own data sets (Data/ReferenceDataVincent,
raw text in tests/golden/vincent.npz): 512-ion NaCl crystal and melt and a
648-site water box, with exact forces (and, for NaCl, total Coulomb
energies) made by the data's authors.

- FP64 Ewald reference forces against the .exact forces, to the data's own
  accuracy (about 1e-6 absolute RMS; the oracle's converged sum agrees with
  them to the same figures).
- P3M with each data file's own parameter header (Mesh, ip = cao - 1,
  alpha, rcut) for all six methods against the oracle on the same folded
  positions: 1e-10 relative RMS, as every FP64 parity test.
- A P3M set-up accurate to ~3e-8 (mesh 64, cao 7, alpha 0.5, rcut 9):
  forces against .exact and the P3M energy against the .exact energy
  column."""
import os

import numpy as np
import pytest

import oracle as O
import p3mg

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
V = np.load(os.path.join(ROOT, "tests", "golden", "vincent.npz"))
EXACT_TOL = {"nacl300": 2e-6, "melt": 3e-7, "water": 1e-6}


def load(tmp_path, key):
    pos, ex = tmp_path / (key + ".dat"), tmp_path / (key + ".exact")
    pos.write_bytes(V[key + "_pos"].tobytes())
    ex.write_bytes(V[key + "_exact"].tobytes())
    x, y, z, q, L = p3mg.read_system(str(pos))
    x, y, z = (np.mod(v, L) for v in (x, y, z))
    f, e = p3mg.read_exact_forces(str(ex), len(x), with_energy=True)
    return x, y, z, q, L, f, e, p3mg.read_system_header(str(pos))


@pytest.mark.parametrize("key", ["nacl300", "melt", "water"])
def test_ewald_reference_matches_exact_forces(gpu, tmp_path, key):
    x, y, z, q, L, ref, _, _ = load(tmp_path, key)
    with p3mg.Context(2, 16, 7, 1) as ctx:
        ctx.set_system(x, y, z, q, L)
        ew = ctx.ewald_reference()
    assert O.abs_rms(ew["f"], ref) <= EXACT_TOL[key]


@pytest.mark.parametrize("method", [0, 1, 2, 3, 6, 7])
@pytest.mark.parametrize("key", ["nacl300", "melt"])
def test_header_settings_match_oracle(gpu, tmp_path, key, method):
    x, y, z, q, L, ref, _, h = load(tmp_path, key)
    mesh, cao, alpha, rcut = h["Mesh"], h["ip"] + 1, h["alpha"], h["rcut"]
    with p3mg.Context(method, mesh, cao, 1) as ctx:
        ctx.set_system(x, y, z, q, L)
        ctx.influence(alpha)
        r = ctx.calculate_forces(rcut)
    o = O.forces(method, mesh, cao, 1, alpha, rcut, x, y, z, q, L)
    assert O.rel_rms(r["f"], o["f"]) <= 1e-10
    assert O.rel_rms(r["f_k"], o["f_k"]) <= 1e-10
    # the same RMS error against the data's exact forces
    assert abs(O.abs_rms(r["f"], ref) - O.abs_rms(o["f"], ref)) <= 1e-10 * O.abs_rms(o["f"], ref)


@pytest.mark.parametrize("method", [2, 7])
@pytest.mark.parametrize("key", ["nacl300", "melt"])
def test_accurate_p3m_forces_and_energy(gpu, tmp_path, key, method):
    x, y, z, q, L, ref, e_exact, _ = load(tmp_path, key)
    alpha, rcut = 0.5, 9.0
    with p3mg.Context(method, 64, 7, 2) as ctx:
        ctx.set_system(x, y, z, q, L)
        assert ctx.error_estimate(alpha, rcut)["total"] < 1e-7
        ctx.influence(alpha)
        f = ctx.calculate_forces(rcut)["f"]
        e = ctx.energy(rcut)
    assert O.abs_rms(f, ref) <= EXACT_TOL[key] + 1e-7
    # the data's energies agree with a converged Ewald sum to 2.0e-6 (crystal)
    # and 1.2e-7 (melt) relative
    assert abs(e["total"] - e_exact) <= 3e-6 * abs(e_exact)
    assert e["neutral"] == 0.0
