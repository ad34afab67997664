"""The reference program's own force step with the GPU plugin.

p3m-standalone_b200/binding/p3m-gpu.c is the method_t table a maintainer adds
to the reference (types.h:306-316).  oracle/build_ref.sh compiles it against
the reference's headers and links it with the reference's objects and
libp3mg.so; the reference's Calculate_forces (common.c:268-327) then runs
once with its CPU table (method_p3m_ik_i, p3m-ik-i.c:40-43, and the other
five) and once with the GPU table on the same system.  Bar: relative RMS
force difference <= 1e-10 (FP64) on f, f_k and f_r, and the same pair
energy; FP32-mixed within 1e-5."""
import pytest

import oracle as O
import p3mg

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not O.ref_binding_available(), reason="oracle/_ref/libp3mref_gpu.so not built")]

CASES = [
    # method, mesh, cao, mc, alpha, rcut, n, L
    (0, 16, 7, 1, 1.1, 3.0, 400, 10.0),
    (1, 32, 7, 1, 0.9, 3.5, 3000, 14.4),
    (2, 16, 5, 2, 1.1, 3.0, 400, 10.0),
    (3, 20, 6, 1, 1.0, 3.0, 500, 11.0),
    (6, 16, 4, 1, 1.2, 3.0, 400, 10.0),
    (7, 16, 7, 2, 1.1, 3.0, 1000, 10.0),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "m%d_mesh%d" % c[:2])
def test_reference_calculate_forces_with_gpu_table(gpu, case):
    method, mesh, cao, mc, alpha, rcut, n, L = case
    x, y, z, q = p3mg.generate_system(0, n, L, seed=500 + method)
    cpu = O.ref_binding_forces(False, method, mesh, cao, mc, alpha, rcut, x, y, z, q, L)
    gpu64 = O.ref_binding_forces(True, method, mesh, cao, mc, alpha, rcut, x, y, z, q, L)
    for k in ("f", "f_k", "f_r"):
        assert O.rel_rms(gpu64[k], cpu[k]) <= 1e-10, k
    assert abs(gpu64["energy"] - cpu["energy"]) <= 1e-10 * abs(cpu["energy"])
    gpu32 = O.ref_binding_forces(True, method, mesh, cao, mc, alpha, rcut, x, y, z, q, L, precision=p3mg.FP32_MIXED)
    assert O.rel_rms(gpu32["f_k"], cpu["f_k"]) <= 1e-5
