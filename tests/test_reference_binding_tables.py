"""The reference-side binding (p3m-standalone_b200/binding/p3m-gpu.c), as
oracle/build_ref.sh links it into the reference's objects: it loads without a
GPU and exports a GPU method_t table beside each of the reference's six P3M
tables (p3m-ik.c, p3m-ik-i.c, p3m-ad.c, p3m-ad-i.c, p3m-ik-real.c,
p3m-ad-real.c), each with the reference's method id (types.h method_t, the
id its first member)."""
import ctypes
import os

import pytest

import oracle as O

TABLES = [("method_p3m_ik", 0), ("method_p3m_ik_i", 1), ("method_p3m_ad", 2), ("method_p3m_ad_i", 3),
          ("method_p3m_ik_r", 6), ("method_p3m_ad_r", 7)]


@pytest.mark.skipif(not O.ref_binding_available(), reason="oracle/_ref/libp3mref_gpu.so not built")
@pytest.mark.parametrize("name,method_id", TABLES)
def test_gpu_table_beside_each_reference_table(name, method_id):
    lib = ctypes.CDLL(os.path.join(os.path.dirname(O.__file__), "_ref", "libp3mref_gpu.so"))
    assert ctypes.c_int.in_dll(lib, name).value == method_id
    assert ctypes.c_int.in_dll(lib, name + "_gpu").value == method_id
