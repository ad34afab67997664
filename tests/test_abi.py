"""The C ABI library: it loads without a GPU, exports every function that
include/p3mg.h declares, and rejects bad arguments before touching CUDA."""
import ctypes
import os
import re

import pytest

import p3mg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    text = open(os.path.join(ROOT, "include", "p3mg.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(p3mg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = p3mg.load()
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_strerror_covers_all_codes():
    lib = p3mg.load()
    for code in range(0, -11, -1):
        s = lib.p3mg_strerror(code).decode()
        assert s and s != "unknown status", code
    assert lib.p3mg_strerror(-99).decode() == "unknown status"


@pytest.mark.parametrize("method,mesh,cao,prec,expected", [
    (5, 16, 7, 0, -2),    # the reference has no method 5 implementation (types.h:115)
    (4, 16, 7, 0, -2),    # Ewald is not a P3M mesh method here
    (8, 16, 7, 0, -2),
    (1, 16, 0, 0, -3),    # cao outside 1..7 (charge-assign.c:209-211)
    (1, 16, 8, 0, -3),
    (1, 2, 1, 0, -4),     # mesh below 4
    (1, 6, 7, 0, -4),     # mesh smaller than cao
    (1, 22, 7, 0, -4),    # prime factor 11
    (7, 15, 3, 0, -4),    # odd mesh with an r2c method
    (1, 1024, 7, 0, -4),  # above the supported maximum
    (1, 16, 7, 2, -9),    # unknown precision
])
def test_create_rejects_bad_arguments_without_cuda(method, mesh, cao, prec, expected):
    lib = p3mg.load()
    h = ctypes.c_void_p()
    assert lib.p3mg_create(ctypes.byref(h), method, mesh, cao, 1, prec) == expected
    assert not h.value


def test_null_context_is_an_argument_error():
    lib = p3mg.load()
    assert lib.p3mg_influence(None, 1.0) == -1
    assert lib.p3mg_compute(None, 3.0) == -1
    assert lib.p3mg_create(None, 1, 16, 7, 1, 0) == -1
    lib.p3mg_destroy(None)
