"""The oracle's DFT restatement (the FFTW3 stand-in) against numpy.fft."""
import ctypes
import os

import numpy as np
import pytest

import oracle as O

_dp = ctypes.POINTER(ctypes.c_double)


def _lib():
    L = O.lib()
    L.oracle_dft_nd.argtypes = [_dp, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
    L.oracle_dft_r2c_3d.argtypes = [_dp, ctypes.c_long, _dp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    L.oracle_dft_c2r_3d.argtypes = [_dp, ctypes.c_long, _dp, ctypes.c_long, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    return L


@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 10, 6), (15, 7, 14), (16, 16, 16), (11, 13, 9)])
@pytest.mark.parametrize("sign", [-1, 1])
def test_c2c_matches_numpy(shape, sign):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    buf = np.ascontiguousarray(np.stack([a.real, a.imag], axis=-1)).ravel()
    dims = (ctypes.c_int * 3)(*shape)
    _lib().oracle_dft_nd(buf.ctypes.data_as(_dp), 3, dims, sign)
    got = buf[0::2] + 1j * buf[1::2]
    ref = np.fft.fftn(a) if sign < 0 else np.fft.ifftn(a) * a.size
    assert np.max(np.abs(got.reshape(shape) - ref)) <= 1e-12 * np.max(np.abs(ref))


@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 10, 6), (16, 14, 10)])
def test_r2c_c2r_roundtrip_and_numpy(shape):
    rng = np.random.default_rng(2)
    n0, n1, n2 = shape
    h = n2 // 2 + 1
    x = rng.standard_normal(shape)
    out = np.zeros(2 * n0 * n1 * h)
    xin = np.ascontiguousarray(x).ravel()
    _lib().oracle_dft_r2c_3d(xin.ctypes.data_as(_dp), n2, out.ctypes.data_as(_dp), h, n0, n1, n2)
    got = (out[0::2] + 1j * out[1::2]).reshape(n0, n1, h)
    ref = np.fft.rfftn(x)
    assert np.max(np.abs(got - ref)) <= 1e-12 * np.max(np.abs(ref))
    back = np.zeros(n0 * n1 * n2)
    _lib().oracle_dft_c2r_3d(out.ctypes.data_as(_dp), h, back.ctypes.data_as(_dp), n2, n0, n1, n2)
    assert np.max(np.abs(back.reshape(shape) / x.size - x)) <= 1e-12
