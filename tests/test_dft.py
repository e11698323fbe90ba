"""The DFT used by the oracle's FFTW shim against numpy.fft.  CPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


@pytest.fixture(scope="module")
def dft():
    from oracle import oracle as O
    L = O.lib()
    f = L.oracle_dft_nd
    f.argtypes = [ctypes.POINTER(ctypes.c_double), ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                  ctypes.c_long, ctypes.c_int]
    return f


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (2, 3, 5, 6), (8, 1, 4, 2), (16, 16)])
@pytest.mark.parametrize("sign", [-1, 1])
def test_dft_matches_numpy(dft, dims, sign):
    rng = np.random.default_rng(7)
    stride = 3
    n = int(np.prod(dims))
    data = rng.standard_normal((n, stride, 2))
    x = data[:, 1, 0] + 1j * data[:, 1, 1]
    ref = (np.fft.fftn if sign < 0 else lambda a: np.fft.ifftn(a) * a.size)(x.reshape(dims))
    buf = np.ascontiguousarray(data)
    ptr = buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    off = ctypes.cast(ctypes.addressof(ptr.contents) + 16, ctypes.POINTER(ctypes.c_double))
    d = (ctypes.c_int * len(dims))(*dims)
    dft(off, len(dims), d, stride, sign)
    got = (buf[:, 1, 0] + 1j * buf[:, 1, 1]).reshape(dims)
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    # untouched interleaved components
    assert np.array_equal(buf[:, 0], data[:, 0]) and np.array_equal(buf[:, 2], data[:, 2])
