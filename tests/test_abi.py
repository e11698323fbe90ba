"""The C ABI library loads and exports every entry point declared in
include/*.h; host-side argument checks that need no GPU.  CPU."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(nspt_[a-z0-9_]+)\s*\(", src))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared()
    for need in ("nspt_create", "nspt_step", "nspt_gauge_wilson", "nspt_zero_modes_subtraction",
                 "nspt_fa_gauge_fixing", "nspt_plaquette_measure", "nspt_upload_links",
                 "nspt_download_links", "nspt_set_noise", "nspt_observables"):
        assert need in names


def test_library_exports_every_declared_symbol(engine_mod):
    from prlgt2020_b200 import _lib
    lib = ctypes.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(declared()) <= set(_lib.SIGNATURES)


def test_error_strings(engine_mod):
    from prlgt2020_b200 import _lib
    lib = _lib.load()
    for code in range(9):
        assert lib.nspt_error_string(code) != b"unknown error"
    assert b"time limit" in lib.nspt_error_string(_lib.NSPT_ERR_TIMEOUT)
    assert lib.nspt_error_string(99) == b"unknown error"


def test_create_rejects_bad_arguments_before_touching_a_device(engine_mod):
    from prlgt2020_b200 import _lib
    lib = _lib.load()
    h = ctypes.c_void_p()
    L = (ctypes.c_int * 4)(4, 4, 4, 4)
    assert lib.nspt_create(L, 0, 0, 0.0, ctypes.byref(h)) == _lib.NSPT_ERR_ORDER
    assert lib.nspt_create(L, _lib.NSPT_MAX_ORDER + 1, 0, 0.0, ctypes.byref(h)) == _lib.NSPT_ERR_ORDER
    assert lib.nspt_create(L, 4, 1 << 12, 0.0, ctypes.byref(h)) == _lib.NSPT_ERR_ARG
    # zero modes / FA with twisted boundaries: not defined by the reference
    assert lib.nspt_create(L, 4, _lib.NSPT_TWIST_Y | _lib.NSPT_ZEROMODE, 0.0,
                           ctypes.byref(h)) == _lib.NSPT_ERR_ARG
    bad = (ctypes.c_int * 4)(4, 1, 4, 4)
    assert lib.nspt_create(bad, 4, 0, 0.0, ctypes.byref(h)) == _lib.NSPT_ERR_ARG
    assert lib.nspt_create(L, 4, 0, 0.0, None) == _lib.NSPT_ERR_ARG


def test_ptgluon_fld_file_format(engine_mod, tmp_path):
    """ptGluon_fld save/load: field bytes then (allocORD+1) complex plaquette,
    size checked like io::load (QCDenvNODEpt_test.h:48-97)."""
    P = engine_mod
    f = P.ptGluon_fld((2, 2, 2, 2), 3)
    f.links[...] = np.random.default_rng(1).standard_normal(f.links.shape)
    plaq = np.arange(8.0).reshape(4, 2)
    p = str(tmp_path / "c.dat")
    f.save(p, plaq)
    assert os.path.getsize(p) == 8 * (16 * 4 * (2 + 18 * 3) + 2 * 4)
    g = P.ptGluon_fld.load(p, (2, 2, 2, 2), 3)
    assert np.array_equal(g.links, f.links)
    assert np.array_equal(g.plaquette_trailer, plaq)
    with pytest.raises(IOError):
        P.ptGluon_fld.load(p, (2, 2, 2, 2), 4)
