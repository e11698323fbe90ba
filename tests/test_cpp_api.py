"""The C++ API (include/nspt_b200.hpp: Cplx, SU3, ptSU3, ptGluon_fld and the
nspt.h function names) through a small program written against it,
prlgt2020_b200/lib/nspt_api_check.  On the GPU its sweeps are compared with
the oracle's on the same start and noise (tolerances of test_gpu_parity.py).
"""
import os
import subprocess

import numpy as np
import pytest

from helpers import obs_close, per_order_rel


@pytest.fixture(scope="module")
def api_check():
    from prlgt2020_b200 import _lib
    _lib.build()
    path = os.path.join(os.path.dirname(_lib.LIB_PATH), "nspt_api_check")
    assert os.path.exists(path)
    return path


def test_api_check_builds_and_reports_usage(api_check):
    r = subprocess.run([api_check], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr


@pytest.mark.gpu
def test_cpp_api_sweeps_match_the_oracle(api_check, oracle_mod, tmp_path):
    O = oracle_mod
    L, N, steps, dt = (4, 4, 4, 4), 4, 2, 0.01
    o = O.Oracle(L, N)
    o.random_start(2718, 0.5)
    O.write_config(str(tmp_path / "start.dat"), o.links, o.plaquette())
    rng = O.Rand55(314)
    noise = [rng.gauss(o.V * 32) for _ in range(steps)]
    np.concatenate(noise).tofile(tmp_path / "noise.bin")
    r = subprocess.run([api_check, *map(str, L), str(N), str(tmp_path / "start.dat"),
                        str(tmp_path / "noise.bin"), str(steps), repr(dt), str(tmp_path / "out.dat")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = {}
    for ln in r.stdout.splitlines():
        key, *vals = ln.split()
        lines.setdefault(key, []).append(np.array(vals, dtype=float).reshape(N + 1, 2))
    for s in range(steps):
        oo = o.sweep(dt, noise[s])
        ok, w = obs_close(lines["plaq"][s], oo.plaq, 1e-12)
        assert ok, ("plaq", s, w)
    links, _ = O.read_config(str(tmp_path / "out.dat"), o.V, N)
    assert per_order_rel(links, o.links, N).max() <= 1e-12
    ok, w = obs_close(lines["measure"][0], o.plaquette(), 1e-12)
    assert ok, ("plaquette_measure", w)
    want22 = o.wilson_loops()[1] * np.array([1.0, -1.0])
    ok, w = obs_close(lines["wl2x2"][0], want22, 1e-12)
    assert ok, ("WL2x2", w)
