"""The C++ host driver (prlgt2020_b200/lib/nspt_quenched), run like the
reference's own program: Quench.cfg and damocle.dag in the working directory,
output files named and formatted as Quenched.cc / nspt.cc write them.

The GPU tests replay every reference fixture in tests/golden through the
driver, with the reference's own noise stream (the driver's host rand55),
and compare the plaquette and norm series it writes, and the configuration
it saves, with what the reference wrote.  Tolerances as in
test_gpu_parity.py; the .nor file carries 6 significant digits (the
reference's default stream precision), so it is held to 1e-5.
"""
import glob
import math
import os
import subprocess

import numpy as np
import pytest

from helpers import obs_close, per_order_rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def driver():
    from prlgt2020_b200 import _lib
    _lib.build()
    path = os.path.join(os.path.dirname(_lib.LIB_PATH), "nspt_quenched")
    assert os.path.exists(path)
    return path


def write_cfg(d, L, sweep, beat, tau_g, alpha, init, N, seed, plaq="plaq", conf="conf",
              nthr=1):
    """Quench.cfg; an OpenMP build reads one seed line per thread
    (Quenched.cc:171-174): seed, seed + 1, ... as the harness seeds them."""
    with open(os.path.join(d, "Quench.cfg"), "w") as f:
        f.write("taglia %d %d %d %d\n" % tuple(L))
        f.write("SWEEP %d\nBEAT %d\ntau_g %r\nalpha %r\ninit_status %d\n" % (sweep, beat, tau_g, alpha,
                                                                             init))
        f.write("plaq_out %s\nlast_conf %s\nPTORD %d\n" % (plaq, conf, N))
        for t in range(nthr):
            f.write("seed %d\n" % (seed + t))


def write_damocle(d, tau_g, alpha, sweep=0, beat=1, save=0, kill=0):
    with open(os.path.join(d, "damocle.dag"), "w") as f:
        f.write("SWEEP %d\nBEAT %d\ntau_g %r\nalpha %r\nsave_config %d\nkill_run %d\n"
                % (sweep, beat, tau_g, alpha, save, kill))


def stem(L, alpha, tau_g, N):
    return "SU3_wil_nf0_%dx%dx%dx%d_a%.2f_tg%.3f_o%d" % (tuple(L) + (abs(alpha), tau_g, N))


def test_driver_reports_missing_inputs(driver, tmp_path):
    r = subprocess.run([driver], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "configurazione" in r.stderr
    r = subprocess.run([driver, "-h"], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0 and "SWEEP" in r.stdout
    write_cfg(tmp_path, (4, 4, 4, 4), 2, 1, 0.01, 0.0, 0, 3, 1)
    r = subprocess.run([driver], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "damocle" in r.stderr
    with open(tmp_path / "Quench.cfg", "w") as f:
        f.write("taglia 4 4 4 4\nSWEEP 2\nBEEP 1\n")
    write_damocle(tmp_path, 0.01, 0.0)
    r = subprocess.run([driver], cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 1 and "BEAT" in r.stderr


@pytest.mark.gpu
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_driver_replays_reference_fixture(driver, oracle_mod, tmp_path, path):
    O = oracle_mod
    g = np.load(path)
    L = tuple(int(x) for x in g["L"])
    N, steps, dt = int(g["N"]), int(g["steps"]), float(g["dt"])
    alpha, seed, start = float(g["alpha"]), int(g["seed"]), int(g["start"])
    twisted, fa, zm = bool(g["twisted"]), bool(g["fa"]), bool(g["zm"])
    V = int(np.prod(L))
    action = {-1.0 / 12.0: "tlsym", -0.331: "iwa", -1.4088: "dbw2"}.get(
        float(g["c1"]) if "c1" in g else 0.0, "wil")
    name = stem(L, alpha, dt, N).replace("SU3_wil", "SU3_" + action[:3])
    grid = tuple(int(x) for x in g["grid"]) if "grid" in g else (1, 1, 1, 1)
    nthr = int(np.prod(grid))
    write_cfg(tmp_path, L, steps, steps, dt, alpha, 1 if start >= 0 else 0, N, seed, nthr=nthr)
    write_damocle(tmp_path, dt, alpha)
    if start >= 0:
        o = O.Oracle(L, N, twist_mask=6 if twisted else 0)
        o.random_start(start, 0.5)
        O.write_config(str(tmp_path / ("conf" + name)), o.links, o.plaquette())
    args = [driver, "-G", ",".join(str(x) for x in grid)]  # the fixture build's thread grid
    if nthr > 1:
        args += ["-M"]  # one noise stream per thread
    if twisted:
        args += ["-T", "yz"]
    else:
        args += ["-W"]
    if fa:
        args += ["-F"]
    if not zm:
        args += ["-Z", "0"]
    if action != "wil":
        args += ["-A", action]
    if "onthefly" in g and bool(g["onthefly"]):
        args += ["-O"]
    r = subprocess.run(args, cwd=tmp_path, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = np.loadtxt(tmp_path / ("plaq_" + name + ".txt"))
    if action != "wil":  # w1 and w2 columns (nspt.cc:586-597)
        w2 = raw[:, 2:].reshape(steps, N + 1, 2)
        raw = raw[:, :2]
        for s in range(steps):
            ok, w = obs_close(w2[s][:N], g["w2"][s][:N], 1e-11)
            assert ok, ("w2", s, w)
    plaq = raw.reshape(steps, N + 1, 2)
    norm = np.loadtxt(tmp_path / (name + ".nor")).reshape(steps, N)
    for s in range(steps):
        ok, w = obs_close(plaq[s], g["plaq"][s], 1e-11)
        assert ok, ("plaq", s, w)
        ok, w = obs_close(norm[s], g["norm"][s], 1e-5)
        assert ok, ("norm", s, w)
    links, trailer = O.read_config(str(tmp_path / ("conf" + name)), V, N)
    rel = per_order_rel(links[: g["links"].shape[0]], g["links"], N)
    bound = (np.array([max(1e-11, 1e-15 * math.factorial(k)) for k in range(1, N + 1)])
             if (zm and start < 0) else 1e-11)
    assert np.all(rel <= bound), rel
    ok, w = obs_close(trailer, g["plaq_final"][: N + 1], 1e-11)
    assert ok, ("saved plaquette", w)
    loops_file = tmp_path / ("plaq_nxm_" + name + ".txt")
    if twisted:
        assert not loops_file.exists()
    else:
        # ComputeLoops after the BEAT and at the end: the last line is the
        # saved field's loops, even orders, 1x2 2x2 2x4 4x4
        lines = np.atleast_2d(np.loadtxt(loops_file))
        assert lines.shape[0] == 2
        o = O.Oracle(L, N)
        o.set_links(links)
        want = o.wilson_loops()[:, ::2, 0]
        got = lines[-1].reshape(4, -1)
        for q in range(4):
            ok, w = obs_close(got[q], want[q], 1e-11)
            assert ok, ("loops", q, w)
        # WL2x2's file: Re Tr of the 2x2 loop, orders 2, 4, ... <= N
        wl = np.atleast_2d(np.loadtxt(tmp_path / ("plaq2x2_" + name + ".txt")))
        assert wl.shape == (2, N // 2)
        ok, w = obs_close(wl[-1], o.wilson_loops()[1, 2::2, 0], 1e-11)
        assert ok, ("wl2x2", w)


@pytest.mark.gpu
@pytest.mark.parametrize("philox", [False, True], ids=["rand55", "philox"])
def test_driver_resumes_a_run_from_its_noise_state_sidecar(driver, tmp_path, philox):
    """A run of 6 sweeps and the same run split into 3 + 3 (hot start from
    the saved configuration and its .rng sidecar) write the same plaquette
    series and save the same configuration, bit for bit."""
    L, N, dt, alpha, seed = (4, 4, 4, 4), 4, 0.01, -0.05, 4242
    extra = ["-P"] if philox else []
    name = stem(L, alpha, dt, N)
    whole, split = tmp_path / "whole", tmp_path / "split"
    for d in (whole, split):
        d.mkdir()
        write_damocle(d, dt, alpha)
    write_cfg(whole, L, 6, 6, dt, alpha, 0, N, seed)
    r = subprocess.run([driver] + extra, cwd=whole, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    write_cfg(split, L, 3, 3, dt, alpha, 0, N, seed)
    r = subprocess.run([driver] + extra, cwd=split, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    assert (split / ("conf" + name + ".rng")).exists()
    write_cfg(split, L, 3, 3, dt, alpha, 1, N, seed)
    r = subprocess.run([driver] + extra, cwd=split, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    for f in ("plaq_" + name + ".txt", "conf" + name, "conf" + name + ".rng"):
        assert (whole / f).read_bytes() == (split / f).read_bytes(), f
