"""The oracle against the reference's own code run live (oracle/_ref), on
cases larger than the committed fixtures.  Needs the reference's sources to
build the binary (or a binary already built); skipped otherwise.  CPU."""
import os
import tempfile

import numpy as np
import pytest

from helpers import obs_close, per_order_rel

def ref_binary(O, N, bc, gf):
    b = O.ref_binary(N, bc, gf)
    if os.path.exists(b):
        return b
    if not os.path.exists(os.path.join(O.reference_dir(), "nspt.cc")):
        pytest.skip("reference sources not available")
    return O.build_reference(N, bc, gf)


@pytest.mark.parametrize("case", [
    dict(L=(4, 4, 4, 4), N=8, bc="pbc", gf="local", steps=20, dt=0.01, alpha=0.0, start=None, zm=True),
    dict(L=(6, 4, 4, 4), N=6, bc="pbc", gf="fa", steps=4, dt=0.02, alpha=-0.05, start=21, zm=True),
    dict(L=(4, 4, 4, 4), N=6, bc="tw", gf="local", steps=6, dt=0.01, alpha=0.0, start=5, zm=False),
], ids=["cold_n8_20steps", "fa_6x4x4x4", "twisted_n6"])
def test_oracle_matches_reference_live(oracle_mod, case):
    O = oracle_mod
    b = ref_binary(O, case["N"], case["bc"], case["gf"])
    tw = 6 if case["bc"] == "tw" else 0
    o = O.Oracle(case["L"], case["N"], twist_mask=tw)
    with tempfile.TemporaryDirectory() as d:
        start = "cold"
        if case["start"] is not None:
            o.random_start(case["start"], 0.5)
            O.write_config(os.path.join(d, "s.dat"), o.links, o.plaquette())
            start = os.path.join(d, "s.dat")
        r = O.run_reference(b, case["L"], case["steps"], case["dt"], case["alpha"], 99, d,
                            start=start, twist_init=tw != 0)
    rng = O.Rand55(99)
    for s in range(case["steps"]):
        nz = rng.gauss(o.V * 32)
        assert np.array_equal(nz, r["noise"][s])
        ob = o.sweep(case["dt"], nz, zero_modes=case["zm"])
        assert obs_close(ob.plaq, r["plaq"][s], 1e-12)[0]
        assert obs_close(ob.norm, r["norm"][s], 1e-12)[0]
        if case["zm"]:
            o.zero_modes()
        if case["gf"] == "fa":
            o.fa_gauge_fix(case["alpha"])
    assert per_order_rel(o.links, r["links"], case["N"]).max() <= 1e-12


@pytest.mark.parametrize("case", [
    dict(L=(4, 4, 4, 4), N=4, bc="pbc", grid=(2, 2, 2), zm=True),
    dict(L=(4, 4, 4, 4), N=5, bc="tw", grid=(1, 1, 1), zm=False),
    dict(L=(4, 4, 4, 4), N=5, bc="tw", grid=(2, 2, 1), zm=False),
], ids=["pbc_grid222", "twisted_sequential", "twisted_grid221"])
def test_oracle_local_gauge_fixing_matches_reference_thread_grid(oracle_mod, case):
    """stochastic_gauge_fixing as the reference's OpenMP build with thread
    grid (ntx, nty, ntz) runs it (nspt.cc:723-815), including the twisted
    boundary updates (nspt.cc:665-720).  dt = 0 makes the sweep an exact
    identity, so the per-thread noise streams of the OpenMP build do not
    enter; what is compared is the gauge fixing (and zero modes)."""
    O = oracle_mod
    N, grid, alpha, steps = case["N"], case["grid"], -0.08, 2
    b = O.ref_binary(N, case["bc"], "local", grid)
    if not os.path.exists(b):
        if not os.path.exists(os.path.join(O.reference_dir(), "nspt.cc")):
            pytest.skip("reference sources not available")
        b = O.build_reference(N, case["bc"], "local", grid)
    tw = 6 if case["bc"] == "tw" else 0
    o = O.Oracle(case["L"], N, twist_mask=tw)
    o.random_start(17, 0.5)
    with tempfile.TemporaryDirectory() as d:
        O.write_config(os.path.join(d, "s.dat"), o.links, o.plaquette())
        r = O.run_reference(b, case["L"], steps, 0.0, alpha, 3, d, start=os.path.join(d, "s.dat"),
                            noise=False, twist_init=tw != 0)
    zeros = np.zeros(o.V * 32)
    for _ in range(steps):
        o.sweep(0.0, zeros, zero_modes=case["zm"])
        if case["zm"]:
            o.zero_modes()
        o.local_gauge_fix(alpha, grid=(1,) + tuple(grid))
    assert per_order_rel(o.links, r["links"], N).max() <= 1e-12


@pytest.mark.parametrize("L,N,start", [((4, 4, 4, 4), 6, 5), ((6, 4, 4, 4), 4, 7)])
def test_oracle_wilson_loops_match_reference(oracle_mod, L, N, start):
    """ComputeLoops (nspt.cc:1148-1312) on a random configuration: the
    reference prints the real parts of the even orders of the 1x2, 2x2, 2x4
    and 4x4 loops (periodic builds).  WL2x2 (nspt.cc:1064-1140) prints the
    2x2 loop traversed the other way round, Re Tr /(18V) of ptU[1], ptU[3],
    ... (orders 2, 4, ...): the real part of the same 2x2 trace."""
    O = oracle_mod
    b = O.ref_binary(N, "pbc", "local")
    if not os.path.exists(b) or os.path.getmtime(b) < os.path.getmtime(
            os.path.join(os.path.dirname(O.__file__), "ref_harness.cc")):
        if not os.path.exists(os.path.join(O.reference_dir(), "nspt.cc")):
            pytest.skip("reference sources not available")
        b = O.build_reference(N, "pbc", "local")
    o = O.Oracle(L, N)
    o.random_start(start, 0.5)
    with tempfile.TemporaryDirectory() as d:
        O.write_config(os.path.join(d, "s.dat"), o.links, o.plaquette())
        loops = os.path.join(d, "loops.txt")
        wl = os.path.join(d, "wl2x2.txt")
        import subprocess
        subprocess.run([b, "--L", *[str(x) for x in L], "--steps", "0", "--start",
                        os.path.join(d, "s.dat"), "--out", os.path.join(d, "r"), "--loops", loops,
                        "--wl2x2", wl], check=True, capture_output=True)
        ref = np.loadtxt(loops).reshape(4, -1)
        ref22 = np.atleast_1d(np.loadtxt(wl))
    got = o.wilson_loops()[:, ::2, 0]
    assert ref.shape == got.shape
    for q in range(4):
        ok, w = obs_close(got[q], ref[q], 1e-12)
        assert ok, (q, w)
    assert ref22.shape == (N // 2,)
    ok, w = obs_close(o.wilson_loops()[1, 2::2, 0], ref22, 1e-12)
    assert ok, ("wl2x2", w)


@pytest.mark.parametrize("action,c1", [("tlsym", -1.0 / 12.0), ("dbw2", -1.4088)])
def test_oracle_improved_action_matches_reference(oracle_mod, action, c1):
    """gauge_wilson with an improved action (nspt.cc:272-308, staple2x1
    QCDenvNODEpt_test.h:579-611): plaquette and rectangle traces per step and
    the links after the sweeps, from a random start with the reference's
    noise."""
    O = oracle_mod
    L, N, steps, dt = (4, 4, 4, 4), 4, 2, 0.01
    b = O.ref_binary(N, "pbc", "local", (1, 1, 1), action)
    if not os.path.exists(b):
        if not os.path.exists(os.path.join(O.reference_dir(), "nspt.cc")):
            pytest.skip("reference sources not available")
        b = O.build_reference(N, "pbc", "local", (1, 1, 1), action)
    o = O.Oracle(L, N)
    o.random_start(23, 0.5)
    o.set_action(c1)
    with tempfile.TemporaryDirectory() as d:
        O.write_config(os.path.join(d, "s.dat"), o.links, o.plaquette())
        r = O.run_reference(b, L, steps, dt, 0.0, 5, d, start=os.path.join(d, "s.dat"))
    rng = O.Rand55(5)
    cum = np.zeros(2)
    for s in range(steps):
        nz = rng.gauss(o.V * 32)
        assert np.array_equal(nz, r["noise"][s])
        ob = o.sweep(dt, nz, zero_modes=True)
        assert obs_close(ob.plaq, r["plaq"][s], 1e-12)[0], s
        w2 = o.last_w2()
        assert obs_close(w2[:N], r["w2"][s][:N], 1e-12)[0], s
        # the reference never resets w2[PTORD] between steps (NsptEvolve,
        # nspt.cc:972-985 zeroes w2[0..PTORD-1] and w1[PTORD] only): its
        # printed top order is the running sum
        cum += w2[N]
        assert np.allclose(r["w2"][s][N], cum, rtol=1e-12, atol=1e-30), s
        o.zero_modes()
    assert per_order_rel(o.links, r["links"], N).max() <= 1e-12


@pytest.mark.parametrize("case", [
    dict(L=(4, 4, 4, 4), N=4, bc="pbc", grid=(1, 1, 1), zm=True, start=None),
    dict(L=(4, 4, 4, 4), N=4, bc="pbc", grid=(2, 2, 2), zm=True, start=21),
    dict(L=(4, 4, 4, 4), N=5, bc="tw", grid=(1, 1, 1), zm=False, start=5),
    dict(L=(4, 4, 4, 4), N=5, bc="tw", grid=(2, 2, 1), zm=False, start=5),
], ids=["pbc_sequential", "pbc_grid222", "twisted_sequential", "twisted_grid221"])
def test_oracle_onthefly_matches_reference(oracle_mod, case):
    """The reference's default build (UPDATE_ONTHEFLY, choices.h:61): links
    updated in place in the thread grid's order (nspt.cc:355-460), with each
    OpenMP thread's own noise stream (the harness replays them by link), then
    zero modes and the local gauge fixing.  With twisted boundaries a read
    across a twisted face sees the copy site of the last twist_boundary
    (nspt.cc:989-1027 calls it only at the end of the step): without that
    the plaquette differs by several per cent."""
    O = oracle_mod
    N, grid, alpha, steps, dt = case["N"], case["grid"], -0.05, 3, 0.01
    b = O.ref_binary(N, case["bc"], "local", grid, update="otf")
    if not os.path.exists(b):
        if not os.path.exists(os.path.join(O.reference_dir(), "nspt.cc")):
            pytest.skip("reference sources not available")
        b = O.build_reference(N, case["bc"], "local", grid, update="otf")
    tw = 6 if case["bc"] == "tw" else 0
    o = O.Oracle(case["L"], N, twist_mask=tw)
    with tempfile.TemporaryDirectory() as d:
        start = "cold"
        if case["start"] is not None:
            o.random_start(case["start"], 0.5)
            O.write_config(os.path.join(d, "s.dat"), o.links, o.plaquette())
            start = os.path.join(d, "s.dat")
        r = O.run_reference(b, case["L"], steps, dt, alpha, 99, d, start=start,
                            twist_init=tw != 0)
    g = (1,) + tuple(grid)
    for s in range(steps):
        ob = o.sweep(dt, r["noise"][s], zero_modes=case["zm"], onthefly=True, grid=g)
        assert obs_close(ob.plaq, r["plaq"][s], 1e-12)[0]
        assert obs_close(ob.norm, r["norm"][s], 1e-12)[0]
        if case["zm"]:
            o.zero_modes()
        o.local_gauge_fix(alpha, grid=g)
        o.twist_boundary()
    assert per_order_rel(o.links, r["links"], N).max() <= 1e-12


@pytest.mark.parametrize("L,grid", [((4, 4, 4, 4), (1, 1, 1)), ((4, 6, 6, 6), (2, 2, 2))],
                         ids=["sequential", "grid222_blocks3"])
def test_oracle_onthefly_improved_action_matches_reference(oracle_mod, L, grid):
    """The reference's on-the-fly build with the tree-level Symanzik action
    (GAUGE_ACTION TLSYM, choices.h:110; staple2x1 QCDenvNODEpt_test.h:
    579-611): plaquette and rectangle traces per step and the final links.
    The rectangles reach two sites, so threads of one barrier step only stay
    apart with blocks of 3 or more: with blocks of 2 the reference's own
    threaded run differs from run to run, and there is nothing to pin."""
    O = oracle_mod
    N, steps, dt, c1 = 4, 2, 0.01, -1.0 / 12.0
    b = O.ref_binary(N, "pbc", "local", grid, "tlsym", "otf")
    if not os.path.exists(b):
        if not os.path.exists(os.path.join(O.reference_dir(), "nspt.cc")):
            pytest.skip("reference sources not available")
        b = O.build_reference(N, "pbc", "local", grid, "tlsym", "otf")
    o = O.Oracle(L, N)
    o.random_start(29, 0.5)
    o.set_action(c1)
    with tempfile.TemporaryDirectory() as d:
        O.write_config(os.path.join(d, "s.dat"), o.links, o.plaquette())
        r = O.run_reference(b, L, steps, dt, 0.0, 47, d, start=os.path.join(d, "s.dat"))
    g = (1,) + tuple(grid)
    for s in range(steps):
        ob = o.sweep(dt, r["noise"][s], zero_modes=True, onthefly=True, grid=g)
        assert obs_close(ob.plaq, r["plaq"][s], 1e-12)[0]
        assert obs_close(o.last_w2()[:N], r["w2"][s][:N], 1e-12)[0]
        o.zero_modes()
        o.local_gauge_fix(0.0, grid=g)
    assert per_order_rel(o.links, r["links"], N).max() <= 1e-12
