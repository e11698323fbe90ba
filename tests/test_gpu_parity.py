"""Parity of the CUDA engine with the oracle and with the reference's golden
fixtures, through the C ABI.  Needs a B200.

Tolerances (FP64 everywhere):
  links, per order k:  max|gpu - oracle| / max|oracle| over the order-k
                       coefficients of all links  <= 1e-12 after 1 step,
                       <= 1e-9 after 100 steps;
  observables:         tests/helpers.obs_close -- per order, relative to the
                       order's magnitude, with orders below 1e-2 of the
                       leading value held to an absolute bound.
"""
import glob
import math
import os

import numpy as np
import pytest

from helpers import flag_diff, obs_close, per_order_rel

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def make_pair(P, O, L, N, twist="", zm=False, fa=False, alpha=0.0, start=None):
    tw = 0
    for d in twist:
        tw |= {"y": 2, "z": 4, "t": 8}[d]
    o = O.Oracle(L, N, twist_mask=tw)
    if start is not None:
        o.random_start(start, 0.5)
    e = P.NsptEngine(L, N, twist=twist, zero_modes=zm, fa=fa, alpha=alpha)
    e.upload(o.links)
    return e, o


def step_both(e, o, dt, rng, zm=False, fa=False, alpha=0.0):
    nz = rng.gauss(o.V * 32)
    e.set_noise(nz)
    eo = e.gauge_wilson(dt)
    oo = o.sweep(dt, nz, zero_modes=zm)
    if zm:
        e.zero_modes_subtraction()
        o.zero_modes()
    if fa:
        e.FAstochastic_gauge_fixing(alpha)
        o.fa_gauge_fix(alpha)
    return eo, oo


def check_obs(eo, oo, tol):
    for name, a, b in (("plaq", eo.plaq, oo.plaq), ("norm", eo.norm, oo.norm),
                       ("tru", eo.tru.transpose(1, 0, 2), oo.tru.transpose(1, 0, 2))):
        ok, w = obs_close(a, b, tol)
        assert ok, (name, w)


@pytest.mark.parametrize("L,N", [((4, 4, 4, 4), 8), ((4, 4, 4, 4), 12), ((2, 4, 2, 4), 24),
                                 ((4, 2, 2, 2), 3), ((2, 2, 2, 2), 1), ((2, 4, 2, 4), 40),
                                 ((2, 2, 4, 2), 48), ((4, 2, 4, 2), 13), ((2, 4, 4, 2), 16),
                                 ((2, 2, 4, 4), 20)])
def test_one_sweep_random_start(engine_mod, oracle_mod, L, N):
    e, o = make_pair(engine_mod, oracle_mod, L, N, start=1234 + N)
    rng = oracle_mod.Rand55(42)
    eo, oo = step_both(e, o, 0.01, rng)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= 1e-12, rel
    assert flag_diff(e.download(), o.links, N) == 0.0
    check_obs(eo, oo, 1e-12)


def cold_bound(N, tol=1e-12):
    """Per-order bound after a cold start with zero modes: the zero-mode step
    takes log(exp(X)), whose orders >= 2 cancel exactly, so any two correct
    FP64 implementations differ there by ~k! * eps relative to the (k!-
    suppressed) order-k coefficient.  test_conditioning.py shows the oracle
    built with and without FMA contraction disagreeing by the same amount."""
    return np.array([max(tol, 1e-15 * math.factorial(k)) for k in range(1, N + 1)])


def test_cold_start_100_steps_zero_modes(engine_mod, oracle_mod):
    """Config 1: 4^4, 8 orders, cold, zero modes, dt = 0.01, 100 steps."""
    L, N = (4, 4, 4, 4), 8
    e, o = make_pair(engine_mod, oracle_mod, L, N, zm=True)
    rng = oracle_mod.Rand55(12345)
    for s in range(100):
        eo, oo = step_both(e, o, 0.01, rng, zm=True)
        if s in (0, 1):
            rel = per_order_rel(e.download(), o.links, N)
            assert np.all(rel <= cold_bound(N)), (s, rel)
        check_obs(eo, oo, 1e-9)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= 1e-9, rel


def test_cold_start_one_sweep_no_zero_modes(engine_mod, oracle_mod):
    """Without the log/exp round trip the cold start meets 1e-12 per order."""
    L, N = (4, 4, 4, 4), 8
    e, o = make_pair(engine_mod, oracle_mod, L, N)
    rng = oracle_mod.Rand55(12345)
    for s in range(2):
        eo, oo = step_both(e, o, 0.01, rng)
        rel = per_order_rel(e.download(), o.links, N)
        assert rel.max() <= 1e-12, (s, rel)
        check_obs(eo, oo, 1e-12)


@pytest.mark.parametrize("L,N,alpha", [((4, 4, 4, 4), 6, -0.05), ((4, 2, 3, 6), 4, -0.1),
                                       ((8, 4, 4, 4), 12, -0.05), ((10, 5, 4, 2), 4, -0.05),
                                       ((2, 12, 4, 6), 4, -0.05), ((16, 2, 2, 8), 3, -0.05),
                                       ((7, 4, 2, 4), 4, -0.05)])
def test_zero_modes_and_fa_gauge_fixing(engine_mod, oracle_mod, L, N, alpha):
    """Sweep + zero modes + FA gauge fixing, three steps.  The extents cover
    the FFT's radix-2, 3, 4 and 5 plans on every axis (10 and 5 on x, y; 12
    and 6 on y, t; 16 and 8 on x, t) and, with 7, the direct transform used
    for extents without a plan."""
    e, o = make_pair(engine_mod, oracle_mod, L, N, zm=True, fa=True, alpha=alpha, start=77)
    rng = oracle_mod.Rand55(3)
    for s in range(3):
        eo, oo = step_both(e, o, 0.01, rng, zm=True, fa=True, alpha=alpha)
        check_obs(eo, oo, 1e-11)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= 1e-11, rel


@pytest.mark.parametrize("twist,N", [("yz", 5), ("yz", 12), ("t", 4), ("yzt", 6)])
def test_twisted_boundaries(engine_mod, oracle_mod, twist, N):
    L = (4, 4, 4, 4)
    e, o = make_pair(engine_mod, oracle_mod, L, N, twist=twist, start=9)
    rng = oracle_mod.Rand55(17)
    eo, oo = step_both(e, o, 0.005, rng)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= 1e-12, rel
    check_obs(eo, oo, 1e-12)
    for s in range(3):
        eo, oo = step_both(e, o, 0.005, rng)
        check_obs(eo, oo, 1e-11)
    assert per_order_rel(e.download(), o.links, N).max() <= 1e-11


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (8, 8, 4, 4), (8, 8, 8, 4)])
def test_headline_combination_one_sweep(engine_mod, oracle_mod, L):
    """The benchmark's combination -- 24 orders, twisted y and z, dt = 0.005 --
    on lattices with every extent >= 4 (so x + mu and x - mu are distinct
    sites) and, at 8 x 8 x 4 x 4, extents above 4 in a twisted direction.
    8 x 8 x 8 x 4 (8192 links) is large enough for the sweep's CTA shape of
    large lattices (22 link groups over 8 warps, launch_sweep) and for
    several of its 4 x 4 x 4 site tiles.  One sweep from a random start:
    <= 1e-12 per order, flags exact (gauge_wilson nspt.cc:362-439, twist
    nspt.cc:163-255)."""
    N = 24
    e, o = make_pair(engine_mod, oracle_mod, L, N, twist="yz", start=2400 + L[0])
    rng = oracle_mod.Rand55(2424)
    eo, oo = step_both(e, o, 0.005, rng)
    got = e.download()
    rel = per_order_rel(got, o.links, N)
    assert rel.max() <= 1e-12, rel
    assert flag_diff(got, o.links, N) == 0.0
    check_obs(eo, oo, 1e-12)


def test_headline_combination_100_steps(engine_mod, oracle_mod):
    """100 sweeps of the benchmark's combination (24 orders, twisted y,z,
    dt = 0.005) from a random start on 4^4: <= 1e-9 per order at the end,
    observables within 1e-9 at every step."""
    L, N = (4, 4, 4, 4), 24
    e, o = make_pair(engine_mod, oracle_mod, L, N, twist="yz", start=2401)
    rng = oracle_mod.Rand55(99)
    for s in range(100):
        eo, oo = step_both(e, o, 0.005, rng)
        check_obs(eo, oo, 1e-9)
        if s == 0:
            assert per_order_rel(e.download(), o.links, N).max() <= 1e-12
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= 1e-9, rel


@pytest.mark.parametrize("L", [(4, 4, 4, 4), (8, 4, 4, 4)])
def test_c2_combination_zero_modes_and_fa(engine_mod, oracle_mod, L):
    """The 16^4 x 20 workload's step at a size the oracle runs in seconds:
    20 orders, random start, sweep + zero modes + FA gauge fixing every
    step (nspt.cc:605-654, 866-948).  One step <= 1e-12 per order."""
    N, alpha = 20, 0.05
    e, o = make_pair(engine_mod, oracle_mod, L, N, zm=True, fa=True, alpha=alpha, start=2000 + L[0])
    rng = oracle_mod.Rand55(2020)
    eo, oo = step_both(e, o, 0.01, rng, zm=True, fa=True, alpha=alpha)
    check_obs(eo, oo, 1e-12)
    got = e.download()
    rel = per_order_rel(got, o.links, N)
    assert rel.max() <= 1e-12, rel
    assert flag_diff(got, o.links, N) == 0.0


def test_c2_combination_100_steps(engine_mod, oracle_mod):
    """100 steps of sweep + zero modes + FA gauge fixing (alpha = +0.05, the
    damping sign) from a random start, 20 orders on 4^4: <= 1e-9 per order."""
    L, N, alpha = (4, 4, 4, 4), 20, 0.05
    e, o = make_pair(engine_mod, oracle_mod, L, N, zm=True, fa=True, alpha=alpha, start=2002)
    rng = oracle_mod.Rand55(7)
    for s in range(100):
        eo, oo = step_both(e, o, 0.01, rng, zm=True, fa=True, alpha=alpha)
        check_obs(eo, oo, 1e-9)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= 1e-9, rel


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))),
                         ids=lambda p: os.path.basename(p)[:-4])
def test_reference_golden_fixture(engine_mod, oracle_mod, path):
    """The engine replays each fixture the reference's own code produced."""
    g = np.load(path)
    local_gf = bool(g["local_gf"])
    L = tuple(int(x) for x in g["L"])
    N = int(g["N"])
    twist = "yz" if bool(g["twisted"]) else ""
    fa, zm, alpha = bool(g["fa"]), bool(g["zm"]), float(g["alpha"])
    action = {-1.0 / 12.0: "tlsym", -0.331: "iwa", -1.4088: "dbw2"}.get(
        float(g["c1"]) if "c1" in g else 0.0, "wil")
    o = oracle_mod.Oracle(L, N, twist_mask=6 if twist else 0)
    if int(g["start"]) >= 0:
        o.random_start(int(g["start"]), 0.5)
    otf = "onthefly" in g and bool(g["onthefly"])
    e = engine_mod.NsptEngine(L, N, twist=twist, zero_modes=zm, fa=fa, alpha=alpha, action=action,
                              update="onthefly" if otf else "jacobi")
    e.upload(o.links)
    ok, w = obs_close(e.plaquette_measure(), g["plaq0"], 1e-12)
    assert ok, ("start plaquette", w)
    grid = tuple(int(x) for x in g["grid"]) if "grid" in g else (1, 1, 1, 1)
    nthr = int(np.prod(grid))
    if local_gf or otf:
        e.set_gf_grid(grid)  # the fixture's reference build's OpenMP thread grid
    if nthr > 1:  # one MyRand per thread, seeded seed + tid
        tn = oracle_mod.ThreadNoise(L, grid, [int(g["seed"]) + t for t in range(nthr)])
        draw = tn.gauss_links
    else:
        rng = oracle_mod.Rand55(int(g["seed"]))
        draw = lambda: rng.gauss(o.V * 32)  # noqa: E731
    for s in range(int(g["steps"])):
        nz = draw()
        e.set_noise(nz)
        ob = e.gauge_wilson(float(g["dt"]))
        for name, a, b in (("plaq", ob.plaq, g["plaq"][s]), ("norm", ob.norm, g["norm"][s])):
            ok, w = obs_close(a, b, 1e-11)
            assert ok, (name, s, w)
        if action != "wil":  # orders below N (the reference's top order is cumulative)
            ok, w = obs_close(e.rect_observables()[:N], g["w2"][s][:N], 1e-11)
            assert ok, ("w2", s, w)
        if zm:
            e.zero_modes_subtraction()
        if fa:
            e.FAstochastic_gauge_fixing(alpha)
        if local_gf:
            e.stochastic_gauge_fixing(alpha)
        e.twist_boundary()
    rel = per_order_rel(e.download()[: g["links"].shape[0]], g["links"], N)
    bound = cold_bound(N, 1e-11) if (zm and int(g["start"]) < 0) else 1e-11
    assert np.all(rel <= bound), rel
    ok, w = obs_close(e.plaquette_measure(), g["plaq_final"][: N + 1], 1e-11)
    assert ok, ("final plaquette", w)


def test_plaquette_measure_matches_oracle(engine_mod, oracle_mod):
    e, o = make_pair(engine_mod, oracle_mod, (4, 4, 2, 4), 10, start=5)
    ok, w = obs_close(e.plaquette_measure(), o.plaquette(), 1e-12)
    assert ok, w


def test_upload_download_roundtrip_wider_alloc(engine_mod):
    P = engine_mod
    rng = np.random.default_rng(0)
    L, N, A = (2, 3, 2, 4), 5, 7
    V = int(np.prod(L))
    host = rng.standard_normal((V, 4, P.series_len(A)))
    with P.NsptEngine(L, N) as e:
        e.upload(host, allocORD=A)
        back = e.download(allocORD=A)
    keep = P.series_len(N)
    assert np.array_equal(back[:, :, :keep], host[:, :, :keep])
    assert np.all(back[:, :, keep:] == 0.0)


def test_save_load_reference_format(engine_mod, oracle_mod, tmp_path):
    P, O = engine_mod, oracle_mod
    e, o = make_pair(P, O, (4, 4, 4, 2), 6, start=8)
    p = str(tmp_path / "conf.dat")
    e.save(p, allocORD=6)
    links, plaq = O.read_config(p, o.V, 6)
    assert np.array_equal(links, o.links)
    assert obs_close(plaq, o.plaquette(), 1e-12)[0]
    e2 = P.NsptEngine((4, 4, 4, 2), 6)
    trailer = e2.load(p, allocORD=6)
    assert np.array_equal(e2.download(), o.links)
    assert np.array_equal(trailer, plaq)


def test_device_noise_statistics_and_determinism(engine_mod):
    """Philox noise: after one sweep from a cold start the order-1 link is
    -sqrt(dt) * SU3rand(eta) (the force vanishes at order 1), so its
    components carry the generator's Gaussians (variance 1/2)."""
    P = engine_mod
    L, N, dt = (8, 8, 8, 8), 2, 0.01
    outs = []
    for seed in (7, 7, 8):
        with P.NsptEngine(L, N) as e:
            e.seed(seed, 0)
            e.gauge_wilson(dt)
            outs.append(e.download())
    assert np.array_equal(outs[0], outs[1])
    assert not np.array_equal(outs[0], outs[2])
    u1 = outs[0][:, :, 2:20].reshape(-1, 9, 2) / (-np.sqrt(dt))
    g0 = u1[:, 1, 1]  # Im P[1] = g1
    g1 = u1[:, 1, 0]  # Re P[1] = g2
    for g in (g0, g1, u1[:, 2, 1], u1[:, 5, 0]):
        assert abs(g.mean()) < 0.02
        assert abs(g.var() - 0.5) < 0.02
    # anti-hermitian, traceless
    m = u1[:, :, 0] + 1j * u1[:, :, 1]
    m = m.reshape(-1, 3, 3)
    assert np.abs(m + np.conj(m.transpose(0, 2, 1))).max() < 1e-12
    assert np.abs(np.trace(m, axis1=1, axis2=2)).max() < 1e-12


def test_two_contexts_with_different_extents_interleaved(engine_mod, oracle_mod):
    """Contexts are independent: two FA contexts of different extents on one
    device, stepped alternately, each match their own oracle run."""
    cases = [((4, 4, 4, 4), 5, -0.05, 21), ((6, 4, 2, 4), 5, -0.08, 22)]
    pairs = [make_pair(engine_mod, oracle_mod, L, N, zm=True, fa=True, alpha=a, start=st)
             for L, N, a, st in cases]
    rngs = [oracle_mod.Rand55(40 + i) for i in range(len(cases))]
    for _ in range(2):
        for (e, o), rng, (_, _, alpha, _) in zip(pairs, rngs, cases):
            eo, oo = step_both(e, o, 0.01, rng, zm=True, fa=True, alpha=alpha)
            check_obs(eo, oo, 1e-11)
    for (e, o), (L, N, _, _) in zip(pairs, cases):
        assert per_order_rel(e.download(), o.links, N).max() <= 1e-11


@pytest.mark.parametrize("L,N,twist,grid", [
    ((4, 4, 4, 4), 4, "", (1, 1, 1, 1)),
    ((4, 4, 4, 4), 6, "", (2, 2, 2, 2)),
    ((4, 6, 4, 4), 5, "", (1, 3, 1, 2)),
    ((4, 4, 4, 4), 5, "yz", (1, 2, 2, 1)),
    ((4, 4, 4, 4), 12, "yzt", (2, 1, 2, 2)),
], ids=["sequential", "grid2222", "grid1312_6x", "twisted_yz_grid1221", "twisted_yzt_n12"])
@pytest.mark.parametrize("form", ["group", "team"])
def test_local_gauge_fixing_matches_oracle_thread_grid(engine_mod, oracle_mod, L, N, twist, grid,
                                                        form):
    """stochastic_gauge_fixing in the order the reference's OpenMP thread grid
    fixes (the oracle is pinned to the reference's builds of those grids),
    by either kernel form."""
    e, o = make_pair(engine_mod, oracle_mod, L, N, twist=twist, start=61)
    alpha = -0.08
    e.set_gf_grid(grid)
    e.set_local_gf_form(form)
    for _ in range(2):
        e.stochastic_gauge_fixing(alpha)
        o.local_gauge_fix(alpha, grid=grid)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= 1e-12, rel
    assert flag_diff(e.download(), o.links, N) == 0.0


def test_local_gauge_fixing_in_the_step_with_default_grid(engine_mod, oracle_mod):
    """nspt_step with NSPT_GF_LOCAL: sweep, zero modes, local gauge fixing;
    the default grid is the finest the reference accepts (blocks of 2)."""
    P, O = engine_mod, oracle_mod
    L, N, alpha = (4, 4, 2, 4), 6, -0.05
    o = O.Oracle(L, N)
    o.random_start(71, 0.5)
    e = P.NsptEngine(L, N, zero_modes=True, local_gf=True, alpha=alpha)
    e.upload(o.links)
    rng = O.Rand55(5)
    for _ in range(2):
        nz = rng.gauss(o.V * 32)
        e.set_noise(nz)
        e.NsptEvolve(0.01, 1, 1)
        oo = o.sweep(0.01, nz, zero_modes=True)
        o.zero_modes()
        o.local_gauge_fix(alpha, grid=(2, 2, 1, 2))
        check_obs(e.observables(), oo, 1e-11)
    assert per_order_rel(e.download(), o.links, N).max() <= 1e-11


@pytest.mark.parametrize("L,N,twist,grid", [
    ((4, 4, 4, 4), 24, "yz", (2, 2, 2, 2)),
    ((6, 4, 4, 8), 8, "yzt", (3, 2, 1, 4)),
], ids=["n24_twisted_yz", "n8_twisted_yzt_grid3214"])
def test_local_gauge_fixing_forms_agree(engine_mod, oracle_mod, L, N, twist, grid):
    """The team and group kernels on the same field: both within 1e-12 of the
    oracle per order, flags exact, and within rounding of each other."""
    P, O = engine_mod, oracle_mod
    alpha = -0.06
    outs = []
    for form in ("group", "team"):
        e, o = make_pair(P, O, L, N, twist=twist, start=83)
        e.set_gf_grid(grid)
        e.set_local_gf_form(form)
        e.stochastic_gauge_fixing(alpha)
        outs.append(e.download())
    o.local_gauge_fix(alpha, grid=grid)
    for out in outs:
        assert per_order_rel(out, o.links, N).max() <= 1e-12
        assert flag_diff(out, o.links, N) == 0.0
    assert per_order_rel(outs[0], outs[1], N).max() <= 1e-13


def test_local_gf_form_rejects_unknown(engine_mod):
    P = engine_mod
    e = P.NsptEngine((4, 4, 4, 4), 3, local_gf=True)
    with pytest.raises(ValueError):
        e.set_local_gf_form("warp")
    assert P.load_library().nspt_set_local_gf_form(e._h, 7) != 0


def test_gf_grid_rejects_what_the_reference_rejects(engine_mod):
    P = engine_mod
    with P.NsptEngine((4, 6, 4, 4), 3) as e:
        for bad in [(3, 1, 1, 1), (1, 6, 1, 1), (0, 1, 1, 1)]:
            with pytest.raises(P.NsptError):
                e.set_gf_grid(bad)
        e.set_gf_grid((2, 3, 2, 2))
    with pytest.raises(P.NsptError):
        P.NsptEngine((4, 4, 4, 4), 3, fa=True, local_gf=True)


@pytest.mark.parametrize("L,N", [((4, 4, 4, 4), 6), ((6, 4, 4, 4), 4), ((4, 4, 4, 4), 12)])
def test_wilson_loops_match_oracle(engine_mod, oracle_mod, L, N):
    """ComputeLoops (nspt.cc:1148-1312): all orders of the four loop traces."""
    e, o = make_pair(engine_mod, oracle_mod, L, N, start=31 + N)
    got, want = e.ComputeLoops(), o.wilson_loops()
    for q in range(4):
        ok, w = obs_close(got[q], want[q], 1e-12)
        assert ok, (q, w)
    # WL2x2 (nspt.cc:1064-1140): the 2x2 loop walked the other way round
    want22 = want[1] * np.array([1.0, -1.0])
    ok, w = obs_close(e.WL2x2(), want22, 1e-12)
    assert ok, ("wl2x2", w)


def test_wilson_loops_need_periodic_boundaries(engine_mod):
    e = engine_mod.NsptEngine((4, 4, 4, 4), 4, twist="yz")
    with pytest.raises(engine_mod.NsptError):
        e.ComputeLoops()
    with pytest.raises(engine_mod.NsptError):
        e.WL2x2()


@pytest.mark.parametrize("action,c1,L,N", [("tlsym", -1.0 / 12.0, (4, 4, 4, 4), 6),
                                           ("iwa", -0.331, (6, 4, 4, 4), 4),
                                           ("dbw2", -1.4088, (4, 4, 4, 4), 8)])
def test_improved_action_sweeps_match_oracle(engine_mod, oracle_mod, action, c1, L, N):
    """gauge_wilson with an improved action (nspt.cc:272-308): links, the
    plaquette and the rectangle traces w2, two sweeps with zero modes."""
    P, O = engine_mod, oracle_mod
    o = O.Oracle(L, N)
    o.random_start(88, 0.5)
    o.set_action(c1)
    e = P.NsptEngine(L, N, zero_modes=True, action=action)
    e.upload(o.links)
    rng = O.Rand55(9)
    for s in range(2):
        nz = rng.gauss(o.V * 32)
        e.set_noise(nz)
        eo = e.gauge_wilson(0.01)
        oo = o.sweep(0.01, nz, zero_modes=True)
        check_obs(eo, oo, 1e-12 if s == 0 else 1e-11)
        ok, w = obs_close(e.rect_observables(), o.last_w2(), 1e-12 if s == 0 else 1e-11)
        assert ok, ("w2", s, w)
        e.zero_modes_subtraction()
        o.zero_modes()
    assert per_order_rel(e.download(), o.links, N).max() <= 1e-11


def test_watchdog_timeout_returns_and_the_context_stays_usable(engine_mod):
    """nspt_set_timeout: a call whose device work outlasts the limit returns
    NSPT_ERR_TIMEOUT while the work runs on; the next call waits for it, and
    the field equals that of a context run without a limit."""
    from prlgt2020_b200 import _lib
    P = engine_mod
    L, N = (16, 16, 16, 16), 12
    a, b = P.NsptEngine(L, N, zero_modes=True), P.NsptEngine(L, N, zero_modes=True)
    for e in (a, b):
        e.seed(77, 0)
    a.set_timeout(1e-6)
    with pytest.raises(P.NsptError) as err:
        a.NsptEvolve(0.01, 3, 1)
    assert err.value.code == _lib.NSPT_ERR_TIMEOUT
    a.set_timeout(0.0)
    a.NsptEvolve(0.01, 1, 1)
    b.NsptEvolve(0.01, 4, 1)
    assert np.array_equal(a.download(), b.download())
    assert np.array_equal(a.observables().plaq, b.observables().plaq)


def test_checkpoint_with_rng_state_resumes_the_same_stream(engine_mod, tmp_path):
    """save + rng_state, then load + seed(seed, counter) in a new context:
    the resumed run equals the uninterrupted one bit for bit."""
    P = engine_mod
    L, N = (4, 4, 4, 4), 6
    kw = dict(zero_modes=True, local_gf=True, alpha=-0.05)
    whole = P.NsptEngine(L, N, **kw)
    whole.seed(31337, 0)
    whole.NsptEvolve(0.01, 5, 1)
    first = P.NsptEngine(L, N, **kw)
    first.seed(31337, 0)
    first.NsptEvolve(0.01, 2, 1)
    path = str(tmp_path / "conf.dat")
    first.save(path)
    state = first.rng_state()
    assert state == (31337, 2)
    resumed = P.NsptEngine(L, N, **kw)
    resumed.load(path)
    resumed.seed(*state)
    resumed.NsptEvolve(0.01, 3, 1)
    assert np.array_equal(whole.download(), resumed.download())
    assert resumed.rng_state() == whole.rng_state() == (31337, 5)
