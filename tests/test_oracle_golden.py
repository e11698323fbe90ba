"""The oracle (oracle/nspt_oracle.c) against the golden fixtures made by the
reference's own code (tests/golden/make_golden.py): noise stream, per-step
plaquette / norm / trU, final links and static plaquette.  CPU only."""
import glob
import os

import numpy as np
import pytest

from helpers import obs_close, per_order_rel, rel_scale

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = sorted(glob.glob(os.path.join(GOLDEN, "*.npz")))
TOL = 1e-12


def replay(O, g):
    L = tuple(int(x) for x in g["L"])
    N = int(g["N"])
    o = O.Oracle(L, N, twist_mask=6 if bool(g["twisted"]) else 0)
    if int(g["start"]) >= 0:
        o.random_start(int(g["start"]), 0.5)
    if "c1" in g:
        o.set_action(float(g["c1"]))
    p0 = o.plaquette()
    grid = tuple(int(x) for x in g["grid"]) if "grid" in g else (1, 1, 1, 1)
    nthr = int(np.prod(grid))
    if nthr > 1:  # an OpenMP build: one MyRand per thread, seeded seed + tid
        tn = O.ThreadNoise(L, grid, [int(g["seed"]) + t for t in range(nthr)])
        draw = tn.gauss_links
    else:
        rng = O.Rand55(int(g["seed"]))
        draw = lambda: rng.gauss(o.V * 32)  # noqa: E731
    obs = []
    noise0 = None
    for s in range(int(g["steps"])):
        nz = draw()
        if s == 0:
            noise0 = nz[:64].copy()
        otf = "onthefly" in g and bool(g["onthefly"])
        ob = o.sweep(float(g["dt"]), nz, zero_modes=bool(g["zm"]), onthefly=otf, grid=grid)
        if "c1" in g:
            ob.w2 = o.last_w2()
        obs.append(ob)
        if bool(g["zm"]):
            o.zero_modes()
        if bool(g["fa"]):
            o.fa_gauge_fix(float(g["alpha"]))
        elif bool(g["local_gf"]):
            o.local_gauge_fix(float(g["alpha"]), grid=grid)
        o.twist_boundary()
    return o, p0, noise0, obs


@pytest.mark.parametrize("path", CASES, ids=[os.path.basename(p)[:-4] for p in CASES])
def test_oracle_matches_reference_golden(oracle_mod, path):
    g = np.load(path)
    o, p0, noise0, obs = replay(oracle_mod, g)
    N = int(g["N"])
    assert np.array_equal(noise0, g["noise0"]), "rand55 stream differs from MyRand"
    ok, w = obs_close(p0, g["plaq0"], TOL)
    assert ok, ("start plaquette", w)
    for s, ob in enumerate(obs):
        for name, a, b in (("plaq", ob.plaq, g["plaq"][s]), ("norm", ob.norm, g["norm"][s]),
                           ("tru", ob.tru.transpose(1, 0, 2), g["tru"][s].transpose(1, 0, 2))):
            ok, w = obs_close(a, b, TOL)
            assert ok, (name, s, w)
        if "c1" in g:  # orders below N; the reference's top order is cumulative
            ok, w = obs_close(ob.w2[:N], g["w2"][s][:N], TOL)
            assert ok, ("w2", s, w)
    rel = per_order_rel(o.links[: g["links"].shape[0]], g["links"], N)
    assert rel.max() <= TOL, rel
    ok, w = obs_close(o.plaquette(), g["plaq_final"][: N + 1], TOL)
    assert ok, ("final plaquette", w)


def test_golden_set_present():
    names = {os.path.basename(p) for p in CASES}
    for need in ("cold_pbc_zm_n8.npz", "rand_pbc_zm_fa_n6.npz", "rand_tw_yz_n5.npz"):
        assert need in names
