"""The reference's default on-the-fly update (UPDATE_ONTHEFLY, choices.h:61)
on the GPU against the oracle, which the CPU suite pins to the reference's
own on-the-fly builds (tests/test_oracle_reference.py).  Links updated in
place in the order of the OpenMP thread grid; with twisted boundaries the
reads across a twisted face, in the sweep and in the local gauge fixing
after it, see the step's start field until twist_boundary.  Needs a B200.

Tolerances as tests/test_gpu_parity.py: per order <= 1e-12 after one step,
observables within tests/helpers.obs_close at 1e-11."""
import numpy as np
import pytest

from helpers import flag_diff, obs_close, per_order_rel

pytestmark = pytest.mark.gpu


def pair(P, O, L, N, twist="", zm=False, local_gf=False, fa=False, alpha=0.0, start=None,
         grid=(1, 1, 1, 1)):
    tw = 0
    for d in twist:
        tw |= {"y": 2, "z": 4, "t": 8}[d]
    o = O.Oracle(L, N, twist_mask=tw)
    if start is not None:
        o.random_start(start, 0.5)
    e = P.NsptEngine(L, N, twist=twist, zero_modes=zm, local_gf=local_gf, fa=fa, alpha=alpha,
                     update="onthefly")
    e.set_gf_grid(grid)
    e.upload(o.links)
    return e, o


def check_obs(eo, oo, tol):
    for name, a, b in (("plaq", eo.plaq, oo.plaq), ("norm", eo.norm, oo.norm),
                       ("tru", eo.tru.transpose(1, 0, 2), oo.tru.transpose(1, 0, 2))):
        ok, w = obs_close(a, b, tol)
        assert ok, (name, w)


@pytest.mark.parametrize("L,N,twist,grid", [
    ((4, 4, 4, 4), 4, "", (1, 1, 1, 1)),
    ((4, 4, 4, 4), 8, "", (2, 2, 2, 2)),
    ((6, 4, 4, 4), 6, "", (3, 2, 1, 2)),
    ((4, 4, 4, 4), 5, "yz", (1, 1, 1, 1)),
    ((4, 4, 4, 4), 6, "yzt", (1, 2, 2, 1)),
    ((4, 4, 4, 4), 24, "yz", (2, 2, 2, 2)),
    ((4, 4, 2, 4), 16, "", (1, 2, 1, 2)),
], ids=["sequential_n4", "grid2222_n8", "grid3212_6x_n6", "twisted_yz_sequential",
        "twisted_yzt_grid1221", "twisted_yz_n24_grid2222", "grid1212_n16"])
@pytest.mark.parametrize("form", ["group", "team"])
def test_onthefly_sweep_matches_oracle(engine_mod, oracle_mod, L, N, twist, grid, form):
    """gauge_wilson on the fly, one sweep, then twist_boundary, by one
    group per reference thread or by a warp of three (one plane's staples
    each; grids with one site per thread and barrier step)."""
    P, O = engine_mod, oracle_mod
    e, o = pair(P, O, L, N, twist=twist, start=500 + N, grid=grid)
    e.set_local_gf_form(form)
    rng = O.Rand55(7)
    for _ in range(2):
        nz = rng.gauss(o.V * 32)
        e.set_noise(nz)
        eo = e.gauge_wilson(0.01)
        oo = o.sweep(0.01, nz, onthefly=True, grid=grid)
        check_obs(eo, oo, 1e-11)
        e.twist_boundary()
        o.twist_boundary()
    out = e.download()
    assert per_order_rel(out, o.links, N).max() <= 1e-12
    assert flag_diff(out, o.links, N) == 0.0


@pytest.mark.parametrize("L,N,twist,zm,grid", [
    ((4, 4, 4, 4), 6, "", True, (2, 2, 2, 2)),
    ((4, 4, 4, 4), 5, "yz", False, (1, 1, 1, 1)),
    ((4, 4, 4, 4), 5, "yz", False, (1, 2, 2, 1)),
    ((4, 4, 4, 4), 14, "yz", False, (2, 2, 2, 2)),
], ids=["zm_grid2222", "twisted_sequential", "twisted_grid1221", "twisted_n14_grid2222"])
def test_onthefly_step_with_local_gauge_fixing(engine_mod, oracle_mod, L, N, twist, zm, grid):
    """NsptEvolve on the fly (nspt.cc:953-1039): sweep in place, zero modes,
    local gauge fixing (reading twisted back links as the step's start
    field), twist_boundary; three steps."""
    P, O = engine_mod, oracle_mod
    alpha = -0.05
    e, o = pair(P, O, L, N, twist=twist, zm=zm, local_gf=True, alpha=alpha, start=77,
                grid=grid)
    rng = O.Rand55(11)
    for _ in range(3):
        nz = rng.gauss(o.V * 32)
        e.set_noise(nz)
        e.NsptEvolve(0.01, 1, 1)
        oo = o.sweep(0.01, nz, zero_modes=zm, onthefly=True, grid=grid)
        if zm:
            o.zero_modes()
        o.local_gauge_fix(alpha, grid=grid)
        o.twist_boundary()
        check_obs(e.observables(), oo, 1e-11)
    out = e.download()
    assert per_order_rel(out, o.links, N).max() <= 1e-11
    assert flag_diff(out, o.links, N) == 0.0


@pytest.mark.parametrize("form", ["group", "team"])
def test_onthefly_twisted_gauge_fixing_forms(engine_mod, oracle_mod, form):
    """Both local gauge fixing kernels read a twisted back link from the
    step's start field after an on-the-fly sweep."""
    P, O = engine_mod, oracle_mod
    L, N, grid, alpha = (4, 4, 4, 4), 8, (2, 2, 2, 2), -0.07
    e, o = pair(P, O, L, N, twist="yz", local_gf=True, alpha=alpha, start=91, grid=grid)
    e.set_local_gf_form(form)
    rng = O.Rand55(3)
    nz = rng.gauss(o.V * 32)
    e.set_noise(nz)
    e.gauge_wilson(0.01)
    e.stochastic_gauge_fixing(alpha)
    e.twist_boundary()
    o.sweep(0.01, nz, onthefly=True, grid=grid)
    o.local_gauge_fix(alpha, grid=grid)
    o.twist_boundary()
    assert per_order_rel(e.download(), o.links, N).max() <= 1e-12


def test_onthefly_with_fa_gauge_fixing(engine_mod, oracle_mod):
    """Periodic boundaries, zero modes and FA gauge fixing after an
    on-the-fly sweep (no copy sites are involved)."""
    P, O = engine_mod, oracle_mod
    L, N, alpha, grid = (4, 4, 4, 4), 6, -0.05, (2, 2, 2, 2)
    e, o = pair(P, O, L, N, zm=True, fa=True, alpha=alpha, start=19, grid=grid)
    rng = O.Rand55(23)
    for _ in range(2):
        nz = rng.gauss(o.V * 32)
        e.set_noise(nz)
        e.NsptEvolve(0.01, 1, 1)
        oo = o.sweep(0.01, nz, zero_modes=True, onthefly=True, grid=grid)
        o.zero_modes()
        o.fa_gauge_fix(alpha)
        check_obs(e.observables(), oo, 1e-11)
    assert per_order_rel(e.download(), o.links, N).max() <= 1e-11


def test_onthefly_rejects_what_is_not_built(engine_mod):
    P = engine_mod
    with pytest.raises(Exception):
        P.NsptEngine((4, 4, 4, 4), 4, update="onthefly", precision="ff")


@pytest.mark.parametrize("action,c1,L,grid", [
    ("tlsym", -1.0 / 12.0, (6, 6, 6, 4), (2, 2, 2, 1)),
    ("dbw2", -1.4088, (4, 4, 4, 4), (1, 1, 1, 1)),
    ("iwa", -0.331, (4, 6, 6, 4), (1, 2, 2, 1)),
    ("tlsym", -1.0 / 12.0, (6, 6, 6, 6), (2, 2, 2, 2)),
], ids=["tlsym_blocks3", "dbw2_sequential", "iwa_blocks3", "tlsym_one_site_per_thread"])
def test_onthefly_improved_action(engine_mod, oracle_mod, action, c1, L, grid):
    """The improved-action sweep on the fly (periodic): plaquette and
    rectangle traces and the links against the oracle, on grids whose
    blocks are at least 3 sites (the rectangles reach two)."""
    P, O = engine_mod, oracle_mod
    N = 5
    o = O.Oracle(L, N)
    o.random_start(41, 0.5)
    o.set_action(c1)
    e = P.NsptEngine(L, N, action=action, update="onthefly")
    e.set_gf_grid(grid)
    e.upload(o.links)
    rng = O.Rand55(13)
    for _ in range(2):
        nz = rng.gauss(o.V * 32)
        e.set_noise(nz)
        eo = e.gauge_wilson(0.01)
        oo = o.sweep(0.01, nz, onthefly=True, grid=grid)
        check_obs(eo, oo, 1e-11)
        ok, w = obs_close(e.rect_observables(), o.last_w2(), 1e-11)
        assert ok, ("w2", w)
    assert per_order_rel(e.download(), o.links, N).max() <= 1e-12


def test_onthefly_improved_action_needs_blocks_of_three(engine_mod):
    """Blocks of 2 would let a thread's rectangles read links another thread
    of the same barrier step updates (the reference's threaded run then
    races): rejected, and the default grid uses blocks of 3 or more."""
    P = engine_mod
    e = P.NsptEngine((4, 4, 4, 4), 3, action="tlsym", update="onthefly")
    with pytest.raises(Exception):
        e.set_gf_grid((2, 2, 2, 2))
    e.set_gf_grid((1, 1, 1, 1))
    P.NsptEngine((4, 4, 4, 4), 3, action="tlsym").set_gf_grid((2, 2, 2, 2))


def test_onthefly_new_field_ends_stale_twisted_reads(engine_mod, oracle_mod):
    """Uploading a field replaces the step's start field as well: a sweep
    right after it, with no twist_boundary between, reads the new field
    across the twisted faces."""
    P, O = engine_mod, oracle_mod
    L, N, grid = (4, 4, 4, 4), 5, (2, 2, 2, 2)
    e, o = pair(P, O, L, N, twist="yz", start=301, grid=grid)
    rng = O.Rand55(5)
    nz = rng.gauss(o.V * 32)
    e.set_noise(nz)
    e.gauge_wilson(0.01)  # leaves the start field for twisted reads
    o2 = O.Oracle(L, N, twist_mask=6)
    o2.random_start(302, 0.5)
    e.upload(o2.links)
    nz = rng.gauss(o.V * 32)
    e.set_noise(nz)
    eo = e.gauge_wilson(0.01)
    oo = o2.sweep(0.01, nz, onthefly=True, grid=grid)
    check_obs(eo, oo, 1e-11)
    assert per_order_rel(e.download(), o2.links, N).max() <= 1e-12
