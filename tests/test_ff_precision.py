"""Float-float Cauchy products (NSPT_PRECISION_FF) against the FP64 oracle.

The float-float sweep computes the staple and U*staples products in pairs of
FP32 numbers (48 significant bits, error-free products and two-sums) with a
per-order scale 2^(e k); exp, log, exp*U and the accumulations stay FP64.
Its per-order error therefore sits a few bits above FP64 rounding: the bound
here is 1e-11 per order after one sweep (FP64 path: 1e-12), in the same
per-order metric as test_gpu_parity.py (max|gpu - oracle| / max|oracle| over
the order-k coefficients of all links).  The same seed on the FP64 engine
gives a different field (the products really ran in float-float), and with
the scale fixed at e = 0 the high orders of a field that grows tenfold per
order overflow FP32 -- the per-order rescaling is what keeps them.
"""
import numpy as np
import pytest

from helpers import flag_diff, obs_close, per_order_rel

pytestmark = pytest.mark.gpu

FF_TOL = 1e-11


def _pair(P, O, L, N, start, precision, twist=""):
    o = O.Oracle(L, N, twist_mask=sum({"y": 2, "z": 4, "t": 8}[d] for d in twist))
    if start is not None:
        o.random_start(start, 0.5)
    e = P.NsptEngine(L, N, precision=precision, twist=twist)
    e.upload(o.links)
    return e, o


def _sweeps(O, e, o, steps, dt, seed):
    rng = O.Rand55(seed)
    for _ in range(steps):
        nz = rng.gauss(o.V * 32)
        e.set_noise(nz)
        eo = e.gauge_wilson(dt)
        oo = o.sweep(dt, nz)
    return eo, oo


@pytest.mark.parametrize("L,N", [((4, 4, 4, 4), 8), ((2, 4, 2, 4), 24)])
def test_ff_one_sweep_random_start(engine_mod, oracle_mod, L, N):
    e, o = _pair(engine_mod, oracle_mod, L, N, 77 + N, "ff")
    d, _ = _pair(engine_mod, oracle_mod, L, N, 77 + N, "fp64")
    start = o.links.copy()
    eo, oo = _sweeps(oracle_mod, e, o, 1, 0.01, 5)
    o2 = oracle_mod.Oracle(L, N)
    o2.set_links(start)
    _sweeps(oracle_mod, d, o2, 1, 0.01, 5)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= FF_TOL, rel
    assert flag_diff(e.download(), o.links, N) == 0.0
    for name, a, b in (("plaq", eo.plaq, oo.plaq), ("norm", eo.norm, oo.norm)):
        ok, w = obs_close(a, b, FF_TOL)
        assert ok, (name, w)
    # the FP64 engine on the same input differs from the float-float one
    assert np.abs(d.download() - e.download()).max() > 0.0
    assert per_order_rel(d.download(), o.links, N).max() <= 1e-12


def test_ff_twisted_boundaries(engine_mod, oracle_mod):
    """The float-float sweep with twisted y,z boundaries (twists applied to
    the staged neighbour links before the float-float products)."""
    L, N = (4, 4, 4, 4), 10
    e, o = _pair(engine_mod, oracle_mod, L, N, 515, "ff", twist="yz")
    eo, oo = _sweeps(oracle_mod, e, o, 2, 0.005, 17)
    rel = per_order_rel(e.download(), o.links, N)
    assert rel.max() <= FF_TOL, rel
    ok, w = obs_close(eo.plaq, oo.plaq, FF_TOL)
    assert ok, w


def test_ff_high_orders_need_the_rescaling(engine_mod, oracle_mod):
    """A random start whose order-k coefficients grow about tenfold per order
    (2e44 at k = 40, above FP32's largest number from k ~ 34 on): with the
    fitted scale every order stays within FF_TOL of the oracle after a
    sweep; with the scale fixed at e = 0 the top orders overflow FP32."""
    L, N = (2, 4, 2, 4), 40
    o = oracle_mod.Oracle(L, N)
    o.random_start(3, 4.0)
    auto = engine_mod.NsptEngine(L, N, precision="ff")
    fixed = engine_mod.NsptEngine(L, N, precision="ff")
    auto.upload(o.links)
    fixed.upload(o.links)
    fixed.set_ff_scale(0)
    nz = oracle_mod.Rand55(9).gauss(o.V * 32)
    for e in (auto, fixed):
        e.set_noise(nz)
        e.gauge_wilson(0.01)
    o.sweep(0.01, nz)
    assert auto.ff_scale() < 0 and fixed.ff_scale() == 0
    rel = per_order_rel(auto.download(), o.links, N)
    assert rel.max() <= FF_TOL, rel
    with np.errstate(invalid="ignore"):
        lost = per_order_rel(fixed.download(), o.links, N)
    assert not np.isfinite(lost[-1]) or lost[-1] > 1e-3, lost


def test_ff_options_checked(engine_mod):
    P = engine_mod
    with pytest.raises(P.NsptError):
        P.NsptEngine((4, 4, 4, 4), 4, action="tlsym", precision="ff")
    e = P.NsptEngine((4, 4, 4, 4), 20, precision="ff")
    with pytest.raises(P.NsptError):
        e.set_ff_scale(51)  # |e| N > 1000
    e.set_ff_scale(-50)
    e.set_ff_scale(None)
    d = P.NsptEngine((4, 4, 4, 4), 4)
    with pytest.raises(P.NsptError):
        d.set_ff_scale(1)
    with pytest.raises(P.NsptError):
        d.ff_scale()


def test_ff_error_after_1_100_1000_steps_is_fp64_rounding_sized(engine_mod):
    """The 24^4 x 40 precision workload's accuracy claim, on 4^4 x 40: from
    a common field (20 FP64 steps from a cold start), float-float and FP64
    engines run on with the same noise (zero modes + FA every step, alpha =
    +0.05), beside a second FP64 run whose dt is larger by one part in 2^52.
    After 1, 100 and 1000 steps, the float-float per-order deviation from
    FP64 (max|ff - fp64| / max|fp64| over the order's coefficients) must be
    within 10x of the deviation that FP64's own rounding-level perturbation
    produces at that order, plus 1e-14: the float-float products cost no
    accuracy beyond what an FP64 run has anyway at every order."""
    P = engine_mod
    L, N, dt, alpha, warm = (4, 4, 4, 4), 40, 0.01, 0.05, 20
    kw = dict(zero_modes=True, fa=True, alpha=alpha)
    with P.NsptEngine(L, N, **kw) as base:
        base.seed(5150, 0)
        base.NsptEvolve(dt, warm, 1)
        start = base.download()
    ff = P.NsptEngine(L, N, precision="ff", **kw)
    ref = P.NsptEngine(L, N, **kw)
    pert = P.NsptEngine(L, N, **kw)
    for e in (ff, ref, pert):
        e.upload(start)
        e.seed(5150, warm)
    done = 0
    for m in (1, 100, 1000):
        ff.NsptEvolve(dt, m - done, 1)
        ref.NsptEvolve(dt, m - done, 1)
        pert.NsptEvolve(dt * (1.0 + 2.0 ** -52), m - done, 1)
        done = m
        r = ref.download()
        assert np.isfinite(r).all()
        e_ff = per_order_rel(ff.download(), r, N)
        e_64 = per_order_rel(pert.download(), r, N)
        bad = np.nonzero(e_ff > 10.0 * e_64 + 1e-14)[0]
        assert bad.size == 0, (m, [(int(k) + 1, float(e_ff[k]), float(e_64[k])) for k in bad])
    for e in (ff, ref, pert):
        e.close()
