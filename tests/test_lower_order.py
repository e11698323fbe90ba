"""loadlowerorder (ptGluon_fld::loadlowerorder, QCDenvNODEpt_test.h:376-426):
a run at N orders started from a configuration saved with fewer orders.
Orders 1..LO come from the file, the orders above are zero, and every link
is unitarised, U = exp(reH(log U)).

The fixture tests/golden/lower/lower_n3_to_n6.npz holds the reference's own
result (its 6-order build loading a 3-order file written from an oracle
random start).  Tolerance: links per order relative to the order's largest
coefficient, <= 1e-12 (the oracle restatement reproduces the reference bit
for bit); flags exact.
"""
import os
import tempfile

import numpy as np
import pytest

from helpers import flag_diff, obs_close, per_order_rel

FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lower",
                   "lower_n3_to_n6.npz")


def _lower_file(O, g, d):
    L, LO = tuple(int(x) for x in g["L"]), int(g["LO"])
    o = O.Oracle(L, LO)
    o.random_start(int(g["start"]), 0.5)
    path = os.path.join(d, "lower.dat")
    O.write_config(path, o.links, o.plaquette())
    return path, o.plaquette()


def test_oracle_lower_order_load_matches_the_reference_fixture(oracle_mod):
    O = oracle_mod
    g = np.load(FIX)
    L, N, LO = tuple(int(x) for x in g["L"]), int(g["N"]), int(g["LO"])
    with tempfile.TemporaryDirectory() as d:
        path, plaq_lo = _lower_file(O, g, d)
        o = O.Oracle(L, N)
        tr = o.load_lower_order(path, LO)
    assert np.array_equal(tr, plaq_lo)
    links = g["links"]
    assert np.array_equal(o.links[: links.shape[0]], links)
    assert np.array_equal(o.plaquette(), g["plaq_final"])


@pytest.mark.gpu
def test_engine_lower_order_load_matches_the_reference(engine_mod, oracle_mod):
    P, O = engine_mod, oracle_mod
    g = np.load(FIX)
    L, N, LO = tuple(int(x) for x in g["L"]), int(g["N"]), int(g["LO"])
    with tempfile.TemporaryDirectory() as d:
        path, plaq_lo = _lower_file(O, g, d)
        o = O.Oracle(L, N)
        o.load_lower_order(path, LO)
        with P.NsptEngine(L, N) as e:
            e.seed(5, 0)
            e.NsptEvolve(0.01, 1, 0)  # a field that is not the cold start
            tr = e.loadlowerorder(path, LO)
            got = e.download()
            pm = e.plaquette_measure()
            with pytest.raises(P.NsptError):
                e.loadlowerorder(path, N + 1)   # more orders than the field holds
            with pytest.raises(P.NsptError):
                e.loadlowerorder(path, LO + 1)  # the file's size says LO orders
    assert np.array_equal(tr, plaq_lo)
    rel = per_order_rel(got, o.links, N)
    assert rel.max() <= 1e-12, rel
    assert flag_diff(got, o.links, N) == 0.0
    links = g["links"]
    assert per_order_rel(got[: links.shape[0]], links, N).max() <= 1e-12
    ok, w = obs_close(pm, g["plaq_final"], 1e-12)
    assert ok, w


@pytest.mark.gpu
@pytest.mark.parametrize("L,N,LO", [((4, 4, 4, 4), 24, 12), ((4, 4, 2, 4), 12, 11)])
def test_engine_lower_order_load_matches_the_oracle(engine_mod, oracle_mod, L, N, LO):
    """The 24-order shapes (paired-run products at N = 24) and the low-order
    ones (N = 12)."""
    P, O = engine_mod, oracle_mod
    with tempfile.TemporaryDirectory() as d:
        o = O.Oracle(L, LO)
        o.random_start(40 + N, 0.5)
        path = os.path.join(d, "lower.dat")
        O.write_config(path, o.links, o.plaquette())
        full = O.Oracle(L, N)
        full.load_lower_order(path, LO)
        with P.NsptEngine(L, N) as e:
            e.loadlowerorder(path, LO)
            got = e.download()
    assert per_order_rel(got, full.links, N).max() <= 1e-12
    assert flag_diff(got, full.links, N) == 0.0
