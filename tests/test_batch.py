"""Batches of replicas in one CUDA graph (nspt_batch_*), through the C ABI.

Every replica of a batch must be bit-identical to a context created, seeded
and stepped alike on its own: the graph replays the same kernels with the
same arguments, and nothing in a step depends on the order the replicas'
kernels run in.  Needs a B200.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = dict(L=[(4, 4, 4, 4), (6, 4, 4, 4), (4, 4, 2, 4)], dt=[0.005, 0.01, 0.02], seeds=[11, 12, 13])


def singles(P, N, steps, **kw):
    out = []
    for L, dt, sd in zip(CASES["L"], CASES["dt"], CASES["seeds"]):
        with P.NsptEngine(L, N, **kw) as e:
            e.seed(sd, 0)
            for n, gf in steps:
                e.NsptEvolve(dt, n, gf)
            out.append((e.download(), e.plaquette_measure()))
    return out


def test_batch_replicas_equal_single_contexts(engine_mod):
    P = engine_mod
    N, kw = 6, dict(zero_modes=True, fa=True, alpha=-0.05)
    want = singles(P, N, [(4, 1)], **kw)
    with P.NsptBatch(CASES["L"], N, CASES["dt"], CASES["seeds"], **kw) as b:
        b.step(2, 1)   # captures the graph
        b.step(2, 1)   # replays it
        plaq = b.plaquettes()
        for r, (links, pm) in enumerate(want):
            assert np.array_equal(b.replicas[r].download(), links), r
            assert np.array_equal(b.replicas[r].plaquette_measure(), pm), r
        assert np.all(np.isfinite(plaq)) and plaq.shape == (3, N + 1, 2)


def test_batch_captures_again_after_a_replica_stepped_alone(engine_mod):
    P = engine_mod
    N, kw = 5, dict(zero_modes=True, fa=True, alpha=-0.05)
    with P.NsptBatch(CASES["L"], N, CASES["dt"], CASES["seeds"], **kw) as b:
        b.step(2, 1)
        b.replicas[0].NsptEvolve(CASES["dt"][0], 1, 1)   # odd: its fields swap
        b.step(2, 1)
        got = [e.download() for e in b.replicas]
    for r, (L, dt, sd) in enumerate(zip(CASES["L"], CASES["dt"], CASES["seeds"])):
        with P.NsptEngine(L, N, **kw) as e:
            e.seed(sd, 0)
            e.NsptEvolve(dt, 5 if r == 0 else 4, 1)
            assert np.array_equal(got[r], e.download()), r


def test_batch_local_gauge_fixing_every_five_steps_twisted(engine_mod):
    P = engine_mod
    N, kw = 4, dict(twist="yz", local_gf=True, alpha=-0.07)
    want = singles(P, N, [(10, 5)], **kw)
    with P.NsptBatch(CASES["L"], N, CASES["dt"], CASES["seeds"], **kw) as b:
        with pytest.raises(P.NsptError):
            b.step(5, 5)   # not a whole graph (10 steps)
        b.step(10, 5)
        for r, (links, _) in enumerate(want):
            assert np.array_equal(b.replicas[r].download(), links), r


def test_batch_tune_restores_the_start(engine_mod):
    P = engine_mod
    N, kw = 6, dict(zero_modes=True, fa=True, alpha=-0.05)
    want = singles(P, N, [(2, 1)], **kw)
    with P.NsptBatch(CASES["L"], N, CASES["dt"], CASES["seeds"], **kw) as b:
        w = b.tune(1)
        assert 1 <= w <= 8
        b.step(2, 1)
        for r, (links, _) in enumerate(want):
            assert np.array_equal(b.replicas[r].download(), links), r


def test_batch_captures_again_after_a_replica_is_reseeded(engine_mod):
    """A replica reseeded between two batch steps, at the same phase of the
    two-step graph, gets its new noise stream: the batch equals single
    contexts seeded alike (the captured sweep holds the seed by value)."""
    P = engine_mod
    N, kw = 5, dict(zero_modes=True, fa=True, alpha=-0.05)
    with P.NsptBatch(CASES["L"], N, CASES["dt"], CASES["seeds"], **kw) as b:
        b.step(2, 1)
        b.replicas[1].seed(999, 2)
        b.step(2, 1)
        got = [e.download() for e in b.replicas]
    for r, (L, dt, sd) in enumerate(zip(CASES["L"], CASES["dt"], CASES["seeds"])):
        with P.NsptEngine(L, N, **kw) as e:
            e.seed(sd, 0)
            e.NsptEvolve(dt, 2, 1)
            if r == 1:
                e.seed(999, 2)
            e.NsptEvolve(dt, 2, 1)
            assert np.array_equal(got[r], e.download()), r


def test_batch_shape_tuner_covers_orders_per_lane_and_warps(engine_mod):
    """nspt_batch_tune_shape times both kernel shapes (8 and 4 orders per
    lane and pass; N = 6 allows both) at every warp count and keeps the
    fastest; the start is restored, and whatever shape it picks, the batch
    equals single contexts bit for bit (the shapes sum in the same order)."""
    P = engine_mod
    N, kw = 6, dict(zero_modes=True, fa=True, alpha=-0.05)
    want = singles(P, N, [(2, 1)], **kw)
    with P.NsptBatch(CASES["L"], N, CASES["dt"], CASES["seeds"], **kw) as b:
        w, mo, table = b.tune_shape(1)
        assert mo in (4, 8)
        assert np.all(table[0, :8] > 0) and np.all(table[1, :6] > 0) and np.all(table[1, 6:] == 0)
        row = 0 if mo == 8 else 1
        assert table[row, w - 1] == table[table > 0].min()
        b.step(2, 1)
        for r, (links, _) in enumerate(want):
            assert np.array_equal(b.replicas[r].download(), links), r
