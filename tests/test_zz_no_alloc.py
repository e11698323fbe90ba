"""The allocation-free plaquette entry point, nspt_plaquette_measure_noalloc,
against the context entry point nspt_plaquette_measure, through the C ABI.

The file name makes pytest collect it last. It must pass in a fresh
process, where its first call sets up the static scratch, and after every
other GPU test has run in the same process.

Tolerance: per order, as in the other observable checks (helpers.obs_close),
1e-12 relative to the order's magnitude. Only the order of the final
summation differs from the context path. Two calls in a row on the same
field must agree bit for bit.
"""
import ctypes

import numpy as np
import pytest

from helpers import obs_close

pytestmark = pytest.mark.gpu

TWIST = {"": 0, "yz": (1 << 1) | (1 << 2), "t": 1 << 3}


def _noalloc(lib, dev_ptr, A, L, N, flags):
    out = np.zeros((N + 1, 2))
    rc = lib.nspt_plaquette_measure_noalloc(
        ctypes.c_void_p(dev_ptr), A, (ctypes.c_int * 4)(*L), N, flags,
        out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), None)
    return rc, out


@pytest.mark.parametrize("twist,L,N,A", [("", (4, 4, 4, 6), 10, 10), ("yz", (4, 4, 4, 4), 7, 9),
                                         ("t", (2, 4, 2, 4), 24, 24),
                                         # 4V = 82944 links: more CTAs than the 1024 partial
                                         # rows, so each CTA loops over many links
                                         ("yz", (12, 12, 12, 12), 2, 3)])
def test_noalloc_plaquette_matches_context_entry(engine_mod, oracle_mod, twist, L, N, A):
    import torch
    P, O = engine_mod, oracle_mod
    lib = P._lib.load()
    o = O.Oracle(L, N, twist_mask=TWIST[twist])
    o.random_start(101 + N, 0.5)
    with P.NsptEngine(L, N, twist=twist) as e:
        e.upload(o.links)
        want = e.plaquette_measure()
    # the caller's own device copy: reference AoS layout, allocORD = A >= N
    host = np.zeros((o.V, 4, 2 * (1 + 9 * A)))
    host[:, :, : 2 * (1 + 9 * N)] = np.asarray(o.links).reshape(o.V, 4, -1)
    dev = torch.from_numpy(host.reshape(-1)).to("cuda")
    torch.cuda.synchronize()
    got = []
    for _ in range(2):
        rc, out = _noalloc(lib, dev.data_ptr(), A, L, N, TWIST[twist])
        assert rc == 0, lib.nspt_error_string(rc).decode()
        got.append(out)
    assert np.array_equal(got[0], got[1])
    for g in got:
        ok, worst = obs_close(g, want, 1e-12)
        assert ok, worst
    # the field was only read
    assert torch.equal(dev.cpu(), torch.from_numpy(host.reshape(-1)))


def test_noalloc_rejects_what_its_scratch_or_arguments_cannot_hold(engine_mod):
    import torch
    P = engine_mod
    lib = P._lib.load()
    L = (2, 2, 2, 2)
    dev = torch.zeros(16 * 4 * 2 * (1 + 9 * 60), dtype=torch.float64, device="cuda")
    p = dev.data_ptr()
    assert _noalloc(lib, p, 60, L, P._lib.NSPT_MAX_ORDER + 1, 0)[0] == P._lib.NSPT_ERR_ORDER
    assert _noalloc(lib, p, 4, L, 5, 0)[0] == P._lib.NSPT_ERR_ARG        # allocORD < N
    assert _noalloc(lib, p, 5, L, 5, 1)[0] == P._lib.NSPT_ERR_ARG        # x twist: no flag
    assert _noalloc(lib, p + 8, 5, L, 5, 0)[0] == P._lib.NSPT_ERR_ARG    # misaligned
    assert _noalloc(lib, 0, 5, L, 5, 0)[0] == P._lib.NSPT_ERR_ARG        # null field
    assert _noalloc(lib, p, 5, (2, 0, 2, 2), 5, 0)[0] == P._lib.NSPT_ERR_ARG
    # a rejected call leaves the next good one intact: a random field gives
    # what the context entry point gives (stale or unwritten scratch would not)
    from oracle import oracle as O
    o = O.Oracle(L, 5)
    o.random_start(313, 0.5)
    with P.NsptEngine(L, 5) as e:
        e.upload(o.links)
        want = e.plaquette_measure()
    host = np.asarray(o.links).reshape(-1)
    dev[: host.size] = torch.from_numpy(host).to("cuda")
    torch.cuda.synchronize()
    rc, out = _noalloc(lib, p, 5, L, 5, 0)
    assert rc == 0
    ok, worst = obs_close(out, want, 1e-12)
    assert ok, worst
