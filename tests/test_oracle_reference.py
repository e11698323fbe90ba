"""The oracle against the reference's own code run live (oracle/_ref), on
cases larger than the committed fixtures.  Needs the reference's sources to
build the binary (or a binary already built); skipped otherwise.  CPU."""
import os
import tempfile

import numpy as np
import pytest

from helpers import obs_close, per_order_rel

REF = os.environ.get("PRLGT_REFERENCE", "/root/reference")


def ref_binary(O, N, bc, gf):
    b = O.ref_binary(N, bc, gf)
    if os.path.exists(b):
        return b
    if not os.path.exists(os.path.join(REF, "nspt.cc")):
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
