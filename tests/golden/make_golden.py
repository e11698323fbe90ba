"""Generate the golden fixtures in tests/golden from the reference's own code.

Runs the reference's NSPT implementation (built from its sources by
oracle/build_ref.sh into oracle/_ref) on small seeded cases and stores what
it prints and saves: per-step plaquette / norm / trU (nspt.cc:570-597), the
final configuration's static plaquette (nspt.cc:1316-1406) and a slice of
the final links, plus the first draws of its noise generator (MyRand.cc).

Random starts are produced by the oracle (oracle.random_start), written in
the reference's binary format and loaded by the reference harness; the
reference's plaquette of that start is stored too, so the fixture pins the
start as well.

    python tests/golden/make_golden.py [NAME ...]   # needs the reference's sources

The reference's location comes from PRLGT_REFERENCE (or REF); with names,
only those fixtures are written.
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, L, N, bc, gf, steps, dt, alpha, noise seed, start (None = cold | seed), zero modes
    dict(name="cold_pbc_zm_n8", L=(4, 4, 4, 4), N=8, bc="pbc", gf="local", steps=5, dt=0.01,
         alpha=0.0, seed=12345, start=None, zm=True),
    dict(name="rand_pbc_zm_fa_n6", L=(4, 4, 4, 4), N=6, bc="pbc", gf="fa", steps=3, dt=0.01,
         alpha=-0.05, seed=777, start=4242, zm=True),
    dict(name="rand_tw_yz_n5", L=(4, 4, 4, 4), N=5, bc="tw", gf="local", steps=3, dt=0.005,
         alpha=0.0, seed=31, start=99, zm=False),
    dict(name="rand_pbc_fa_odd_n4", L=(4, 2, 3, 6), N=4, bc="pbc", gf="fa", steps=2, dt=0.02,
         alpha=-0.1, seed=5, start=11, zm=True),
    dict(name="rand_pbc_localgf_n4", L=(4, 4, 4, 4), N=4, bc="pbc", gf="local", steps=2,
         dt=0.01, alpha=-0.05, seed=8, start=3, zm=True),
    dict(name="rand_pbc_tlsym_n4", L=(4, 4, 4, 4), N=4, bc="pbc", gf="local", steps=2,
         dt=0.01, alpha=0.0, seed=19, start=13, zm=True, action="tlsym"),
    # the benchmark's combination: 24 orders, twisted y,z, dt = 0.005
    dict(name="rand_tw_yz_n24", L=(4, 4, 4, 4), N=24, bc="tw", gf="local", steps=2,
         dt=0.005, alpha=0.0, seed=2424, start=24, zm=False),
    # the 16^4 x 20 workload's step: 20 orders, zero modes + FA every step
    dict(name="rand_pbc_zm_fa_n20", L=(4, 4, 4, 4), N=20, bc="pbc", gf="fa", steps=2,
         dt=0.01, alpha=0.05, seed=2020, start=20, zm=True),
    # the reference's default on-the-fly update (UPDATE_ONTHEFLY), one thread
    dict(name="rand_pbc_otf_localgf_n6", L=(4, 4, 4, 4), N=6, bc="pbc", gf="local", steps=3,
         dt=0.01, alpha=-0.05, seed=61, start=16, zm=True, update="otf"),
    dict(name="rand_tw_otf_localgf_n5", L=(4, 4, 4, 4), N=5, bc="tw", gf="local", steps=3,
         dt=0.01, alpha=-0.05, seed=62, start=17, zm=False, update="otf"),
    # ... and its OpenMP build with thread grid (2,2,2): thread tid draws from
    # its own MyRand, seeded seed + tid by the harness
    dict(name="rand_pbc_otf_grid222_n4", L=(4, 4, 4, 4), N=4, bc="pbc", gf="local", steps=3,
         dt=0.01, alpha=-0.05, seed=63, start=18, zm=True, update="otf", grid=(2, 2, 2)),
]
C1 = {"wil": 0.0, "tlsym": -1.0 / 12.0, "iwa": -0.331, "dbw2": -1.4088}

LINK_SITES = 6  # sites of the final field kept in the fixture


def make_case(c: dict) -> dict:
    action = c.get("action", "wil")
    binary = O.build_reference(c["N"], c["bc"], c["gf"], c.get("grid", (1, 1, 1)), action,
                               c.get("update", "jacobi"))
    with tempfile.TemporaryDirectory() as d:
        start = "cold"
        twist_mask = 6 if c["bc"] == "tw" else 0
        if c["start"] is not None:
            o = O.Oracle(c["L"], c["N"], twist_mask=twist_mask)
            o.random_start(c["start"], 0.5)
            O.write_config(os.path.join(d, "start.dat"), o.links, o.plaquette())
            start = os.path.join(d, "start.dat")
        r = O.run_reference(binary, c["L"], c["steps"], c["dt"], c["alpha"], c["seed"], d,
                            start=start, noise=True, twist_init=(c["bc"] == "tw"))
    out = dict(
        plaq=r["plaq"], norm=r["norm"], tru=r["tru"], plaq0=r["plaq0"],
        plaq_final=r["plaq_final"], links=r["links"][:LINK_SITES],
        noise0=r["noise"][0][:64],
    )
    if action != "wil":
        # rectangle traces; the reference's top order is a running sum over
        # the steps (w2[PTORD] is never reset), the others are per step
        out["w2"] = r["w2"]
        out["c1"] = C1[action]
    return out


# loadlowerorder (QCDenvNODEpt_test.h:376-426): the reference at N orders
# starts from a file saved with LO < N orders (an oracle random start)
LOWER = dict(name="lower_n3_to_n6", L=(4, 4, 2, 4), N=6, LO=3, start=33)


def make_lower(c: dict) -> dict:
    binary = O.build_reference(c["N"], "pbc", "fa", (1, 1, 1))
    with tempfile.TemporaryDirectory() as d:
        o = O.Oracle(c["L"], c["LO"])
        o.random_start(c["start"], 0.5)
        path = os.path.join(d, "lower.dat")
        O.write_config(path, o.links, o.plaquette())
        r = O.run_reference(binary, c["L"], 0, 0.01, 0.0, 1, d, start=path, noise=False,
                            lower=c["LO"])
    return dict(links=r["links"][:LINK_SITES], plaq_final=r["plaq_final"],
                L=np.array(c["L"]), N=c["N"], LO=c["LO"], start=c["start"])


def main():
    meta = []
    only = set(sys.argv[1:])
    if not only or LOWER["name"] in only:
        os.makedirs(os.path.join(OUT, "lower"), exist_ok=True)
        path = os.path.join(OUT, "lower", LOWER["name"] + ".npz")
        np.savez_compressed(path, **make_lower(LOWER))
        meta.append((LOWER["name"], os.path.getsize(path)))
    for c in CASES:
        if only and c["name"] not in only:
            continue
        res = make_case(c)
        path = os.path.join(OUT, c["name"] + ".npz")
        np.savez_compressed(path, **res, L=np.array(c["L"]), N=c["N"], steps=c["steps"],
                            dt=c["dt"], alpha=c["alpha"], seed=c["seed"],
                            start=-1 if c["start"] is None else c["start"],
                            twisted=c["bc"] == "tw", fa=c["gf"] == "fa", zm=c["zm"],
                            local_gf=c["gf"] == "local" and c["alpha"] != 0.0,
                            onthefly=c.get("update", "jacobi") == "otf",
                            grid=np.array((1,) + tuple(c.get("grid", (1, 1, 1)))))
        meta.append((c["name"], os.path.getsize(path)))
    for name, size in meta:
        print("%-28s %8d bytes" % (name, size))


if __name__ == "__main__":
    main()
