"""Generate tests/golden/stat/*.npz: long runs of the reference's own code,
for the statistical comparison of the plaquette series (test_statistics.py).

The reference's default program (Quenched.cc with choices.h as shipped:
periodic boundaries, zero-mode subtraction, local stochastic gauge fixing,
the on-the-fly update and its rand55 noise), its Jacobi build (the parity
build, UPDATE_ONTHEFLY off) and its on-the-fly build with OpenMP thread grid
(2,2,2) each run R independent replicas from a cold
start: THERM steps, then MEAS steps whose plaquette coefficients
(nspt.cc:570-597) are averaged per replica.  Only the per-replica averages
are stored, so the fixture is small.

    python tests/golden/make_stat_ref.py   # needs the reference sources (PRLGT_REFERENCE), ~4 min on 16 cores
"""
from __future__ import annotations

import os
import sys
import tempfile
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
from oracle import oracle as O  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "stat")

CFG = dict(L=(4, 4, 4, 4), N=6, dt=0.01, alpha=-0.05, therm=500, meas=5000, reps=16,
           seed0=9001)


def replica_means(binary, seed, cfg):
    with tempfile.TemporaryDirectory() as d:
        r = O.run_reference(binary, cfg["L"], cfg["therm"] + cfg["meas"], cfg["dt"], cfg["alpha"],
                            seed, d, noise=False)
    return r["plaq"][cfg["therm"]:].mean(axis=0)  # (N+1, 2)


def main():
    os.makedirs(OUT, exist_ok=True)
    cfg = CFG
    seeds = [cfg["seed0"] + 17 * r for r in range(cfg["reps"])]
    res = {}
    # the default on-the-fly build (one thread), the Jacobi build, and the
    # on-the-fly build with OpenMP thread grid (2,2,2): blocks of 2 sites
    for upd, grid in (("otf", (1, 1, 1)), ("jacobi", (1, 1, 1)), ("otf_grid222", (2, 2, 2))):
        b = O.build_reference(cfg["N"], "pbc", "local", grid, "wil", upd.split("_")[0])
        # a threaded build runs its replicas one at a time: its OpenMP
        # barriers crawl when the cores are oversubscribed
        workers = os.cpu_count() if grid == (1, 1, 1) else 1
        with ThreadPoolExecutor(max_workers=workers) as ex:
            means = list(ex.map(lambda s: replica_means(b, s, cfg), seeds))
        res[upd] = np.array(means)
        m = res[upd].mean(axis=0)[:, 0]
        e = res[upd].std(axis=0, ddof=1)[:, 0] / np.sqrt(cfg["reps"])
        print(upd, " ".join("%.5f(%.5f)" % (a, b_) for a, b_ in zip(m, e)))
    np.savez_compressed(os.path.join(OUT, "ref_longrun_pbc_n6.npz"),
                        L=np.array(cfg["L"]), N=cfg["N"], dt=cfg["dt"], alpha=cfg["alpha"],
                        therm=cfg["therm"], meas=cfg["meas"], seeds=np.array(seeds),
                        means_otf=res["otf"], means_jacobi=res["jacobi"],
                        means_otf_grid222=res["otf_grid222"])


if __name__ == "__main__":
    main()
