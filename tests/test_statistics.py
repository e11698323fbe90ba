"""Statistical agreement of long runs with the reference's own long runs.

The engine's production path (device Philox noise, Jacobi update, zero-mode
subtraction and local stochastic gauge fixing every step) against the
reference's program run the same way, with its own rand55 noise
(tests/golden/stat, made by make_stat_ref.py from the reference's code):
16 independent replicas each, 500 steps from a cold start to thermalise,
then the plaquette coefficients of 5000 steps averaged per replica.  The
means over replicas, with their standard errors, must agree order by order
within Z_MAX combined standard errors: against the reference's Jacobi build
(the same algorithm with other noise) and against its default on-the-fly
build.  The on-the-fly update (Gauss-Seidel order inside a sweep) integrates
the same Langevin equation with other O(dt) corrections: the reference's
two builds, run on the same seeds, differ by 0.0034 in the order-2
coefficient at dt = 0.01 (-2.0041 vs -2.0006, errors 0.0013).  That
measured difference enters the on-the-fly comparison as a systematic error.
The engine's own on-the-fly update is compared, with no systematic, with
the reference's on-the-fly build of the same OpenMP thread grid.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "stat",
                       "ref_longrun_pbc_n6.npz")
Z_MAX = 4.5


def mean_err(per_replica):
    """Mean over replicas and its standard error, real parts, per order."""
    x = np.asarray(per_replica)[:, :, 0]
    return x.mean(axis=0), x.std(axis=0, ddof=1) / np.sqrt(x.shape[0])


def test_plaquette_series_agree_with_the_reference_long_runs(engine_mod):
    P = engine_mod
    g = np.load(FIXTURE)
    L = tuple(int(x) for x in g["L"])
    N, dt, alpha = int(g["N"]), float(g["dt"]), float(g["alpha"])
    therm, meas, reps = int(g["therm"]), int(g["meas"]), len(g["seeds"])
    ours = []
    for r in range(reps):
        e = P.NsptEngine(L, N, zero_modes=True, local_gf=True, alpha=alpha)
        e.seed(424242 + 1000003 * r, 0)
        e.NsptEvolve(dt, therm, 1)
        acc = np.zeros((N + 1, 2))
        for _ in range(meas):
            e.NsptEvolve(dt, 1, 1)
            acc += e.observables().plaq
        ours.append(acc / meas)
        e.close()
    m, s = mean_err(ours)
    # the O(dt) difference between the reference's two updates, same seeds
    syst = np.abs(mean_err(g["means_jacobi"])[0] - mean_err(g["means_otf"])[0])
    for build in ("jacobi", "otf"):
        mr, sr = mean_err(g["means_" + build])
        extra = syst if build == "otf" else 0.0
        z = np.abs(m - mr) / np.sqrt(s ** 2 + sr ** 2 + extra ** 2 + 1e-300)
        # order 0 is the exact flag 1; order 1 vanishes identically
        assert np.all(z[2:] <= Z_MAX), (build, m, mr, s, sr, z)
        assert abs(m[0] - 1.0) < 1e-12


def test_onthefly_plaquette_series_agree_with_the_reference_long_runs(engine_mod):
    """The engine's on-the-fly update against the reference's on-the-fly
    build with the same OpenMP thread grid (1,2,2,2), so that both run the
    same algorithm with different noise: no systematic error enters.  The
    16 replicas run as one batch (one CUDA graph per step)."""
    P = engine_mod
    g = np.load(FIXTURE)
    if "means_otf_grid222" not in g:
        pytest.skip("fixture without the threaded on-the-fly runs")
    L = tuple(int(x) for x in g["L"])
    N, dt, alpha = int(g["N"]), float(g["dt"]), float(g["alpha"])
    therm, meas, reps = int(g["therm"]), int(g["meas"]), len(g["seeds"])
    b = P.NsptBatch([L] * reps, N, [dt] * reps, [515151 + 7919 * r for r in range(reps)],
                    zero_modes=True, local_gf=True, alpha=alpha, update="onthefly")
    for e in b.replicas:
        e.set_gf_grid((1, 2, 2, 2))
    b.step(therm, 1)
    # the batch graph advances two steps: the plaquette of every 2nd step
    acc = np.zeros((reps, N + 1, 2))
    for _ in range(meas // 2):
        b.step(2, 1)
        acc += b.plaquettes()
    b.close()
    m, s = mean_err(acc / (meas // 2))
    mr, sr = mean_err(g["means_otf_grid222"])
    z = np.abs(m - mr) / np.sqrt(s ** 2 + sr ** 2 + 1e-300)
    assert np.all(z[2:] <= Z_MAX), (m, mr, s, sr, z)
    assert abs(m[0] - 1.0) < 1e-12
