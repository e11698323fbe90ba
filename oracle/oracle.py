"""TEST INFRASTRUCTURE (oracle).  ctypes binding of liboracle.so.

liboracle.so is the plain-C restatement of the reference's Langevin step
(nspt_oracle.c).  Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` import this module, and only as the checker.

Also drives the reference's own code built by ``build_ref.sh`` (``oracle/_ref``)
when that binary is present: ``run_reference`` runs it and parses its outputs.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build() -> str:
    """Compile liboracle.so (gcc, seconds)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return os.path.join(HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "nspt_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        L.oracle_create.restype = P
        L.oracle_create.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int]
        L.oracle_destroy.argtypes = [P]
        L.oracle_links.restype = D
        L.oracle_links.argtypes = [P]
        L.oracle_volume.restype = ctypes.c_long
        L.oracle_volume.argtypes = [P]
        L.oracle_cold_start.argtypes = [P]
        L.oracle_random_start.argtypes = [P, ctypes.c_long, ctypes.c_double]
        L.oracle_unitarise.argtypes = [P]
        L.oracle_sweep.argtypes = [P, ctypes.c_double, D, D, D, D, ctypes.c_int]
        L.oracle_sweep_onthefly.argtypes = [P, ctypes.c_double, D, ctypes.POINTER(ctypes.c_int),
                                            D, D, D, ctypes.c_int]
        L.oracle_sweep_onthefly.restype = ctypes.c_int
        L.oracle_twist_boundary.argtypes = [P]
        L.oracle_zero_modes.argtypes = [P]
        L.oracle_fa_gauge_fix.argtypes = [P, ctypes.c_double]
        L.oracle_local_gauge_fix.argtypes = [P, ctypes.c_double]
        L.oracle_local_gauge_fix_grid.argtypes = [P, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
        L.oracle_local_gauge_fix_grid.restype = ctypes.c_int
        L.oracle_wilson_loops.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
        L.oracle_set_action.argtypes = [P, ctypes.c_double]
        L.oracle_set_action.restype = ctypes.c_int
        L.oracle_last_w2.argtypes = [P, ctypes.POINTER(ctypes.c_double)]
        L.oracle_plaquette.argtypes = [P, D]
        for f in ("oracle_ser_mul",):
            getattr(L, f).argtypes = [ctypes.c_int, D, D, D]
        for f in ("oracle_ser_exp", "oracle_ser_log", "oracle_ser_dag"):
            getattr(L, f).argtypes = [ctypes.c_int, D, D]
        L.oracle_ser_reH.argtypes = [ctypes.c_int, D]
        L.oracle_rng_create.restype = P
        L.oracle_rng_create.argtypes = [ctypes.c_long]
        L.oracle_rng_destroy.argtypes = [P]
        L.oracle_rng_gauss.argtypes = [P, D, ctypes.c_long]
        L.oracle_su3rand.argtypes = [D, D]
        _LIB = L
    return _LIB


def _dp(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def series_len(N: int) -> int:
    """Doubles per series: flag + N orders x 9 complex."""
    return 2 + 18 * N


class Rand55:
    """The reference's MyRand generator (rand55 + Box-Muller, MyRand.cc)."""

    def __init__(self, seed: int):
        self._h = lib().oracle_rng_create(int(seed))

    def gauss(self, n: int) -> np.ndarray:
        out = np.empty(int(n), dtype=np.float64)
        lib().oracle_rng_gauss(self._h, _dp(out), int(n))
        return out

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.oracle_rng_destroy(h)
            self._h = None


class ThreadNoise:
    """The noise of the reference's OpenMP build with thread grid
    grid = (ntt, ntx, nty, ntz): thread tid draws from its own MyRand,
    seeded with seeds[tid], the 8 Gaussians of every link of its block
    (blocks as Quenched.cc:518-531), sites in the block's lexicographic order
    and mu inner (nspt.cc:355-440).  gauss_links() gives one step's V*4*8
    draws by link (site lexicographic, mu inner)."""

    def __init__(self, L, grid, seeds):
        self.L = tuple(int(x) for x in L)
        self.grid = tuple(int(x) for x in grid)
        nthr = int(np.prod(self.grid))
        if len(seeds) < nthr:
            raise ValueError("one seed per thread")
        self.rngs = [Rand55(int(seeds[t])) for t in range(nthr)]
        bs = [l // n for l, n in zip(self.L, self.grid)]
        s3, s2, s1 = self.L[3], self.L[2] * self.L[3], self.L[1] * self.L[2] * self.L[3]
        self.blocks = []
        for tid in range(nthr):
            b = (tid // (self.grid[1] * self.grid[2] * self.grid[3]),
                 (tid // (self.grid[2] * self.grid[3])) % self.grid[1],
                 (tid // self.grid[3]) % self.grid[2], tid % self.grid[3])
            sites = [(x0 * s1 + x1 * s2 + x2 * s3 + x3)
                     for x0 in range(b[0] * bs[0], (b[0] + 1) * bs[0])
                     for x1 in range(b[1] * bs[1], (b[1] + 1) * bs[1])
                     for x2 in range(b[2] * bs[2], (b[2] + 1) * bs[2])
                     for x3 in range(b[3] * bs[3], (b[3] + 1) * bs[3])]
            self.blocks.append(np.array(sites, dtype=np.int64))
        self.V = s1 * self.L[0]

    def gauss_links(self) -> np.ndarray:
        out = np.empty((self.V, 32))
        for rng, sites in zip(self.rngs, self.blocks):
            out[sites] = rng.gauss(sites.size * 32).reshape(-1, 32)
        return out.reshape(-1)


@dataclass
class SweepObs:
    plaq: np.ndarray  # (N+1, 2)
    norm: np.ndarray  # (N,)
    tru: np.ndarray  # (4, N, 2)


class Oracle:
    """One lattice field on the host, reference AoS layout."""

    def __init__(self, L, N: int, twist_mask: int = 0):
        self.L = tuple(int(x) for x in L)
        self.N = int(N)
        arr = (ctypes.c_int * 4)(*self.L)
        self._h = lib().oracle_create(arr, self.N, int(twist_mask))
        if not self._h:
            raise ValueError("oracle_create rejected the lattice")
        self.V = int(lib().oracle_volume(self._h))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _LIB is not None:
            _LIB.oracle_destroy(h)
            self._h = None

    @property
    def links(self) -> np.ndarray:
        """View (V, 4, 2+18N) of the field (reference byte layout)."""
        p = lib().oracle_links(self._h)
        n = self.V * 4 * series_len(self.N)
        flat = np.ctypeslib.as_array(p, shape=(n,))
        return flat.reshape(self.V, 4, series_len(self.N))

    def set_links(self, a: np.ndarray):
        self.links[...] = np.asarray(a, dtype=np.float64).reshape(self.links.shape)

    def cold_start(self):
        lib().oracle_cold_start(self._h)

    def random_start(self, seed: int, sigma: float = 0.5):
        lib().oracle_random_start(self._h, int(seed), float(sigma))

    def unitarise(self):
        """U = exp(reH(log U)) per link (QCDenvNODEpt_test.h:414-417)."""
        lib().oracle_unitarise(self._h)

    def load_lower_order(self, path: str, loworder: int) -> np.ndarray:
        """loadlowerorder (QCDenvNODEpt_test.h:376-426): a configuration
        file holding `loworder` <= N orders fills orders 1..loworder, the
        orders above are zero, and every link is unitarised.  Returns the
        file's loworder + 1 plaquette values.  (The reference's zeroing loop
        starts one order too high, at ptU[loworder+1]: order loworder + 1
        keeps what the field held before the call, zero after a cold start,
        which is what this restatement gives.)"""
        lo = int(loworder)
        if not 1 <= lo <= self.N:
            raise ValueError("loworder must be in 1..N")
        links, plaq = read_config(path, self.V, lo)
        full = np.zeros(self.links.shape)
        full[:, :, : series_len(lo)] = links
        self.set_links(full)
        self.unitarise()
        return plaq

    def sweep(self, dt: float, noise: np.ndarray, zero_modes: bool = False,
              onthefly: bool = False, grid=(1, 1, 1, 1)) -> SweepObs:
        """gauge_wilson: the Jacobi update (Umu = Fmu after the sweep), or
        with onthefly the reference's default in-place update in the order
        of the OpenMP thread grid (ntt, ntx, nty, ntz).  noise: V*4*8
        Gaussians by link (site lexicographic, mu inner)."""
        N = self.N
        noise = np.ascontiguousarray(noise, dtype=np.float64)
        assert noise.size == self.V * 4 * 8
        plaq = np.zeros((N + 1, 2))
        norm = np.zeros(N)
        tru = np.zeros((4, N, 2))
        if onthefly:
            g = (ctypes.c_int * 4)(*[int(x) for x in grid])
            if lib().oracle_sweep_onthefly(self._h, float(dt), _dp(noise), g, _dp(plaq), _dp(norm),
                                           _dp(tru), 1 if zero_modes else 0) != 0:
                raise ValueError("thread grid %r rejected" % (tuple(grid),))
        else:
            lib().oracle_sweep(self._h, float(dt), _dp(noise), _dp(plaq), _dp(norm), _dp(tru),
                               1 if zero_modes else 0)
        return SweepObs(plaq, norm, tru)

    def twist_boundary(self):
        """twist_boundary (nspt.cc:163-255): after an on-the-fly sweep, reads
        across a twisted face see the current field again."""
        lib().oracle_twist_boundary(self._h)

    def zero_modes(self):
        lib().oracle_zero_modes(self._h)

    def fa_gauge_fix(self, alpha: float):
        lib().oracle_fa_gauge_fix(self._h, float(alpha))

    def set_action(self, c1: float):
        """Improved gauge action c1 (Quenched.cc:311-322), periodic only."""
        if lib().oracle_set_action(self._h, float(c1)) != 0:
            raise ValueError("improved actions need periodic boundaries")

    def last_w2(self) -> np.ndarray:
        out = np.zeros((self.N + 1, 2))
        lib().oracle_last_w2(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def wilson_loops(self) -> np.ndarray:
        """ComputeLoops (nspt.cc:1148-1312): [4, N+1, 2] traces of the 1x2,
        2x2, 2x4, 4x4 loops, normalised as the reference prints them."""
        out = np.zeros((4, self.N + 1, 2))
        lib().oracle_wilson_loops(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return out

    def local_gauge_fix(self, alpha: float, grid=(1, 1, 1, 1)):
        """stochastic_gauge_fixing as the reference built with the OpenMP
        thread grid (ntt, ntx, nty, ntz) runs it (nspt.cc:660-862)."""
        g = (ctypes.c_int * 4)(*grid)
        if lib().oracle_local_gauge_fix_grid(self._h, float(alpha), g) != 0:
            raise ValueError("thread grid %r does not tile the lattice" % (tuple(grid),))

    def plaquette(self) -> np.ndarray:
        out = np.zeros((self.N + 1, 2))
        lib().oracle_plaquette(self._h, _dp(out))
        return out


def ser_op(name: str, N: int, *args: np.ndarray) -> np.ndarray:
    out = np.zeros(series_len(N))
    fn = getattr(lib(), "oracle_ser_" + name)
    fn(int(N), *[_dp(np.ascontiguousarray(a, dtype=np.float64)) for a in args], _dp(out))
    return out


# ---------------------------------------------------------------------------
# The reference's own code (oracle/_ref, built by build_ref.sh)
# ---------------------------------------------------------------------------

def reference_dir() -> str:
    """The reference's source tree: $PRLGT_REFERENCE, else $REF, else a
    directory named `reference` beside the repository."""
    for var in ("PRLGT_REFERENCE", "REF"):
        if os.environ.get(var):
            return os.environ[var]
    return os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def ref_binary(N: int, bc: str = "pbc", gf: str = "local", grid=(1, 1, 1),
               action: str = "wil", update: str = "jacobi") -> str:
    name = "ref_N%d_%s_%s_t%d%d%d" % ((N, bc, gf) + tuple(grid))
    if action != "wil":
        name += "_" + action
    if update != "jacobi":
        name += "_" + update
    return os.path.join(HERE, "_ref", name, "ref_harness")


def build_reference(N: int, bc: str = "pbc", gf: str = "local", grid=(1, 1, 1),
                    action: str = "wil", update: str = "jacobi") -> str:
    """update: "jacobi" (UPDATE_ONTHEFLY off, the parity builds) or "otf"
    (the reference's default on-the-fly update, choices.h:61)."""
    subprocess.run([os.path.join(HERE, "build_ref.sh"), str(N), bc, gf] +
                   [str(g) for g in grid] + [action, update], check=True,
                   stdout=subprocess.DEVNULL, env=dict(os.environ, REF=reference_dir()))
    return ref_binary(N, bc, gf, grid, action, update)


def read_config(path: str, V: int, N: int):
    """Reference configuration file: V*4 series + (N+1) complex plaquette."""
    raw = np.fromfile(path, dtype=np.float64)
    nl = V * 4 * series_len(N)
    assert raw.size == nl + 2 * (N + 1), (raw.size, nl)
    return raw[:nl].reshape(V, 4, series_len(N)), raw[nl:].reshape(N + 1, 2)


def write_config(path: str, links: np.ndarray, plaq: np.ndarray):
    with open(path, "wb") as f:
        np.ascontiguousarray(links, dtype=np.float64).tofile(f)
        np.ascontiguousarray(plaq, dtype=np.float64).tofile(f)


def run_reference(binary: str, L, steps: int, dt: float, alpha: float, seed: int,
                  workdir: str, start: str = "cold", noise: bool = True,
                  twist_init: bool = False, project: bool = False, timing: bool = False,
                  wl2x2: bool = False, sweep_only: bool = False, lower: int = 0):
    """Run the reference harness; returns dict of parsed outputs."""
    out = os.path.join(workdir, "ref")
    cmd = [binary, "--L", *[str(x) for x in L], "--steps", str(steps), "--dt", repr(dt),
           "--alpha", repr(alpha), "--seed", str(seed), "--start", start, "--out", out]
    if noise:
        cmd += ["--noise", out + ".noise"]
    if twist_init:
        cmd.append("--twist-init")
    if project:
        cmd.append("--project")
    if timing:
        cmd.append("--time")
    if sweep_only:
        cmd.append("--sweep-only")
    if lower:
        cmd += ["--lower", str(lower)]
    if wl2x2:
        cmd += ["--wl2x2", out + ".wl2x2"]
    p = subprocess.run(cmd, check=True, capture_output=True, text=True)
    V = int(np.prod(L))
    res = {"stdout": p.stdout}
    for ln in p.stdout.splitlines():
        if ln.startswith("step_seconds"):
            res["step_seconds"] = [float(x) for x in ln.split()[1:]]
    if steps == 0:  # a load only: the start's plaquette and the saved field
        p0 = np.loadtxt(out + ".plaq0").reshape(-1, 2)
        res["plaq0"] = p0
        res["links"], res["plaq_final"] = read_config(out + ".dat", V, p0.shape[0] - 1)
        return res
    N = None
    raw = np.loadtxt(out + ".plaq")
    if raw.ndim == 2 and raw.shape[1] == 4:  # improved action: w1 and w2 (nspt.cc:586-597)
        res["w2"] = raw[:, 2:].reshape(steps, -1, 2)
        raw = raw[:, :2]
    plaq = raw.reshape(steps, -1, 2)
    N = plaq.shape[1] - 1
    res["plaq"] = plaq
    res["norm"] = np.loadtxt(out + ".nor").reshape(steps, N)
    res["tru"] = np.loadtxt(out + ".tru").reshape(steps, N, 4, 2).transpose(0, 2, 1, 3)
    res["plaq0"] = np.loadtxt(out + ".plaq0").reshape(N + 1, 2)
    res["links"], res["plaq_final"] = read_config(out + ".dat", V, N)
    if noise:
        res["noise"] = np.fromfile(out + ".noise", dtype=np.float64).reshape(steps, V * 4 * 8)
    if wl2x2:  # WL2x2 (nspt.cc:1118-1124): Re Tr /(18V) of ptU[1], ptU[3], ...
        res["wl2x2"] = np.atleast_1d(np.loadtxt(out + ".wl2x2"))
    return res
