"""prlgt2020_b200 -- B200 NSPT Langevin engine behind the reference's API.

Host-side mirror of the PRlgt2020 hot path (nspt.h:55-94): the names and the
argument meaning follow the reference, the work runs in the CUDA engine
(libnspt_b200.so, C ABI in include/nspt_b200.h).  There is no CPU fallback:
without the built library or a CUDA device every compute call raises.

    eng = NsptEngine((4, 4, 4, 4), N=8, zero_modes=True)
    eng.cold_start()
    obs = eng.gauge_wilson(dt=0.01)        # one Jacobi sweep
    eng.zero_modes_subtraction()
    plaq = eng.plaquette_measure()

Field data on the host use the reference's AoS layout (ptGluon_fld,
QCDenvNODEpt_test.h:331-338): shape (V, 4, 2 + 18*allocORD) float64 =
site (t fastest), mu, {flag re/im, order 1 [3x3 row major re/im], ...}.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import (NSPT_GF_FA, NSPT_GF_LOCAL, NSPT_TWIST_T, NSPT_TWIST_Y, NSPT_TWIST_Z, NSPT_ZEROMODE,
                   NsptError, build as build_library, check, load as load_library)

__all__ = ["NsptEngine", "ptGluon_fld", "SweepObservables", "build", "series_len",
           "NsptError", "fp64_peak_tflops", "NsptBatch"]

_DIRS = {"x": 0, "y": 1, "z": 2, "t": 3}


def build(verbose: bool = False) -> str:
    return build_library(verbose)


def series_len(allocORD: int) -> int:
    """Doubles in one ptSU3 (QCDpt.h:47-48): flag + allocORD 3x3 complex."""
    return 2 + 18 * int(allocORD)


def _dp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@dataclass
class SweepObservables:
    """Per-sweep output of gauge_wilson (nspt.cc:570-597)."""
    plaq: np.ndarray  # (N+1, 2): Tr(U * staples) / 72V per order (re, im)
    norm: np.ndarray  # (N,):     Re Tr(U_k U_k^dag) / 12V
    tru: np.ndarray   # (4, N, 2): Tr U_k / 3V per mu


class ptGluon_fld:
    """Host gauge field in the reference's layout and file format.

    Mirrors ptGluon_fld (QCDenvNODEpt_test.h:331-426): `links` is
    (V, 4, 2 + 18*allocORD) float64; save/load use the binary format of
    ptGluon_fld::save(char*, Cplx*) -- the field then (allocORD+1) complex
    plaquette values -- and load checks the byte count like io::load.
    """

    def __init__(self, L, allocORD: int, links: np.ndarray | None = None):
        self.L = tuple(int(x) for x in L)
        self.allocORD = int(allocORD)
        self.V = int(np.prod(self.L))
        shape = (self.V, 4, series_len(self.allocORD))
        if links is None:
            self.links = np.zeros(shape)
            self.links[:, :, 0] = 1.0  # cold start: flag = VACUUM = 1
        else:
            self.links = np.ascontiguousarray(links, dtype=np.float64).reshape(shape)

    def id(self):
        """Cold configuration (ptSU3::id, QCDpt.h:69-72)."""
        self.links[...] = 0.0
        self.links[:, :, 0] = 1.0

    def save(self, path: str, plaquette: np.ndarray | None = None):
        trailer = np.zeros((self.allocORD + 1, 2))
        if plaquette is not None:
            p = np.asarray(plaquette, dtype=np.float64).reshape(-1, 2)
            trailer[: p.shape[0]] = p
        with open(path, "wb") as f:
            self.links.tofile(f)
            trailer.tofile(f)

    @classmethod
    def load(cls, path: str, L, allocORD: int):
        V = int(np.prod(L))
        n = V * 4 * series_len(allocORD)
        want = 8 * (n + 2 * (allocORD + 1))
        size = os.path.getsize(path)
        if size != want:
            raise IOError("%s: %d bytes, expected %d for L=%s allocORD=%d"
                          % (path, size, want, tuple(L), allocORD))
        raw = np.fromfile(path, dtype=np.float64)
        fld = cls(L, allocORD, raw[:n])
        fld.plaquette_trailer = raw[n:].reshape(allocORD + 1, 2)
        return fld


def fp64_peak_tflops() -> float:
    """Measured FP64 FMA throughput of the current device (TFLOP/s)."""
    out = ctypes.c_double(0.0)
    check(load_library().nspt_measure_fp64_peak(ctypes.byref(out)), "nspt_measure_fp64_peak")
    return out.value


class NsptEngine:
    """One lattice on the current CUDA device (a context of the C ABI).

    L           lattice extents (x, y, z, t), lattice.h:139
    N           perturbative order PTORD (device allocORD == N)
    twist       twisted directions, subset of "yzt" (choices.h:45-50)
    zero_modes  REMOVE_GLUON_ZEROMOM (choices.h:82-84), periodic only
    fa          Fourier-accelerated Landau gauge fixing (nspt.cc:866-948)
    alpha       act_pars.alpha as in Quench.cfg (negative in the reference
                config; FA multiplies by -alpha/p^2)
    local_gf    local stochastic gauge fixing (nspt.cc:660-862)
    action      "wil", or an improved action "tlsym", "iwa", "dbw2"
                (Quenched.cc:311-322)
    precision   "fp64", or "ff": the sweep's Cauchy products in compensated
                float-float with a per-order scale (Wilson action)
    """

    def __init__(self, L, N: int, twist: str = "", zero_modes: bool = False, fa: bool = False,
                 alpha: float = 0.0, local_gf: bool = False, action: str = "wil",
                 precision: str = "fp64", update: str = "jacobi"):
        """update: "jacobi" (F = exp(W1) U, then U = F) or "onthefly", the
        reference's default UPDATE_ONTHEFLY: links updated in place in the
        order of the OpenMP thread grid (set_gf_grid)."""
        lib = load_library()
        self.L = tuple(int(x) for x in L)
        if len(self.L) != 4:
            raise ValueError("L must have 4 extents")
        self.N = int(N)
        self.V = int(np.prod(self.L))
        flags = 0
        for d in twist:
            flags |= {"y": NSPT_TWIST_Y, "z": NSPT_TWIST_Z, "t": NSPT_TWIST_T}[d]
        if zero_modes:
            flags |= NSPT_ZEROMODE
        if fa:
            flags |= NSPT_GF_FA
        if local_gf:
            flags |= NSPT_GF_LOCAL
        flags |= {"wil": 0, "tlsym": _lib.NSPT_ACTION_TLSYM, "iwa": _lib.NSPT_ACTION_IWA,
                  "dbw2": _lib.NSPT_ACTION_DBW2}[action]
        flags |= {"fp64": 0, "ff": _lib.NSPT_PRECISION_FF}[precision]
        flags |= {"jacobi": 0, "onthefly": _lib.NSPT_UPDATE_ONTHEFLY}[update]
        self.flags = flags
        self.alpha = float(alpha)
        arr = (ctypes.c_int * 4)(*self.L)
        h = ctypes.c_void_p()
        check(lib.nspt_create(arr, self.N, flags, self.alpha, ctypes.byref(h)), "nspt_create")
        self._h = h
        self._owned = True

    @classmethod
    def _view(cls, h, L, N, flags, alpha):
        """A context owned elsewhere (a replica of an NsptBatch)."""
        e = cls.__new__(cls)
        e.L, e.N, e.V = tuple(L), int(N), int(np.prod(L))
        e.flags, e.alpha = flags, float(alpha)
        e._h, e._owned = h, False
        return e

    # -- lifetime -------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            if getattr(self, "_owned", True):
                load_library().nspt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, code, where):
        check(code, where, self._h)

    @property
    def device_bytes(self) -> int:
        return int(load_library().nspt_device_bytes(self._h))

    # -- field transfer -------------------------------------------------
    def cold_start(self):
        self._check(load_library().nspt_cold_start(self._h), "nspt_cold_start")

    def upload(self, links, allocORD: int | None = None):
        """Copy a host field (reference AoS layout) to the device."""
        if isinstance(links, ptGluon_fld):
            allocORD, links = links.allocORD, links.links
        A = self.N if allocORD is None else int(allocORD)
        a = np.ascontiguousarray(links, dtype=np.float64)
        if a.size != self.V * 4 * series_len(A):
            raise ValueError("field has %d doubles, expected %d" % (a.size, self.V * 4 * series_len(A)))
        self._check(load_library().nspt_upload_links(self._h, a.ctypes.data, A), "nspt_upload_links")

    def download(self, allocORD: int | None = None) -> np.ndarray:
        A = self.N if allocORD is None else int(allocORD)
        out = np.empty((self.V, 4, series_len(A)))
        self._check(load_library().nspt_download_links(self._h, out.ctypes.data, A),
                    "nspt_download_links")
        return out

    def save(self, path: str, allocORD: int | None = None):
        A = self.N if allocORD is None else int(allocORD)
        self._check(load_library().nspt_save_config(self._h, path.encode(), A), "nspt_save_config")

    def load(self, path: str, allocORD: int | None = None) -> np.ndarray:
        A = self.N if allocORD is None else int(allocORD)
        trailer = np.zeros((A + 1, 2))
        self._check(load_library().nspt_load_config(self._h, path.encode(), A, _dp(trailer)),
                    "nspt_load_config")
        return trailer

    def loadlowerorder(self, path: str, loworder: int) -> np.ndarray:
        """ptGluon_fld::loadlowerorder (QCDenvNODEpt_test.h:376-426): start
        from a file saved with loworder <= N orders; the orders above are
        zero and every link is unitarised, U = exp(reH(log U)).  Returns the
        file's loworder + 1 plaquette values."""
        lo = int(loworder)
        trailer = np.zeros((max(lo, 0) + 1, 2))
        self._check(load_library().nspt_load_lower_order(self._h, path.encode(), lo, _dp(trailer)),
                    "nspt_load_lower_order")
        return trailer

    # -- noise ------------------------------------------------------------
    def set_noise(self, eta: np.ndarray):
        """Inject the 8 Gaussians per link SU3rand draws (V, 4, 8) for the next sweep."""
        a = np.ascontiguousarray(eta, dtype=np.float64)
        if a.size != self.V * 32:
            raise ValueError("noise needs V*4*8 values")
        self._check(load_library().nspt_set_noise(self._h, _dp(a)), "nspt_set_noise")

    def seed(self, seed: int, counter: int = 0):
        self._check(load_library().nspt_seed(self._h, int(seed), int(counter)), "nspt_seed")

    def rng_state(self):
        """(seed, counter) of the device noise generator: with seed(seed,
        counter) a context loaded from a saved configuration continues the
        same noise stream."""
        s, c = ctypes.c_uint64(0), ctypes.c_uint64(0)
        self._check(load_library().nspt_get_seed(self._h, ctypes.byref(s), ctypes.byref(c)),
                    "nspt_get_seed")
        return int(s.value), int(c.value)

    # -- the reference's hot-path functions (nspt.h:55-94) -----------------
    def gauge_wilson(self, dt: float) -> SweepObservables:
        """One Jacobi Langevin sweep (nspt.cc:258-600); dt = tau_g of Quench.cfg."""
        self._check(load_library().nspt_gauge_wilson(self._h, float(dt)), "nspt_gauge_wilson")
        return self.observables()

    def zero_modes_subtraction(self):
        self._check(load_library().nspt_zero_modes_subtraction(self._h),
                    "nspt_zero_modes_subtraction")

    def FAstochastic_gauge_fixing(self, alpha: float | None = None):
        a = self.alpha if alpha is None else float(alpha)
        self._check(load_library().nspt_fa_gauge_fixing(self._h, a), "nspt_fa_gauge_fixing")

    def stochastic_gauge_fixing(self, alpha: float | None = None):
        """Local stochastic gauge fixing (nspt.cc:660-862) with the thread grid
        set by set_gf_grid (default: the finest the reference accepts)."""
        a = self.alpha if alpha is None else float(alpha)
        self._check(load_library().nspt_local_gauge_fixing(self._h, a),
                    "nspt_local_gauge_fixing")

    def set_gf_grid(self, grid):
        """The reference's OpenMP thread grid (ntt, ntx, nty, ntz), which fixes
        the order of the local gauge fixing (choices.h:124-128)."""
        g = (ctypes.c_int * 4)(*[int(x) for x in grid])
        self._check(load_library().nspt_set_gf_grid(self._h, g), "nspt_set_gf_grid")

    def set_local_gf_form(self, form: str):
        """Kernel of the local gauge fixing: "group" (one 9-lane link group
        per reference thread), "team" (a warp of three groups per thread) or
        "auto" (the team form when the barrier step's teams all fit on the
        GPU at once).  Both forms give the same links."""
        code = {"auto": 0, "group": 1, "team": 2}.get(form)
        if code is None:
            raise ValueError(f"local gauge fixing form {form!r}: auto, group or team")
        self._check(load_library().nspt_set_local_gf_form(self._h, code),
                    "nspt_set_local_gf_form")

    def twist_boundary(self):
        """twist_boundary (nspt.cc:163-255).  Twists are applied inside every
        neighbour read, so this only ends what an on-the-fly sweep on twisted
        boundaries leaves: reads across a twisted face seeing the step's start
        field, as the reference's copy sites do.  NsptEvolve calls it at the
        end of every step."""
        self._check(load_library().nspt_twist_boundary(self._h), "nspt_twist_boundary")

    def NsptEvolve(self, dt: float, beat: int = 1, gf_every: int = 1):
        """Beat Langevin steps (nspt.cc:953-1039)."""
        self._check(load_library().nspt_step(self._h, float(dt), int(beat), int(gf_every)),
                    "nspt_step")

    def plaquette_measure(self) -> np.ndarray:
        out = np.zeros((self.N + 1, 2))
        self._check(load_library().nspt_plaquette_measure(self._h, _dp(out)),
                    "nspt_plaquette_measure")
        return out

    def rect_observables(self) -> np.ndarray:
        """Improved actions: rectangle traces w2 of the last sweep (/72V)."""
        out = np.zeros((self.N + 1, 2))
        self._check(load_library().nspt_rect_observables(self._h, _dp(out)),
                    "nspt_rect_observables")
        return out

    def set_timeout(self, seconds: float = 0.0):
        """Wait at most `seconds` for a call's device work (0: no limit);
        past it the call raises NsptError with code NSPT_ERR_TIMEOUT while
        the work runs on, and the next call waits for it first."""
        self._check(load_library().nspt_set_timeout(self._h, float(seconds)), "nspt_set_timeout")

    def set_ff_scale(self, e=None):
        """Float-float products: fixed per-order scale exponent e (order k
        multiplied by 2^(e k) before the split), or None to fit it to the
        field every sweep (the default)."""
        lib = load_library()
        if e is None:
            self._check(lib.nspt_set_ff_scale(self._h, 1, 0), "nspt_set_ff_scale")
        else:
            self._check(lib.nspt_set_ff_scale(self._h, 0, int(e)), "nspt_set_ff_scale")

    def ff_scale(self) -> int:
        """Scale exponent the last float-float sweep used."""
        e = ctypes.c_int(0)
        self._check(load_library().nspt_get_ff_scale(self._h, ctypes.byref(e)),
                    "nspt_get_ff_scale")
        return e.value

    def WL2x2(self) -> np.ndarray:
        """WL2x2 of nspt.cc:1064-1140: [N+1, 2] trace of the 2x2 loop per
        order, /(18V); the reference prints the real parts of orders 2, 4, ..."""
        out = np.zeros((self.N + 1, 2))
        self._check(load_library().nspt_wl2x2(self._h, _dp(out)), "nspt_wl2x2")
        return out

    def ComputeLoops(self) -> np.ndarray:
        """Wilson loops of nspt.cc:1148-1312: [4, N+1, 2] traces of the 1x2,
        2x2, 2x4 and 4x4 loops, normalised as the reference prints them."""
        out = np.zeros((4, self.N + 1, 2))
        self._check(load_library().nspt_wilson_loops(self._h, _dp(out)), "nspt_wilson_loops")
        return out

    def observables(self) -> SweepObservables:
        N = self.N
        plaq = np.zeros((N + 1, 2))
        norm = np.zeros(N)
        tru = np.zeros((4, N, 2))
        self._check(load_library().nspt_observables(self._h, _dp(plaq), _dp(norm), _dp(tru)),
                    "nspt_observables")
        return SweepObservables(plaq, norm, tru)

    def last_step_ms(self) -> float:
        """Device time of the last step / sweep / zero-mode / gauge-fixing / loops call."""
        return float(load_library().nspt_last_step_ms(self._h))

    def last_kernel_ms(self) -> float:
        """Average sweep-kernel launch of the last NsptEvolve / gauge_wilson."""
        return float(load_library().nspt_last_kernel_ms(self._h))


class NsptBatch:
    """Independent replicas advanced together in one CUDA graph
    (nspt_batch_* in include/nspt_b200.h): replica r has extents L[r], time
    step dt[r] and noise seed seeds[r]; all share N, the flags and alpha."""

    def __init__(self, L, N: int, dt, seeds, zero_modes: bool = False, fa: bool = False,
                 local_gf: bool = False, alpha: float = 0.0, twist: str = "",
                 update: str = "jacobi"):
        lib = load_library()
        L = [tuple(int(x) for x in l) for l in L]
        n = len(L)
        if len(dt) != n or len(seeds) != n:
            raise ValueError("L, dt and seeds need one entry per replica")
        flags = 0
        for d in twist:
            flags |= {"y": NSPT_TWIST_Y, "z": NSPT_TWIST_Z, "t": NSPT_TWIST_T}[d]
        flags |= (NSPT_ZEROMODE if zero_modes else 0) | (NSPT_GF_FA if fa else 0)
        flags |= NSPT_GF_LOCAL if local_gf else 0
        flags |= {"jacobi": 0, "onthefly": _lib.NSPT_UPDATE_ONTHEFLY}[update]
        self.N, self.n = int(N), n
        Ls = (ctypes.c_int * (4 * n))(*[x for l in L for x in l])
        dts = (ctypes.c_double * n)(*[float(x) for x in dt])
        sds = (ctypes.c_uint64 * n)(*[int(x) for x in seeds])
        h = ctypes.c_void_p()
        check(lib.nspt_batch_create(n, Ls, self.N, flags, float(alpha), dts, sds, ctypes.byref(h)),
              "nspt_batch_create")
        self._h = h
        self.replicas = []
        for r in range(n):
            c = ctypes.c_void_p()
            check(lib.nspt_batch_context(h, r, ctypes.byref(c)), "nspt_batch_context")
            self.replicas.append(NsptEngine._view(c, L[r], self.N, flags, alpha))

    def step(self, nsteps: int, gf_every: int = 1):
        check(load_library().nspt_batch_step(self._h, int(nsteps), int(gf_every)), "nspt_batch_step")

    def last_step_ms(self) -> float:
        return float(load_library().nspt_batch_last_step_ms(self._h))

    def plaquettes(self) -> np.ndarray:
        out = np.zeros((self.n, self.N + 1, 2))
        check(load_library().nspt_batch_observables(self._h, _dp(out)), "nspt_batch_observables")
        return out

    def tune(self, gf_every: int = 1) -> int:
        w = ctypes.c_int()
        check(load_library().nspt_batch_tune(self._h, int(gf_every), ctypes.byref(w)),
              "nspt_batch_tune")
        return w.value

    def tune_shape(self, gf_every: int = 1):
        """Autotune the tile shape: (warps per CTA, orders per lane and pass,
        table of step times in ms [orders 8 / 4][warps 1..8], 0 = not tried)."""
        w, mo = ctypes.c_int(), ctypes.c_int()
        table = (ctypes.c_float * 16)()
        check(load_library().nspt_batch_tune_shape(self._h, int(gf_every), ctypes.byref(w),
                                                   ctypes.byref(mo), table),
              "nspt_batch_tune_shape")
        return w.value, mo.value, np.array(list(table), dtype=np.float64).reshape(2, 8)

    def close(self):
        if getattr(self, "_h", None):
            for e in self.replicas:
                e._h = None
            load_library().nspt_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
