"""Python binding of the B200-native checkerboard SU(2) sweep (libqcd2d.so).

The library is C/CUDA behind the C ABI in include/qcd2d.h; this module only
wraps that ABI with ctypes so that tests and the benchmark can drive it.  It
loads the in-tree ``libqcd2d.so`` and raises if it is missing: there is no
Python or CPU fallback for any operation.

Mapping to the reference (fezquerro/QCD_2d_GPU):

=========================  ====================================================
``Lattice(...)``           struct lattice + setup_kernel (lattice_setup.h:2-21)
``init_cold/init_hot``     id_init2 / rand_init2 / rand_init2_pcc
``sweep(n)``               mc_up_per / mc_up_pcc / mc_up_pmc, n times
``overrelax(n)``           mc_up_per(..., update=1)
``normalize()``            normalize (lattice_setup.h:202-207)
``measure()``              en_av<PMC> (observables.h:99-141)
``store/load_config``      save_conf / read_conf layout (output.h:77-94)
``accept_counts()``        the accept array read by mean_lattice
=========================  ====================================================
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libqcd2d.so")

METROPOLIS, HEATBATH = 0, 1
PERIODIC, PCC, PMC = 0, 1, 2
FP64, FP32 = 0, 1
SCHED_AUTO, SCHED_PHASES, SCHED_WAVEFRONT, SCHED_PAIRS = 0, 1, 2, 3
_SCHED_NAME = {SCHED_PHASES: "phases", SCHED_WAVEFRONT: "wavefront", SCHED_PAIRS: "pairs"}

_BC = {"periodic": PERIODIC, "per": PERIODIC, "pcc": PCC, "pmc": PMC}
_ALGO = {"metropolis": METROPOLIS, "metro": METROPOLIS, "heatbath": HEATBATH, "hb": HEATBATH}
_PREC = {"fp64": FP64, "fp32": FP32}

QCD_OK = 0
_STATUS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "out of device memory",
    -4: "links not unitary",
    -5: "device wait timed out",
    -6: "configuration I/O error",
    -7: "unsupported combination",
}


class QcdError(RuntimeError):
    """A qcd_* call returned a non-zero status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{_STATUS.get(status, 'error')} ({status}): {message}")
        self.status = status


class Params(ctypes.Structure):
    """qcd_params (include/qcd2d.h)."""

    _fields_ = [
        ("lt", ctypes.c_int),
        ("lx", ctypes.c_int),
        ("ly", ctypes.c_int),
        ("beta", ctypes.c_float),
        ("epsilon", ctypes.c_float),
        ("upd", ctypes.c_int),
        ("algo", ctypes.c_int),
        ("boundary", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("n_or", ctypes.c_int),
        ("renorm_every", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
    ]


class Tuning(ctypes.Structure):
    """qcd_tuning (include/qcd2d.h)."""

    _fields_ = [
        ("schedule", ctypes.c_int),
        ("chunk_sites", ctypes.c_int),
        ("passes_per_launch", ctypes.c_int),
        ("fronts", ctypes.c_int),
        ("ms_per_sweep", ctypes.c_double),
    ]


class Replica(ctypes.Structure):
    """qcd_replica (include/qcd2d.h)."""

    _fields_ = [
        ("lt", ctypes.c_int),
        ("lx", ctypes.c_int),
        ("ly", ctypes.c_int),
        ("beta", ctypes.c_float),
        ("boundary", ctypes.c_int),
        ("hot", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
        ("stream_offset", ctypes.c_longlong),
    ]


TAPE_DTYPE = np.dtype(
    [
        ("ud", "<f8"),
        ("uf", "<f4"),
        ("log_uf", "<f4"),
        ("cospi_2uf", "<f4"),
        ("sc_sin", "<f4"),
        ("sc_cos", "<f4"),
        ("same_step", "<u4"),
    ]
)

_lib = None

# exported symbols of include/qcd2d.h: name -> (restype, argtypes)
_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_DP = ctypes.POINTER(ctypes.c_double)
_SIGS = {
    "qcd_params_default": (None, [ctypes.POINTER(Params), _I, _I, _I]),
    "qcd_create": (_I, [ctypes.POINTER(Params), ctypes.POINTER(_P)]),
    "qcd_destroy": (_I, [_P]),
    "qcd_set_stream": (_I, [_P, _P]),
    "qcd_get_stream": (_P, [_P]),
    "qcd_init_cold": (_I, [_P]),
    "qcd_init_hot": (_I, [_P]),
    "qcd_load_config": (_I, [_P, _P]),
    "qcd_store_config": (_I, [_P, _P]),
    "qcd_load_config_device": (_I, [_P, _P]),
    "qcd_store_config_device": (_I, [_P, _P]),
    "qcd_sweep": (_I, [_P, _I]),
    "qcd_overrelax": (_I, [_P, _I]),
    "qcd_normalize": (_I, [_P]),
    "qcd_measure": (_I, [_P, _DP, _DP]),
    "qcd_series_reserve": (_I, [_P, _I]),
    "qcd_measure_into_series": (_I, [_P, _I]),
    "qcd_series_read": (_I, [_P, _P, _P, _I]),
    "qcd_accept_counts": (_I, [_P, _P]),
    "qcd_accept_reset": (_I, [_P]),
    "qcd_check_unitarity": (_I, [_P, _D, _DP]),
    "qcd_volume": (ctypes.c_longlong, [_P]),
    "qcd_get_params": (_I, [_P, ctypes.POINTER(Params)]),
    "qcd_link_store": (_I, [_P, ctypes.POINTER(_P), ctypes.POINTER(ctypes.c_size_t)]),
    "qcd_last_error": (ctypes.c_char_p, [_P]),
    "qcd_status_string": (ctypes.c_char_p, [_I]),
    "qcd_rng_tape": (_I, [ctypes.c_ulonglong, ctypes.c_longlong, _I, _I, _P]),
    "qcd_measure_aos_noalloc": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "qcd_set_schedule": (_I, [_P, _I]),
    "qcd_get_schedule": (_I, [_P]),
    "qcd_set_pair_layout": (_I, [_P, _I]),
    "qcd_get_pair_layout": (_I, [_P]),
    "qcd_wave_plan": (_I, [_P, _P, _I, _P, _P, _P]),
    "qcd_wave_selftest_timeout": (_I, [_P]),
    "qcd_set_wave_tuning": (_I, [_P, _I, _I, _I]),
    "qcd_set_pair_tuning": (_I, [_P, _I]),
    "qcd_rng_words": (ctypes.c_longlong, [_P]),
    "qcd_philox4x32": (None, [_P, _P, _P]),
    "qcd_store_rng": (_I, [_P, _P]),
    "qcd_load_rng": (_I, [_P, _P]),
    "qcd_autotune": (_I, [_P, _I, ctypes.POINTER(Tuning)]),
    "qcd_batch_create": (_I, [_P, _I, ctypes.POINTER(Params), ctypes.POINTER(_P)]),
    "qcd_batch_destroy": (_I, [_P]),
    "qcd_batch_set_stream": (_I, [_P, _P]),
    "qcd_batch_init": (_I, [_P]),
    "qcd_batch_reserve": (_I, [_P, _I]),
    "qcd_batch_run": (_I, [_P, _I, _I, _I]),
    "qcd_batch_synchronize": (_I, [_P]),
    "qcd_batch_set_groups": (_I, [_P, ctypes.c_longlong]),
    "qcd_batch_groups": (_I, [_P]),
    "qcd_batch_set_lanes": (_I, [_P, _I]),
    "qcd_batch_autotune": (_I, [_P, _I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(ctypes.c_int), _DP]),
    "qcd_batch_measured": (_I, [_P]),
    "qcd_batch_series": (_I, [_P, _I, _P, _P, _I]),
    "qcd_batch_store_config": (_I, [_P, _I, _P]),
    "qcd_batch_sites": (ctypes.c_longlong, [_P]),
    "qcd_batch_last_error": (ctypes.c_char_p, [_P]),
    "qcd_stats_mean_variance": (_I, [_P, _I, _DP, _DP]),
    "qcd_stats_autocorrelation": (_I, [_P, _I, _I, _D, _D, _P]),
    "qcd_stats_binned": (_I, [_P, _I, _I, _DP, _DP]),
    "qcd_stats_tau_int": (_I, [_P, _I, _D, _DP, ctypes.POINTER(ctypes.c_int), _DP]),
}


def exported_symbols() -> list[str]:
    """Names the C ABI exports (the declarations of include/qcd2d.h)."""
    return sorted(_SIGS)


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load libqcd2d.so; raises if it has not been built."""
    global _lib
    if _lib is not None and path == LIB_PATH:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"{path} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
            "(there is no fallback implementation)"
        )
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path == LIB_PATH:
        _lib = lib
    return lib


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data)


class Lattice:
    """One lattice on the GPU (a qcd_lattice handle)."""

    def __init__(
        self,
        lt: int,
        lx: int,
        ly: int,
        beta: float,
        *,
        algo: str | int = "heatbath",
        boundary: str | int = "periodic",
        precision: str | int = "fp64",
        epsilon: float = 0.1,
        upd: int = 1,
        n_or: int = 0,
        renorm_every: int = 0,
        seed: int = 1234,
        lib: ctypes.CDLL | None = None,
    ):
        self._lib = lib or load_library()
        p = Params()
        self._lib.qcd_params_default(ctypes.byref(p), lt, lx, ly)
        p.beta = beta
        p.epsilon = epsilon
        p.upd = upd
        p.algo = _ALGO[algo] if isinstance(algo, str) else int(algo)
        p.boundary = _BC[boundary] if isinstance(boundary, str) else int(boundary)
        p.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
        p.n_or = n_or
        p.renorm_every = renorm_every
        p.seed = seed
        self.params = p
        h = ctypes.c_void_p()
        rc = self._lib.qcd_create(ctypes.byref(p), ctypes.byref(h))
        if rc != QCD_OK:
            raise QcdError(rc, f"qcd_create({lt}x{lx}x{ly})")
        self._h = h
        self.V = lt * lx * ly

    # -- plumbing ---------------------------------------------------------
    def _check(self, rc: int, what: str) -> None:
        if rc != QCD_OK:
            msg = self._lib.qcd_last_error(self._h)
            raise QcdError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.qcd_destroy(self._h)
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

    @property
    def handle(self) -> ctypes.c_void_p:
        return self._h

    def set_stream(self, stream_ptr: int | None) -> None:
        self._check(self._lib.qcd_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)), "set_stream")

    def set_schedule(self, mode: int | str) -> None:
        m = {"auto": SCHED_AUTO, "phases": SCHED_PHASES, "wavefront": SCHED_WAVEFRONT, "pairs": SCHED_PAIRS}.get(mode, mode)
        self._check(self._lib.qcd_set_schedule(self._h, int(m)), "set_schedule")

    def schedule(self) -> str:
        return _SCHED_NAME[self._lib.qcd_get_schedule(self._h)]

    def set_pair_layout(self, on: bool) -> None:
        """FP32, Lt % 4 == 0: allow (True, the default) or forbid the site-pair store."""
        self._check(self._lib.qcd_set_pair_layout(self._h, int(bool(on))), "set_pair_layout")

    def pair_layout(self) -> bool:
        return self._lib.qcd_get_pair_layout(self._h) == 1

    def set_wave_tuning(self, chunk_sites: int = 0, passes_per_launch: int = 0, fronts: int = 0) -> None:
        self._check(self._lib.qcd_set_wave_tuning(self._h, chunk_sites, passes_per_launch, fronts),
                    "set_wave_tuning")

    def set_pair_tuning(self, slices_per_cta: int = 0) -> None:
        self._check(self._lib.qcd_set_pair_tuning(self._h, slices_per_cta), "set_pair_tuning")

    def autotune(self, sweeps_per_trial: int = 0) -> dict:
        """Pick the fastest schedule for this lattice (state is preserved)."""
        t = Tuning()
        self._check(self._lib.qcd_autotune(self._h, sweeps_per_trial, ctypes.byref(t)), "autotune")
        return {"schedule": _SCHED_NAME[t.schedule],
                "chunk_sites": t.chunk_sites, "passes_per_launch": t.passes_per_launch, "fronts": t.fronts,
                "ms_per_sweep": t.ms_per_sweep}

    def wave_selftest_timeout(self) -> int:
        """Run the bounded-wait self-test; returns the status (expected -5)."""
        return self._lib.qcd_wave_selftest_timeout(self._h)

    # -- the path ---------------------------------------------------------
    def init_cold(self) -> None:
        self._check(self._lib.qcd_init_cold(self._h), "init_cold")

    def init_hot(self) -> None:
        self._check(self._lib.qcd_init_hot(self._h), "init_hot")

    def sweep(self, n: int = 1) -> None:
        self._check(self._lib.qcd_sweep(self._h, n), "sweep")

    def overrelax(self, n: int = 1) -> None:
        self._check(self._lib.qcd_overrelax(self._h, n), "overrelax")

    def normalize(self) -> None:
        self._check(self._lib.qcd_normalize(self._h), "normalize")

    def measure(self) -> tuple[float, float]:
        e, p = ctypes.c_double(), ctypes.c_double()
        self._check(self._lib.qcd_measure(self._h, ctypes.byref(e), ctypes.byref(p)), "measure")
        return e.value, p.value

    def series_reserve(self, n: int) -> None:
        self._check(self._lib.qcd_series_reserve(self._h, n), "series_reserve")

    def measure_into_series(self, i: int) -> None:
        self._check(self._lib.qcd_measure_into_series(self._h, i), "measure_into_series")

    def series_read(self, n: int) -> tuple[np.ndarray, np.ndarray]:
        e = np.zeros(n)
        p = np.zeros(n)
        self._check(self._lib.qcd_series_read(self._h, _ptr(e), _ptr(p), n), "series_read")
        return e, p

    def store_config(self) -> np.ndarray:
        out = np.empty(self.V * 12, dtype=np.float64)
        self._check(self._lib.qcd_store_config(self._h, _ptr(out)), "store_config")
        return out

    def load_config(self, aos: np.ndarray) -> None:
        a = np.ascontiguousarray(aos, dtype=np.float64)
        if a.size != self.V * 12:
            raise ValueError(f"configuration has {a.size} doubles, expected {self.V * 12}")
        self._check(self._lib.qcd_load_config(self._h, _ptr(a)), "load_config")

    def store_rng(self) -> np.ndarray:
        """The generator checkpoint (MRG32k3a words + the FP32 draws' counter and key)."""
        out = np.empty(self._lib.qcd_rng_words(self._h), dtype=np.uint32)
        self._check(self._lib.qcd_store_rng(self._h, _ptr(out)), "store_rng")
        return out

    def load_rng(self, words: np.ndarray) -> None:
        a = np.ascontiguousarray(words, dtype=np.uint32)
        if a.size != self._lib.qcd_rng_words(self._h):
            raise ValueError("generator state has the wrong size")
        self._check(self._lib.qcd_load_rng(self._h, _ptr(a)), "load_rng")

    def accept_counts(self) -> np.ndarray:
        out = np.empty(self.V, dtype=np.int32)
        self._check(self._lib.qcd_accept_counts(self._h, _ptr(out)), "accept_counts")
        return out

    def accept_reset(self) -> None:
        self._check(self._lib.qcd_accept_reset(self._h), "accept_reset")

    def check_unitarity(self, tol: float = 1e-10) -> float:
        m = ctypes.c_double()
        self._check(self._lib.qcd_check_unitarity(self._h, tol, ctypes.byref(m)), "check_unitarity")
        return m.value

    def link_store(self) -> tuple[int, int]:
        p = ctypes.c_void_p()
        n = ctypes.c_size_t()
        self._check(self._lib.qcd_link_store(self._h, ctypes.byref(p), ctypes.byref(n)), "link_store")
        return p.value or 0, n.value


class Batch:
    """Many replicas advanced by shared launches (a qcd_batch handle).

    replicas: sequence of dicts with keys lt, lx, ly, beta, boundary, hot, seed,
    stream_offset (defaults: periodic, cold, seed 1234, offset 0).
    """

    def __init__(self, replicas, *, algo="heatbath", precision="fp32", epsilon=0.1, upd=1, n_or=0,
                 renorm_every=0, lib: ctypes.CDLL | None = None):
        self._lib = lib or load_library()
        arr = (Replica * len(replicas))()
        for i, r in enumerate(replicas):
            bc = r.get("boundary", PERIODIC)
            arr[i] = Replica(r["lt"], r["lx"], r["ly"], r["beta"], _BC[bc] if isinstance(bc, str) else int(bc),
                             int(r.get("hot", 0)), int(r.get("seed", 1234)), int(r.get("stream_offset", 0)))
        p = Params()
        self._lib.qcd_params_default(ctypes.byref(p), 2, 2, 2)
        p.algo = _ALGO[algo] if isinstance(algo, str) else int(algo)
        p.precision = _PREC[precision] if isinstance(precision, str) else int(precision)
        p.epsilon = epsilon
        p.upd = upd
        p.n_or = n_or
        p.renorm_every = renorm_every
        h = ctypes.c_void_p()
        rc = self._lib.qcd_batch_create(arr, len(replicas), ctypes.byref(p), ctypes.byref(h))
        if rc != QCD_OK:
            raise QcdError(rc, "qcd_batch_create")
        self._h = h
        self.replicas = [dict(r) for r in replicas]
        self.n = len(replicas)

    def _check(self, rc, what):
        if rc != QCD_OK:
            msg = self._lib.qcd_batch_last_error(self._h)
            raise QcdError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.qcd_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr):
        self._check(self._lib.qcd_batch_set_stream(self._h, ctypes.c_void_p(stream_ptr or 0)), "set_stream")

    def init(self):
        self._check(self._lib.qcd_batch_init(self._h), "init")

    def reserve(self, capacity):
        self._check(self._lib.qcd_batch_reserve(self._h, capacity), "reserve")

    def run(self, sweeps, measure_every=1, graph=True):
        self._check(self._lib.qcd_batch_run(self._h, sweeps, measure_every, int(graph)), "run")

    def synchronize(self):
        self._check(self._lib.qcd_batch_synchronize(self._h), "synchronize")

    def set_groups(self, bytes_per_group):
        """Sweep the replicas in groups of at most this many bytes of links (0: one group)."""
        self._check(self._lib.qcd_batch_set_groups(self._h, int(bytes_per_group)), "set_groups")

    def groups(self):
        return self._lib.qcd_batch_groups(self._h)

    def set_lanes(self, lanes):
        """Run groups on this many streams at the same time (1..4)."""
        self._check(self._lib.qcd_batch_set_lanes(self._h, int(lanes)), "set_lanes")

    def autotune(self, sweeps_per_trial=0):
        """Pick the fastest grouping and lanes (the batch's state is preserved)."""
        nb, nl, ms = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_double()
        self._check(self._lib.qcd_batch_autotune(self._h, sweeps_per_trial, ctypes.byref(nb), ctypes.byref(nl),
                                                 ctypes.byref(ms)), "autotune")
        return {"bytes_per_group": nb.value, "groups": self.groups(), "lanes": nl.value, "ms_per_sweep": ms.value}

    def measured(self):
        k = self._lib.qcd_batch_measured(self._h)
        if k < 0:
            self._check(k, "measured")
        return k

    def series(self, replica, n=None):
        n = self.measured() if n is None else n
        e, p = np.zeros(n), np.zeros(n)
        self._check(self._lib.qcd_batch_series(self._h, replica, _ptr(e), _ptr(p), n), "series")
        return e, p

    def store_config(self, replica):
        r = self.replicas[replica]
        out = np.empty(r["lt"] * r["lx"] * r["ly"] * 12)
        self._check(self._lib.qcd_batch_store_config(self._h, replica, _ptr(out)), "store_config")
        return out

    @property
    def sites(self):
        return self._lib.qcd_batch_sites(self._h)


def rng_tape(seed: int, first: int, n_streams: int, n_draws: int, lib: ctypes.CDLL | None = None) -> np.ndarray:
    """First draws of MRG32k3a streams curand_init(seed, id, 0), see qcd_rng_tape."""
    lib = lib or load_library()
    out = np.zeros(n_streams * n_draws, dtype=TAPE_DTYPE)
    rc = lib.qcd_rng_tape(seed, first, n_streams, n_draws, _ptr(out))
    if rc != QCD_OK:
        raise QcdError(rc, "qcd_rng_tape")
    return out.reshape(n_streams, n_draws)


def philox4x32(ctr, key, lib: ctypes.CDLL | None = None) -> np.ndarray:
    """One Philox4x32-10 block (the FP32 sweep's generator), computed on the host."""
    lib = lib or load_library()
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    if c.size != 4 or k.size != 2:
        raise ValueError("ctr has 4 words, key 2")
    out = np.empty(4, dtype=np.uint32)
    lib.qcd_philox4x32(_ptr(c), _ptr(k), _ptr(out))
    return out


def wave_plan(mu, par, lib: ctypes.CDLL | None = None):
    """Host-side wavefront plan (seam, start, need[3][P]) of a phase program."""
    lib = lib or load_library()
    m = np.ascontiguousarray(mu, dtype=np.int32)
    p = np.ascontiguousarray(par, dtype=np.int32)
    n = len(m)
    seam = np.zeros(n, np.int32)
    start = np.zeros(n, np.int32)
    need = np.zeros(3 * n, np.int32)
    rc = lib.qcd_wave_plan(_ptr(m), _ptr(p), n, _ptr(seam), _ptr(start), _ptr(need))
    if rc != QCD_OK:
        raise QcdError(rc, "qcd_wave_plan")
    return seam, start, need.reshape(3, n)


# -- statistics of measurement series (host code of the library) ------------
def _series(x):
    return np.ascontiguousarray(x, dtype=np.float64)


def mean_variance(x):
    """The reference's naive mean and population variance (statistics.h:30-39)."""
    lib = load_library()
    a = _series(x)
    m, v = ctypes.c_double(), ctypes.c_double()
    if lib.qcd_stats_mean_variance(_ptr(a), len(a), ctypes.byref(m), ctypes.byref(v)):
        raise QcdError(-1, "mean_variance")
    return m.value, v.value


def autocorrelation(x, w, mean, var):
    """The reference's normalised autocorrelation of lags 1..w (statistics.h:41-51)."""
    lib = load_library()
    a = _series(x)
    out = np.zeros(w)
    if lib.qcd_stats_autocorrelation(_ptr(a), len(a), w, mean, var, _ptr(out)):
        raise QcdError(-1, "autocorrelation")
    return out


def binned(x, bin_size):
    lib = load_library()
    a = _series(x)
    m, e = ctypes.c_double(), ctypes.c_double()
    if lib.qcd_stats_binned(_ptr(a), len(a), bin_size, ctypes.byref(m), ctypes.byref(e)):
        raise QcdError(-1, "binned")
    return m.value, e.value


def tau_int(x, c=6.0):
    """Integrated autocorrelation time, Madras-Sokal window: (tau, W, dtau)."""
    lib = load_library()
    a = _series(x)
    t, d = ctypes.c_double(), ctypes.c_double()
    w = ctypes.c_int()
    if lib.qcd_stats_tau_int(_ptr(a), len(a), c, ctypes.byref(t), ctypes.byref(w), ctypes.byref(d)):
        raise QcdError(-1, "tau_int")
    return t.value, w.value, d.value
