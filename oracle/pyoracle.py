"""ctypes binding of the CPU oracle (liboracle.so) — TEST INFRASTRUCTURE.

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module; the product (qcd_2d_gpu_b200) never does.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_HARNESS = os.path.join(HERE, "_ref", "ref_harness")

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


class OraParams(ctypes.Structure):
    _fields_ = [
        ("lt", ctypes.c_int),
        ("lx", ctypes.c_int),
        ("ly", ctypes.c_int),
        ("beta", ctypes.c_float),
        ("epsilon", ctypes.c_float),
        ("upd", ctypes.c_int),
        ("algo", ctypes.c_int),
        ("boundary", ctypes.c_int),
        ("seed", ctypes.c_ulonglong),
    ]


_lib = None


def build() -> None:
    """Compile liboracle.so with the recipe in oracle/Makefile."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB):
        build()
    lib = ctypes.CDLL(LIB)
    P = ctypes.c_void_p
    lib.ora_create.restype = P
    lib.ora_create.argtypes = [ctypes.POINTER(OraParams), P, ctypes.c_int, ctypes.c_int]
    lib.ora_destroy.argtypes = [P]
    for n in ("ora_init_cold", "ora_init_hot", "ora_normalize"):
        getattr(lib, n).argtypes = [P]
        getattr(lib, n).restype = ctypes.c_int
    lib.ora_load.argtypes = [P, P]
    lib.ora_phase.argtypes = [P, ctypes.c_int, ctypes.c_int]
    lib.ora_sweep.argtypes = [P, ctypes.c_int]
    lib.ora_overrelax.argtypes = [P, ctypes.c_int]
    lib.ora_measure.argtypes = [P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]
    lib.ora_field.restype = ctypes.POINTER(ctypes.c_double)
    lib.ora_field.argtypes = [P]
    lib.ora_accept.restype = ctypes.POINTER(ctypes.c_int)
    lib.ora_accept.argtypes = [P]
    lib.ora_volume.restype = ctypes.c_longlong
    lib.ora_volume.argtypes = [P]
    lib.ora_max_draws.restype = ctypes.c_longlong
    lib.ora_max_draws.argtypes = [P]
    lib.ora_phase32.argtypes = [P, ctypes.c_int, ctypes.c_int, ctypes.c_ulonglong, ctypes.c_ulonglong, ctypes.c_int,
                                P]
    lib.ora_phase32.restype = ctypes.c_int
    lib.ora_philox4x32.argtypes = [P, P, P]
    lib.ora_philox4x32.restype = None
    lib.ora_set_threads.argtypes = [ctypes.c_int]
    lib.ora_set_threads.restype = ctypes.c_int
    lib.ora_get_threads.restype = ctypes.c_int
    _lib = lib
    return lib


class OracleError(RuntimeError):
    pass


class Oracle:
    """CPU restatement of one reference lattice (AoS FP64)."""

    def __init__(self, lt, lx, ly, beta, *, algo=1, boundary=0, epsilon=0.1, upd=1, seed=1234, tape=None):
        self.lib = load()
        p = OraParams(lt, lx, ly, beta, epsilon, upd, algo, boundary, seed)
        self._tape = None
        if tape is not None:
            t = np.ascontiguousarray(tape, dtype=TAPE_DTYPE)
            if t.ndim != 2:
                raise ValueError("tape must be (streams, draws)")
            self._tape = t
            h = self.lib.ora_create(ctypes.byref(p), ctypes.c_void_p(t.ctypes.data), t.shape[0], t.shape[1])
        else:
            h = self.lib.ora_create(ctypes.byref(p), None, 0, 0)
        if not h:
            raise OracleError(f"ora_create({lt}x{lx}x{ly}) failed")
        self.h = ctypes.c_void_p(h)
        self.V = lt * lx * ly

    def _rc(self, rc, what):
        if rc != 0:
            raise OracleError(f"{what}: status {rc}" + (" (tape exhausted)" if rc == -2 else ""))

    def close(self):
        if self.h:
            self.lib.ora_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def init_cold(self):
        self._rc(self.lib.ora_init_cold(self.h), "init_cold")

    def init_hot(self):
        self._rc(self.lib.ora_init_hot(self.h), "init_hot")

    def load(self, aos):
        a = np.ascontiguousarray(aos, dtype=np.float64)
        self._rc(self.lib.ora_load(self.h, ctypes.c_void_p(a.ctypes.data)), "load")

    def phase(self, k, kind):
        self._rc(self.lib.ora_phase(self.h, k, kind), f"phase {k}")

    def sweep(self, n=1):
        self._rc(self.lib.ora_sweep(self.h, n), "sweep")

    def phase32(self, k, kind, key=0, phase=0, renorm=False, hb_tries=None):
        """One phase of the FP32 path (float links, FP64 fix-ups, Philox draws
        of counter (site, block, phase) under `key`); hb_tries, an int32 array
        of V entries, receives the heat-bath rejection-loop trips per site."""
        t = None
        if hb_tries is not None:
            assert hb_tries.dtype == np.int32 and hb_tries.size == self.V and hb_tries.flags.c_contiguous
            t = ctypes.c_void_p(hb_tries.ctypes.data)
        self._rc(self.lib.ora_phase32(self.h, k, kind, key, phase, int(renorm), t), f"phase32 {k}")

    def sweep32(self, n=1, kind=1, key=0, phase=0, renorm_last=False):
        """n passes of the six phases in the FP32 path, drawing phases
        phase, phase + 1, ... (six per heat-bath or Metropolis pass)."""
        for s in range(n):
            for k in range(6):
                self.phase32(k, kind, key, phase + 6 * s + k, renorm_last and s == n - 1)

    def overrelax(self, n=1):
        self._rc(self.lib.ora_overrelax(self.h, n), "overrelax")

    def normalize(self):
        self._rc(self.lib.ora_normalize(self.h), "normalize")

    def measure(self):
        e, p = ctypes.c_double(), ctypes.c_double()
        self._rc(self.lib.ora_measure(self.h, ctypes.byref(e), ctypes.byref(p)), "measure")
        return e.value, p.value

    def field(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.lib.ora_field(self.h), shape=(self.V * 12,)).copy()

    def accept(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.lib.ora_accept(self.h), shape=(self.V,)).copy()

    def max_draws(self) -> int:
        return int(self.lib.ora_max_draws(self.h))


def set_threads(n: int) -> int:
    return load().ora_set_threads(n)


def philox4x32(ctr, key) -> np.ndarray:
    """One Philox4x32-10 block of the oracle's FP32 restatement."""
    lib = load()
    c = np.ascontiguousarray(ctr, dtype=np.uint32)
    k = np.ascontiguousarray(key, dtype=np.uint32)
    out = np.empty(4, dtype=np.uint32)
    lib.ora_philox4x32(ctypes.c_void_p(c.ctypes.data), ctypes.c_void_p(k.ctypes.data), ctypes.c_void_p(out.ctypes.data))
    return out
