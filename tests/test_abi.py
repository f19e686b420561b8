"""The C ABI library: loads, exports every declared entry point, and validates
arguments on the host (no GPU needed: no compute call is made here)."""
import ctypes
import os
import re
import subprocess
import tempfile

import pytest

import qcd_2d_gpu_b200 as q
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "qcd2d.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(qcd_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    lib = q.load_library()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    # and the Python binding wraps exactly the declared set
    assert set(names) == set(q.exported_symbols())


def test_params_layout_matches_c():
    prog = r"""
#include <stdio.h>
#include <stddef.h>
#include "qcd2d.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu\n", sizeof(qcd_params), offsetof(qcd_params, beta),
         offsetof(qcd_params, precision), offsetof(qcd_params, seed), sizeof(qcd_tape_record));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "p.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "p")
        subprocess.run(["/usr/bin/gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        size, beta, prec, seed, tape = map(int, subprocess.check_output([exe]).split())
    P = q.Params
    assert ctypes.sizeof(P) == size
    assert P.beta.offset == beta and P.precision.offset == prec and P.seed.offset == seed
    assert q.TAPE_DTYPE.itemsize == tape


@pytest.mark.parametrize(
    "dims,kw",
    [
        ((3, 4, 4), {}),              # odd Lt (kernel.cu:61-64)
        ((4, 5, 4), {}),              # odd Lx
        ((4, 4, 7), {}),              # odd Ly
        ((0, 4, 4), {}),              # empty
        ((4, 4, 4), {"algo": 5}),
        ((4, 4, 4), {"boundary": 3}),
        ((4, 4, 4), {"precision": 9}),
        ((4, 4, 4), {"beta": 0.0}),
        ((4, 4, 4), {"algo": "metro", "epsilon": 1.5}),
    ],
)
def test_create_rejects_bad_parameters_on_host(dims, kw):
    kw = dict(kw)
    beta = kw.pop("beta", 2.0)
    with pytest.raises(q.QcdError) as e:
        q.Lattice(*dims, beta, **kw)
    assert e.value.status == -1


def test_status_strings():
    lib = q.load_library()
    assert lib.qcd_status_string(0) == b"ok"
    assert lib.qcd_status_string(-4) == b"links not unitary"
    assert lib.qcd_status_string(-5) == b"device wait timed out"


def test_defaults_match_reference_knobs():
    lib = q.load_library()
    p = q.Params()
    lib.qcd_params_default(ctypes.byref(p), 96, 96, 4)
    # kernel.cu:24-46
    assert (p.lt, p.lx, p.ly) == (96, 96, 4)
    assert p.beta == 20.0 and abs(p.epsilon - 0.1) < 1e-7 and p.upd == 1
    assert p.algo == q.HEATBATH and p.boundary == q.PERIODIC and p.precision == q.FP64


def test_noalloc_measurement_refuses_on_the_host():
    # argument checks of qcd_measure_aos_noalloc happen before any CUDA call
    # (the pointers below are never dereferenced)
    lib = q.load_library()
    fake = ctypes.c_void_p(256)
    assert lib.qcd_measure_aos_noalloc(fake, 1024, 1024, 1024, 0, fake, None) == -7  # V/2 beyond 32-bit indices
    assert lib.qcd_measure_aos_noalloc(fake, 1 << 30, 1 << 30, 1 << 30, 0, fake, None) == -7  # product overflows
    assert lib.qcd_measure_aos_noalloc(fake, 8, 6, 5, 0, fake, None) == -1
    assert lib.qcd_measure_aos_noalloc(fake, 8, 8, 8, -1, fake, None) == -1
    assert lib.qcd_measure_aos_noalloc(fake, 8, 8, 8, 0, None, None) == -1


def test_batch_refuses_stream_offsets_beyond_the_seeding_tables():
    # the streams of a replica are seeded by jumps of up to 2^40 subsequences
    with pytest.raises(q.QcdError) as ei:
        q.Batch([dict(lt=4, lx=4, ly=4, beta=5.0, stream_offset=(1 << 40) - 10)])
    assert ei.value.status == -1
