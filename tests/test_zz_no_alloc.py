"""qcd_measure_aos_noalloc: the measurement for callers that cannot allocate.

Such a caller (a lattice that fills the GPU, device memory owned by a host
framework's pool, a loop that must not synchronise on cudaMalloc/cudaFree)
holds its configuration in device memory in the reference's AoS layout and
gets energy and plaquette back without the library allocating anything.
This file runs last so that a failure here cannot hide the other tests.
"""
import ctypes

import numpy as np
import pytest

import qcd_2d_gpu_b200 as q

pytestmark = pytest.mark.gpu

TOL = 1e-14  # same summation order as qcd_measure: equal up to the last bit


def _dev_ptr(t):
    return ctypes.c_void_p(t.data_ptr())


@pytest.mark.parametrize("bc", [0, 1, 2])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_noalloc_matches_measure_on_two_calls(bc, precision):
    import torch

    lib = q.load_library()
    lt, lx, ly = 8, 6, 10
    L = q.Lattice(lt, lx, ly, 7.0, boundary=bc, precision=precision, seed=99 + bc)
    L.init_hot()
    L.sweep(3)
    phi = torch.empty(lt * lx * ly * 12, dtype=torch.float64, device="cuda")
    assert lib.qcd_store_config_device(L.handle, _dev_ptr(phi)) == 0
    L.measure()  # synchronises the handle's stream
    # the existing entry point on the same FP64 links (an FP32 lattice's links
    # are exact in FP64): qcd_measure of an FP64 handle holding them
    R = q.Lattice(lt, lx, ly, 7.0, boundary=bc, precision="fp64", seed=1)
    assert lib.qcd_load_config_device(R.handle, _dev_ptr(phi)) == 0
    e_ref, p_ref = R.measure()
    R.close()
    torch.cuda.synchronize()
    out = torch.empty(2, dtype=torch.float64, device="cuda")
    for _ in range(2):  # the scratch keeps the previous call's contents
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        rc = lib.qcd_measure_aos_noalloc(_dev_ptr(phi), lt, lx, ly, bc, _dev_ptr(out), None)
        assert rc == 0
        torch.cuda.synchronize()
        e, p = out.cpu().tolist()
        assert abs(e - e_ref) <= TOL and abs(p - p_ref) <= TOL
    L.close()


def test_noalloc_allocates_nothing_after_first_call():
    import torch

    lib = q.load_library()
    lt = lx = ly = 16
    L = q.Lattice(lt, lx, ly, 6.0, seed=5)
    L.init_cold()
    L.sweep(2)
    phi = torch.empty(lt * lx * ly * 12, dtype=torch.float64, device="cuda")
    out = torch.empty(2, dtype=torch.float64, device="cuda")
    assert lib.qcd_store_config_device(L.handle, _dev_ptr(phi)) == 0
    ref = L.measure()
    torch.cuda.synchronize()
    assert lib.qcd_measure_aos_noalloc(_dev_ptr(phi), lt, lx, ly, 0, _dev_ptr(out), None) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(5):
        assert lib.qcd_measure_aos_noalloc(_dev_ptr(phi), lt, lx, ly, 0, _dev_ptr(out), None) == 0
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert np.allclose(out.cpu().numpy(), ref, rtol=0, atol=TOL)
    L.close()


def test_noalloc_large_lattice_matches_measure():
    # 256^3 (V/2 = 8,388,608 sites): the scratch holds one partial per CTA and
    # a measurement launches at most QCD_NOALLOC_MAX_BLOCKS CTAs whatever the
    # size, so a lattice this large is measured too, with the sums of qcd_measure
    import torch

    lib = q.load_library()
    n = 256
    L = q.Lattice(n, n, n, 9.0, boundary=2, precision="fp64", seed=17)
    L.init_hot()
    phi = torch.empty(n ** 3 * 12, dtype=torch.float64, device="cuda")
    assert lib.qcd_store_config_device(L.handle, _dev_ptr(phi)) == 0
    e_ref, p_ref = L.measure()  # synchronises the handle's stream
    out = torch.empty(2, dtype=torch.float64, device="cuda")
    for _ in range(2):
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        assert lib.qcd_measure_aos_noalloc(_dev_ptr(phi), n, n, n, 2, _dev_ptr(out), None) == 0
        torch.cuda.synchronize()
        e, p = out.cpu().tolist()
        assert abs(e - e_ref) <= TOL and abs(p - p_ref) <= TOL
    L.close()
    del phi


def test_noalloc_refuses_bad_arguments_before_touching_the_device():
    lib = q.load_library()
    # every case below is refused on the host: the pointers are never dereferenced
    fake = ctypes.c_void_p(256)
    # V/2 = 536,870,912 sites exceeds the 32-bit site indices (QCD_NOALLOC_MAX_HALF_SITES)
    assert lib.qcd_measure_aos_noalloc(fake, 1024, 1024, 1024, 2, fake, None) == -7
    # extents whose product overflows 64 bits
    big = 1 << 30
    assert lib.qcd_measure_aos_noalloc(fake, big, big, big, 0, fake, None) == -7
    assert lib.qcd_measure_aos_noalloc(fake, 8, 7, 8, 0, fake, None) == -1  # odd extent
    assert lib.qcd_measure_aos_noalloc(fake, 8, 8, 8, 3, fake, None) == -1  # no such boundary
    assert lib.qcd_measure_aos_noalloc(None, 8, 8, 8, 0, fake, None) == -1
    assert lib.qcd_measure_aos_noalloc(ctypes.c_void_p(264), 8, 8, 8, 0, fake, None) == -1  # not 16-B aligned
