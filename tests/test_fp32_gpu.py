"""FP32 links + FP64 fix-ups: statistical parity with the FP64 path.

The FP64 path reproduces the reference's kernels bit for bit (test_parity_gpu),
so FP64 runs stand for the reference's long runs.  The FP32 path cannot match
bit for bit (different rounding, hardware transcendentals in the heat-bath);
its thermalised averages must agree with FP64 within the binned statistical
error.  The test uses 3 sigma so that a correct build fails it with
probability ~0.3% per comparison; the accuracy study reports the 2-sigma
criterion at the full sizes.
"""
import numpy as np
import pytest

import qcd_2d_gpu_b200 as q

pytestmark = pytest.mark.gpu


def binned(series, nbins=20):
    s = np.asarray(series)
    n = len(s) // nbins * nbins
    b = s[:n].reshape(nbins, -1).mean(1)
    return b.mean(), b.std(ddof=1) / np.sqrt(nbins)


def run(precision, bc, beta, n_or, seed, dims=(16, 16, 16), therm=150, meas=600):
    L = q.Lattice(*dims, beta, boundary=bc, precision=precision, n_or=n_or,
                  renorm_every=1 if precision == "fp32" else 0, seed=seed)
    L.init_hot()
    L.sweep(therm)
    L.series_reserve(meas)
    for i in range(meas):
        L.sweep(1)
        L.measure_into_series(i)
    e, p = L.series_read(meas)
    L.close()
    return e, p


@pytest.mark.parametrize("bc,beta,n_or", [(0, 4.0, 0), (2, 8.0, 3), (1, 6.0, 1)])
def test_fp32_matches_fp64_statistically(bc, beta, n_or):
    e64, p64 = run("fp64", bc, beta, n_or, seed=11)
    e32, p32 = run("fp32", bc, beta, n_or, seed=12)
    for a, b in ((p64, p32), (e64, e32)):
        ma, sa = binned(a)
        mb, sb = binned(b)
        assert abs(ma - mb) < 3 * np.hypot(sa, sb), (ma, sa, mb, sb)


def test_fp32_links_stay_on_the_group():
    L = q.Lattice(12, 12, 12, 6.0, boundary=2, precision="fp32", n_or=3, renorm_every=1, seed=3)
    L.init_hot()
    L.sweep(50)
    assert abs(L.check_unitarity(2e-6) - 1.0) < 1e-6


def test_fp32_overrelaxation_conserves_action_to_float_accuracy():
    L = q.Lattice(12, 12, 12, 6.0, boundary=0, precision="fp32", seed=4)
    L.init_hot()
    L.sweep(20)
    p0 = L.measure()[1]
    L.overrelax(10)
    assert abs(L.measure()[1] - p0) < 1e-5
