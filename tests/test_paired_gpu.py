"""The FP32 site-pair store (Lt % 4 == 0) against one float4 plane per class.

Both layouts run the same link updates with the same counter-based draws.
The paired kernels form the quaternion products with packed two-lane
multiply-adds, so the two agree to float rounding; a rounding difference can
move a heat-bath rejection or Metropolis decision, which then changes that
link (and the staples it feeds later in the pass) by more, so those links
are counted, not bounded.  Every lattice has the seams of the row ring
(t = Lt/2 - 1 -> Lt/2 and Lt - 1 -> 0, where the two sites of a pair trade
places); with Lt = 4 every row is a seam row.
"""
import numpy as np
import pytest

import qcd_2d_gpu_b200 as q

pytestmark = pytest.mark.gpu

TOL = 2e-5          # one pass, per link (as the FP32 oracle checks)
FLIP_TOL = 1e-3     # a link beyond this moved a decision
MAX_FLIPPED = 64
MEAS_TOL = 2e-7     # energy / plaquette means: FP32 plaquette products, FP64 sums
DIMS = [(4, 4, 4), (8, 6, 10), (16, 16, 16), (12, 10, 6), (20, 18, 34), (4, 2, 2)]


def twins(dims, bc, beta=7.0, **kw):
    # the same thermalised links (three sweeps of one twin copied into the
    # other) and the same draw counters: over-relaxation of a hot start
    # (random links, small staples) amplifies rounding within one pass
    kw = dict(boundary=bc, precision="fp32", seed=41, **kw)
    a = q.Lattice(*dims, beta, **kw)
    b = q.Lattice(*dims, beta, **kw)
    b.set_pair_layout(False)
    assert a.pair_layout() and not b.pair_layout()
    for L in (a, b):
        L.init_hot()
        L.sweep(3)
    b.load_config(a.store_config())
    assert np.array_equal(a.store_config(), b.store_config())
    return a, b


def link_dev(a, b):
    return np.abs(a.reshape(-1, 4) - b.reshape(-1, 4)).max(axis=1)


def test_layout_follows_lt_and_precision():
    assert q.Lattice(8, 4, 4, 6.0, precision="fp32").pair_layout()
    assert not q.Lattice(6, 4, 4, 6.0, precision="fp32").pair_layout()
    assert not q.Lattice(8, 4, 4, 6.0, precision="fp64").pair_layout()


@pytest.mark.parametrize("dims", DIMS)
def test_layout_change_keeps_every_link(dims):
    L = q.Lattice(*dims, 6.0, boundary=1, precision="fp32", seed=5)
    L.init_hot()
    L.sweep(2)
    c0 = L.store_config()
    L.set_pair_layout(False)
    assert np.array_equal(L.store_config(), c0)
    L.set_schedule("wavefront")
    L.set_schedule("phases")
    assert not L.pair_layout()  # forbidden stays forbidden
    L.set_pair_layout(True)
    assert L.pair_layout() and np.array_equal(L.store_config(), c0)
    L.set_schedule("wavefront")
    assert not L.pair_layout() and np.array_equal(L.store_config(), c0)
    L.set_schedule("auto")
    assert L.pair_layout() and np.array_equal(L.store_config(), c0)


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("bc", [0, 1, 2])
def test_paired_overrelaxation_matches(dims, bc):
    a, b = twins(dims, bc)
    a.overrelax(1)
    b.overrelax(1)
    d = link_dev(a.store_config(), b.store_config())
    assert d.max() <= TOL, d.max()


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("bc", [0, 1, 2])
def test_paired_heatbath_matches(dims, bc):
    a, b = twins(dims, bc, beta=9.0, renorm_every=1)
    a.sweep(1)
    b.sweep(1)
    d = link_dev(a.store_config(), b.store_config())
    assert (d > TOL).sum() <= MAX_FLIPPED, (d > TOL).sum()
    assert (d > FLIP_TOL).sum() <= MAX_FLIPPED


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("bc", [0, 1, 2])
def test_paired_metropolis_matches(dims, bc):
    a, b = twins(dims, bc, algo="metro", epsilon=0.3, upd=3)
    a.sweep(1)
    b.sweep(1)
    d = link_dev(a.store_config(), b.store_config())
    assert (d > TOL).sum() <= MAX_FLIPPED, (d > TOL).sum()
    assert (a.accept_counts() != b.accept_counts()).sum() <= 4


@pytest.mark.parametrize("bc", [0, 1, 2])
def test_paired_measurement_and_unitarity(bc):
    a, b = twins((16, 12, 20), bc, n_or=2, renorm_every=1)
    a.sweep(3)
    b.load_config(a.store_config())  # the same links in both layouts
    ea, pa = a.measure()
    eb, pb = b.measure()
    assert abs(ea - eb) <= MEAS_TOL and abs(pa - pb) <= MEAS_TOL
    assert abs(a.check_unitarity(1e-5) - 1.0) < 1e-6
    a.normalize()
    b.normalize()
    assert np.array_equal(a.store_config(), b.store_config())


def test_paired_sweeps_track_unpaired_statistically():
    # many sweeps: the chains decorrelate (float rounding grows) but sample
    # the same distribution
    res = []
    for paired in (True, False):
        L = q.Lattice(16, 16, 16, 6.0, boundary=2, precision="fp32", n_or=2, renorm_every=1, seed=3)
        L.set_pair_layout(paired)
        L.init_cold()
        L.sweep(100)
        p = []
        for _ in range(200):
            L.sweep(1)
            p.append(L.measure()[1])
        res.append(np.array(p))
        L.close()
    m = [x.mean() for x in res]
    err = [x.std(ddof=1) / np.sqrt(len(x) / 10.0) for x in res]  # generous: tau_int <= 5
    assert abs(m[0] - m[1]) <= 4 * np.hypot(*err), (m, err)


def test_autotune_on_the_pair_store_restores_links_layout_and_counters():
    # the candidates include schedules that rewrite the store into float4
    # planes; the tuner puts back the links, their layout and the draw counter
    kw = dict(boundary=2, precision="fp32", n_or=1, renorm_every=1, seed=21)
    a = q.Lattice(12, 10, 14, 7.0, **kw)
    b = q.Lattice(12, 10, 14, 7.0, **kw)
    for L in (a, b):
        L.init_hot()
        L.sweep(2)
    t = a.autotune(1)
    assert np.array_equal(a.store_config(), b.store_config())
    assert a.pair_layout() == (t["schedule"] == "phases")
    a.set_schedule("phases")
    b.set_schedule("phases")
    assert a.pair_layout() and b.pair_layout()
    a.sweep(2)
    b.sweep(2)
    assert np.array_equal(a.store_config(), b.store_config())
