"""The fused-pair schedule of the FP32 sweep against the per-phase launches.

Both run the same link updates with the same Philox draws; the pairs gather
the staples from shared memory, so the two agree to float rounding (the
compiler contracts multiply-adds per kernel).  Lattices are chosen so that
tiles, windows and stream segments are ragged, wrap around the lattice or
cover it several times over; all three boundary conditions and the three
update kinds are covered.  The per-phase kernels themselves are pinned to
the oracle (test_fp32_oracle_gpu) and, in FP64, to the reference's kernels.
"""
import numpy as np
import pytest

import qcd_2d_gpu_b200 as q

pytestmark = pytest.mark.gpu

TOL = 2e-5
FLIP_TOL = 1e-3
MAX_FLIPPED = 64

DIMS = [(16, 16, 16), (20, 18, 34), (6, 10, 4), (2, 2, 2), (4, 2, 6), (34, 26, 62), (64, 48, 96)]


def pair_and_phases(dims, bc, beta=8.0, seg=0, **kw):
    kw = dict(boundary=bc, precision="fp32", seed=31, **kw)
    a = q.Lattice(*dims, beta, **kw)
    b = q.Lattice(*dims, beta, **kw)
    for L in (a, b):
        L.init_hot()
        L.sweep(3)
    b.set_schedule("pairs")
    b.set_pair_tuning(seg)
    return a, b


def link_dev(a, b):
    return np.abs(a.reshape(-1, 4) - b.reshape(-1, 4)).max(axis=1)


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("bc", [0, 1, 2])
def test_pairs_overrelaxation_matches_phases(dims, bc):
    a, b = pair_and_phases(dims, bc)
    assert np.array_equal(a.store_config(), b.store_config())
    a.overrelax(1)
    b.overrelax(1)
    assert b.schedule() == "pairs"
    d = link_dev(a.store_config(), b.store_config())
    a.close()
    b.close()
    assert d.max() <= TOL, d.max()


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("bc", [0, 1, 2])
def test_pairs_heatbath_matches_phases(dims, bc):
    a, b = pair_and_phases(dims, bc, beta=9.0, renorm_every=1)
    a.sweep(1)
    b.sweep(1)
    d = link_dev(a.store_config(), b.store_config())
    a.close()
    b.close()
    flipped = int((d > FLIP_TOL).sum())
    assert flipped <= MAX_FLIPPED, flipped
    assert np.sort(d)[len(d) - flipped - 1] <= TOL


@pytest.mark.parametrize("dims", DIMS[:4])
@pytest.mark.parametrize("bc", [0, 1, 2])
def test_pairs_metropolis_matches_phases_with_accept_counts(dims, bc):
    a, b = pair_and_phases(dims, bc, beta=6.0, algo="metro", epsilon=0.3, upd=2)
    a.accept_reset()
    b.accept_reset()
    a.sweep(1)
    b.sweep(1)
    d = link_dev(a.store_config(), b.store_config())
    ca, cb = a.accept_counts(), b.accept_counts()
    a.close()
    b.close()
    flipped = int((d > FLIP_TOL).sum())
    assert flipped <= MAX_FLIPPED, flipped
    assert np.sort(d)[len(d) - flipped - 1] <= TOL
    assert int((ca != cb).sum()) <= 4 and ca.sum() > 0


@pytest.mark.parametrize("seg", [1, 2, 3, 5, 16])
def test_pairs_stream_segments_of_any_length(seg):
    # short segments: the pipeline start (even links of slice s0 - 1) and end
    # (slice s1) are recomputed at every segment boundary
    a, b = pair_and_phases((24, 22, 30), 2, seg=seg)
    a.overrelax(2)
    b.overrelax(2)
    d = link_dev(a.store_config(), b.store_config())
    a.close()
    b.close()
    assert d.max() <= 4 * TOL


def test_pairs_headline_sweep_shape_and_measurement():
    # 1 heat-bath + 3 over-relaxation passes, re-projected every sweep; the
    # store alternates between the two copies (an even number of passes per
    # sweep here), and measurement and configuration reads see the current one
    a, b = pair_and_phases((32, 32, 48), 2, beta=10.0, n_or=3, renorm_every=1)
    for L in (a, b):
        L.sweep(2)
    ea, pa = a.measure()
    eb, pb = b.measure()
    assert abs(pa - pb) < 1e-4 and abs(ea - eb) < 1e-4
    assert abs(b.check_unitarity(2e-6) - 1.0) < 1e-6
    b.overrelax(1)  # an odd number of passes: the other store is current
    a.overrelax(1)
    d = link_dev(a.store_config(), b.store_config())
    assert np.sort(d)[-MAX_FLIPPED - 1] <= 1e-3
    a.close()
    b.close()


def test_pairs_sweeps_replayed_from_a_captured_graph():
    import torch

    kw = dict(boundary=1, precision="fp32", n_or=1, renorm_every=1, seed=8)
    direct = q.Lattice(16, 12, 20, 7.0, **kw)
    direct.set_schedule("pairs")
    direct.init_hot()
    direct.sweep(3)
    s = torch.cuda.Stream()
    G = q.Lattice(16, 12, 20, 7.0, **kw)
    G.set_schedule("pairs")
    G.set_stream(s.cuda_stream)
    G.init_hot()
    G.sweep(1)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        G.sweep(1)  # two passes: the stores swap twice, so each replay starts where the last ended
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(G.store_config(), direct.store_config())
    for L in (direct, G):
        L.close()


def test_pairs_checkpoint_and_config_round_trip():
    kw = dict(boundary=2, precision="fp32", n_or=1, renorm_every=1)
    a = q.Lattice(12, 14, 18, 7.5, seed=5, **kw)
    a.set_schedule("pairs")
    a.init_hot()
    a.sweep(4)
    cfg, rng = a.store_config(), a.store_rng()
    a.sweep(3)
    b = q.Lattice(12, 14, 18, 7.5, seed=6, **kw)
    b.set_schedule("pairs")
    b.load_config(cfg)
    b.load_rng(rng)
    b.sweep(3)
    assert np.array_equal(a.store_config(), b.store_config())
    a.close()
    b.close()


def test_pairs_refused_for_fp64():
    L = q.Lattice(8, 8, 8, 6.0, precision="fp64")
    with pytest.raises(q.QcdError) as ei:
        L.set_schedule("pairs")
    assert ei.value.status == -7
    L.close()


def test_autotune_considers_pairs_and_restores_the_lattice():
    kw = dict(boundary=2, precision="fp32", n_or=3, renorm_every=1, seed=12)
    a = q.Lattice(64, 64, 64, 10.0, **kw)
    a.init_hot()
    a.sweep(1)
    before = a.store_config()
    rng = a.store_rng()
    t = a.autotune(1)
    assert t["schedule"] in ("phases", "wavefront", "pairs")
    assert np.array_equal(a.store_config(), before)
    assert np.array_equal(a.store_rng(), rng)
    a.close()
