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


# ---- the counter-based draws of the FP32 sweep ------------------------------
@pytest.mark.parametrize("algo,bc,n_or", [("hb", 2, 3), ("metro", 1, 1)])
def test_fp32_generator_checkpoint_resumes_the_chain_exactly(algo, bc, n_or):
    kw = dict(algo=algo, boundary=bc, precision="fp32", n_or=n_or, renorm_every=1, epsilon=0.3, upd=2)
    a = q.Lattice(8, 8, 12, 6.5, seed=21, **kw)
    a.init_hot()
    a.sweep(10)
    b = q.Lattice(8, 8, 12, 6.5, seed=21, **kw)
    b.init_hot()
    b.sweep(5)
    cfg, rng = b.store_config(), b.store_rng()
    c = q.Lattice(8, 8, 12, 6.5, seed=999, **kw)  # the key comes from the checkpoint
    c.load_config(cfg)
    c.load_rng(rng)
    c.sweep(5)
    assert np.array_equal(c.store_config(), a.store_config())
    # accept counts are not part of the checkpoint: c counted only its own 5 sweeps
    assert np.array_equal(c.accept_counts(), a.accept_counts() - b.accept_counts())
    for L in (a, b, c):
        L.close()


def test_fp32_sweeps_replayed_from_a_captured_graph_draw_fresh_numbers():
    # the drawing-phase counter lives on the device: each replay of a captured
    # sweep advances it, so two replays equal two sweeps run directly
    import torch

    kw = dict(boundary=2, precision="fp32", n_or=1, renorm_every=1, seed=8)
    direct = q.Lattice(8, 8, 16, 7.0, **kw)
    direct.init_hot()
    direct.sweep(3)
    s = torch.cuda.Stream()
    G = q.Lattice(8, 8, 16, 7.0, **kw)
    G.set_stream(s.cuda_stream)
    G.init_hot()
    G.sweep(1)  # the first sweep runs directly
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        G.sweep(1)  # captured, not run
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert np.array_equal(G.store_config(), direct.store_config())
    for L in (direct, G):
        L.close()


def test_fp32_seeds_give_different_chains():
    f = []
    for seed in (1, 2):
        L = q.Lattice(8, 8, 8, 6.0, precision="fp32", seed=seed)
        L.init_cold()  # the same start: only the draws differ
        L.sweep(2)
        f.append(L.store_config())
        L.close()
    assert not np.array_equal(f[0], f[1])


def test_headline_lattice_full_size_properties():
    # the 384^3 PMC lattice of the benchmark: one sweep of 1 heat-bath + 3
    # over-relaxation passes keeps every FP32 link on the group and gives a
    # plaquette inside (0, 1); over-relaxation then conserves the total action
    # (the plaquette average), while the energy observable (the x-t plaquettes
    # alone) may move between planes
    L = q.Lattice(384, 384, 384, 10.0, algo="hb", boundary="pmc", precision="fp32", n_or=3, renorm_every=1,
                  seed=1234)
    L.init_hot()
    L.sweep(1)
    assert abs(L.check_unitarity(2e-6) - 1.0) < 1e-6
    _, p0 = L.measure()
    assert 0.0 < p0 < 1.0
    L.overrelax(2)
    _, p1 = L.measure()
    assert abs(p1 - p0) < 1e-6
    L.close()
