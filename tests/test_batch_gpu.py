"""Batched replicas against single lattices (bit for bit, on the store layout
the replicas use: one float4 plane per link class) and the oracle."""
import numpy as np
import pytest

import pyoracle as po
import qcd_2d_gpu_b200 as q

pytestmark = pytest.mark.gpu

REPS = [
    dict(lt=8, lx=8, ly=16, beta=6.0, boundary=0, hot=1, seed=11),
    dict(lt=4, lx=6, ly=8, beta=3.5, boundary=1, hot=0, seed=12),
    dict(lt=10, lx=10, ly=4, beta=11.0, boundary=2, hot=1, seed=13),
    dict(lt=2, lx=2, ly=2, beta=5.0, boundary=2, hot=1, seed=14),
    dict(lt=16, lx=16, ly=32, beta=8.0, boundary=1, hot=1, seed=15),
]


@pytest.mark.parametrize("precision,algo,n_or", [("fp64", "hb", 0), ("fp32", "hb", 2), ("fp64", "metro", 1)])
@pytest.mark.parametrize("graph", [True, False])
def test_batch_matches_single_lattices(precision, algo, n_or, graph):
    kw = dict(algo=algo, precision=precision, epsilon=0.25, upd=2, n_or=n_or,
              renorm_every=1 if precision == "fp32" else 0)
    B = q.Batch(REPS, **kw)
    B.init()
    B.reserve(8)
    B.run(6, measure_every=1, graph=graph)
    assert B.measured() == 6
    for i, r in enumerate(REPS):
        L = q.Lattice(r["lt"], r["lx"], r["ly"], r["beta"], boundary=r["boundary"], seed=r["seed"], **kw)
        L.set_pair_layout(False)  # the replicas' store: one float4 plane per class
        L.init_hot() if r["hot"] else L.init_cold()
        ser = []
        for _ in range(6):
            L.sweep(1)
            ser.append(L.measure())
        e, p = B.series(i, 6)
        assert np.array_equal(e, [s[0] for s in ser]) and np.array_equal(p, [s[1] for s in ser])
        assert np.array_equal(B.store_config(i), L.store_config())
        L.close()
    B.close()


def test_stream_offsets_follow_the_subsequence_mapping():
    # a replica at offset o draws from curand_init(seed, o + id, 0): replay
    # that tape through the oracle
    seed, off = 99, 5000
    r = dict(lt=6, lx=4, ly=8, beta=7.0, boundary=2, hot=1, seed=seed, stream_offset=off)
    B = q.Batch([dict(r, stream_offset=0), r], algo="hb", precision="fp64")
    B.init()
    B.run(3, measure_every=0)
    B.synchronize()
    vh = 6 * 4 * 8 // 2
    tape = q.rng_tape(seed, off, vh, 24 + 3 * 6 * 12)
    o = po.Oracle(6, 4, 8, 7.0, algo=1, boundary=2, seed=seed, tape=tape)
    o.init_hot()
    o.sweep(3)
    assert np.abs(B.store_config(1) - o.field()).max() <= 1e-12
    assert not np.array_equal(B.store_config(0), B.store_config(1))


def test_batch_of_96_uneven_replicas_runs_and_thermalises():
    rng = np.random.default_rng(1234)
    reps = []
    for i in range(96):
        lt = int(rng.choice(np.arange(8, 65, 2)))
        reps.append(dict(lt=lt, lx=lt, ly=int(rng.choice(np.arange(8, 129, 2))), beta=float(rng.uniform(3, 12)),
                         boundary=i % 3, hot=int(i % 2 == 0), seed=1234, stream_offset=0))
    off = 0
    for r in reps:  # disjoint subsequence blocks under one seed
        r["stream_offset"] = off
        off += r["lt"] * r["lx"] * r["ly"] // 2
    B = q.Batch(reps, algo="hb", precision="fp32")
    B.init()
    B.reserve(20)
    B.run(20, measure_every=1)
    assert B.measured() == 20
    for i in (0, 37, 95):
        e, p = B.series(i)
        assert np.all(np.isfinite(p)) and 0.2 < p[-1] < 1.0
    B.close()


@pytest.mark.parametrize("precision,algo,n_or", [("fp32", "hb", 1), ("fp64", "metro", 0)])
def test_groups_give_the_same_results_as_one_group(precision, algo, n_or):
    # one replica per group (1 byte per group) on three lanes, then a
    # regrouping in the middle of the run: every replica draws and records
    # exactly as in one group
    kw = dict(algo=algo, precision=precision, epsilon=0.25, upd=2, n_or=n_or,
              renorm_every=1 if precision == "fp32" else 0)
    A, G = q.Batch(REPS, **kw), q.Batch(REPS, **kw)
    A.set_groups(0)
    G.set_groups(1)
    G.set_lanes(3)  # groups on three streams at once
    assert A.groups() == 1 and G.groups() == len(REPS)
    for B in (A, G):
        B.init()
        B.reserve(10)
        B.run(4, measure_every=1, graph=True)
    G.set_groups(3 * 1024 * 16)
    for B in (A, G):
        B.run(4, measure_every=2, graph=False)
        B.run(2, measure_every=1, graph=True)
    assert A.measured() == G.measured() == 8
    for i in range(len(REPS)):
        ea, pa = A.series(i, 8)
        eg, pg = G.series(i, 8)
        assert np.array_equal(ea, eg) and np.array_equal(pa, pg)
        assert np.array_equal(A.store_config(i), G.store_config(i))
    A.close()
    G.close()


def test_batch_autotune_restores_the_batch():
    kw = dict(algo="hb", precision="fp32", renorm_every=1)
    A, T = q.Batch(REPS, **kw), q.Batch(REPS, **kw)
    for B in (A, T):
        B.init()
        B.reserve(12)
        B.run(3, measure_every=1)
    t = T.autotune(4)
    assert t["groups"] >= 1 and t["ms_per_sweep"] > 0
    assert T.measured() == 3
    for B in (A, T):
        B.run(3, measure_every=1)
    for i in range(len(REPS)):
        assert np.array_equal(A.series(i, 6)[1], T.series(i, 6)[1])
        assert np.array_equal(A.store_config(i), T.store_config(i))
    A.close()
    T.close()


def test_c4_batch_matches_lone_lattices():
    # the benchmark's 96 replicas (shapes 8^3 to 64x64x128, beta in [3, 12],
    # boundary r mod 3, hot for even r), each with a seed of its own so that a
    # lone lattice (whose streams start at 0) can reproduce it; FP32 heat-bath
    # re-projected every sweep, grouped on lanes as the benchmark runs them:
    # every replica's links and series are those of the same lattice run alone
    import bench

    reps = [dict(r, seed=1234 + i, stream_offset=0) for i, r in enumerate(bench.c4_replicas())]
    sweeps = 4
    kw = dict(algo="hb", precision="fp32", renorm_every=1)
    B = q.Batch(reps, **kw)
    B.set_groups(16 << 20)
    B.set_lanes(4)
    B.init()
    B.reserve(sweeps)
    B.run(sweeps, measure_every=1, graph=True)
    assert B.measured() == sweeps
    for i, r in enumerate(reps):
        L = q.Lattice(r["lt"], r["lx"], r["ly"], r["beta"], boundary=r["boundary"], seed=r["seed"], **kw)
        L.set_pair_layout(False)  # the replicas' store: one float4 plane per class
        L.init_hot() if r["hot"] else L.init_cold()
        ser = []
        for _ in range(sweeps):
            L.sweep(1)
            ser.append(L.measure())
        e, p = B.series(i, sweeps)
        assert np.array_equal(e, [s[0] for s in ser]) and np.array_equal(p, [s[1] for s in ser]), i
        assert np.array_equal(B.store_config(i), L.store_config()), i
        L.close()
    B.close()
