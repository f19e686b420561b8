"""Parity of the CUDA path (through the C ABI) with the reference and the oracle.

1. Against the golden fixtures made by the reference's own kernels: the FP64
   path reproduces heat-bath and over-relaxation bit for bit and Metropolis
   to within a few ulp (nvcc contracts one multiply-add differently in the
   proposal arithmetic), with identical accept/reject decisions.
2. Against the CPU oracle replaying the same cuRAND draws (qcd_rng_tape) at
   sizes and boundary conditions the fixtures do not cover.
The parity bound is max|dU| <= 1e-12 after 10 sweeps.
"""
import numpy as np
import pytest

import pyoracle as po
import qcd_2d_gpu_b200 as q
from cases import CASES, SWEEPS
from conftest import load_case

pytestmark = pytest.mark.gpu

FIELD_TOL = 1e-12
METRO_BITS_TOL = 1e-14  # few-ulp difference of the Metropolis proposal arithmetic
OBS_TOL = 1e-14


def make(case, **kw):
    lt, lx, ly, algo, bc, hot, beta, eps, upd, seed, _ = case
    L = q.Lattice(lt, lx, ly, beta, algo="metro" if algo == "metro" else "hb", boundary=bc, epsilon=eps,
                  upd=upd, seed=seed, **kw)
    L.init_hot() if hot else L.init_cold()
    return L


@pytest.mark.parametrize("name", list(CASES))
def test_fp64_matches_reference_kernels(name):
    g = load_case(name)
    case = g["case"]
    algo = case[3]
    L = make(case)
    step = L.overrelax if algo == "or" else L.sweep
    obs = []
    for s in range(1, SWEEPS + 1):
        step(1)
        obs.append(L.measure())
        if s == 1:
            f1 = L.store_config()
    fN = L.store_config()
    if algo == "metro":
        assert np.abs(f1 - g["field_1"]).max() <= METRO_BITS_TOL
        assert np.abs(fN - g["field_N"]).max() <= METRO_BITS_TOL
    else:
        assert np.array_equal(f1, g["field_1"]), "heat-bath / over-relaxation must be bit-identical"
        assert np.array_equal(fN, g["field_N"])
    assert np.abs(np.array(obs) - g["obs"]).max() <= OBS_TOL
    assert np.array_equal(L.accept_counts(), g["accept"])
    L.close()


ORACLE_CASES = [
    # lt, lx, ly, algo, bc, hot, beta, eps, upd
    (8, 8, 8, "hb", 0, 0, 6.0, 0.1, 1),
    (8, 8, 8, "hb", 1, 0, 8.0, 0.1, 1),
    (8, 8, 8, "hb", 2, 0, 10.0, 0.1, 1),
    (10, 6, 4, "hb", 2, 0, 4.0, 0.1, 1),
    (8, 8, 8, "metro", 0, 0, 6.0, 0.2, 4),
    (8, 8, 8, "metro", 1, 0, 8.0, 0.2, 4),
    (6, 10, 12, "metro", 2, 0, 5.0, 0.3, 2),
    (16, 16, 16, "hb", 1, 0, 8.0, 0.1, 1),
    (8, 8, 16, "metro", 1, 1, 8.0, 0.2, 4),
    (12, 8, 6, "hb", 0, 1, 9.0, 0.1, 1),
]


@pytest.mark.parametrize("case", ORACLE_CASES, ids=lambda c: "_".join(map(str, c[:6])))
def test_fp64_matches_oracle(case):
    lt, lx, ly, algo, bc, hot, beta, eps, upd = case
    seed = 20261203
    vh = lt * lx * ly // 2
    draws = 24 + SWEEPS * 6 * (4 * upd if algo == "metro" else 12)
    tape = q.rng_tape(seed, 0, vh, draws)
    o = po.Oracle(lt, lx, ly, beta, algo=0 if algo == "metro" else 1, boundary=bc, epsilon=eps, upd=upd,
                  seed=seed, tape=tape)
    L = q.Lattice(lt, lx, ly, beta, algo=algo, boundary=bc, epsilon=eps, upd=upd, seed=seed)
    if hot:
        o.init_hot()
        L.init_hot()
    else:
        o.init_cold()
        L.init_cold()
    for s in range(SWEEPS):
        o.sweep(1)
        L.sweep(1)
        eo, po_ = o.measure()
        eg, pg = L.measure()
        assert abs(eo - eg) <= 1e-13 and abs(po_ - pg) <= 1e-13
    assert np.abs(L.store_config() - o.field()).max() <= FIELD_TOL
    assert np.array_equal(L.accept_counts(), o.accept())
    L.close()


def test_over_relaxation_extension_matches_oracle():
    # PCC / PMC over-relaxation has no reference kernel (mc_updates_pcc.h and
    # _pmc.h have no update flag); it uses the same boundary-masked staples.
    for bc in (1, 2):
        seed = 77
        tape = q.rng_tape(seed, 0, 4 * 4 * 6 // 2, 64)
        o = po.Oracle(4, 4, 6, 7.0, algo=1, boundary=bc, seed=seed, tape=tape)
        L = q.Lattice(4, 4, 6, 7.0, boundary=bc, seed=seed)
        o.init_cold()
        L.init_cold()
        o.sweep(1)  # heat-bath to leave the trivial configuration
        L.sweep(1)
        o.overrelax(1)
        L.overrelax(1)
        assert np.abs(L.store_config() - o.field()).max() <= 1e-13
        p0 = L.measure()[1]
        L.overrelax(5)
        assert abs(L.measure()[1] - p0) < 1e-12  # action conserved


def test_config_round_trip_and_determinism():
    a = q.Lattice(8, 6, 10, 5.0, boundary=2, seed=5)
    b = q.Lattice(8, 6, 10, 5.0, boundary=2, seed=5)
    for L in (a, b):
        L.init_hot()
        L.sweep(3)
    fa, fb = a.store_config(), b.store_config()
    assert np.array_equal(fa, fb)
    assert a.measure() == b.measure()  # fixed-order sums: bitwise reproducible
    c = q.Lattice(8, 6, 10, 5.0, boundary=2, seed=5)
    c.load_config(fa)
    assert np.array_equal(c.store_config(), fa)
    assert c.measure() == a.measure()


def test_normalize_and_unitarity_check():
    L = q.Lattice(8, 8, 8, 6.0, seed=3)
    L.init_hot()
    f = L.store_config().reshape(-1, 4)
    f *= 1 + 1e-6 * np.arange(len(f))[:, None] / len(f)  # drift off the group manifold
    L.load_config(f.ravel())
    with pytest.raises(q.QcdError) as e:
        L.check_unitarity(1e-9)
    assert e.value.status == -4
    L.normalize()
    assert abs(L.check_unitarity(1e-14) - 1.0) < 1e-15
    g = L.store_config().reshape(-1, 4)
    ref = f / np.sqrt((f ** 2).sum(1))[:, None]
    assert np.abs(g - ref).max() < 1e-15


def test_nan_link_is_reported_not_trapped():
    L = q.Lattice(4, 4, 4, 6.0, seed=3)
    L.init_cold()
    f = L.store_config()
    f[17] = np.nan
    L.load_config(f)
    with pytest.raises(q.QcdError) as e:
        L.check_unitarity(1e-9)
    assert e.value.status == -4


def test_vanishing_staple_is_reported_not_spun():
    # links of norm 1e-20 make every staple sum ~1e-60: the heat-bath scale
    # 1/(2 beta |A|) overflows float, the rejection loop cannot accept, stops
    # at its bound and flags the error instead of spinning
    L = q.Lattice(4, 4, 4, 6.0, seed=3)
    L.load_config(np.tile([1e-20, 0.0, 0.0, 0.0], 4 * 4 * 4 * 3))
    L.sweep(1)
    with pytest.raises(q.QcdError) as e:
        L.measure()
    assert e.value.status == -4


def test_series_matches_synchronous_measure():
    L = q.Lattice(8, 8, 8, 6.0, seed=11)
    L.init_cold()
    L.series_reserve(5)
    ref = []
    for i in range(5):
        L.sweep(2)
        L.measure_into_series(i)
        ref.append(L.measure())
    e, p = L.series_read(5)
    assert np.array_equal(e, [r[0] for r in ref]) and np.array_equal(p, [r[1] for r in ref])


def test_accept_counts_heatbath_pcc():
    L = q.Lattice(4, 4, 6, 6.0, boundary=1, seed=1)
    L.init_cold()
    L.sweep(3)
    acc = L.accept_counts().reshape(2, -1)
    # 3 links per site per sweep, 1 at y = 0 under PCC (mc_updates_pcc.h:29)
    lyh = 3
    for par in range(2):
        for i in range(acc.shape[1]):
            yq, x, t = i % lyh, (i // lyh) % 4, i // (lyh * 4)
            y = 2 * yq + (((t + x) & 1) ^ par)
            assert acc[par, i] == (3 if y == 0 else 9)
    L.accept_reset()
    assert not L.accept_counts().any()


def test_generator_checkpoint_resumes_the_chain_exactly():
    kw = dict(boundary=1, precision="fp64", seed=21)
    a = q.Lattice(8, 8, 12, 6.5, **kw)
    a.init_hot()
    a.sweep(10)
    b = q.Lattice(8, 8, 12, 6.5, **kw)
    b.init_hot()
    b.sweep(5)
    cfg, rng = b.store_config(), b.store_rng()
    c = q.Lattice(8, 8, 12, 6.5, **dict(kw, seed=999))  # seeded differently on purpose
    c.load_config(cfg)
    c.load_rng(rng)
    c.sweep(5)
    assert np.array_equal(c.store_config(), a.store_config())
