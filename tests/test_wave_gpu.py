"""The wavefront schedule against the per-phase schedule (bit for bit).

Both run the same per-link code in the same sequential order, so every link,
every random draw and every accept count must be identical; any missed
dependency in the wavefront would show up as a difference (a race).
"""
import numpy as np
import pytest

import qcd_2d_gpu_b200 as q

pytestmark = pytest.mark.gpu

CASES = [
    # dims, precision, algo, boundary, n_or, sweeps[, (chunk, passes, fronts)]
    ((16, 16, 16), "fp64", "hb", 0, 0, 4),
    ((16, 16, 16), "fp64", "metro", 1, 0, 3),
    ((12, 8, 16), "fp64", "hb", 2, 2, 3),
    ((2, 8, 8), "fp64", "hb", 0, 1, 3),
    ((4, 6, 2), "fp64", "metro", 2, 0, 3),
    ((24, 32, 64), "fp32", "hb", 2, 3, 3),
    ((20, 16, 32), "fp32", "metro", 1, 1, 2),
    ((6, 64, 128), "fp32", "hb", 0, 3, 2),
    ((32, 48, 96), "fp64", "hb", 1, 1, 2),
    ((16, 16, 32), "fp64", "hb", 2, 1, 3, (256, 2, 8)),
    ((24, 32, 64), "fp32", "hb", 0, 3, 2, (512, 4, 12)),
    ((12, 16, 16), "fp64", "metro", 1, 0, 3, (256, 1, 3)),
    ((8, 16, 16), "fp32", "hb", 2, 2, 2, (256, 3, 4)),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{'x'.join(map(str, c[0]))}_{c[1]}_{c[2]}_bc{c[3]}_or{c[4]}_{len(c)}")
def test_wavefront_is_bit_identical_to_phases(case):
    dims, prec, algo, bc, n_or, sweeps = case[:6]
    tuning = case[6] if len(case) > 6 else None
    out = []
    for mode in ("phases", "wavefront"):
        L = q.Lattice(*dims, 7.0, algo=algo, boundary=bc, precision=prec, n_or=n_or, epsilon=0.3, upd=2,
                      renorm_every=1 if prec == "fp32" else 0, seed=31)
        L.set_pair_layout(False)  # FP32: the store layout the wavefront uses, for bit identity
        L.set_schedule(mode)
        assert L.schedule() == mode
        if tuning and mode == "wavefront":
            L.set_wave_tuning(*tuning)
        L.init_hot()
        L.sweep(sweeps)
        L.overrelax(1)
        out.append((L.store_config(), L.accept_counts(), L.measure()))
        L.close()
    (fa, aa, ma), (fb, ab, mb) = out
    assert np.array_equal(fa, fb)
    assert np.array_equal(aa, ab)
    assert ma == mb


def test_wavefront_matches_reference_golden_case():
    # the reference's own 16^3 heat-bath run, reproduced through the wavefront
    from conftest import load_case

    g = load_case("hb_per_cold_16")
    L = q.Lattice(16, 16, 16, 6.0, algo="hb", boundary=0, seed=1234)
    L.set_schedule("wavefront")
    L.init_cold()
    L.sweep(10)
    assert np.array_equal(L.store_config(), g["field_N"])


def test_bounded_wait_reports_timeout_and_context_survives():
    L = q.Lattice(16, 16, 32, 6.0, precision="fp32", seed=2)
    L.set_schedule("wavefront")
    L.init_cold()
    assert L.wave_selftest_timeout() == -5
    # the context is still usable: re-initialise and run normally
    L.init_cold()
    L.sweep(2)
    e, p = L.measure()
    assert 0.0 < p < 1.0
    L.close()


def test_autotune_keeps_the_lattice_and_picks_a_schedule():
    kw = dict(boundary=2, precision="fp32", n_or=1, renorm_every=1, seed=8)
    a = q.Lattice(24, 16, 32, 7.0, **kw)
    b = q.Lattice(24, 16, 32, 7.0, **kw)
    for L in (a, b):
        L.set_pair_layout(False)  # the layout every candidate schedule shares
        L.init_hot()
        L.sweep(2)
    t = a.autotune(2)
    assert t["schedule"] in ("phases", "wavefront") and t["ms_per_sweep"] > 0
    # tuning left no trace: both lattices continue identically (all schedules are bit-identical)
    a.sweep(3)
    b.sweep(3)
    assert np.array_equal(a.store_config(), b.store_config())
    assert np.array_equal(a.accept_counts(), b.accept_counts())
    # a second handle of the same shape reuses the cached choice
    c = q.Lattice(24, 16, 32, 7.0, **kw)
    c.set_pair_layout(False)
    assert c.autotune(2) == t
