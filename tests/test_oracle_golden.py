"""Pin the CPU oracle against the reference's own outputs (no GPU needed).

The fixtures in tests/golden were produced by the reference's kernels
(oracle/_ref/ref_harness, see make_golden.py).  The oracle replays the
recorded cuRAND tape and must reproduce the reference's link field, energy,
plaquette and accept array.

Tolerances: the oracle rounds every double operation as written while nvcc
fuses some multiply-adds, and CUDA's rsqrt is within 1 ulp of 1/sqrt; those
last-bit differences stay below 1e-12 after 10 heat-bath or Metropolis sweeps
(the parity bound of the FP64 path).  Over-relaxation from a hot start is a
chaotic map (the normalised staple of a random field can be short), so it is
compared after one pass, and its exact invariant — the total Wilson action —
is checked over all passes.
"""
import numpy as np
import pytest

import pyoracle as po
from cases import CASES, SWEEPS
from conftest import load_case

FIELD_TOL = 1e-12   # north-star parity bound, max |dU| after 10 sweeps
OBS_TOL = 1e-13     # energy / plaquette per sweep
OR_ONE_PASS_TOL = 1e-13

TAPE_CASES = [n for n, c in CASES.items() if c[10]]


def run_oracle(name, tapes):
    lt, lx, ly, algo, bc, hot, beta, eps, upd, seed, _ = CASES[name]
    o = po.Oracle(lt, lx, ly, beta, algo=0 if algo == "metro" else 1, boundary=bc, epsilon=eps, upd=upd,
                  seed=seed, tape=tapes[seed])
    o.init_hot() if hot else o.init_cold()
    step = o.overrelax if algo == "or" else o.sweep
    obs = []
    fields = {}
    for s in range(1, SWEEPS + 1):
        step(1)
        obs.append(o.measure())
        if s in (1, SWEEPS):
            fields[s] = o.field()
    return o, np.array(obs), fields


def test_tape_flavours_advance_together(tapes):
    # curand_uniform and curand_uniform_double move the MRG32k3a stream by the
    # same single step, so one record per draw serves both flavours
    for seed, t in tapes.items():
        assert t["same_step"].all(), seed
        assert np.all((t["ud"] > 0) & (t["ud"] <= 1))
        assert np.all((t["uf"] > 0) & (t["uf"] <= 1))


@pytest.mark.parametrize("name", TAPE_CASES)
def test_oracle_matches_reference(name, tapes):
    g = load_case(name)
    o, obs, fields = run_oracle(name, tapes)
    algo = CASES[name][3]
    if algo == "or":
        assert np.abs(fields[1] - g["field_1"]).max() <= OR_ONE_PASS_TOL
        assert np.abs(obs[0] - g["obs"][0]).max() <= OBS_TOL
        assert np.abs(obs[:, 1] - g["obs"][:, 1]).max() <= OBS_TOL  # conserved plaquette
    else:
        assert np.abs(fields[1] - g["field_1"]).max() <= FIELD_TOL
        assert np.abs(fields[SWEEPS] - g["field_N"]).max() <= FIELD_TOL
        assert np.abs(obs - g["obs"]).max() <= OBS_TOL
    assert np.array_equal(o.accept(), g["accept"])


def test_overrelaxation_conserves_action(tapes):
    # over-relaxation keeps Re tr(U A) of every updated link, so the total
    # Wilson action (the average plaquette) is the same after every pass
    g = load_case("or_per_hot_4")
    o, obs, _ = run_oracle("or_per_hot_4", tapes)
    assert np.ptp(g["obs"][:, 1]) < 1e-13
    assert np.ptp(obs[:, 1]) < 1e-13


def test_reference_fields_are_unitary():
    for name in CASES:
        g = load_case(name)
        det = (g["field_N"].reshape(-1, 4) ** 2).sum(1)
        assert np.abs(det - 1).max() < 1e-13, name


def test_cold_start_observables():
    o = po.Oracle(6, 4, 8, 5.0, algo=1, boundary=2)
    o.init_cold()
    assert o.measure() == (0.0, 1.0)
    assert np.array_equal(o.field().reshape(-1, 4), np.tile([1.0, 0, 0, 0], (6 * 4 * 8 * 3, 1)))


def test_pcc_hot_start_pins_boundary_links(tapes):
    # rand_init2_pcc: x and t links of the plane y = 0 are the identity
    lt, lx, ly = 4, 4, 4
    o = po.Oracle(lt, lx, ly, 8.0, algo=1, boundary=1, tape=tapes[1234])
    o.init_hot()
    f = o.field().reshape(2, lt * lx * ly // 2, 3, 4)
    lyh = ly // 2
    for par in range(2):
        for i in range(lt * lx * lyh):
            yq, x, t = i % lyh, (i // lyh) % lx, i // (lyh * lx)
            y = 2 * yq + (((t + x) & 1) ^ par)
            if y == 0:
                assert np.array_equal(f[par, i, 1:], [[1, 0, 0, 0]] * 2)
            else:
                assert not np.array_equal(f[par, i, 1], [1, 0, 0, 0])


def test_own_generator_streams_differ_and_thermalise():
    # the OWN generator (L'Ecuyer MRG32k3a, used for the CPU baseline) gives a
    # thermalised plaquette in the expected range and different streams per seed
    a = po.Oracle(8, 8, 8, 6.0, algo=1, boundary=0, seed=1)
    b = po.Oracle(8, 8, 8, 6.0, algo=1, boundary=0, seed=2)
    for o in (a, b):
        o.init_cold()
        o.sweep(30)
    pa, pb = a.measure()[1], b.measure()[1]
    assert pa != pb
    assert 0.78 < pa < 0.86 and 0.78 < pb < 0.86
