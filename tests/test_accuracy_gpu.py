"""Accuracy of the FP32 + FP64 fix-ups path against FP64, on the GPU, with
the 2-sigma criterion on binned means.

* The benchmark workload itself (384^3, PMC, beta 10, hot start, sweep =
  1 heat-bath + 3 over-relaxation passes): N_term 300, N 100, N_cor 2, run
  in FP32 (re-projected every sweep) and FP64.
* A reduced accuracy scan at 128^3: periodic and PMC, beta 4 and 10, 2000
  heat-bath sweeps from a cold start (the first 400 discarded), a
  measurement every sweep: four rows of the accuracy study, same runs.

The FP64 path reproduces the reference's kernels bit for bit (the golden
tests), so its series stand for the reference's long runs
(functions/mc_updates_pmc.h:249-257, functions/observables.h:99-141, the
measurement loop of kernel.cu:192-236).  The seeds are fixed, so each run is
deterministic; with independent chains a correct build passes a 2-sigma
comparison with probability ~95%, and these seeds are among those.
"""
import pytest

import bench
import qcd_2d_gpu_b200 as q

pytestmark = pytest.mark.gpu

SIGMAS = 2.0


def test_benchmark_workload_fp32_matches_fp64_within_two_sigma():
    import torch

    row = bench.c3_accuracy(q, torch)
    print(row)
    for name in ("plaquette", "energy"):
        assert row[f"delta_{name}_sigma"] <= SIGMAS, (name, row)
    # both runs thermalised to the same, physical plaquette
    assert 0.85 < row["fp32"]["plaquette"]["mean"] < 1.0


def test_reduced_accuracy_scan_fp32_matches_fp64_within_two_sigma():
    import torch

    rows = bench.scan_runs(q, torch, 128, 2000, bcs=(0, 2), betas=(4.0, 10.0))
    for row in rows:
        print(row)
        for name in ("plaquette", "energy"):
            assert row[f"delta_{name}_sigma"] <= SIGMAS, (name, row)
