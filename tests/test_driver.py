"""The drop-in program qcd2d: argument and configuration-file failures are
caught on the host before any GPU work (no GPU needed)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

DRIVER = os.path.join(ROOT, "qcd_2d_gpu_b200", "qcd2d")


@pytest.fixture(scope="module")
def driver():
    from qcd_2d_gpu_b200.build import build_driver

    build_driver()
    return DRIVER


def run(driver, *args, cwd=None):
    return subprocess.run([driver, *map(str, args)], capture_output=True, text=True, cwd=cwd, timeout=60)


def test_odd_extent_is_rejected_like_the_reference(driver):
    r = run(driver, "--dt", 5, "--dx", 4, "--dy", 4)
    assert r.returncode == 1
    assert "Lt, Lx and Ly must be even" in r.stdout  # kernel.cu:61-64


def test_unknown_flag_prints_usage(driver):
    r = run(driver, "--no-such-knob", 1)
    assert r.returncode == 2 and "usage" in r.stderr


def test_missing_configuration_fails_before_the_gpu(driver, tmp_path):
    r = run(driver, "--dt", 4, "--dx", 4, "--dy", 4, "--readconf", 1, "--outdir", tmp_path)
    assert r.returncode == 1
    assert "Error creating the file" in r.stdout  # read_conf, lattice_setup.h:87-90


@pytest.mark.parametrize("defect", ["short", "long", "bad_sidecar"])
def test_corrupt_configuration_is_rejected(driver, tmp_path, defect):
    lt = lx = ly = 4
    V = lt * lx * ly
    name = f"Config_{lt}_{lx}_{ly}_B_6.00_per_1"
    phi = np.tile([1.0, 0, 0, 0], V * 3)
    if defect == "short":
        phi = phi[:-5]
    elif defect == "long":
        phi = np.concatenate([phi, [0.0]])
    phi.tofile(tmp_path / f"{name}.txt")
    (tmp_path / f"{name}_data.txt").write_text("garbage" if defect == "bad_sidecar" else
                                               "N_termalization 10 Type_termalization 1")
    r = run(driver, "--dt", lt, "--dx", lx, "--dy", ly, "--beta", 6, "--boundary", 0, "--readconf", 2,
            "--outdir", tmp_path)
    assert r.returncode == 1
    assert "Error" in r.stdout
