"""qcd2d against the reference's own run loop, file by file.

oracle/_ref/ref_harness `main` replays kernel.cu's loop (kernel.cu:49-268)
with the reference's own kernels, statistics and output functions; qcd2d is
the drop-in.  Run with the same knobs and seed, they must leave the same
files: the text outputs byte for byte, the Config_ binary bit for bit for the
heat-bath (Metropolis: within 1e-14, the proposal rounding of the FP64 path),
and the same stdout apart from the wall-clock lines.
"""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT

pytestmark = pytest.mark.gpu

DRIVER = os.path.join(ROOT, "qcd_2d_gpu_b200", "qcd2d")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "ref_harness")

RUNS = [
    # algo, dt, dx, dy, beta, bc, init, N_term, N, N_cor, Nsave, W, eps, upd
    ("hb", 8, 8, 8, 6.0, 0, 1, 20, 30, 2, 3, 5, 0.1, 1),
    ("hb", 6, 4, 8, 9.0, 2, 0, 12, 20, 1, 2, 4, 0.1, 1),
    ("metro", 8, 8, 16, 8.0, 1, 0, 15, 24, 3, 4, 6, 0.2, 4),
    # C1 of the benchmark configurations: 16^3 periodic, beta 6, cold start, N_term 200, N 100, N_cor 5
    ("hb", 16, 16, 16, 6.0, 0, 1, 200, 100, 5, 4, 10, 0.1, 1),
]


def knobs(r):
    algo, dt, dx, dy, beta, bc, init, n_term, n, n_cor, n_save, w, eps, upd = r
    return ["--dt", dt, "--dx", dx, "--dy", dy, "--beta", beta, "--boundary", bc, "--init", init, "--N-term", n_term,
            "--N", n, "--N-cor", n_cor, "--Nsave", n_save, "--W", w, "--epsilon", eps, "--upd", upd, "--seed", 4242,
            "--N-block", 5, "--Nblock-term", 4]


def harness_args(r, extra):
    # the harness spells a few knobs differently
    algo, dt, dx, dy, beta, bc, init, n_term, n, n_cor, n_save, w, eps, upd = r
    return ["main", "--algo", algo, "--lt", dt, "--lx", dx, "--ly", dy, "--beta", beta, "--bc", bc, "--hot",
            1 - init, "--N-term", n_term, "--N", n, "--N-cor", n_cor, "--Nsave", n_save, "--W", w, "--eps", eps,
            "--upd", upd, "--seed", 4242, "--N-block", 5, "--Nblock-term", 4] + extra


def stable_stdout(text):
    return [ln for ln in text.splitlines() if "Time" not in ln and "nblocks" not in ln]


def same_text(ta, tb):
    """Equal token by token; decimals may differ by one unit of their last
    printed digit: the reference's en_av adds block sums with atomicAdd in
    arbitrary order (observables.h:137-140), so its own plaquette series move
    at ~1e-16 from run to run, enough to flip the 10th decimal of a derived
    autocorrelation once in a while."""
    la, lb = ta.split(), tb.split()
    if len(la) != len(lb):
        return False
    for x, y in zip(la, lb):
        if x == y:
            continue
        if "." not in x or "." not in y:
            return False
        digits = len(x.split(".")[1])
        if abs(float(x) - float(y)) > 1.01 * 10.0 ** (-digits):
            return False
    return True


def compare_dirs(a, b, algo):
    fa, fb = sorted(os.listdir(a)), sorted(os.listdir(b))
    assert fa == fb and len(fa) >= 7, (fa, fb)
    for name in fa:
        pa, pb = os.path.join(a, name), os.path.join(b, name)
        if name.startswith("Config_") and not name.endswith("_data.txt"):
            x, y = np.fromfile(pa), np.fromfile(pb)
            if algo == "hb":
                assert np.array_equal(x, y), name
            else:
                assert x.shape == y.shape and np.abs(x - y).max() <= 1e-14, name
        else:
            assert same_text(open(pa).read(), open(pb).read()), name


@pytest.mark.parametrize("r", RUNS, ids=lambda r: f"{r[0]}_bc{r[5]}_{r[1]}x{r[2]}x{r[3]}")
def test_driver_leaves_the_reference_files(r, tmp_path):
    if not os.path.exists(HARNESS):
        pytest.skip("reference harness not built (needs the reference checkout at build time)")
    from qcd_2d_gpu_b200.build import build_driver

    build_driver()
    ref, ours = tmp_path / "ref", tmp_path / "ours"
    ref.mkdir()
    ours.mkdir()
    a = subprocess.run([HARNESS, *map(str, harness_args(r, []))], cwd=ref, capture_output=True, text=True,
                       timeout=300)
    b = subprocess.run([DRIVER, "--algo", r[0], *map(str, knobs(r)), "--outdir", str(ours)], capture_output=True,
                       text=True, timeout=300)
    assert a.returncode == 0, a.stderr
    assert b.returncode == 0, b.stderr + b.stdout
    compare_dirs(ref, ours, r[0])
    assert same_text("\n".join(stable_stdout(a.stdout)), "\n".join(stable_stdout(b.stdout)))
    # resume without thermalisation from the saved configuration (readconf = 2)
    ra, rb = tmp_path / "ref2", tmp_path / "ours2"
    for src, dst in ((ref, ra), (ours, rb)):
        dst.mkdir()
        for name in os.listdir(src):
            if name.startswith("Config_"):
                (dst / name).write_bytes((src / name).read_bytes())
    a = subprocess.run([HARNESS, *map(str, harness_args(r, ["--readconf", 2, "--nsave", 2]))], cwd=ra,
                       capture_output=True, text=True, timeout=300)
    b = subprocess.run([DRIVER, "--algo", r[0], *map(str, knobs(r)), "--readconf", "2", "--nsave", "2", "--outdir",
                        str(rb)], capture_output=True, text=True, timeout=300)
    assert a.returncode == 0 and b.returncode == 0, (a.stderr, b.stderr)
    if r[0] == "hb":
        compare_dirs(ra, rb, r[0])
        assert same_text("\n".join(stable_stdout(a.stdout)), "\n".join(stable_stdout(b.stdout)))
    # read the configuration and thermalise further (readconf = 1): N_term
    # accumulates into the _data.txt of the saved configuration
    if r[0] == "hb":
        rc, rd = tmp_path / "ref3", tmp_path / "ours3"
        for src, dst in ((ref, rc), (ours, rd)):
            dst.mkdir()
            for name in os.listdir(src):
                if name.startswith("Config_"):
                    (dst / name).write_bytes((src / name).read_bytes())
        a = subprocess.run([HARNESS, *map(str, harness_args(r, ["--readconf", 1, "--nsave", 3]))], cwd=rc,
                           capture_output=True, text=True, timeout=300)
        b = subprocess.run([DRIVER, "--algo", r[0], *map(str, knobs(r)), "--readconf", "1", "--nsave", "3",
                            "--outdir", str(rd)], capture_output=True, text=True, timeout=300)
        assert a.returncode == 0 and b.returncode == 0, (a.stderr, b.stderr)
        compare_dirs(rc, rd, r[0])
        assert same_text("\n".join(stable_stdout(a.stdout)), "\n".join(stable_stdout(b.stdout)))


def test_fp32_driver_run_with_report(tmp_path):
    from qcd_2d_gpu_b200.build import build_driver

    build_driver()
    b = subprocess.run([DRIVER, *map(str, ["--dt", 16, "--dx", 16, "--dy", 16, "--beta", 6, "--boundary", 2, "--N-term", 50,
                        "--N", 200, "--N-cor", 1, "--W", 10, "--precision", "fp32", "--n-or", 3, "--renorm-every", 1,
                        "--seed", 7, "--report", "--outdir", str(tmp_path)])], capture_output=True, text=True,
                       timeout=300)
    assert b.returncode == 0, b.stderr
    assert "report Plaquette" in b.stdout
    assert any(n.startswith("Check_16_16_16_B_6.00_pmc_1") for n in os.listdir(tmp_path))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_driver_resume_with_generator_state(tmp_path, precision):
    # FP64: the MRG32k3a words; FP32: also the counter and key of its Philox draws
    from qcd_2d_gpu_b200.build import build_driver

    build_driver()
    common = ["--dt", 8, "--dx", 8, "--dy", 8, "--beta", 6, "--boundary", 0, "--N", 12, "--N-cor", 2, "--W", 3,
              "--Nsave", 1, "--seed", 5, "--rng-state", 1, "--outdir", str(tmp_path), "--precision", precision]
    if precision == "fp32":
        common += ["--n-or", 2, "--renorm-every", 1]
    a = subprocess.run([DRIVER, *map(str, common + ["--N-term", 10])], capture_output=True, text=True, timeout=300)
    assert a.returncode == 0, a.stderr
    assert any(n.endswith("_rng.bin") for n in os.listdir(tmp_path))
    first = (tmp_path / "Check_8_8_8_B_6.00_per_1.txt").read_text()
    b = subprocess.run([DRIVER, *map(str, common + ["--readconf", 2, "--nsave", 2])], capture_output=True, text=True,
                       timeout=300)
    assert b.returncode == 0, b.stderr + b.stdout
    # resumed from the saved links and generator words: the same measurement chain
    second = (tmp_path / "Check_8_8_8_B_6.00_per_2.txt").read_text()
    assert first.splitlines()[2:] == second.splitlines()[2:]
