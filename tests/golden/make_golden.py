"""Generate the golden fixtures from the reference's own kernels.

Runs on a machine with a GPU and the reference harness built
(`make -C oracle ref`, which compiles the reference's headers where they lie
with oracle/ref_harness.cu).  For every case in cases.py it runs the reference
sweep and stores, in <out>/<case>.npz:

  field_1, field_N   link field (reference AoS FP64 layout) after 1 and N sweeps
  obs                (N, 2) energy and plaquette after every sweep (en_av)
  accept             the reference's accept array after N sweeps
  params             the case tuple

and, per seed, <out>/tape_<seed>.npy: the first TAPE_DRAWS draws of each
MRG32k3a stream curand_init(seed, id, 0) in both flavours with the CUDA float
transcendentals of each draw (see include/qcd2d.h, qcd_rng_tape).

    python tests/golden/make_golden.py --out tests/golden
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from cases import CASES, SWEEPS, TAPE_DRAWS, tape_seeds, tape_streams  # noqa: E402
from pyoracle import REF_HARNESS, TAPE_DTYPE  # noqa: E402


def run(args: list[str]) -> dict:
    out = subprocess.run([REF_HARNESS] + args, check=True, capture_output=True, text=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=HERE)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    if not os.path.exists(REF_HARNESS):
        sys.exit(f"{REF_HARNESS} missing: build it with `make -C oracle ref` where the reference is present")
    os.makedirs(a.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as tmp:
        for seed in tape_seeds():
            n = tape_streams(seed)
            pre = os.path.join(tmp, f"tape{seed}")
            info = run(["tape", "--seed", str(seed), "--streams", str(n), "--draws", str(TAPE_DRAWS), "--out", pre])
            tape = np.fromfile(pre + "_tape.bin", dtype=TAPE_DTYPE).reshape(n, TAPE_DRAWS)
            np.save(os.path.join(a.out, f"tape_{seed}.npy"), tape)
            print(f"tape seed {seed}: {info}")
        for name, c in CASES.items():
            if a.only and a.only not in name:
                continue
            lt, lx, ly, algo, bc, hot, beta, eps, upd, seed, _tape = c
            pre = os.path.join(tmp, name)
            info = run(
                [
                    "run", "--lt", str(lt), "--lx", str(lx), "--ly", str(ly),
                    "--algo", algo, "--bc", str(bc), "--hot", str(hot),
                    "--beta", repr(beta), "--eps", repr(eps), "--upd", str(upd),
                    "--seed", str(seed), "--sweeps", str(SWEEPS),
                    "--dumps", f"1,{SWEEPS}", "--out", pre,
                ]
            )
            V = lt * lx * ly
            f1 = np.fromfile(f"{pre}_field_1.bin", dtype=np.float64)
            fN = np.fromfile(f"{pre}_field_{SWEEPS}.bin", dtype=np.float64)
            obs = np.fromfile(f"{pre}_obs.bin", dtype=np.float64).reshape(SWEEPS, 2)
            acc = np.fromfile(f"{pre}_accept.bin", dtype=np.int32)
            assert f1.size == V * 12 and fN.size == V * 12 and acc.size == V
            np.savez(
                os.path.join(a.out, f"{name}.npz"),
                field_1=f1,
                field_N=fN,
                obs=obs,
                accept=acc,
                params=np.array(json.dumps(c)),
            )
            print(f"{name}: {info}")


if __name__ == "__main__":
    main()
