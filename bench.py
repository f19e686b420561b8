"""Benchmark of the checkerboard SU(2) sweep on one B200 (one JSON line).

Workload (value): a 384^3 lattice with PMC boundary, hot start, one sweep =
1 Kennedy-Pendleton heat-bath pass + 3 over-relaxation passes over the six
checkerboard phases, FP32 links with FP64 fix-ups, links re-projected every
sweep, energy/plaquette measured every 2 sweeps (N_cor = 2).  One step = one
measurement interval = 2 sweeps + 1 measurement.  Metric = link updates/s,
counting every heat-bath and over-relaxation update (12 V per sweep).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica of the lattice (the sweep
has no cross-replica exchange); value = all ranks' updates / max rank time.
`--impl reference` times the reference's own kernels (mc_up_pmc + en_av from
fezquerro/QCD_2d_GPU, built for sm_100a by oracle/Makefile) on the same
lattice; the reference has no over-relaxation for PMC and no FP32 path, so its
sweep is its heat-bath PMC sweep in FP64.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LT = LX = LY = 384
BETA = 10.0
N_OR = 3
N_COR = 2
L2_BYTES = 126 * 1024 * 1024


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples taken during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.p:
            self.p.terminate()
            try:
                self.out, _ = self.p.communicate(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in (getattr(self, "out", "") or "").splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


C4_SWEEPS = 200


def c4_replicas():
    """96 replicas: Nt = Nx uniform over even 8..64, Ny over even 8..128, beta
    uniform in [3, 12], boundary r mod 3, hot start for even r (numpy's PCG64
    seeded with 1234 draws the shapes).  Every replica has its own block of
    MRG32k3a subsequences under the one seed 1234: replica r's streams are
    curand_init(1234, offset_r + id, 0) with offset_r the half-sites of the
    replicas before it, so no two streams of the batch coincide (the same
    offsets separate the Philox site counters of the FP32 draws)."""
    import numpy as np

    rng = np.random.default_rng(1234)
    reps = []
    offset = 0
    for r in range(96):
        lt = int(rng.choice(np.arange(8, 65, 2)))
        ly = int(rng.choice(np.arange(8, 129, 2)))
        beta = float(rng.uniform(3.0, 12.0))
        reps.append(dict(lt=lt, lx=lt, ly=ly, beta=beta, boundary=r % 3, hot=int(r % 2 == 0), seed=1234,
                         stream_offset=offset))
        offset += lt * lt * ly // 2
    return reps


def run_batch_c4(q, torch, stream, rank=0, world=1, dist=None):
    """Batched replicas: the 96 lattices in shared launches, FP32 heat-bath,
    a measurement every sweep, the interval replayed as a CUDA graph; timed
    from the seeding of the streams to the last measurement.  Under torchrun
    the replicas are shared out between the ranks (no collective on the data
    path); the rate is all replicas / the slowest rank's time."""
    from qcd_2d_gpu_b200.replicas import job_rate, shard

    all_reps = c4_replicas()
    reps = shard(all_reps, rank, world)
    sites = sum(r["lt"] * r["lx"] * r["ly"] for r in reps)
    B = q.Batch(reps, algo="hb", precision="fp32", renorm_every=1)
    B.set_stream(stream.cuda_stream)
    B.reserve(C4_SWEEPS)
    B.init()
    B.run(3, measure_every=1)  # warm-up: graph capture and first launches
    B.synchronize()
    # the grouping of the replicas (each group sweeps while its links sit in
    # L2), chosen by the library's autotuner on this batch; state is restored
    tune = B.autotune(10)
    B.reserve(C4_SWEEPS)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    B.init()
    B.run(C4_SWEEPS, measure_every=1, graph=True)
    e1.record(stream)
    B.synchronize()
    ms = e0.elapsed_time(e1)
    assert B.measured() == C4_SWEEPS
    B.close()
    rate, ms_max = job_rate(float(len(reps)), ms, dist, device="cuda")
    ups, _ = job_rate(3.0 * sites * C4_SWEEPS, ms, dist, device="cuda")
    return {"workload": f"96 replicas (Nt=Nx in 8..64, Ny in 8..128, beta in [3,12], bc r mod 3, half hot), "
                        f"FP32 heat-bath, {C4_SWEEPS} sweeps with a measurement each, CUDA graph"
                        + (f", shared out over {world} ranks" if world > 1 else ""),
            "replicas_per_s": rate, "link_updates_per_s": ups, "ms": ms_max, "grouping": tune,
            "sites": sum(r["lt"] * r["lx"] * r["ly"] for r in all_reps)}


def reference_accuracy(args):
    """The reference's own build on the accuracy-scan runs: its link updates/s
    per (boundary, beta) at the scan size (heat-bath sweeps with en_av each)."""
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    if not os.path.exists(harness):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/ref_harness not built"}))
        return 0
    L3 = args.scan_size
    for bc in (0, 2):
        for beta in (4.0, 6.0, 8.0, 10.0, 12.0):
            out = subprocess.run([harness, "bench", "--lt", str(L3), "--lx", str(L3), "--ly", str(L3), "--algo", "hb",
                                  "--bc", str(bc), "--hot", "0", "--beta", str(beta), "--sweeps", "200", "--warmup",
                                  "20"], capture_output=True, text=True, check=True)
            r = json.loads(out.stdout.strip().splitlines()[-1])
            ms = r["ms_per_sweep"] + r["ms_measure"]
            print(json.dumps({"impl": "reference", "lattice": [L3] * 3, "boundary": bc, "beta": beta,
                              "link_updates_per_s": 3.0 * L3 ** 3 / (ms * 1e-3), "ms_per_sweep_with_measure": ms}))
    return 0


def reference_batch_c4(harness):
    import tempfile

    reps = c4_replicas()
    with tempfile.NamedTemporaryFile("w", suffix=".txt", delete=False) as f:
        for r in reps:
            f.write(f"{r['lt']} {r['lx']} {r['ly']} {r['beta']!r} {r['boundary']} {r['hot']} {r['seed']}\n")
        name = f.name
    try:
        out = subprocess.run([harness, "batch", "--list", name, "--sweeps", str(C4_SWEEPS)], capture_output=True,
                             text=True, check=True)
    finally:
        os.unlink(name)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    return {"workload": f"the same 96 replicas run one after the other by the reference's kernels (FP64 "
                        f"heat-bath, {C4_SWEEPS} sweeps, en_av each sweep)",
            "replicas_per_s": r["replicas_per_s"], "link_updates_per_s": r["link_updates_per_s"], "ms": r["ms_total"],
            "sites": r["sites"]}


def chain_stats(e, p):
    """Binned means and errors (bins of ceil(4 tau_int), tau_int by the
    Madras-Sokal window with c = 6) of an energy and a plaquette series."""
    import numpy as np

    import qcd_2d_gpu_b200 as q

    res = {}
    for name, x in (("plaquette", p), ("energy", e)):
        tau, w, dtau = q.tau_int(x, 6.0)
        b = max(1, int(np.ceil(4 * tau)))
        m, err = q.binned(x, b)
        res[name] = {"mean": m, "err": err, "tau_int": tau, "dtau": dtau, "bin": b}
    return res


def compare_stats(a, b):
    """|delta| and |delta| / sigma of the plaquette and energy means of two runs."""
    import numpy as np

    out = {}
    for name in ("plaquette", "energy"):
        d = abs(a[name]["mean"] - b[name]["mean"])
        out[f"delta_{name}"] = d
        out[f"delta_{name}_sigma"] = d / float(np.hypot(a[name]["err"], b[name]["err"]))
    return out


def scan_runs(q, torch, size, sweeps, bcs=(0, 2), betas=(4.0, 6.0, 8.0, 10.0, 12.0), seed=2026, emit=None):
    """FP32 + FP64 fix-ups against FP64 at size^3: `sweeps` heat-bath sweeps
    from a cold start (the first fifth discarded), a measurement every sweep;
    binned means and errors, tau_int and link updates/s per variant.  The
    FP64 path reproduces the reference's build bit for bit (the golden
    tests), so its series stand for the reference's long runs."""
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    therm = sweeps // 5
    out = []
    for bc in bcs:
        for beta in betas:
            row = {"lattice": [size] * 3, "boundary": bc, "beta": beta, "sweeps": sweeps, "discarded": therm}
            for prec in ("fp64", "fp32"):
                lat = q.Lattice(size, size, size, beta, boundary=bc, precision=prec,
                                renorm_every=1 if prec == "fp32" else 0, seed=seed)
                lat.set_stream(stream.cuda_stream)
                lat.init_cold()
                lat.series_reserve(sweeps)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                for i in range(sweeps):
                    if prec == "fp64" and (i + 1) % 100 == 0:
                        lat.normalize()  # the reference re-projects every 100 sweeps
                    lat.sweep(1)
                    lat.measure_into_series(i)
                e1.record(stream)
                e, p = lat.series_read(sweeps)
                ms = e0.elapsed_time(e1)
                lat.close()
                res = chain_stats(e[therm:], p[therm:])
                res["link_updates_per_s"] = 3.0 * size ** 3 * sweeps / (ms * 1e-3)
                row[prec] = res
            row.update(compare_stats(row["fp64"], row["fp32"]))
            out.append(row)
            if emit:
                emit(row)
    torch.cuda.set_stream(torch.cuda.default_stream())
    return out


def accuracy_scan(args, q, torch):
    """The accuracy scan (C5): 128^3, periodic and PMC, beta in {4, 6, 8, 10,
    12}, FP32 + FP64 fix-ups against FP64 (see scan_runs)."""
    out = scan_runs(q, torch, args.scan_size, args.scan_sweeps, emit=lambda r: print(json.dumps(r), flush=True))
    n2 = sum(1 for r in out for k in ("plaquette", "energy") if r[f"delta_{k}_sigma"] <= 2.0)
    print(json.dumps({"summary": f"{n2} of {2 * len(out)} FP32-vs-FP64 comparisons within 2 sigma",
                      "max_delta_plaquette": max(r["delta_plaquette"] for r in out),
                      "max_delta_energy": max(r["delta_energy"] for r in out)}))
    return 0


def c3_accuracy(q, torch, size=LT, n_term=300, n_meas=100, n_cor=2, seed=1234):
    """The benchmark's own workload at matched accuracy: the 384^3 PMC lattice
    at beta 10 from the same hot start, sweep = 1 heat-bath + 3
    over-relaxation passes, run in FP32 + FP64 fix-ups (links re-projected
    every sweep) and in FP64 (re-projected every 100 sweeps like the
    reference's run loop), each with n_term thermalisation sweeps, then n_meas
    measurements n_cor sweeps apart; binned means and errors and tau_int
    of the plaquette and the energy, and |delta| / sigma between the two."""
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    row = {"lattice": [size] * 3, "boundary": "pmc", "beta": BETA, "n_or": N_OR, "n_term": n_term, "n_meas": n_meas,
           "n_cor": n_cor, "start": "hot", "seed": seed}
    for prec in ("fp32", "fp64"):
        lat = q.Lattice(size, size, size, BETA, algo="hb", boundary="pmc", precision=prec, n_or=N_OR,
                        renorm_every=1 if prec == "fp32" else 100, seed=seed)
        lat.set_stream(stream.cuda_stream)
        lat.init_hot()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lat.sweep(n_term)
        lat.series_reserve(n_meas)
        for i in range(n_meas):
            lat.sweep(n_cor)
            lat.measure_into_series(i)
        e1.record(stream)
        e, p = lat.series_read(n_meas)
        ms = e0.elapsed_time(e1)
        lat.close()
        res = chain_stats(e, p)
        res["link_updates_per_s"] = 3.0 * size ** 3 * (1 + N_OR) * (n_term + n_meas * n_cor) / (ms * 1e-3)
        res["seconds"] = ms * 1e-3
        row[prec] = res
    row.update(compare_stats(row["fp64"], row["fp32"]))
    torch.cuda.set_stream(torch.cuda.default_stream())
    return row


def same_work(q, torch, stream, precision, steps, warmup=3, rank=0):
    """The reference arm's exact workload on our kernels: the 384^3 PMC
    lattice from a hot start, heat-bath sweeps only (the reference's
    mc_up_pmc, mc_updates_pmc.h:249-257), one measurement every N_COR sweeps
    (en_av, observables.h:99-141); link updates/s over `steps` measurement
    intervals."""
    L = q.Lattice(LT, LX, LY, BETA, algo="hb", boundary="pmc", precision=precision, n_or=0,
                  renorm_every=1 if precision == "fp32" else 0, seed=1234 + rank)
    L.set_stream(stream.cuda_stream)
    L.init_hot()
    L.series_reserve(1)
    for _ in range(warmup):
        L.sweep(N_COR)
        L.measure_into_series(0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        L.sweep(N_COR)
        L.measure_into_series(0)
    e1.record(stream)
    torch.cuda.synchronize()
    L.close()
    ms = e0.elapsed_time(e1)
    return 3.0 * LT * LX * LY * N_COR * steps / (ms * 1e-3), ms / steps


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def run_cpu_baseline(seconds_hint: float = 20.0):
    """The C oracle (the reference's FP64 sweep restated, own MRG32k3a, OpenMP
    over all host cores) on a bounded sample: one 1 HB + 3 OR sweep of a
    96 x 384 x 384 slab of the workload (a quarter of the lattice)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po

    cores = po.set_threads(os.cpu_count() or 1)
    lt = 96
    o = po.Oracle(lt, LX, LY, BETA, algo=1, boundary=2, seed=1234)
    o.init_hot()
    t0 = time.perf_counter()
    o.sweep(1)
    o.overrelax(N_OR)
    dt = time.perf_counter() - t0
    o.close()
    ups = 3.0 * lt * LX * LY * (1 + N_OR) / dt
    return {"value": ups, "unit": "link updates/s", "cores": cores, "kind": "port",
            "sample": f"1 sweep (1 HB + {N_OR} OR, FP64) of a {lt}x{LX}x{LY} PMC slab of the workload, "
                      f"{dt:.1f} s"}


def reference_arm(args, ws, rank):
    if rank != 0:
        return 0
    harness = os.path.join(ROOT, "oracle", "_ref", "ref_harness")
    base = {"impl": "reference", "metric": "link updates/s", "unit": "link updates/s",
            "higher_is_better": True}
    if not os.path.exists(harness):
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/ref_harness not built (needs the reference checkout "
                                         "at build time: make -C oracle ref)"}))
        return 0
    cmd = [harness, "bench", "--lt", str(LT), "--lx", str(LX), "--ly", str(LY), "--algo", "hb", "--bc", "2",
           "--hot", "1", "--beta", str(BETA), "--sweeps", str(args.steps * N_COR), "--warmup",
           str(args.warmup * N_COR)]
    out = subprocess.run(cmd, capture_output=True, text=True, check=True)
    r = json.loads(out.stdout.strip().splitlines()[-1])
    sweeps = args.steps * N_COR
    # one step = N_COR sweeps + one en_av measurement, as in our arm
    step_ms = r["ms_per_sweep"] * N_COR + r["ms_measure"]
    ups = 3.0 * LT * LX * LY * N_COR / (step_ms * 1e-3)
    line = dict(base)
    line.update({
        "value": ups, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (hot start)",
        "config": {"workload": f"{LT}x{LX}x{LY} PMC hot, reference sweep = heat-bath only (the reference "
                               f"has no PMC over-relaxation and no FP32 path), FP64, measure every {N_COR} "
                               "sweeps", "lattice": [LT, LX, LY], "boundary": "pmc", "precision": "fp64",
                   "n_or": 0, "n_cor": N_COR, "l2": "inputs larger than L2 (5.4 GB link field)"},
        # the reference's implementation of the path is CUDA only: this line
        # times its kernels on the B200, and no CPU number belongs to it (the
        # CPU transcription of its sweep is our arm's cpu_baseline)
        "cpu_baseline": {"value": None, "unit": "link updates/s", "cores": 0, "kind": "reference",
                         "sample": f"none: the reference has no CPU implementation; this arm ran its kernels "
                                   f"(mc_up_pmc + en_av) built for sm_100a on the B200, {sweeps} sweeps timed "
                                   "with CUDA events"},
        "e2e": {"value": ups, "unit": "link updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "heatbath_pass_link_updates_per_s": 3.0 * LT * LX * LY / (r["ms_per_sweep"] * 1e-3),
        "reference_raw": r,
        "batched": reference_batch_c4(harness),
    })
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-replica measurement")
    ap.add_argument("--lattice", type=int, nargs=3, default=None, help="override (testing only)")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "accuracy", "c3-accuracy", "batch"])
    ap.add_argument("--schedule", default="auto", choices=["auto", "phases", "wavefront", "pairs"])
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"],
                    help="link precision of the timed workload (fp32 is the benchmark; fp64 for profiling)")
    ap.add_argument("--wave-tuning", type=int, nargs=3, default=None, metavar=("CHUNK", "PASSES", "FRONTS"))
    ap.add_argument("--scan-size", type=int, default=128)
    ap.add_argument("--scan-sweeps", type=int, default=2000)
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_env()
    if args.lattice:
        global LT, LX, LY
        LT, LX, LY = args.lattice

    if args.workload == "accuracy":
        if args.impl == "reference":
            return reference_accuracy(args)
        import torch

        import qcd_2d_gpu_b200 as q

        return accuracy_scan(args, q, torch)
    if args.workload == "batch" and args.impl == "ours":
        import torch

        import qcd_2d_gpu_b200 as q

        stream = torch.cuda.Stream()
        print(json.dumps(run_batch_c4(q, torch, stream)))
        return 0
    if args.workload == "c3-accuracy":
        import torch

        import qcd_2d_gpu_b200 as q

        print(json.dumps(c3_accuracy(q, torch, size=LT)))
        return 0
    if args.impl == "reference":
        return reference_arm(args, ws, rank)

    import numpy as np
    import torch

    import qcd_2d_gpu_b200 as q

    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    # a dedicated stream: the library launches on it and the CUDA events are
    # recorded on it (torch's default stream is the legacy stream 0, which does
    # not order work on the library's own non-blocking stream)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    V = LT * LX * LY

    PREC = args.precision
    L = q.Lattice(LT, LX, LY, BETA, algo="hb", boundary="pmc", precision=PREC, n_or=N_OR,
                  renorm_every=1, seed=1234 + rank)
    L.set_stream(stream.cuda_stream)
    L.set_schedule(args.schedule)
    if args.wave_tuning:
        L.set_wave_tuning(*args.wave_tuning)
    L.init_hot()

    L_schedule = L.schedule()
    L_paired = L.pair_layout()  # FP32 with Lt % 4 == 0: the site-pair store and its kernels

    def step():
        L.sweep(N_COR)
        L.measure_into_series(0)

    L.series_reserve(1)
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if dist:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    ms_step = ms / args.steps
    updates_per_step = 3.0 * V * (1 + N_OR) * N_COR
    value = updates_per_step * args.steps * ws / (ms * 1e-3)
    # launches of one pass: six phase kernels (the wavefront runs passes in
    # persistent launches); the re-projection rides on the last pass, the
    # measurement is one launch
    per_pass = {"phases": 6, "pairs": 3}.get(L_schedule)
    # + one one-thread launch per heat-bath pass advancing the FP32 draws' counter
    launches_per_step = N_COR * (per_pass * (1 + N_OR) + 1) + 1 if per_pass else None

    # ---- dominant kernel: the over-relaxation pass, timed live -----------
    # one qcd_overrelax pass = 6 phase launches (3 fused-pair launches)
    reps = 5
    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a0.record(stream)
    L.overrelax(reps)
    a1.record(stream)
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    L.close()
    L2h = q.Lattice(LT, LX, LY, BETA, algo="hb", boundary="pmc", precision=PREC, n_or=0, seed=99)
    L2h.set_stream(stream.cuda_stream)
    L2h.set_schedule(args.schedule)
    if args.wave_tuning:
        L2h.set_wave_tuning(*args.wave_tuning)
    torch.cuda.synchronize()
    L2h.init_hot()
    b0.record(stream)
    L2h.sweep(reps)
    b1.record(stream)
    torch.cuda.synchronize()
    n_launch = per_pass or 6
    or_pass_ms = a0.elapsed_time(a1) / reps
    hb_pass_ms = b0.elapsed_time(b1) / reps
    or_launch_ms = or_pass_ms / n_launch
    hb_launch_ms = hb_pass_ms / n_launch
    L2h.close()
    # strict algorithmic bytes: each FP32 link read once and written once per
    # pass, 32 B per update (the FP32 heat-bath draws keep no generator state);
    # a pass is 3V updates
    # (FP64: 2 x 32 B per update, and the heat-bath reads and writes its site's
    # 24-B MRG32k3a state once per six updates)
    link_b = 16.0 if PREC == "fp32" else 32.0
    or_bytes = 2 * link_b * 3 * V / n_launch
    hb_bytes = (2 * link_b + (0.0 if PREC == "fp32" else 2 * 24.0 / 6)) * 3 * V / n_launch
    hbm, peak_kind = peaks()
    or_gbs = or_bytes / (or_launch_ms * 1e-3) / 1e9
    kname = ("pair32<mu, PMC, OR> (fused over-relaxation pair)" if L_schedule == "pairs"
             else "phase32p<mu, par, PMC, OR> (over-relaxation phase, site-pair store)" if L_paired
             else f"phase{PREC[2:]}<mu, par, PMC, OR> (over-relaxation phase)")
    roofline = {"kernel": kname, "bound": "hbm", "achieved": or_gbs,
                "peak": hbm, "unit": "GB/s", "frac": or_gbs / hbm, "peak_source": peak_kind,
                "traffic": None, "algorithmic_bytes_per_launch": or_bytes, "launch_ms": or_launch_ms,
                "launches_per_pass": n_launch,
                "heatbath": {"launch_ms": hb_launch_ms, "achieved": hb_bytes / (hb_launch_ms * 1e-3) / 1e9}}
    traffic_file = os.path.join(ROOT, "profiles", "dram_traffic.json")
    if os.path.exists(traffic_file) and PREC == "fp32" and L_schedule == "phases":
        try:
            key = "phase32p_or_bytes_per_launch" if L_paired else "phase32_or_bytes_per_launch"
            roofline["traffic"] = json.load(open(traffic_file)).get(key)
        except Exception:
            pass
    if roofline["traffic"]:
        # the DRAM bytes a launch really moves (ncu) over its live time: how close
        # the kernel runs to HBM for the traffic of its per-phase design
        roofline["traffic_gbs"] = roofline["traffic"] / (or_launch_ms * 1e-3) / 1e9
        roofline["traffic_frac"] = roofline["traffic_gbs"] / hbm

    # ---- the reference arm's workload on our kernels ------------------------
    # (heat-bath only, a measurement every N_COR sweeps): the like-for-like
    # rates against the reference arm's line, in both precisions
    sw = {"workload": f"{LT}x{LX}x{LY} PMC hot, heat-bath sweeps only, one measurement every {N_COR} sweeps "
                      "(the reference arm's workload)", "steps": args.steps}
    for prec in ("fp64", "fp32"):
        rate, ms_s = same_work(q, torch, stream, prec, args.steps, rank=rank)
        sw[prec] = {"link_updates_per_s": rate, "ms_per_step": ms_s}

    # ---- end to end through the C ABI with host buffers -------------------
    # one host configuration in the reference's AoS FP64 layout is uploaded
    # (pinned host -> device, converted to FP32 SoA) at the start of the timed
    # region; every step reads its (energy, plaquette) back to the host.
    host_cfg = torch.empty(V * 12, dtype=torch.float64, pin_memory=True)
    hv = host_cfg.numpy()
    hv[:] = 0.0
    hv[0::4] = 1.0  # a cold configuration
    E = q.Lattice(LT, LX, LY, BETA, algo="hb", boundary="pmc", precision=PREC, n_or=N_OR,
                  renorm_every=1, seed=4321 + rank)
    E.set_stream(stream.cuda_stream)
    E.load_config(hv)  # allocate the staging buffer outside the timed region
    E.sweep(N_COR)
    E.measure()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    E.load_config(hv)
    for _ in range(args.steps):
        E.sweep(N_COR)
        E.measure()
    t1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = t0.elapsed_time(t1)
    if dist:
        t = torch.tensor([e2e_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = updates_per_step * args.steps * ws / (e2e_ms * 1e-3)
    E.close()

    batched = run_batch_c4(q, torch, stream, rank, ws, dist) if not args.no_batch else None

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cpu = run_cpu_baseline()

    if rank == 0:
        line = {
            "metric": "link updates/s",
            "value": value,
            "unit": "link updates/s",
            "n_gpus": ws,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_step,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32+f64-fixups" if PREC == "fp32" else "f64",
            "data": "synthetic (hot start from seeded MRG32k3a streams; FP32 draws from Philox4x32-10)",
            "config": {"workload": f"{LT}x{LX}x{LY} PMC, hot start, sweep = 1 heat-bath + {N_OR} "
                                   f"over-relaxation, "
                                   + ("FP32 links + FP64 fix-ups, " if PREC == "fp32" else "FP64 links, ")
                                   + "renormalise every sweep, "
                                   f"measure every {N_COR} sweeps",
                       "lattice": [LT, LX, LY], "boundary": "pmc", "precision": PREC, "n_or": N_OR,
                       "n_cor": N_COR, "beta": BETA,
                       "l2": f"inputs larger than L2 ({V * 48 / 1e9:.2f} GB FP32 link store)",
                       "parallelism": f"replicas x{ws}"},
            # one heat-bath pass alone (timed live above): the rate comparable
            # with the reference's heat-bath-only sweep
            "heatbath_pass_link_updates_per_s": 3.0 * V / (hb_pass_ms * 1e-3),
            "same_work_as_reference": sw,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "link updates/s",
                    "h2d_bytes_per_step": V * 12 * 8 / args.steps, "d2h_bytes_per_step": 16,
                    "note": "one AoS FP64 configuration uploaded from pinned host memory per timed run "
                            "(amortised over the steps); one (energy, plaquette) readback per step"},
            "gpu_launches": launches_per_step * args.steps if launches_per_step else None,
            "schedule": L_schedule,
            "batched": batched,
            "clocks": clk.summary(),
        }
        print(json.dumps(line))
    if dist:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
