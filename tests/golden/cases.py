"""Golden cases: small lattices run through the reference's own kernels.

Each case is one reference run (oracle/_ref/ref_harness, the reference's
mc_up_per/pcc/pmc + en_av compiled for sm_100a) of SWEEPS sweeps; the fixture
holds the link field after sweep 1 and after sweep SWEEPS, the per-sweep
energy/plaquette and the accept array.  Cases with `tape` set can be replayed
by the CPU oracle from the committed random-number tape of that seed.
"""

SWEEPS = 10
TAPE_DRAWS = 1100  # draws per stream kept in the tape fixtures

# name: (lt, lx, ly, algo, bc, hot, beta, eps, upd, seed, tape)
#   algo: "hb", "metro" or "or" (the reference's over-relaxation, periodic only)
CASES = {
    "hb_per_cold_4": (4, 4, 4, "hb", 0, 0, 6.0, 0.1, 1, 1234, True),
    "hb_per_hot_4": (4, 4, 4, "hb", 0, 1, 3.0, 0.1, 1, 1234, True),
    "metro_per_hot_4": (4, 4, 4, "metro", 0, 1, 8.0, 0.2, 4, 1234, True),
    "hb_pcc_hot_4": (4, 4, 4, "hb", 1, 1, 8.0, 0.1, 1, 1234, True),
    "metro_pcc_hot_4": (4, 4, 4, "metro", 1, 1, 8.0, 0.2, 4, 1234, True),
    "hb_pmc_hot_4": (4, 4, 4, "hb", 2, 1, 10.0, 0.1, 1, 1234, True),
    "metro_pmc_cold_4": (4, 4, 4, "metro", 2, 0, 5.0, 0.3, 2, 1234, True),
    "hb_pmc_hot_648": (6, 4, 8, "hb", 2, 1, 10.0, 0.1, 1, 1234, True),
    "metro_pcc_cold_648": (6, 4, 8, "metro", 1, 0, 4.0, 0.5, 1, 1234, True),
    "hb_per_hot_2": (2, 2, 2, "hb", 0, 1, 2.0, 0.1, 1, 1234, True),
    "hb_pcc_hot_246": (2, 4, 6, "hb", 1, 1, 6.0, 0.1, 1, 1234, True),
    "metro_pmc_hot_246": (2, 4, 6, "metro", 2, 1, 6.0, 0.2, 3, 1234, True),
    "or_per_hot_4": (4, 4, 4, "or", 0, 1, 6.0, 0.1, 1, 1234, True),
    "hb_per_hot_seed_4": (4, 4, 4, "hb", 0, 1, 5.0, 0.1, 1, 4321, True),
    # the reference's CPU-runnable configuration shape (16^3 periodic, beta 6, cold)
    "hb_per_cold_16": (16, 16, 16, "hb", 0, 0, 6.0, 0.1, 1, 1234, False),
    # Metropolis PCC, hot, eps 0.2, 4 hits on a 32x32x64-shaped smaller lattice
    "metro_pcc_hot_8816": (8, 8, 16, "metro", 1, 1, 8.0, 0.2, 4, 1234, False),
}


def tape_streams(seed: int) -> int:
    """Streams needed from the tape of `seed` (the largest V/2 among its cases)."""
    return max(lt * lx * ly // 2 for (lt, lx, ly, *_r, s, tp) in CASES.values() if s == seed and tp)


def tape_seeds() -> list:
    return sorted({c[9] for c in CASES.values() if c[10]})
