"""The FP32 sweep's counter-based generator, Philox4x32-10, on the host.

Pinned by the published known-answer vectors of the algorithm (Salmon et al.,
SC'11, and its reference implementation's test vectors) and by an
independent numpy restatement over many counters.  No GPU: qcd_philox4x32 is
the same __host__ __device__ code the FP32 kernels run.
"""
import numpy as np
import pytest

import qcd_2d_gpu_b200 as q

KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_known_answer_vectors(ctr, key, out):
    assert tuple(int(v) for v in q.philox4x32(ctr, key)) == out


def philox_np(ctr, key):
    """Philox4x32-10 over arrays of counters: ten rounds of two 32x32->64-bit
    products, round keys bumped by the Weyl increments between rounds."""
    x = [c.astype(np.uint64) for c in ctr]
    k0, k1 = np.uint64(key[0]), np.uint64(key[1])
    m = np.uint64(0xFFFFFFFF)
    for r in range(10):
        if r:
            k0 = (k0 + np.uint64(0x9E3779B9)) & m
            k1 = (k1 + np.uint64(0xBB67AE85)) & m
        p0 = np.uint64(0xD2511F53) * x[0]
        p1 = np.uint64(0xCD9E8D57) * x[2]
        x = [((p1 >> np.uint64(32)) ^ x[1] ^ k0) & m, p1 & m, ((p0 >> np.uint64(32)) ^ x[3] ^ k1) & m, p0 & m]
    return np.stack(x).astype(np.uint32)


def test_matches_an_independent_restatement():
    rng = np.random.default_rng(7)
    ctr = rng.integers(0, 2 ** 32, size=(4, 200), dtype=np.uint64)
    key = (0x12345678, 0x9ABCDEF0)
    ref = philox_np(list(ctr), key)
    for i in range(ctr.shape[1]):
        assert np.array_equal(q.philox4x32(ctr[:, i].astype(np.uint32), key), ref[:, i])


def test_site_and_phase_counters_give_uniform_words():
    # the FP32 draws of sites 0..4095 in one drawing phase: the top 24 bits of
    # the first word, mapped to (0, 1], are uniform (chi-square over 16 bins)
    sites = np.arange(4096, dtype=np.uint64)
    z = np.zeros_like(sites)
    w = philox_np([sites, z, z + 5, z], (1234, 0))[0]
    u = ((w >> 8).astype(np.float64) + 1) / 2 ** 24
    assert u.min() > 0 and u.max() <= 1
    h, _ = np.histogram(u, bins=16, range=(0, 1))
    chi2 = ((h - 256.0) ** 2 / 256.0).sum()
    assert chi2 < 40  # 15 degrees of freedom: p ~ 5e-4


@pytest.mark.parametrize("ctr,key,out", KAT)
def test_oracle_restatement_matches_the_known_answers(ctr, key, out):
    # the CPU oracle's own Philox (the checker of the FP32 kernels) is pinned
    # to the same published vectors
    import pyoracle as po

    assert tuple(int(v) for v in po.philox4x32(ctr, key)) == out


def test_oracle_restatement_matches_the_library_on_many_counters():
    import pyoracle as po

    rng = np.random.default_rng(5)
    for _ in range(200):
        c = rng.integers(0, 2 ** 32, 4, dtype=np.uint64).astype(np.uint32)
        k = rng.integers(0, 2 ** 32, 2, dtype=np.uint64).astype(np.uint32)
        assert np.array_equal(po.philox4x32(c, k), q.philox4x32(c, k))
