"""The oracle's FP32 restatement (the checker of the FP32 kernels) against its
own FP64 restatement of the reference, on the CPU.

Over-relaxation is deterministic, so one pass in float from a float-exact
configuration must agree with the FP64 pass to float accuracy; the
heat-bath draws differ between the two paths (Philox here, MRG32k3a there),
so its float restatement is checked through exact properties: links stay on
the group, the first draw of every site is consumed, and PCC leaves the
frozen links alone.
"""
import numpy as np
import pytest

import pyoracle as po


def hot_float_config(dims, bc, seed=3):
    o = po.Oracle(*dims, 6.0, algo=1, boundary=bc, seed=seed)
    o.init_hot()
    o.sweep(2)
    cfg = o.field().astype(np.float32).astype(np.float64)
    o.close()
    return cfg


@pytest.mark.parametrize("bc", [0, 1, 2])
def test_float_overrelaxation_agrees_with_double(bc):
    dims = (8, 6, 10)
    cfg = hot_float_config(dims, bc)
    a = po.Oracle(*dims, 6.0, algo=1, boundary=bc)
    b = po.Oracle(*dims, 6.0, algo=1, boundary=bc)
    a.load(cfg)
    b.load(cfg)
    for k in range(6):
        a.phase32(k, 2)
        b.phase(k, 2)
    d = np.abs(a.field() - b.field()).max()
    a.close()
    b.close()
    assert d < 2e-5, d


@pytest.mark.parametrize("bc", [0, 1, 2])
def test_float_heatbath_keeps_links_on_the_group_and_pcc_frozen(bc):
    dims = (8, 6, 10)
    cfg = hot_float_config(dims, bc)
    o = po.Oracle(*dims, 8.0, algo=1, boundary=bc)
    o.load(cfg)
    tries = np.zeros(np.prod(dims), np.int32)
    for k in range(6):
        o.phase32(k, 1, key=99, phase=k, renorm=True, hb_tries=tries)
    f = o.field().reshape(-1, 3, 4)
    o.close()
    det = (f ** 2).sum(-1)
    assert np.abs(det - 1).max() < 1e-6
    assert tries.min() >= 1 and tries.max() < 64
    changed = np.abs(f - cfg.reshape(-1, 3, 4)).max(-1) > 0
    if bc == 1:
        # x and t links on the plane y = 0 are never updated (mc_updates_pcc.h:29)
        lt, lx, ly = dims
        vh = lt * lx * ly // 2
        for p in range(2):
            for i in range(vh):
                yq, r = i % (ly // 2), i // (ly // 2)
                x, t = r % lx, r // lx
                if yq == 0 and ((t + x) & 1) ^ p == 0:
                    assert not changed[p * vh + i, 1] and not changed[p * vh + i, 2]
    assert changed[:, 0].all()
