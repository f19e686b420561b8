"""The wavefront plan (host code, no GPU) checked by an independent model.

Every pair of tasks that conflict (one writes a link class the other reads or
writes, at slices t+o and t) must be ordered by the ring schedule
tau(n, t) = T_n + ((t - s_n) mod Lt) for every slice t of every ring size, and
the plan's `need` table must name the latest conflicting earlier phase.
The read sets below are written from the staple sites of the reference's
kernels (mc_updates.h:158-176 and siblings), independently of the C++ code.
"""
import numpy as np
import pytest

import qcd_2d_gpu_b200 as q

Y, X, T = 0, 1, 2


def reads(mu, p):
    o = 1 - p
    if mu != T:
        nu = 1 - mu
        # plane (mu, nu): U_nu(x+mu) U_mu(x+nu) U_nu(x) | U_nu(x+mu-nu) U_mu(x-nu) U_nu(x-nu)
        r = {(nu, o, 0), (mu, o, 0), (nu, p, 0), (nu, p, 0), (mu, o, 0), (nu, o, 0)}
        # plane (mu, t): U_t(x+mu) U_mu(x+t) U_t(x) | U_t(x+mu-t) U_mu(x-t) U_t(x-t)
        r |= {(T, o, 0), (mu, o, 1), (T, p, 0), (T, p, -1), (mu, o, -1), (T, o, -1)}
    else:
        r = set()
        for nu in (Y, X):
            # plane (t, nu): U_nu(x+t) U_t(x+nu) U_nu(x) | U_nu(x+t-nu) U_t(x-nu) U_nu(x-nu)
            r |= {(nu, o, 1), (T, o, 0), (nu, p, 0), (nu, p, 1), (T, o, 0), (nu, o, 0)}
    r.add((mu, p, 0))  # over-relaxation / Metropolis read their own link
    return r


def conflict(m, n, o):
    (mum, pm), (mun, pn) = m, n
    return (mum, pm, o) in reads(mun, pn) or (mun, pn, -o) in reads(mum, pm) or ((mum, pm) == (mun, pn) and o == 0)


REF_ORDER = [(Y, 0), (Y, 1), (X, 0), (X, 1), (T, 0), (T, 1)]


@pytest.mark.parametrize("passes", [1, 2, 3, 4])
def test_plan_orders_every_conflict_on_every_ring(passes):
    prog = REF_ORDER * passes
    seam, start, need = q.wave_plan([m for m, _ in prog], [p for _, p in prog])
    P = len(prog)
    for n in range(P):
        for o in (-1, 0, 1):
            latest = max([m for m in range(n) if conflict(prog[m], prog[n], o)], default=-1)
            assert need[o + 1, n] == latest
    for lt in (2, 4, 6, 10, 16, 30):
        tau = lambda n, t: start[n] + ((t - seam[n]) % lt)  # noqa: E731
        for n in range(P):
            for m in range(n):
                for o in (-1, 0, 1):
                    if conflict(prog[m], prog[n], o):
                        for t in range(lt):
                            assert tau(m, (t + o) % lt) < tau(n, t), (passes, lt, n, m, o, t)


def test_plan_phases_complete_in_program_order_per_slice():
    # each phase depends on the previous one at the same slice, which is what
    # lets one arrival counter per slice stand for "phase m is done there"
    prog = REF_ORDER * 4
    _, _, need = q.wave_plan([m for m, _ in prog], [p for _, p in prog])
    assert all(need[1, n] == n - 1 for n in range(1, len(prog)))


def test_plan_window_is_small():
    # a t-slice stays live from its first to its last phase of a pass: about
    # 10 time steps, so ~11 slices (+ neighbours) are resident at a time
    seam, start, _ = q.wave_plan([m for m, _ in REF_ORDER], [p for _, p in REF_ORDER])
    assert (start[-1] - seam[-1]) - (start[0] - seam[0]) <= 10
