"""Batched solves in one persistent kernel (pmgb_batch_solve): calculations
of uneven grid sizes solved together agree with the same calculations
solved one at a time, in mixed precision and against FP64."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import FP64, MIXED, PmgbError, Vpmg, batch_solve

pytestmark = pytest.mark.gpu


def _jobs():
    out = []
    for i, (dime, natoms, rad) in enumerate([(33, 120, 6.0), (65, 400, 11.0), (49, 250, 9.0),
                                             (33, 80, 5.0), (65, 600, 12.0), (49, 200, 8.0)]):
        m = synth.cluster(natoms, rad, seed=40 + i, net_charge=float(i % 3 - 1))
        span = float(np.ptp(m.xyz, axis=0).max()) + 14.0
        conc = 0.05 * i
        ions = ((1.0, conc, 2.0), (-1.0, conc, 2.0)) if conc > 0 else ()
        out.append((synth.mg_manual(dime, span / (dime - 1), m.center(), ions=ions), m))
    return out


def _alone(p, m, prec):
    with Vpmg(p, prec) as pmg:
        pmg.fillco(m)
        pmg.solve()
        return pmg.energy(), pmg.u, pmg.stats()


def test_batch_matches_solves_one_at_a_time():
    jobs = _jobs()
    calcs = [Vpmg(p, MIXED) for p, _ in jobs]
    try:
        for c, (p, m) in zip(calcs, jobs):
            c.fillco(m)
        for rep in range(2):          # twice: the second call reuses every hierarchy
            batch_solve(calcs)
            got = [(c.energy(), c.u, c.stats()) for c in calcs]
            for (p, m), (e, u, st) in zip(jobs, got):
                e_mx, u_mx, st_mx = _alone(p, m, MIXED)
                e_64, u_64, _ = _alone(p, m, FP64)
                assert abs(e - e_mx) <= 1e-8 * abs(e_mx)
                assert abs(e - e_64) <= 1e-6 * abs(e_64)
                assert np.abs(u - u_64).max() <= 1e-5 * np.abs(u_64).max()
                assert abs(st["vcycles"] - st_mx["vcycles"]) <= 1
                assert st["rel_residual"] <= (p.etol if p.etol > 0 else 1e-6)
    finally:
        for c in calcs:
            c.close()


def test_batch_refuses_what_it_cannot_run():
    m = synth.cluster(100, 6.0, seed=2)
    p = synth.mg_manual(33, 0.5, m.center())
    with Vpmg(p, FP64) as c:
        c.fillco(m)
        with pytest.raises(PmgbError):
            batch_solve([c])             # FP64 calculations take pmgb_solve
    big = synth.mg_manual(161, 0.4, m.center())
    with Vpmg(big, MIXED) as c:
        c.fillco(m)
        with pytest.raises(PmgbError):
            batch_solve([c])             # level 1 (81^3) is above the tail limit
