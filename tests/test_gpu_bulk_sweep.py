"""The bulk-staged single-pass sweep (apbs_b200/csrc/gs7_rb_bulk.cuh) on the
GPU: the same iterates as the unstaged single-pass sweep, bit for bit, in
the mixed path's FP32 inner cycles, for odd and even sweep counts and grids
whose windows reach past the arrays (guarded loads) as well as ones that
only use bulk copies."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import (MIXED, K_GS7_BULK_FP32, TUNE_GS7_COLOUR_PASSES,
                            TUNE_MIXED_FINE_SWEEPS, Vpmg)

pytestmark = pytest.mark.gpu


def _solve(p, m, mode, sweeps):
    with Vpmg(p, MIXED) as pmg:
        pmg.set_tuning(TUNE_GS7_COLOUR_PASSES, mode)
        pmg.set_tuning(TUNE_MIXED_FINE_SWEEPS, sweeps)
        pmg.fillco(m)
        pmg.solve()
        return pmg.u, pmg.residual_history(), pmg.energy()


@pytest.mark.parametrize("dime,npbe", [(33, True), (65, False), (97, True), (129, False)])
def test_bulk_sweep_equals_single_pass(dime, npbe):
    m = synth.cluster(300, 10.0, seed=dime, net_charge=3.0)
    p = synth.mg_manual(dime, 32.0 / (dime - 1), m.center(), npbe=npbe,
                        ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    for sweeps in (1, 2, 3):
        want = _solve(p, m, 2, sweeps)
        got = _solve(p, m, 3, sweeps)
        assert np.array_equal(got[0], want[0]), sweeps
        assert np.array_equal(got[1], want[1]), sweeps
        assert got[2] == want[2], sweeps


def test_bulk_sweep_timing_runs():
    m = synth.cluster(300, 10.0, seed=3, net_charge=3.0)
    p = synth.mg_manual(97, 0.4, m.center(), ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    with Vpmg(p, MIXED) as pmg:
        pmg.fillco(m)
        pmg.solve()
        ms, nbytes = pmg.time_kernel(K_GS7_BULK_FP32, 5)
    assert ms > 0.0 and nbytes == 28.0 * 95 ** 3
