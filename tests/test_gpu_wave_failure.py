"""Failure path of the plane-parallel GS27 wavefronts, made without a device
fault: one plane's step counter is shifted (a testing hook) so that its
neighbours' bounded waits run out -- with step counters (k_gs27_planes) the
neighbours wait for a count that never comes, with the mailbox
(k_gs27_mail) the plane tags its slots with a value nobody waits for.  The
solve fails with an error naming the waits, the counters restart (and the
mailboxes are zeroed), and the next solve on the same calculation gives the
normal answer."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import FP64, TUNE_GS27_PLANES, PmgbError, Vpmg, lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("planes", [0, 2], ids=["mailbox", "counters"])
def test_wavefront_wait_runs_out_and_recovers(planes):
    m = synth.cluster(200, 9.0, seed=3)
    p = synth.mg_manual(65, 0.5, m.center())
    with Vpmg(p, FP64) as pmg:
        pmg.set_tuning(TUNE_GS27_PLANES, planes)
        pmg.fillco(m)
        pmg.solve()
        e0, u0 = pmg.energy(), pmg.u
        # level 1 (33^3) runs the plane kernel; shift plane 10's counter back
        assert lib().pmgb_debug_shift_wave_counter(pmg._h, 1, 10, -1000) == 1
        with pytest.raises(PmgbError, match="bounded device waits ran out"):
            pmg.solve()
        pmg.solve()
        assert pmg.energy() == e0
        assert np.array_equal(pmg.u, u0)
