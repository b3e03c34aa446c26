"""Failure path of the plane-parallel GS27 wavefront, made without a device
fault: one plane's step counter is shifted (a testing hook) so that its
neighbours' bounded waits run out.  The solve fails with an error naming
the waits, the counters restart, and the next solve on the same calculation
gives the normal answer."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import FP64, PmgbError, Vpmg, lib

pytestmark = pytest.mark.gpu


def test_wavefront_wait_runs_out_and_recovers():
    m = synth.cluster(200, 9.0, seed=3)
    p = synth.mg_manual(65, 0.5, m.center())
    with Vpmg(p, FP64) as pmg:
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
