"""Per-calculation launch-shape tuning on the device: the FP64 variants give
bitwise the same solve, the mixed ones agree to round-off, two calculations
in one process keep their own settings, and the tuner returns a setting from
its candidates."""
import numpy as np
import pytest

from apbs_b200 import autotune, synth
from apbs_b200.vpmg import (FP64, MIXED, TUNE_GS27_CLUSTER, TUNE_GS27_CLUSTER_MID,
                            TUNE_GS27_LAG, TUNE_GS27_PLANES, TUNE_GS27_PLANES_POLL, TUNE_GS7_COLOUR_PASSES,
                            TUNE_GS7_SWEEP_KCHUNK, TUNE_GS7_SWEEP_SHAPE,
                            TUNE_TAIL_MAX_POINTS, Vpmg, get_tuning)

pytestmark = pytest.mark.gpu


def _solve(p, m, prec, tune):
    with Vpmg(p, prec) as pmg:
        for k, v in tune.items():
            pmg.set_tuning(k, v)
        pmg.fillco(m)
        pmg.solve()
        return pmg.energy(), pmg.u, pmg.residual_history()


def test_fp64_launch_shapes_do_not_change_the_solve():
    """The plane-parallel and one-cluster GS27 wavefronts, the plane
    wavefront's lag between half-sweeps (4 is lockstep), cluster sizes and
    fine-smoother shapes: bitwise the same FP64 solve (NPBE, 129^3: GS27 on
    the 65^3, 33^3 and 17^3 levels)."""
    m = synth.cluster(400, 11.0, seed=12, net_charge=2.0)
    p = synth.mg_manual(129, 0.4, m.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    e0, u0, h0 = _solve(p, m, FP64, {})
    for tune in ({TUNE_GS27_LAG: 4}, {TUNE_GS27_LAG: 5}, {TUNE_GS27_LAG: 12},
                 {TUNE_GS27_LAG: 16, TUNE_GS27_PLANES_POLL: 1},
                 {TUNE_GS27_PLANES: 1}, {TUNE_GS27_PLANES: 2}, {TUNE_GS27_PLANES_POLL: 1},
                 {TUNE_GS27_PLANES: 1, TUNE_GS27_CLUSTER: 4},
                 {TUNE_GS27_PLANES: 1, TUNE_GS27_CLUSTER_MID: 16},
                 {TUNE_GS7_SWEEP_KCHUNK: 3}, {TUNE_GS7_SWEEP_KCHUNK: 32}, {TUNE_GS7_SWEEP_KCHUNK: 0},
                 {TUNE_GS7_SWEEP_SHAPE: 0x01}, {TUNE_GS7_SWEEP_SHAPE: 0x12},
                 {TUNE_GS7_SWEEP_SHAPE: 0x41}, {TUNE_GS7_COLOUR_PASSES: 1}):
        e, u, h = _solve(p, m, FP64, tune)
        assert e == e0 and np.array_equal(u, u0) and np.array_equal(h, h0), tune


def test_mixed_tail_limit_changes_only_round_off():
    m = synth.cluster(400, 11.0, seed=12)
    p = synth.mg_manual(129, 0.4, m.center())
    e0, u0, _ = _solve(p, m, MIXED, {})
    for lim in (20000, 200000):
        e, u, _ = _solve(p, m, MIXED, {TUNE_TAIL_MAX_POINTS: lim})
        assert abs(e - e0) <= 1e-9 * abs(e0)


def test_tuning_is_per_calculation():
    m = synth.cluster(200, 9.0, seed=3)
    p = synth.mg_manual(65, 0.5, m.center())
    with Vpmg(p, FP64) as a, Vpmg(p, FP64) as b:
        default = get_tuning(TUNE_GS7_SWEEP_KCHUNK)
        a.set_tuning(TUNE_GS7_SWEEP_KCHUNK, default + 4)
        assert a.get_tuning(TUNE_GS7_SWEEP_KCHUNK) == default + 4
        assert b.get_tuning(TUNE_GS7_SWEEP_KCHUNK) == default
        for s in (a, b):
            s.fillco(m)
            s.solve()
        assert a.energy() == b.energy()


def test_tuner_returns_a_candidate():
    m = synth.cluster(200, 9.0, seed=3)
    p = synth.mg_manual(65, 0.5, m.center())
    cands = {TUNE_GS7_SWEEP_KCHUNK: [16, 8], TUNE_GS7_COLOUR_PASSES: [0, 1]}
    e = autotune.tune(p, m, FP64, reps=2, candidates=cands)
    assert int(e["tune"][str(TUNE_GS7_SWEEP_KCHUNK)]) in (16, 8)
    assert 0.0 < e["ms"] <= e["default_ms"]
    assert len(e["trials"]) == 3


def test_mixed_cooperative_smoother_matches_per_colour():
    """The 8-colour GS of a large level as one launch per colour (default) or
    one cooperative launch per call: the same updates in the same order."""
    from apbs_b200.vpmg import TUNE_MC_COOPERATIVE
    m = synth.cluster(300, 10.0, seed=4)
    p = synth.mg_manual(161, 0.4, m.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    e0, u0, h0 = _solve(p, m, MIXED, {})
    e1, u1, h1 = _solve(p, m, MIXED, {TUNE_MC_COOPERATIVE: 1})
    assert e0 == e1 and np.array_equal(u0, u1) and np.array_equal(h0, h1)


def test_mixed_smoothing_counts_reach_the_same_solution():
    """The inner FP32 V-cycle's smoothing counts change the path, not the
    converged answer: every setting meets the stopping test and the energy
    agrees with FP64 to the mixed-precision tolerance."""
    from apbs_b200.vpmg import TUNE_MIXED_COARSE_SWEEPS, TUNE_MIXED_FINE_SWEEPS
    m = synth.cluster(400, 11.0, seed=12, net_charge=2.0)
    for npbe in (False, True):
        p = synth.mg_manual(97, 0.4, m.center(), npbe=npbe, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
        e64, _, _ = _solve(p, m, FP64, {})
        for tune in ({TUNE_MIXED_COARSE_SWEEPS: 1}, {TUNE_MIXED_FINE_SWEEPS: 1},
                     {TUNE_MIXED_COARSE_SWEEPS: 3, TUNE_MIXED_FINE_SWEEPS: 3}):
            e, _, _ = _solve(p, m, MIXED, tune)
            assert abs(e - e64) <= 1e-6 * abs(e64), (npbe, tune)
