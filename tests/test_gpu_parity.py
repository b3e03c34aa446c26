"""Parity of the CUDA PMG path (through the C ABI) with the reference
compiled from source (oracle/_ref) and with the C restatement (oracle/)."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import FP64, Vpmg
from oracle import port, ref

pytestmark = pytest.mark.gpu

REL_U = 1e-9       # potential, relative to max |u|  (FP64 drop-in bar)
REL_E = 1e-9       # total energy, relative


def _checker():
    return ref if ref.available() else port


def _cases():
    m0, p0 = synth.config0()
    m1 = synth.cluster(300, 10.0, seed=5, net_charge=3.0)
    p1 = synth.mg_manual(65, 0.5, m1.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    m2 = synth.cluster(400, 12.0, seed=7)
    p2 = synth.mg_manual(97, 0.4, m2.center())
    p3 = synth.mg_manual(49, 0.8, m2.center(), srfm=synth.SRFM_MOL)
    m4 = synth.cluster(120, 6.0, seed=11, net_charge=-2.0)
    p4 = synth.mg_manual(33, 0.6, m4.center(), npbe=True, ions=((2, 0.05, 2.0), (-1, 0.1, 1.8)))
    m5 = synth.cluster(150, 8.0, seed=11, net_charge=2.0)
    p5 = synth.mg_manual(33, 0.6, m5.center(), bcfl=synth.BCFL_MDH)
    p6 = synth.mg_manual(65, 0.4, m5.center(), bcfl=synth.BCFL_MDH, npbe=True)
    p6.chgm = synth.CHGM_TRIL
    p7 = synth.mg_manual(49, 0.5, m5.center(), ions=())
    p7.chgm = synth.CHGM_TRIL
    return [("config0_lpbe65", m0, p0), ("npbe65", m1, p1), ("lpbe97_band", m2, p2),
            ("lpbe49_mol", m2, p3), ("npbe33_2to1", m4, p4), ("lpbe33_mdh", m5, p5),
            ("npbe65_mdh_spl0", m5, p6), ("lpbe49_spl0_noions", m5, p7)]


CASES = _cases()


@pytest.mark.parametrize("name,mol,params", CASES, ids=[c[0] for c in CASES])
def test_fill_maps(name, mol, params):
    want = port.fill(params, mol)
    with Vpmg(params, FP64) as pmg:
        pmg.fillco(mol)
        got = pmg.maps()
    for k in ("epsx", "epsy", "epsz", "kappa"):
        assert np.array_equal(got[k], want[k]), k
    # the charge gather adds each point's terms in atom order, as the
    # reference's atom loop does: bitwise
    assert np.array_equal(got["charge"], want["charge"])
    # boundary values go through exp(): CUDA libdevice vs glibc, round-off apart
    fscale = np.abs(want["faces"]).max()
    assert np.abs(got["faces"] - want["faces"]).max() <= 1e-13 * fscale


@pytest.mark.parametrize("name,mol,params", CASES, ids=[c[0] for c in CASES])
def test_solve_matches_reference(name, mol, params):
    want = _checker().run(params, mol)
    with Vpmg(params, FP64) as pmg:
        pmg.fillco(mol)
        pmg.solve()
        e = pmg.energy()
        u = pmg.u
        hist = pmg.residual_history()
    scale = np.abs(want["u"]).max()
    assert np.abs(u - want["u"]).max() <= REL_U * scale
    assert abs(e - want["energy_kT"]) <= REL_E * abs(want["energy_kT"])
    # same iteration history as the reference (its log has 7 digits)
    assert len(hist) == len(want["reslog"])
    np.testing.assert_allclose(hist, want["reslog"], rtol=2e-6)


def test_set_coefficients_dropin():
    """Vpmg_solve drop-in: maps filled on the host, solve on the GPU."""
    mol, params = synth.config0()
    want = _checker().run(params, mol, want_maps=True, want_faces=True)
    with Vpmg(params, FP64) as pmg:
        pmg.set_coefficients(want["charge"], want["epsx"], want["epsy"], want["epsz"],
                             want["kappa"], want["faces"])
        pmg.solve()
        u = pmg.u
    scale = np.abs(want["u"]).max()
    assert np.abs(u - want["u"]).max() <= REL_U * scale


def test_repeat_solve_is_deterministic():
    mol, params = synth.config0()
    with Vpmg(params, FP64) as pmg:
        pmg.fillco(mol)
        pmg.solve()
        e1, u1 = pmg.energy(), pmg.u
        pmg.fillco(mol)
        pmg.solve()
        e2, u2 = pmg.energy(), pmg.u
    assert abs(e1 - e2) <= 1e-13 * abs(e1)
    assert np.abs(u1 - u2).max() <= 1e-13 * np.abs(u1).max()


def test_exact_coarse_solve_matches_band():
    """Above 512 coarsest unknowns the FP64 LPBE path solves the coarsest level
    by exact refinement instead of the reference's banded Cholesky; both are
    exact to round-off, so the two runs agree far inside the parity bar."""
    from apbs_b200.vpmg import TUNE_BAND_ALWAYS, get_tuning, set_tuning
    m = synth.cluster(400, 12.0, seed=7)
    p = synth.mg_manual(49, 0.8, m.center())
    out = {}
    old = get_tuning(TUNE_BAND_ALWAYS)
    try:
        for band in (1, 0):
            set_tuning(TUNE_BAND_ALWAYS, band)
            with Vpmg(p, FP64) as pmg:
                pmg.fillco(m)
                pmg.solve()
                out[band] = (pmg.energy(), pmg.u, pmg.residual_history(), pmg.stats())
    finally:
        set_tuning(TUNE_BAND_ALWAYS, old)
    assert out[1][3]["coarse_method"] == 1 and out[0][3]["coarse_method"] == 3
    assert len(out[1][2]) == len(out[0][2])
    np.testing.assert_allclose(out[0][2], out[1][2], rtol=1e-9)
    scale = np.abs(out[1][1]).max()
    assert np.abs(out[0][1] - out[1][1]).max() <= 1e-12 * scale
    assert abs(out[0][0] - out[1][0]) <= 1e-12 * abs(out[1][0])


def test_single_pass_sweep_matches_colour_passes():
    """The fine smoother's single-pass sweep (gs7_rb.cuh: flat pair slots,
    the first colour of the next plane in a shared-memory ring) computes the
    same red-black sweep as one launch per colour: bitwise equal FP64 solves
    (LPBE and NPBE) for every launch shape and plane chunk, including ranges
    that split rows and chunks of one plane.  In FP32 (the mixed path's
    inner cycles) every shape gives the same iterates and the solve meets
    the mixed-precision tolerance."""
    from apbs_b200.vpmg import (MIXED, TUNE_GS7_COLOUR_PASSES, TUNE_GS7_SWEEP_KCHUNK,
                                TUNE_GS7_SWEEP_SHAPE, TUNE_MIXED_FINE_SWEEPS)
    m = synth.cluster(300, 10.0, seed=5, net_charge=3.0)
    shapes = ((0x00, 8), (0x01, 8), (0x02, 8), (0x12, 18), (0x41, 8), (0x10, 1), (0x21, 5))
    for npbe in (False, True):
        p = synth.mg_manual(65, 0.5, m.center(), npbe=npbe, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
        out = {}
        for key in (("colour",),) + shapes:
            with Vpmg(p, FP64) as pmg:
                if key == ("colour",):
                    pmg.set_tuning(TUNE_GS7_COLOUR_PASSES, 1)
                else:
                    pmg.set_tuning(TUNE_GS7_COLOUR_PASSES, 0)
                    pmg.set_tuning(TUNE_GS7_SWEEP_SHAPE, key[0])
                    pmg.set_tuning(TUNE_GS7_SWEEP_KCHUNK, key[1])
                pmg.fillco(m)
                pmg.solve()
                out[key] = (pmg.u, pmg.residual_history(), pmg.energy())
        for key in shapes:
            assert np.array_equal(out[key][0], out[("colour",)][0]), (npbe, key)
            assert np.array_equal(out[key][1], out[("colour",)][1]), (npbe, key)
            assert out[key][2] == out[("colour",)][2], (npbe, key)
    # FP32 inner cycles of the mixed path
    p = synth.mg_manual(65, 0.5, m.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    with Vpmg(p, FP64) as pmg:
        pmg.fillco(m)
        pmg.solve()
        e64 = pmg.energy()
    res = {}
    for shape, kchunk in shapes:
        with Vpmg(p, MIXED) as pmg:
            pmg.set_tuning(TUNE_GS7_COLOUR_PASSES, 2)
            pmg.set_tuning(TUNE_MIXED_FINE_SWEEPS, 2)
            pmg.set_tuning(TUNE_GS7_SWEEP_SHAPE, shape)
            pmg.set_tuning(TUNE_GS7_SWEEP_KCHUNK, kchunk)
            pmg.fillco(m)
            pmg.solve()
            res[(shape, kchunk)] = (pmg.u, pmg.residual_history(), pmg.energy())
    first = res[shapes[0]]
    for key in shapes[1:]:
        assert np.array_equal(res[key][0], first[0]), key
        assert np.array_equal(res[key][1], first[1]), key
    assert abs(first[2] - e64) <= 1e-6 * abs(e64)
