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
    # spline charges are scattered with FP64 atomics: equal to round-off
    scale = np.abs(want["charge"]).max()
    assert np.abs(got["charge"] - want["charge"]).max() <= 1e-14 * scale
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
    """The fine smoother's single-pass sweep kernels (ring tiles, the default;
    ring tiles staged by cp.async; one thread per column marching up k, on
    32x16 and 32x8 tiles; whole-row pair tiles, with and without the next
    plane's coefficients loaded ahead) and the one-launch-per-colour kernels compute the
    same red-black sweep: bitwise equal FP64 solves, and bitwise equal FP32
    inner cycles of the mixed path."""
    from apbs_b200.vpmg import (MIXED, TUNE_GS7_COLOUR_PASSES, TUNE_GS7_SWEEP_KERNEL,
                                TUNE_MIXED_FINE_SWEEPS, get_tuning, set_tuning)
    m = synth.cluster(300, 10.0, seed=5, net_charge=3.0)
    out = {}
    old = get_tuning(TUNE_GS7_COLOUR_PASSES)
    kernels = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9)
    try:
        for npbe in (False, True):
            p = synth.mg_manual(65, 0.5, m.center(), npbe=npbe, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
            for passes, kern in ((1, 0),) + tuple((0, k) for k in kernels):
                set_tuning(TUNE_GS7_COLOUR_PASSES, passes)
                with Vpmg(p, FP64) as pmg:
                    pmg.set_tuning(TUNE_GS7_SWEEP_KERNEL, kern)
                    pmg.fillco(m)
                    pmg.solve()
                    out[(npbe, passes, kern)] = (pmg.u, pmg.residual_history())
    finally:
        set_tuning(TUNE_GS7_COLOUR_PASSES, old)
    for npbe in (False, True):
        for var in tuple((0, k) for k in kernels):
            assert np.array_equal(out[(npbe,) + var][0], out[(npbe, 1, 0)][0]), var
            assert np.array_equal(out[(npbe,) + var][1], out[(npbe, 1, 0)][1]), var
    # FP32 (mixed inner cycles): every sweep kernel gives the same iterates
    p = synth.mg_manual(65, 0.5, m.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    res = {}
    for kern in kernels:
        with Vpmg(p, MIXED) as pmg:
            pmg.set_tuning(TUNE_GS7_COLOUR_PASSES, 2)
            pmg.set_tuning(TUNE_MIXED_FINE_SWEEPS, 2)
            pmg.set_tuning(TUNE_GS7_SWEEP_KERNEL, kern)
            pmg.fillco(m)
            pmg.solve()
            res[kern] = (pmg.u, pmg.residual_history())
    for kern in kernels[1:]:
        assert np.array_equal(res[kern][0], res[0][0]), kern
        assert np.array_equal(res[kern][1], res[0][1]), kern
