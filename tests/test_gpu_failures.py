"""Failures made on the host, and the solver's defined behaviour for each:

* non-finite atom data: the fill refuses it (naming the atom), the
  calculation stays unfilled and a following solve fails too; the same
  calculation then solves a good molecule normally;
* a non-finite value in coefficient maps handed in by the caller: the solve
  stops at the first non-finite residual and returns 0, and the calculation
  recovers on the next good fill;
* an iteration limit too small to converge (itmax = 1): as Vpmg_solve
  (the reference only sets ierror, src/pmgc/mgcsd.c:564), the solve returns
  success with the last iterate, and that iterate is the reference's own
  after the same number of steps; the stats report converged = 0;
* one bad request in a serving mix: it fails with its message, every other
  request gives the result it gives alone.
No device fault is involved in any of them."""
import numpy as np
import pytest

from apbs_b200 import serve, synth
from apbs_b200.vpmg import FP64, MIXED, PmgbError, Vpmg
from oracle import ref

pytestmark = pytest.mark.gpu

REL_SAME = 1e-10


def _small():
    m = synth.cluster(200, 8.0, seed=31, net_charge=2.0)
    return m, synth.mg_manual(33, 0.6, m.center(), npbe=True,
                              ions=((1.0, 0.1, 2.0), (-1.0, 0.1, 2.0)))


def _poisoned(mol, atom, what):
    xyz, q, r = mol.xyz.copy(), mol.charge.copy(), mol.radius.copy()
    if what == "x":
        xyz[atom, 0] = np.nan
    elif what == "charge":
        q[atom] = np.inf
    else:
        r[atom] = np.nan
    return synth.Molecule(xyz, q, r)


@pytest.mark.parametrize("what", ["x", "charge", "radius"])
@pytest.mark.parametrize("precision", [FP64, MIXED], ids=["fp64", "mixed"])
def test_non_finite_atoms_are_refused(what, precision):
    mol, params = _small()
    with Vpmg(params, precision) as pmg:
        pmg.fillco(mol)
        pmg.solve()
        e_good = pmg.energy()
        bad = _poisoned(mol, 17, what)
        with pytest.raises(PmgbError, match="atom 17 has a non-finite"):
            pmg.fillco(bad)
        with pytest.raises(PmgbError, match="fillco first"):
            pmg.solve()
        pmg.fillco(mol)
        pmg.solve()
        assert abs(pmg.energy() - e_good) <= REL_SAME * abs(e_good)


def test_non_finite_map_stops_the_solve():
    mol, params = _small()
    params.nonlin = 0
    want = ref.run(params, mol, want_maps=True, want_faces=True) if ref.available() else None
    with Vpmg(params, FP64) as pmg:
        pmg.fillco(mol)
        maps = pmg.maps()
        charge = maps["charge"].copy()
        charge[16, 16, 16] = np.nan
        pmg.set_coefficients(charge, maps["epsx"], maps["epsy"], maps["epsz"], maps["kappa"],
                             maps["faces"])
        with pytest.raises(PmgbError, match="non-finite residual"):
            pmg.solve()
        pmg.fillco(mol)
        pmg.solve()
        if want is not None:
            scale = np.abs(want["u"]).max()
            assert np.abs(pmg.u - want["u"]).max() <= 1e-9 * scale


@pytest.mark.skipif(not ref.available(), reason="oracle/_ref not built")
@pytest.mark.parametrize("npbe", [False, True], ids=["lpbe", "npbe"])
def test_iteration_limit_returns_the_reference_iterate(npbe):
    mol, params = _small()
    params.nonlin = 1 if npbe else 0
    params.itmax = 1
    want = ref.run(params, mol)
    with Vpmg(params, FP64) as pmg:
        pmg.fillco(mol)
        pmg.solve()                      # success, as Vpmg_solve returns 1
        st = pmg.stats()
        u, e, hist = pmg.u, pmg.energy(), pmg.residual_history()
    assert st["converged"] == 0 and st["rel_residual"] > 1e-6
    assert (st["newton_iters"] if npbe else st["vcycles"]) == 1
    scale = np.abs(want["u"]).max()
    assert np.abs(u - want["u"]).max() <= 1e-9 * scale
    assert abs(e - want["energy_kT"]) <= 1e-9 * abs(want["energy_kT"])
    np.testing.assert_allclose(hist, want["reslog"], rtol=2e-6)
    # mixed precision stops at the same limit, also with success
    with Vpmg(params, MIXED) as pmg:
        pmg.fillco(mol)
        pmg.solve()
        st = pmg.stats()
    assert st["converged"] == 0
    # and the default limit converges
    params.itmax = 0
    with Vpmg(params, FP64) as pmg:
        pmg.fillco(mol)
        pmg.solve()
        assert pmg.stats()["converged"] == 1


@pytest.mark.parametrize("precision", [MIXED, FP64], ids=["mixed", "fp64"])
def test_bad_request_in_a_serving_mix(precision):
    rng = np.random.default_rng(12)
    jobs = []
    for i in range(8):
        dime = int(rng.choice([33, 49, 65]))
        mol = synth.cluster(int(rng.integers(80, 300)), 7.0, seed=200 + i)
        span = float(np.ptp(mol.xyz, axis=0).max()) + 14.0
        jobs.append((synth.mg_manual(dime, span / (dime - 1), mol.center(), npbe=(i == 5)),
                     mol))
    alone = []
    for p, m in jobs:
        with Vpmg(p, precision) as pmg:
            pmg.fillco(m)
            pmg.solve()
            alone.append(pmg.energy())
    bad_at = 3
    sub = list(jobs)
    sub[bad_at] = (jobs[bad_at][0], _poisoned(jobs[bad_at][1], 5, "x"))
    with serve.Server(precision, max_inflight=3) as srv:
        res = [srv.wait(i) for i in [srv.submit(p, m) for p, m in sub]]
        st = srv.stats()
    assert res[bad_at]["status"] == -1
    assert "non-finite" in res[bad_at]["error"]
    for k, (r, e0) in enumerate(zip(res, alone)):
        if k == bad_at:
            continue
        assert r["status"] == 1, r["error"]
        assert abs(r["energy_kT"] - e0) <= REL_SAME * abs(e0)
    assert st["failed"] == 1 and st["done"] == len(jobs) - 1
