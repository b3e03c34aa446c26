"""Mixed precision (FP32 V-cycles, FP64 refinement) against the FP64 path:
energy within 1e-6 relative, potential within 1e-5 of max |u|, and the same
stopping rule satisfied."""
import numpy as np
import pytest

from apbs_b200 import synth
from apbs_b200.vpmg import FP64, MIXED, Vpmg

pytestmark = pytest.mark.gpu

TOL_E = 1e-6
TOL_U = 1e-5


def _cases():
    m0, p0 = synth.config0()
    m1 = synth.cluster(300, 10.0, seed=5, net_charge=3.0)
    p1 = synth.mg_manual(65, 0.5, m1.center(), npbe=True, ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    m2 = synth.cluster(400, 12.0, seed=7)
    p2 = synth.mg_manual(97, 0.4, m2.center())
    m4 = synth.cluster(120, 6.0, seed=11, net_charge=-2.0)
    p4 = synth.mg_manual(33, 0.6, m4.center(), npbe=True, ions=((2, 0.05, 2.0), (-1, 0.1, 1.8)))
    p5 = synth.mg_manual(49, 0.8, m2.center(), npbe=True)
    # three levels: the mixed hierarchy is extended to a 6^3 (216 unknowns)
    # or 7^3 (343) coarsest level whose dense inverse runs on a 2- or 8-CTA
    # cluster (the matrix does not fit one CTA's shared memory)
    p6 = synth.mg_manual(57, 0.6, m1.center(), npbe=True, nlev=3,
                         ions=((1, 0.1, 2.0), (-1, 0.1, 2.0)))
    p7 = synth.mg_manual(65, 0.5, m0.center(), nlev=3)
    return [("lpbe65", m0, p0), ("npbe65", m1, p1), ("lpbe97", m2, p2),
            ("npbe33_2to1", m4, p4), ("npbe49", m2, p5), ("npbe57_dense216", m1, p6),
            ("lpbe65_dense343", m0, p7)]


CASES = _cases()


def _solve(params, mol, prec):
    with Vpmg(params, prec) as pmg:
        pmg.fillco(mol)
        pmg.solve()
        return pmg.energy(), pmg.u, pmg.stats()


@pytest.mark.parametrize("name,mol,params", CASES, ids=[c[0] for c in CASES])
def test_mixed_matches_fp64(name, mol, params):
    e64, u64, _ = _solve(params, mol, FP64)
    emx, umx, st = _solve(params, mol, MIXED)
    assert abs(emx - e64) <= TOL_E * abs(e64)
    assert np.abs(umx - u64).max() <= TOL_U * np.abs(u64).max()
    assert st["rel_residual"] <= 1e-6


@pytest.mark.parametrize("npbe", [False, True], ids=["lpbe", "npbe"])
def test_solver_reuse_across_molecules(npbe):
    """A calculation refilled with another molecule gives the answer of a
    fresh one (the FP32 hierarchy follows every operator rebuild)."""
    ions = ((1, 0.1, 2.0), (-1, 0.1, 2.0))
    ma = synth.cluster(150, 8.0, seed=21)
    mb = synth.cluster(150, 8.0, seed=22, net_charge=2.0)
    p = synth.mg_manual(33, 0.6, ma.center(), npbe=npbe, ions=ions)
    for prec in (FP64, MIXED):
        fresh = {}
        for name, m in (("a", ma), ("b", mb)):
            with Vpmg(p, prec) as pmg:
                pmg.fillco(m)
                pmg.solve()
                fresh[name] = pmg.energy()
        with Vpmg(p, prec) as pmg:
            for name, m in (("a", ma), ("b", mb), ("a", ma)):
                pmg.fillco(m)
                pmg.solve()
                e = pmg.energy()
                assert abs(e - fresh[name]) <= 1e-10 * abs(fresh[name]), (prec, name)
