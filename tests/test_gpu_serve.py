"""The serving loop on the device: every result is the same alone and in the
mix, admission stays within the memory budget, and the binding-energy sweep
through the loop in mixed precision agrees with per-solve FP64."""
import numpy as np
import pytest

from apbs_b200 import serve, synth
from apbs_b200.vpmg import FP64, MIXED, Vpmg

pytestmark = pytest.mark.gpu

REL_SAME = 1e-10     # alone vs in the mix (only FP64 atomic-add order differs)
KCAL_PER_KT = 0.5924838  # kT at 298.15 K in kcal/mol (k_B T N_A / 4184)


def _mix(n=12, seed=8):
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n):
        dime = int(rng.choice([33, 49, 65, 97]))
        natoms = int(rng.integers(100, 800))
        mol = synth.cluster(natoms, 9.0 * (natoms / 300) ** (1 / 3), seed=100 + i,
                            net_charge=float(rng.integers(-3, 4)))
        span = float(np.ptp(mol.xyz, axis=0).max()) + 14.0
        conc = float(rng.uniform(0.0, 0.3))
        ions = ((1.0, conc, 2.0), (-1.0, conc, 2.0))
        jobs.append((synth.mg_manual(dime, span / (dime - 1), mol.center(),
                                     npbe=bool(i % 4 == 3), ions=ions), mol))
    return jobs


@pytest.mark.parametrize("precision", [MIXED, FP64], ids=["mixed", "fp64"])
def test_results_same_alone_and_in_mix(precision):
    jobs = _mix()
    alone = []
    for p, m in jobs:
        with Vpmg(p, precision) as pmg:
            pmg.fillco(m)
            pmg.solve()
            alone.append((pmg.energy(), pmg.u))
    outs = [np.empty((p.nz, p.ny, p.nx)) for p, _ in jobs]
    budget = 3 * max(serve.footprint(p, precision, m.natoms) for p, m in jobs)
    with serve.Server(precision, max_inflight=4, hbm_budget_bytes=budget) as srv:
        ids = [srv.submit(p, m, u_out=o) for (p, m), o in zip(jobs, outs)]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for (e0, u0), r, u in zip(alone, res, outs):
        assert r["status"] == 1, r["error"]
        assert abs(r["energy_kT"] - e0) <= REL_SAME * abs(e0)
        assert np.abs(u - u0).max() <= REL_SAME * np.abs(u0).max()
    assert st["done"] == len(jobs)
    assert st["bytes_peak"] <= budget
    assert st["inflight_peak"] > 1           # requests overlapped on the device
    if precision == MIXED:                   # small LPBE requests shared persistent kernels
        assert st["batched"] >= 2 and st["batch_peak"] >= 2


def test_mixed_in_mix_matches_fp64_alone():
    jobs = _mix(6, seed=9)
    with serve.Server(MIXED, max_inflight=3) as srv:
        res = [srv.wait(i) for i in [srv.submit(p, m) for p, m in jobs]]
    for (p, m), r in zip(jobs, res):
        with Vpmg(p, FP64) as pmg:
            pmg.fillco(m)
            pmg.solve()
            e64 = pmg.energy()
        assert abs(r["energy_kT"] - e64) <= 1e-6 * abs(e64)


def test_binding_sweep_through_the_loop_matches_fp64():
    """A reduced binding sweep (4 poses, 97^3 complexes) solved to a 1e-9
    relative residual: dG from mixed precision through the loop agrees with
    per-solve FP64 to 0.01 kcal/mol."""
    rec, pairs = synth.binding_sweep(npose=4, rec_atoms=600, rec_radius=11.0, rec_dime=97,
                                     lig_dimes=(33, 49), h=0.6, etol=1e-9)
    jobs = [rec] + [j for pr in pairs for j in pr]
    with serve.Server(MIXED, max_inflight=4) as srv:
        res = [srv.wait(i) for i in [srv.submit(p, m) for p, m in jobs]]
    e_mx = [r["energy_kT"] for r in res]
    e_64 = []
    for p, m in jobs:
        with Vpmg(p, FP64) as pmg:
            pmg.fillco(m)
            pmg.solve()
            e_64.append(pmg.energy())
    for k in range(len(pairs)):
        dg_mx = e_mx[1 + 2 * k] - e_mx[0] - e_mx[2 + 2 * k]
        dg_64 = e_64[1 + 2 * k] - e_64[0] - e_64[2 + 2 * k]
        assert abs(dg_mx - dg_64) * KCAL_PER_KT <= 0.01


def test_tuned_loop_matches_tuned_solves():
    """With the B200 tuning table applied per grid shape (as the benchmark
    runs the loop), every request succeeds and gives the energy of the same
    calculation solved alone with the same table, in mixed precision: the
    batched kernel takes the tuned calculations too (it widens a tail limit
    that would keep level 1 outside its cluster)."""
    from apbs_b200 import autotune
    table = autotune.load_table()
    jobs = _mix(10, seed=21)
    alone = []
    for p, m in jobs:
        with Vpmg(p, MIXED) as pmg:
            autotune.apply(pmg, table)
            pmg.fillco(m)
            pmg.solve()
            alone.append(pmg.energy())
    with serve.Server(MIXED, max_inflight=4) as srv:
        srv.apply_table(table, MIXED)
        res = [srv.wait(i) for i in [srv.submit(p, m) for p, m in jobs]]
        st = srv.stats()
    for r, e0 in zip(res, alone):
        assert r["status"] == 1, r["error"]
        assert abs(r["energy_kT"] - e0) <= 1e-9 * abs(e0)
    assert st["failed"] == 0 and st["batched"] >= 2
