"""Runs the reference's regression decks (fixtures in tests/golden/, made by
tests/golden/make_fixtures.py) through a solver and checks the energies the
way the reference's test harness does (tests/apbs_check_results.py:27-54 in
the APBS tree: both values rounded to 6 significant figures, equal or within
1e-4 relative).

A deck is a list of ELEC blocks.  An mg-manual block is one calculation; an
mg-auto block is the focusing chain NOsh_setupCalcMGAUTO makes of it
(apbs_b200.mgauto).  The values are every calculation's total energy in
kJ/mol, in order (energyMG, src/routines.c:1756-1760), then every print
statement's sum (printElecEnergy, src/routines.c:3082-3105), which takes the
last calculation of each named block."""
import json
import math
import os

import numpy as np

from apbs_b200 import mgauto, synth

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
FIXTURES = sorted(f[:-5] for f in os.listdir(HERE) if f.endswith(".json"))

_SRFM = {"mol": synth.SRFM_MOL, "smol": synth.SRFM_SMOL, "spl2": synth.SRFM_SPL2,
         "spl4": synth.SRFM_SPL4}
_CHGM = {"spl0": synth.CHGM_TRIL, "spl2": synth.CHGM_SPL2}
_BCFL = {"zero": synth.BCFL_ZERO, "sdh": synth.BCFL_SDH, "mdh": synth.BCFL_MDH,
         "focus": synth.BCFL_FOCUS}


def load(name):
    with open(os.path.join(HERE, name + ".json")) as f:
        return json.load(f)


def molecule(fx, index):
    """Molecule `index` (1-based, as the deck's "mol N") of the read block."""
    a = np.array(fx["molecules"][index - 1]["atoms"], dtype=np.float64).reshape(-1, 5)
    return synth.Molecule(a[:, :3].copy(), a[:, 3].copy(), a[:, 4].copy())


def _center(fx, spec):
    if isinstance(spec, dict):
        return molecule(fx, spec["mol"]).center()
    return np.array(spec, dtype=np.float64)


def block_levels(fx, blk):
    """The calculations of one ELEC block: a list of pmgb_params (coarse
    first; one entry for mg-manual) and the block's molecule."""
    dime = [int(d) for d in blk["dime"]]
    base = synth.mg_manual(dime, (1.0, 1.0, 1.0), (0.0, 0.0, 0.0),
                           npbe=(blk.get("eq") == "npbe"), srfm=_SRFM[blk["srfm"]],
                           bcfl=_BCFL[blk["bcfl"]], pdie=blk["pdie"], sdie=blk["sdie"],
                           srad=blk["srad"], sdens=blk["sdens"], temp=blk["temp"],
                           ions=[tuple(i) for i in blk["ions"]])
    base.chgm = _CHGM[blk["chgm"]]
    base.swin = blk["swin"]
    if blk["type"] == "mg-auto":
        levels = mgauto.chain_params(base, dime, blk["cglen"], blk["fglen"],
                                     _center(fx, blk["cgcent"]), _center(fx, blk["fgcent"]))
    else:
        grid = blk["grid"] if "grid" in blk else [blk["glen"][j] / (dime[j] - 1)
                                                  for j in range(3)]
        base.hx, base.hy, base.hz = grid
        c = _center(fx, blk["gcent"])
        for j in range(3):
            base.center[j] = c[j]
        levels = [base]
    return levels, molecule(fx, blk["mol"])


def deck_values(fx, solve_chain):
    """All values the reference's harness compares, in kJ/mol.
    solve_chain(levels, mol) returns the total energy (kT) of every level."""
    kb, na = fx["units"]["Vunit_kb"], fx["units"]["Vunit_Na"]
    values, last = [], {}
    for blk in fx["elec"]:
        levels, mol = block_levels(fx, blk)
        e_kt = solve_chain(levels, mol)
        for e in e_kt:
            values.append(kb * blk["temp"] * (1e-3) * na * e)
        last[blk["name"]] = (e_kt[-1], blk["temp"])
    for terms in fx["print"]:
        tot = 0.0
        for k, (sign, name) in enumerate(terms):
            e, temp = last[name]
            v = kb * (1e-3) * na * temp * e
            tot = v if k == 0 else tot + sign * v
        values.append(tot)
    return values


def round_sigfigs(x, sig):
    return round(x, sig - int(math.floor(math.log10(abs(x)))) - 1)


def mismatches(computed, expected):
    """(index, computed, expected, relative error) of every value the
    reference's rule rejects."""
    bad = []
    for i, (c, e) in enumerate(zip(computed, expected)):
        cr, er = round_sigfigs(c, 6), round_sigfigs(e, 6)
        err = abs((cr - er) / er)
        if not (cr == er or err < 1e-4):
            bad.append((i, c, e, err))
    if len(computed) != len(expected):
        bad.append(("count", len(computed), len(expected), None))
    return bad
