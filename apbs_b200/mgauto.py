"""Geometry of an ``mg-auto`` focusing chain.

An mg-auto ELEC block (dime, cglen, fglen, cgcent, fgcent) becomes a chain
of mg-manual calculations: the first on the coarse box with the block's own
boundary condition, every later one focused (bcfl focus) on the one before.
The number of levels and the per-level boxes follow
NOsh_setupCalcMGAUTO (src/generic/nosh.c:1828-2101):

* spacings cgrid = cglen/(dime-1), fgrid = fglen/(dime-1);
* the spacing never shrinks by more than VREDFRAC = 0.25 per level
  (src/generic/vhal.h:392): nfocus = ceil(log(fgrid/cgrid)/log(0.25)) + 1
  on an axis where fgrid/cgrid < 0.25, else 2, the largest over the axes;
* each level's spacing and length are the previous ones times
  redrat = (fgrid/cgrid)^(1/(nfocus-1));
* the first level is centred on cgcent, the last on fgcent, the ones
  between start on fgcent and are shifted back inside the previous box
  where they stick out (by at least VSMALL = 1e-9);
* the finest box must lie inside the one before (the reference asserts).

``chain_params`` turns the chain into ``pmgb_params`` blocks for the CUDA
library (pmgb_create + pmgb_focus + pmgb_fillco + pmgb_solve per level).
"""
from __future__ import annotations

import math

from . import synth

VREDFRAC = 0.25
VSMALL = 1.0e-9


def focus_levels(dime, cglen, fglen, ccenter, fcenter):
    """The chain's boxes: a list of dicts with ``grid`` (spacing), ``glen``
    (box length) and ``center``, coarse first (NOsh_setupCalcMGAUTO)."""
    dime = [int(d) for d in dime]
    cgrid = [cglen[j] / float(dime[j] - 1) for j in range(3)]
    fgrid = [fglen[j] / float(dime[j] - 1) for j in range(3)]
    tnfocus = []
    for j in range(3):
        if fgrid[j] / cgrid[j] < VREDFRAC:
            redfrac = fgrid[j] / cgrid[j]
            td = math.log(redfrac) / math.log(VREDFRAC)
            tnfocus.append(int(math.ceil(td)) + 1)
        else:
            tnfocus.append(2)
    nfocus = max(tnfocus)
    redrat = [math.pow(fgrid[j] / cgrid[j], 1.0 / (float(nfocus) - 1.0)) for j in range(3)]
    levels = []
    for ifocus in range(nfocus):
        if ifocus == 0:
            grid = list(cgrid)
            glen = [float(cglen[j]) for j in range(3)]
            center = [float(ccenter[j]) for j in range(3)]
        else:
            prev = levels[-1]
            grid = [redrat[j] * prev["grid"][j] for j in range(3)]
            glen = [redrat[j] * prev["glen"][j] for j in range(3)]
            center = [float(fcenter[j]) for j in range(3)]
            for j in range(3):
                # fallen off the lower end of the previous mesh?
                dofix = False
                minf = center[j] - 0.5 * glen[j]
                minc = prev["center"][j] - 0.5 * prev["glen"][j]
                d = minc - minf
                if d >= VSMALL:
                    if ifocus == nfocus - 1:
                        raise ValueError("finest mesh has fallen off the coarser meshes")
                    center[j] += d
                    dofix = True
                maxf = center[j] + 0.5 * glen[j]
                maxc = prev["center"][j] + 0.5 * prev["glen"][j]
                d = maxf - maxc
                if d >= VSMALL:
                    if ifocus == nfocus - 1:
                        raise ValueError("finest mesh has fallen off the coarser meshes")
                    if dofix:
                        raise ValueError("both ends of the finer mesh do not fit the coarser one")
                    center[j] -= d
        levels.append({"grid": grid, "glen": glen, "center": center})
    return levels


def chain_params(base: "synth.PmgbParams", dime, cglen, fglen, ccenter, fcenter):
    """pmgb_params of every level of the chain: `base` carries the block's
    physics and its boundary condition (used on the first level); the grid,
    spacing and centre come from focus_levels, later levels get bcfl focus."""
    out = []
    for i, lv in enumerate(focus_levels(dime, cglen, fglen, ccenter, fcenter)):
        p = synth.PmgbParams.from_buffer_copy(base)
        p.nx, p.ny, p.nz = (int(d) for d in dime)
        p.nlev = min(synth.mgparm_nlev(int(d)) for d in dime)
        p.hx, p.hy, p.hz = lv["grid"]
        for j in range(3):
            p.center[j] = lv["center"][j]
        if i > 0:
            p.bcfl = synth.BCFL_FOCUS
        out.append(p)
    return out
