"""Autotuner for the launch shapes of the PMG kernels.

Each calculation carries its own launch-shape tunables (PMGB_TUNE_* in
include/apbs_b200.h): which ordered 27-point wavefront runs on which levels
(one CTA per plane or one cluster) and the cluster size on the middle levels, the fine smoother's kernel and its plane chunk,
and the size limit of the one-cluster coarse V-cycle tail of the
mixed-precision path, and the smoothing counts of the mixed path's inner FP32
V-cycle.  The FP64 keys change no result at all; the mixed keys change the
path to the converged solution (the same stopping test holds), so the best
values are a speed question that depends on the grid shape and the device.

The tuner times whole solves of the actual problem (device time of
pmgb_solve from CUDA events, best of a few after a warm-up solve that
captures the V-cycle graph) and searches by coordinate descent: one key at a
time over its candidate values, keeping a change only if it is faster by
more than a margin.  Results go to a table keyed by grid shape, precision
and equation, stored as JSON (apbs_b200/tuning/b200.json holds the table
made on a B200 for the benchmark's shapes); `apply` sets a calculation's
tunables from it and the serving loop applies it per shape.

    python -m apbs_b200.autotune --out apbs_b200/tuning/b200.json
"""
from __future__ import annotations

import argparse
import json
import os
from typing import Callable

from . import vpmg
from .vpmg import (FP64, MIXED, TUNE_GS27_CLUSTER, TUNE_GS27_CLUSTER_MID, TUNE_GS27_PLANES,
                   TUNE_GS7_COLOUR_PASSES, TUNE_GS7_SWEEP_KCHUNK, TUNE_GS7_SWEEP_SHAPE,
                   TUNE_MC_COOPERATIVE, TUNE_MIXED_CHEBYSHEV, TUNE_MIXED_COARSE_SWEEPS,
                   TUNE_MIXED_FINE_SWEEPS, TUNE_TAIL_MAX_POINTS)

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_TABLE = os.path.join(HERE, "tuning", "b200.json")

# candidate values per key; the first value of each list is the default
CANDIDATES = {
    FP64: {
        vpmg.TUNE_GS27_LAG: [6, 4, 8, 12],
        TUNE_GS27_PLANES: [0, 2, 1],
        TUNE_GS27_CLUSTER_MID: [0, 4, 16],
        TUNE_GS7_COLOUR_PASSES: [0, 1],
        TUNE_GS7_SWEEP_SHAPE: [0x12, 0x11, 0x02, 0x21],
        TUNE_GS7_SWEEP_KCHUNK: [0, 8, 10, 12],
    },
    MIXED: {
        TUNE_MIXED_CHEBYSHEV: [2, 0, 4],
        TUNE_TAIL_MAX_POINTS: [70000, 20000, 5000],
        TUNE_MIXED_FINE_SWEEPS: [2, 1, 3, 4],
        TUNE_MIXED_COARSE_SWEEPS: [2, 1, 3],
        TUNE_GS7_COLOUR_PASSES: [0, 2],
        TUNE_GS7_SWEEP_SHAPE: [0x12, 0x21, 0x11],
        TUNE_GS7_SWEEP_KCHUNK: [0, 6, 8],
        TUNE_GS27_CLUSTER_MID: [0, 4, 16],
    },
}

KEY_NAMES = {TUNE_GS27_CLUSTER: "gs27_cluster", TUNE_GS27_CLUSTER_MID: "gs27_cluster_mid",
             vpmg.TUNE_GS27_LAG: "gs27_lag",
             TUNE_GS27_PLANES: "gs27_planes",
             TUNE_GS7_COLOUR_PASSES: "gs7_colour_passes", TUNE_GS7_SWEEP_KCHUNK: "gs7_sweep_kchunk",
             TUNE_TAIL_MAX_POINTS: "tail_max_points", TUNE_MC_COOPERATIVE: "mc_cooperative",
             TUNE_MIXED_COARSE_SWEEPS: "mixed_coarse_sweeps",
             TUNE_MIXED_FINE_SWEEPS: "mixed_fine_sweeps",
             vpmg.TUNE_GS7_SWEEP_SHAPE: "gs7_sweep_shape",
             vpmg.TUNE_MIXED_CHEBYSHEV: "mixed_chebyshev"}


def shape_key(params, precision: int) -> str:
    """Table key: grid, level count, precision and equation."""
    return "%dx%dx%d/%d/%s/%s" % (params.nx, params.ny, params.nz, params.nlev,
                                  "mixed" if precision == MIXED else "fp64",
                                  "npbe" if params.nonlin else "lpbe")


def coordinate_descent(candidates: dict, measure: Callable[[dict], float],
                       margin: float = 0.02) -> tuple[dict, float, list]:
    """Search `candidates` ({key: [default, alternatives...]}) one key at a
    time; `measure(config)` returns a time (lower is better) for a full
    config {key: value}.  A change is kept only if it beats the current best
    by more than `margin` (relative).  Returns (best config, its time, the
    list of (config, time) measured)."""
    best = {k: v[0] for k, v in candidates.items()}
    best_t = measure(dict(best))
    trials = [(dict(best), best_t)]
    for key, values in candidates.items():
        for v in values[1:]:
            cfg = dict(best)
            cfg[key] = v
            t = measure(cfg)
            trials.append((cfg, t))
            if t < best_t * (1.0 - margin):
                best, best_t = cfg, t
    return best, best_t, trials


def solve_time_ms(pmg: "vpmg.Vpmg", mol, reps: int = 3) -> float:
    """Best device time of pmgb_solve over `reps` solves after one warm-up."""
    pmg.fillco(mol)
    pmg.solve()
    best = float("inf")
    for _ in range(reps):
        pmg.solve()
        best = min(best, pmg.stats()["t_solve_ms"])
    return best


def tune(params, mol, precision: int, reps: int = 3, candidates: dict | None = None) -> dict:
    """Tune one problem on the current device; returns a table entry."""
    cands = candidates if candidates is not None else CANDIDATES[precision]
    with vpmg.Vpmg(params, precision) as pmg:
        def measure(cfg):
            for k, v in cfg.items():
                pmg.set_tuning(k, v)
            return solve_time_ms(pmg, mol, reps)
        best, best_t, trials = coordinate_descent(cands, measure)
    default_t = trials[0][1]
    return {"tune": {str(k): int(v) for k, v in best.items()}, "ms": best_t,
            "default_ms": default_t,
            "trials": [{"tune": {KEY_NAMES.get(k, str(k)): v for k, v in c.items()}, "ms": t}
                       for c, t in trials]}


def load_table(path: str = DEFAULT_TABLE) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f).get("entries", {})


def save_table(entries: dict, path: str = DEFAULT_TABLE, device: str = "") -> None:
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "w") as f:
        json.dump({"device": device, "entries": entries}, f, indent=1, sort_keys=True)


def lookup(table: dict, params, precision: int) -> dict:
    """{key: value} for this shape, or {} (defaults)."""
    e = table.get(shape_key(params, precision))
    return {int(k): int(v) for k, v in e["tune"].items()} if e else {}


def apply(pmg: "vpmg.Vpmg", table: dict) -> dict:
    """Set a calculation's tunables from the table; returns what was set."""
    cfg = lookup(table, pmg.params, pmg.precision)
    for k, v in cfg.items():
        pmg.set_tuning(k, v)
    return cfg


def _bench_problems():
    """The benchmark's shapes: the 161^3 NPBE workload, the focusing and
    binding-sweep grids, and the serving stream's grid sizes (LPBE)."""
    from . import synth
    mol1, p1 = synth.config1()
    out = [(p1, mol1)]
    p_l = synth.mg_manual(161, 0.4, mol1.center(), ions=((1.0, 0.1, 2.0), (-1.0, 0.1, 2.0)))
    out.append((p_l, mol1))
    for dime in (33, 65, 97, 129, 225):
        natoms = {33: 500, 65: 1500, 97: 3000, 129: 4000, 225: 6000}[dime]
        m = synth.cluster(natoms, 12.0 * (natoms / 500.0) ** (1.0 / 3.0), seed=dime)
        span = float((m.xyz.max(axis=0) - m.xyz.min(axis=0)).max()) + 14.0
        for npbe in (False, True):
            out.append((synth.mg_manual(dime, span / (dime - 1), m.center(), npbe=npbe,
                                        ions=((1.0, 0.1, 2.0), (-1.0, 0.1, 2.0))), m))
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    import torch
    dev = torch.cuda.get_device_name(0)
    entries = load_table(args.out)
    for params, mol in _bench_problems():
        for prec in (MIXED, FP64):
            key = shape_key(params, prec)
            e = tune(params, mol, prec, args.reps)
            entries[key] = e
            print(json.dumps({"shape": key, "ms": round(e["ms"], 3),
                              "default_ms": round(e["default_ms"], 3), "tune": e["tune"]}),
                  flush=True)
    save_table(entries, args.out, dev)


if __name__ == "__main__":
    main()
