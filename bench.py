#!/usr/bin/env python
"""Benchmark of the B200 PMG solve path: PB solves/s and p50/p99 latency,
mixed precision (FP32 V-cycles + FP64 refinement) against plain FP64.

Workload (default): mg-manual NPBE, 161^3 grid, 0.4 A spacing, 5000-atom
seeded globular cluster (25 A radius, net charge +12), 0.1 M 1:1 salt,
spl2 / smol / sdh, pdie 2, sdie 78.54 -- the synthetic stand-in for the
benchmark's config of the same shape.  One step = one full calculation:
coefficient fill from device-resident atoms, operator build, solve, energy.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun (N > 1) every rank solves independent calculations (replicas;
the path has no data-path collective) and the job throughput is the sum.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "PB solves/s & p50/p99 latency, mixed vs FP64 GPU PMG at 1e-6 rel energy"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
TRAFFIC_FILE = os.path.join(ROOT, "profiles", "traffic.json")
FALLBACK_HBM_GBS = 6650.0


def workload(name: str):
    from apbs_b200 import synth
    if name == "c1":
        mol, params = synth.config1()
        desc = ("mg-manual NPBE 161^3 h=0.4A, 5000-atom cluster r=25A net +12 (seed 1), "
                "0.1M 1:1 salt, spl2/smol/sdh, pdie 2 sdie 78.54")
    elif name == "c0":
        mol, params = synth.config0()
        desc = ("mg-manual LPBE 65^3 h=0.5A, 500-atom cluster r=12A net 0 (seed 0), "
                "0.15M 1:1 salt, spl2/smol/sdh, pdie 2 sdie 78.54")
    else:
        raise SystemExit("unknown workload " + name)
    return mol, params, desc


def peak_hbm():
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def start(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()

    def _run(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.samples.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        if not self.samples:
            return None
        sm = sorted(float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit())
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for s in self.samples:
            for name, v in zip(names, s[3:7]):
                if v.strip().lower() == "active":
                    reasons.add(name)
        mx = float(self.samples[0][1]) if self.samples[0][1].replace(".", "").isdigit() else None
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(self.samples)}


def run_reference(args, rank):
    """The reference's own CPU PMG (compiled unchanged in oracle/_ref) on the
    same workload, every host thread, one full calculation per step."""
    if rank != 0:
        return
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    from oracle import ref
    mol, params, desc = workload(args.workload)
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref not built"}))
        return
    for _ in range(args.warmup):
        ref.run(params, mol)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.run(params, mol)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    v = args.steps / total
    cores = int(os.environ.get("OMP_NUM_THREADS", ncores))
    line = {
        "metric": METRIC, "impl": "reference", "value": v, "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "implementation": "reference APBS CPU PMG, OpenMP"},
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "reference",
                         "sample": "%d full calculations (ctor+fillco+solve+energy)" % args.steps},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def cpu_baseline_sample(args, n=None):
    """Reference CPU PMG timed on a bounded sample (n calculations of the
    workload).  Returns the baseline record and the last calculation's
    result (potential and energy), which the GPU results are checked
    against."""
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    try:
        from oracle import ref
        if not ref.available():
            return None, None
        mol, params, _ = workload(args.workload)
        if n is None:
            n = 2 if args.workload == "c1" else 10
        t0 = time.perf_counter()
        for _ in range(n):
            res = ref.run(params, mol)
        dt = time.perf_counter() - t0
        return ({"value": n / dt, "unit": "solves/s",
                 "cores": int(os.environ.get("OMP_NUM_THREADS", ncores)), "kind": "reference",
                 "sample": "%d full calculations of the same workload" % n}, res)
    except Exception as e:  # the baseline must not break the GPU line
        return ({"value": None, "unit": "solves/s", "cores": ncores, "kind": "reference",
                 "sample": "failed: %s" % e}, None)


def errors_vs_reference(u, e, want):
    """Potential and energy error of one GPU result against the reference's
    result for the same calculation (relative to max |u| and to |E|)."""
    import numpy as np
    ur = want["u"].reshape(-1)
    d = np.abs(u.reshape(-1) - ur)
    scale = float(np.abs(ur).max())
    return {"u_rel_max": float(d.max()) / scale,
            "u_rel_rms": float(np.sqrt(np.mean(d * d))) / scale,
            "energy_rel": abs(e - want["energy_kT"]) / abs(want["energy_kT"]),
            "energy_kT": e, "reference_energy_kT": want["energy_kT"]}


def serving_measurements(args):
    """The batched and served workloads through the native serving loop:
    the Poisson request stream (LPBE/NPBE 80/20, grids 33^3-225^3) and the
    binding-energy sweep (1 receptor + 64 complexes at 129^3, 64 ligands at
    33^3-65^3), each in mixed precision and in FP64."""
    import numpy as np

    from apbs_b200 import autotune, serve, synth
    from apbs_b200.vpmg import FP64, MIXED
    out = {}
    if args.serve_n > 0:
        stream = serve.serving_stream(args.serve_n, seed=4, rate=200.0)
        rec = {"workload": "Poisson arrivals 200/s, %d requests, LPBE/NPBE 80/20, dime "
                           "{33,65,97,129,161,225}^3, 200-8000 atoms, I ~ U[0,0.3] M (seed 4)"
                           % args.serve_n,
               "server": "8 worker streams, mixed LPBE up to 65^3 batched up to 16 per "
                         "persistent kernel, budget 80%% of free HBM, warm pools (the stream "
                         "replayed once untimed so every grid shape is resident)",
               "timed_replays": "%d, the median one reported; counters per replay" % args.serve_reps,
               "sustained": "the same stream replayed at 60%% of the precision's measured "
                            "throughput (an arrival rate the server keeps up with): "
                            "latency without queue growth"}
        counters = ("reused", "created", "evicted", "batched", "batches", "done", "failed")
        for name, prec in (("mixed", MIXED), ("fp64", FP64)):
            with serve.Server(prec, max_inflight=8) as srv:
                srv.apply_table(autotune.load_table(), prec)
                serve.replay(srv, stream, time_scale=0.0)     # resident calculations
                # the makespan of one replay hangs on where the largest requests
                # land: replay several times and keep the median run
                runs = []
                for _ in range(max(1, args.serve_reps)):
                    before = srv.stats()
                    r = serve.replay(srv, stream)
                    after = srv.stats()
                    r["counters"] = {c: after[c] - before[c] for c in counters}
                    runs.append(r)
                ordered = sorted(runs, key=lambda x: x["solves_per_s"])
                r = ordered[len(ordered) // 2]
                st = srv.stats()
                # at a sustainable arrival rate
                rate = 0.6 * r["solves_per_s"]
                sus = serve.replay(srv, stream, time_scale=200.0 / rate)
            pts = sum(q.params.nx * q.params.ny * q.params.nz for q in stream)
            errors = sorted({x["error"] for x in r["results"] if x["status"] != 1})
            rec[name] = {"solves_per_s": r["solves_per_s"],
                         "solves_per_s_runs": [x["solves_per_s"] for x in runs],
                         "p50_ms": r["p50_ms"],
                         "p99_ms": r["p99_ms"], "failed": r["failed"], "errors": errors,
                         "wall_s": r["wall_s"],
                         "grid_points_per_s": pts / r["wall_s"],
                         "mean_service_ms": st["mean_service_ms"],
                         "inflight_peak": st["inflight_peak"], "bytes_peak": st["bytes_peak"],
                         "reported_replay": r["counters"],
                         "sustained": {"arrivals_per_s": rate,
                                       "solves_per_s": sus["solves_per_s"],
                                       "p50_ms": sus["p50_ms"], "p99_ms": sus["p99_ms"],
                                       "failed": sus["failed"]}}
            rec[name + "_energies"] = [x["energy_kT"] for x in r["results"]]
        e_mx = np.array(rec.pop("mixed_energies"))
        e_64 = np.array(rec.pop("fp64_energies"))
        both = (e_mx != 0.0) & (e_64 != 0.0)
        rec["energy_rel_err_max"] = float(np.max(np.abs(e_mx[both] - e_64[both]) /
                                                 np.abs(e_64[both])))
        rec["mixed_vs_fp64"] = rec["mixed"]["solves_per_s"] / rec["fp64"]["solves_per_s"]
        out["serving"] = rec
    if args.sweep_poses > 0:
        rec_job, pairs = synth.binding_sweep(args.sweep_poses, etol=1e-9)
        jobs = [rec_job] + [j for pr in pairs for j in pr]
        rec = {"workload": "binding sweep: 3000-atom receptor + %d poses of a 40-atom ligand, "
                           "complexes 129^3 at 0.55 A, ligands 33-65^3 on the same lattice, "
                           "%d LPBE solves to a 1e-9 relative residual"
                           % (args.sweep_poses, len(jobs))}
        energies = {}
        for name, prec in (("mixed", MIXED), ("fp64", FP64)):
            with serve.Server(prec, max_inflight=8) as srv:
                srv.apply_table(autotune.load_table(), prec)
                # untimed pass first: every grid shape resident, as for the stream
                serve.replay(srv, [serve.StreamRequest(0.0, p, m) for p, m in jobs], 0.0)
                t0 = time.perf_counter()
                ids = [srv.submit(p, m) for p, m in jobs]
                res = [srv.wait(i) for i in ids]
                wall = time.perf_counter() - t0
                st = srv.stats()
            energies[name] = np.array([x["energy_kT"] for x in res])
            pts = sum(p.nx * p.ny * p.nz for p, _ in jobs)
            rec[name] = {"solves_per_s": len(jobs) / wall, "wall_s": wall,
                         "grid_points_per_s": pts / wall,
                         "failed": sum(1 for x in res if x["status"] != 1),
                         "batched_requests": st["batched"], "batch_launches": st["batches"]}
        kcal = 1.380662e-23 * 298.15 * 6.022045e23 / 4184.0
        dg = {}
        for name, e in energies.items():
            dg[name] = np.array([e[1 + 2 * k] - e[0] - e[2 + 2 * k] for k in range(len(pairs))])
        rec["dG_max_abs_diff_kcal"] = float(np.max(np.abs(dg["mixed"] - dg["fp64"])) * kcal)
        rec["dG_range_kcal"] = [float(dg["fp64"].min() * kcal), float(dg["fp64"].max() * kcal)]
        rec["mixed_vs_fp64"] = rec["mixed"]["solves_per_s"] / rec["fp64"]["solves_per_s"]
        out["batch"] = rec
    return out


def profile_batch(args):
    """Profiling mode: the binding sweep's 64 ligands (33-65^3 LPBE, mixed)
    solved by the persistent batched kernel, `--warmup` untimed launches and
    `--steps` timed ones."""
    import torch

    from apbs_b200 import synth
    from apbs_b200.vpmg import MIXED, Vpmg, batch_solve
    _, pairs = synth.binding_sweep(64)
    ligs = [pr[1] for pr in pairs]
    calcs = [Vpmg(p, MIXED) for p, _ in ligs]
    for c, (_, m) in zip(calcs, ligs):
        c.fillco(m)
    for _ in range(max(args.warmup, 1)):
        batch_solve(calcs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        batch_solve(calcs)
    torch.cuda.synchronize()
    ms = 1e3 * (time.perf_counter() - t0) / max(args.steps, 1)
    print(json.dumps({"profile_run": "batch", "calculations": len(calcs), "ms_per_launch": ms,
                      "solves_per_s": len(calcs) / (ms * 1e-3)}), flush=True)
    for c in calcs:
        c.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="c1", choices=["c1", "c0"])
    ap.add_argument("--headline", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-n", type=int, default=300,
                    help="requests in the serving-stream measurement (0 skips it)")
    ap.add_argument("--serve-reps", type=int, default=5,
                    help="timed replays of the request stream (the median one is reported)")
    ap.add_argument("--sweep-poses", type=int, default=64,
                    help="poses of the binding-energy sweep measurement (0 skips it)")
    ap.add_argument("--only", choices=["mixed", "fp64", "batch"], default=None,
                    help="profiling mode: run the steps of one precision (or the batched "
                         "kernel on the binding sweep's ligands) and nothing else")
    ap.add_argument("--tune", action="append", default=[], metavar="KEY=VALUE",
                    help="override one launch-shape tunable of the benchmark calculations "
                         "after the tuning table (names as in the JSON line's config.tuning, "
                         "e.g. gs7_sweep_shape=1)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.only == "batch":
        profile_batch(args)
        return

    import numpy as np
    import torch
    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    from apbs_b200 import vpmg

    mol, params, desc = workload(args.workload)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.Stream(device=dev)
    d_xyz = torch.tensor(mol.xyz.reshape(-1), dtype=torch.float64, device=dev)
    d_q = torch.tensor(mol.charge, dtype=torch.float64, device=dev)
    d_r = torch.tensor(mol.radius, dtype=torch.float64, device=dev)
    # pinned host copies for the end-to-end leg
    h_xyz = torch.tensor(mol.xyz.reshape(-1), dtype=torch.float64).pin_memory()
    h_q = torch.tensor(mol.charge, dtype=torch.float64).pin_memory()
    h_r = torch.tensor(mol.radius, dtype=torch.float64).pin_memory()

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    from apbs_b200 import replicas
    if world > 1:
        max_over_ranks, sum_over_ranks = replicas.torch_reducers(dist, dev)
    else:
        max_over_ranks = sum_over_ranks = (lambda x: x)

    results = {}
    potentials = {}
    precisions = [("fp64", vpmg.FP64), ("mixed", vpmg.MIXED)]
    if args.only:
        precisions = [p for p in precisions if p[0] == args.only]
    from apbs_b200 import autotune
    table = autotune.load_table()
    solvers = {}
    tuned = {}
    for name, prec in precisions:
        s = vpmg.Vpmg(params, prec)
        tuned[name] = autotune.apply(s, table)   # launch shapes from the autotuner's table
        for kv in args.tune:
            key, val = kv.split("=")
            ids = [k for k, n in autotune.KEY_NAMES.items() if n == key]
            if not ids:
                raise SystemExit("--tune: unknown key %r" % key)
            s.set_tuning(ids[0], int(val, 0))
            tuned[name][ids[0]] = int(val, 0)
        s.set_stream(stream.cuda_stream)
        solvers[name] = s

    def step(s):
        s.fillco_device(mol.natoms, d_xyz.data_ptr(), d_q.data_ptr(), d_r.data_ptr())
        s.solve()
        return s.energy()

    clocks = None
    for name, prec in precisions:
        s = solvers[name]
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                e = step(s)
        barrier()
        sampler = ClockSampler(local_rank) if name == args.headline else None
        if sampler:
            sampler.start()
        vpmg.lib().pmgb_launch_count(1)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
        with torch.cuda.stream(stream):
            ev[0].record(stream)
            for i in range(args.steps):
                e = step(s)
                ev[i + 1].record(stream)
        barrier()
        launches = vpmg.lib().pmgb_launch_count(1)
        if sampler:
            clocks = sampler.stop()
        lat = [ev[i].elapsed_time(ev[i + 1]) for i in range(args.steps)]
        rate, total_ms = replicas.aggregate(args.steps, ev[0].elapsed_time(ev[-1]),
                                            max_over_ranks, sum_over_ranks)
        st = s.stats()
        potentials[name] = s.u
        results[name] = {
            "solves_per_s": rate,
            "ms_per_step": total_ms / args.steps,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "energy_kT": e, "vcycles": st["vcycles"], "newton_iters": st["newton_iters"],
            "rel_residual": st["rel_residual"], "t_fill_ms": st["t_fill_ms"],
            "t_setup_ms": st["t_setup_ms"], "t_solve_ms": st["t_solve_ms"],
            "gpu_launches": int(launches),
        }

    if args.only:
        for s in solvers.values():
            s.close()
        if rank == 0:
            print(json.dumps({"profile_run": args.only, **results[args.only]}), flush=True)
        return

    head = results[args.headline]
    e64 = results["fp64"]["energy_kT"]
    emix = results["mixed"]["energy_kT"]

    # end to end through the C ABI from pinned host buffers (H2D of the atoms,
    # D2H of the energy), headline precision
    s = solvers[args.headline]
    class _HostMol:
        natoms = mol.natoms
        xyz = h_xyz.numpy()      # pinned memory, shared with the torch tensors
        charge = h_q.numpy()
        radius = h_r.numpy()
    hm = _HostMol()
    # the potential comes back every step, as Vpmg_solve leaves it in thee->u
    h_u = torch.empty(params.nx * params.ny * params.nz, dtype=torch.float64).pin_memory()
    h_u_np = h_u.numpy()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for _ in range(args.steps):
            s.fillco(hm)
            s.solve()
            s.energy()
            s.potential_into(h_u_np)
        ev1.record(stream)
    barrier()
    e2e_rate, e2e_ms = replicas.aggregate(args.steps, ev0.elapsed_time(ev1), max_over_ranks,
                                          sum_over_ranks)
    e2e = {"value": e2e_rate, "unit": "solves/s",
           "h2d_bytes_per_step": int(8 * (h_xyz.numel() + h_q.numel() + h_r.numel())),
           "d2h_bytes_per_step": int(8 + 8 * h_u.numel()),
           "returns": "energy (8 B) and the potential grid (nx*ny*nz doubles) to pinned "
                      "host memory every step"}

    # roofline of the dominant kernel of the headline path (largest share of
    # the ncu launch list in profiles/: the FP32 fine smoother of the mixed
    # path, the ordered GS27 wavefront of the FP64 one), timed live on the
    # headline stream
    peak, peak_kind = peak_hbm()
    if args.headline == "mixed":
        # the fine smoother the tuned calculation runs: FP32 single-pass
        # sweeps or one launch per colour
        ksolver = solvers["mixed"]
        if ksolver.get_tuning(vpmg.TUNE_GS7_COLOUR_PASSES) == 2:
            kern, kname = vpmg.K_GS7_SWEEP_FP32, "k_gs7_rb<float>"
        else:
            kern, kname = vpmg.K_GS7_FP32, "k_gs7_f32"
    else:
        kern, kname, ksolver = vpmg.K_GS27_WAVE, "k_gs27_wave", solvers["fp64"]
    ms, nbytes = ksolver.time_kernel(kern, 10)
    achieved = nbytes / (ms * 1e-3) / 1e9
    traffic = None
    try:
        with open(TRAFFIC_FILE) as f:
            traffic = json.load(f).get(kname)
    except Exception:
        pass
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic,
                "bytes_per_launch": nbytes, "ms_per_launch": ms,
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs, burst copy)"}
    # the fine-level smoothers (HBM-bound), FP64 and FP32
    smoothers = {}
    for nm, sv, k in (("k_gs7_rb<double>", solvers["fp64"], vpmg.K_GS7_SWEEP_FP64),
                      ("k_gs7_rb<float>", solvers["mixed"], vpmg.K_GS7_SWEEP_FP32),
                      ("k_gs7_colour", solvers["fp64"], vpmg.K_GS7_FP64),
                      ("k_gs7_f32", solvers["mixed"], vpmg.K_GS7_FP32)):
        ms_k, b_k = sv.time_kernel(k, 20)
        ach = b_k / (ms_k * 1e-3) / 1e9
        smoothers[nm] = {"achieved": ach, "frac": ach / peak, "ms_per_launch": ms_k,
                         "bytes_per_launch": b_k}

    extra = {}
    if world == 1:
        for sv in solvers.values():
            sv.close()
        extra = serving_measurements(args)

    cpu, err_ref = None, None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, want = cpu_baseline_sample(args)
        if want is not None:
            # error of every GPU result against the reference's own run of
            # the same calculation
            err_ref = {name: errors_vs_reference(potentials[name], results[name]["energy_kT"],
                                                 want)
                       for name in results}

    if rank == 0:
        line = {
            "metric": METRIC, "value": head["solves_per_s"], "unit": "solves/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64" if args.headline == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": desc, "headline": args.headline,
                       "step": "fillco (device atoms) + build + solve + energy",
                       "l2": "working set ~1 GB per calculation, larger than L2",
                       "parallelism": "replicas x%d" % world,
                       "tuning": {"table": "apbs_b200/tuning/b200.json",
                                  "mixed": {autotune.KEY_NAMES.get(k, str(k)): v
                                            for k, v in tuned.get("mixed", {}).items()},
                                  "fp64": {autotune.KEY_NAMES.get(k, str(k)): v
                                           for k, v in tuned.get("fp64", {}).items()}}},
            "latency_ms": head["latency_ms"],
            "fp64": results["fp64"], "mixed": results["mixed"],
            "mixed_vs_fp64": {"speedup": results["mixed"]["solves_per_s"] /
                              results["fp64"]["solves_per_s"],
                              "energy_rel_err": abs(emix - e64) / abs(e64)},
            "err_vs_reference": err_ref,
            "e2e": e2e, "gpu_launches": head["gpu_launches"],
            "roofline": roofline, "smoothers": smoothers,
            "cpu_baseline": cpu, "clocks": clocks, **extra,
        }
        print(json.dumps(line), flush=True)

    for s in solvers.values():
        s.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
