"""ctypes binding of the serving loop (pmgb_server_* in include/apbs_b200.h)
and the request streams it is measured on.

The loop itself is native (apbs_b200/csrc/serve.cu): worker threads with
their own CUDA streams, admission by device footprint, a pool of resident
calculations reused per grid shape.  This module submits requests, waits for
them and replays arrival schedules.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np

from . import synth
from .vpmg import FP64, MIXED, PmgbStats, lib as _core_lib  # noqa: F401

_bound = False


class ServerConfig(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int), ("max_inflight", ctypes.c_int),
                ("hbm_budget_bytes", ctypes.c_size_t), ("pool_per_shape", ctypes.c_int),
                ("max_batch", ctypes.c_int)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("energy_kT", ctypes.c_double),
                ("latency_ms", ctypes.c_double), ("queue_ms", ctypes.c_double),
                ("service_ms", ctypes.c_double), ("admit_order", ctypes.c_longlong),
                ("stats", PmgbStats),
                ("error", ctypes.c_char * 256)]

    def as_dict(self):
        return {"status": self.status, "energy_kT": self.energy_kT,
                "latency_ms": self.latency_ms, "queue_ms": self.queue_ms,
                "service_ms": self.service_ms, "admit_order": self.admit_order,
                "stats": self.stats.as_dict(),
                "error": self.error.decode(errors="replace")}


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_longlong), ("done", ctypes.c_longlong),
                ("failed", ctypes.c_longlong), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("mean_service_ms", ctypes.c_double), ("bytes_in_use", ctypes.c_size_t),
                ("bytes_peak", ctypes.c_size_t), ("budget", ctypes.c_size_t),
                ("created", ctypes.c_longlong), ("reused", ctypes.c_longlong),
                ("evicted", ctypes.c_longlong), ("inflight_peak", ctypes.c_int),
                ("batches", ctypes.c_longlong), ("batched", ctypes.c_longlong),
                ("batch_peak", ctypes.c_int)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


FOOTPRINT = ctypes.CFUNCTYPE(ctypes.c_size_t, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                             ctypes.c_int)
CREATE = ctypes.CFUNCTYPE(ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int)
RECONFIGURE = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p)
RUN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                       ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))
DESTROY = ctypes.CFUNCTYPE(None, ctypes.c_void_p, ctypes.c_void_p)


class Backend(ctypes.Structure):
    """Mirror of pmgb_server_backend: the device side as callbacks."""
    _fields_ = [("ctx", ctypes.c_void_p), ("footprint", FOOTPRINT), ("create", CREATE),
                ("reconfigure", RECONFIGURE), ("run", RUN), ("destroy", DESTROY)]


def lib():
    global _bound
    L = _core_lib()
    if not _bound:
        vp, dp = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        L.pmgb_server_create.argtypes = [ctypes.POINTER(ServerConfig), ctypes.POINTER(vp)]
        L.pmgb_server_create.restype = ctypes.c_int
        L.pmgb_server_create_ex.argtypes = [ctypes.POINTER(ServerConfig),
                                            ctypes.POINTER(Backend), ctypes.POINTER(vp)]
        L.pmgb_server_create_ex.restype = ctypes.c_int
        L.pmgb_server_submit.argtypes = [vp, vp, ctypes.c_int, dp, dp, dp, dp]
        L.pmgb_server_submit.restype = ctypes.c_longlong
        L.pmgb_server_poll.argtypes = [vp, ctypes.c_longlong, ctypes.POINTER(Result)]
        L.pmgb_server_poll.restype = ctypes.c_int
        L.pmgb_server_wait.argtypes = [vp, ctypes.c_longlong, ctypes.POINTER(Result)]
        L.pmgb_server_wait.restype = ctypes.c_int
        L.pmgb_server_drain.argtypes = [vp]
        L.pmgb_server_drain.restype = ctypes.c_int
        L.pmgb_server_get_stats.argtypes = [vp, ctypes.POINTER(ServerStats)]
        L.pmgb_server_get_stats.restype = ctypes.c_int
        L.pmgb_server_destroy.argtypes = [vp]
        L.pmgb_server_destroy.restype = None
        L.pmgb_server_set_shape_tuning.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int]
        L.pmgb_server_set_shape_tuning.restype = ctypes.c_int
        L.pmgb_footprint.argtypes = [vp, ctypes.c_int, ctypes.c_int]
        L.pmgb_footprint.restype = ctypes.c_size_t
        _bound = True
    return L


def footprint(params, precision, natoms) -> int:
    """Device bytes of one calculation (pmgb_footprint)."""
    return int(lib().pmgb_footprint(ctypes.byref(params), precision, natoms))


def _dp(a):
    return None if a is None else a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Server:
    """Native serving loop.  With `backend` (a Backend structure), the device
    calls are replaced by callbacks, which runs the loop without a GPU."""

    def __init__(self, precision=MIXED, max_inflight=4, hbm_budget_bytes=0, pool_per_shape=0,
                 backend: Backend | None = None, max_batch=0):
        self._h = ctypes.c_void_p()
        cfg = ServerConfig(precision, max_inflight, hbm_budget_bytes, pool_per_shape, max_batch)
        self._keep = {}
        if backend is None:
            ok = lib().pmgb_server_create(ctypes.byref(cfg), ctypes.byref(self._h))
        else:
            self._backend = backend
            ok = lib().pmgb_server_create_ex(ctypes.byref(cfg), ctypes.byref(backend),
                                             ctypes.byref(self._h))
        if ok != 1:
            raise RuntimeError("pmgb_server_create failed")

    def submit(self, params, mol, u_out: np.ndarray | None = None) -> int:
        xyz = np.ascontiguousarray(mol.xyz, dtype=np.float64).reshape(-1)
        q = np.ascontiguousarray(mol.charge, dtype=np.float64)
        r = np.ascontiguousarray(mol.radius, dtype=np.float64)
        rid = lib().pmgb_server_submit(self._h, ctypes.byref(params), mol.natoms, _dp(xyz),
                                       _dp(q), _dp(r), _dp(u_out))
        if rid <= 0:
            raise RuntimeError("request does not fit the device budget")
        if u_out is not None:
            self._keep[rid] = u_out
        return int(rid)

    def set_shape_tuning(self, params, key: int, value: int):
        """Tunable for every calculation of this grid shape built from now on."""
        if lib().pmgb_server_set_shape_tuning(self._h, ctypes.byref(params), key, value) != 1:
            raise RuntimeError("pmgb_server_set_shape_tuning failed")

    def apply_table(self, table: dict, precision: int) -> int:
        """Apply an autotuner table (apbs_b200.autotune) per grid shape; where
        LPBE and NPBE entries of a shape differ, the LPBE one wins.  Returns
        the number of shapes tuned."""
        shapes = {}
        for key, e in table.items():
            dims, nlev, prec, eq = key.split("/")
            if prec != ("mixed" if precision == MIXED else "fp64"):
                continue
            if dims + nlev in shapes and eq == "npbe":
                continue
            shapes[dims + nlev] = (dims, int(nlev), e["tune"])
        for dims, nlev, tune in shapes.values():
            p = synth.PmgbParams()
            p.nx, p.ny, p.nz = (int(d) for d in dims.split("x"))
            p.nlev = nlev
            for k, v in tune.items():
                self.set_shape_tuning(p, int(k), int(v))
        return len(shapes)

    def poll(self, rid: int) -> dict:
        res = Result()
        lib().pmgb_server_poll(self._h, rid, ctypes.byref(res))
        return res.as_dict()

    def wait(self, rid: int) -> dict:
        res = Result()
        lib().pmgb_server_wait(self._h, rid, ctypes.byref(res))
        self._keep.pop(rid, None)
        return res.as_dict()

    def drain(self):
        lib().pmgb_server_drain(self._h)

    def stats(self) -> dict:
        st = ServerStats()
        lib().pmgb_server_get_stats(self._h, ctypes.byref(st))
        return st.as_dict()

    def close(self):
        if self._h:
            lib().pmgb_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Request streams
# ---------------------------------------------------------------------------
@dataclass
class StreamRequest:
    t_arrival: float          # seconds after the start of the stream
    params: object            # PmgbParams
    mol: object               # synth.Molecule


DIMES = (33, 65, 97, 129, 161, 225)


def serving_stream(n: int, seed: int = 4, rate: float = 200.0, dimes=DIMES,
                   npbe_frac: float = 0.2) -> list[StreamRequest]:
    """Poisson arrivals (mean `rate` per second) of calculations mixing LPBE
    and NPBE (npbe_frac NPBE), grids drawn uniformly from `dimes`, seeded
    200-8000-atom clusters generated as the 65^3 LPBE case is (ball radius
    scaled to keep the atom density), grid spacing chosen so the molecule
    fits with at least 5 A of margin, ionic strength uniform in 0-0.3 M
    (1:1 salt).  Every draw comes from `seed`."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        dime = int(rng.choice(dimes))
        natoms = int(rng.integers(200, 8001))
        radius = 12.0 * (natoms / 500.0) ** (1.0 / 3.0)
        npbe = bool(rng.random() < npbe_frac)
        conc = float(rng.uniform(0.0, 0.3))
        mol = synth.cluster(natoms, radius, seed=int(rng.integers(1 << 30)))
        # extent of the atom cloud plus radii, 5 A margin on every side
        span = float((mol.xyz.max(axis=0) - mol.xyz.min(axis=0)).max()) + 2 * 2.0 + 10.0
        h = span / (dime - 1)
        ions = ((1.0, conc, 2.0), (-1.0, conc, 2.0)) if conc > 0 else ()
        params = synth.mg_manual(dime, h, mol.center(), npbe=npbe, ions=ions)
        out.append(StreamRequest(t, params, mol))
    return out


def stream_request(dime: int, natoms: int, npbe: bool, conc: float, seed: int):
    """One calculation drawn by the rules of `serving_stream` with its grid,
    size, equation and ionic strength given: a seeded `natoms`-atom cluster
    (ball radius scaled to keep the atom density), the spacing that fits it
    with 5 A of margin, 1:1 salt of concentration `conc` M."""
    radius = 12.0 * (natoms / 500.0) ** (1.0 / 3.0)
    mol = synth.cluster(natoms, radius, seed=seed)
    span = float((mol.xyz.max(axis=0) - mol.xyz.min(axis=0)).max()) + 2 * 2.0 + 10.0
    ions = ((1.0, conc, 2.0), (-1.0, conc, 2.0)) if conc > 0 else ()
    return synth.mg_manual(dime, span / (dime - 1), mol.center(), npbe=npbe, ions=ions), mol


def replay(server: Server, stream: list[StreamRequest], time_scale: float = 1.0) -> dict:
    """Submit each request at its arrival time and wait for all of them.
    Returns per-request results, the wall time from the first arrival to the
    last completion and the solves/s over it."""
    t0 = time.perf_counter()
    ids = []
    for rq in stream:
        delay = rq.t_arrival * time_scale - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        ids.append(server.submit(rq.params, rq.mol))
    results = [server.wait(i) for i in ids]
    wall = time.perf_counter() - t0
    ok = [r for r in results if r["status"] == 1]
    lat = np.array([r["latency_ms"] for r in ok]) if ok else np.zeros(1)
    return {"results": results, "wall_s": wall, "solves_per_s": len(ok) / wall,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "failed": len(results) - len(ok)}
