"""Host logic of the serving loop (apbs_b200/csrc/serve.cu): queueing in
arrival order, admission by device footprint, pooling and reuse of resident
calculations, release of idle ones under memory pressure.  The device calls
are replaced by Python callbacks (pmgb_server_create_ex), so no GPU is
needed; the library itself is the real one."""
import ctypes
import threading
import time

import numpy as np
import pytest

from apbs_b200 import serve, synth
from apbs_b200.synth import PmgbParams

try:
    serve.lib()
    HAVE_LIB = True
except OSError:
    HAVE_LIB = False

pytestmark = pytest.mark.skipif(not HAVE_LIB, reason="libapbs_b200.so not built")


class FakeDevice:
    """Calculations as host records: bytes = 8 per grid point, a run sleeps
    `service_s` and returns sum(charge) + natoms as its energy."""

    def __init__(self, service_s=0.01):
        self.service_s = service_s
        self.lock = threading.Lock()
        self.live = {}
        self.next = 1
        self.running = 0
        self.max_running = 0
        self.created = 0
        self.peak_live = 0
        self.order = []          # natoms of each run, in start order
        self.bad_reconfigure = 0

        def footprint(ctx, pp, precision, natoms):
            p = ctypes.cast(pp, ctypes.POINTER(PmgbParams)).contents
            return p.nx * p.ny * p.nz * 8

        def create(ctx, pp, precision):
            p = ctypes.cast(pp, ctypes.POINTER(PmgbParams)).contents
            with self.lock:
                h = self.next
                self.next += 1
                self.live[h] = ((p.nx, p.ny, p.nz, p.nlev), p.nx * p.ny * p.nz * 8)
                self.created += 1
                self.peak_live = max(self.peak_live, sum(b for _, b in self.live.values()))
            return h

        def reconfigure(ctx, calc, pp):
            p = ctypes.cast(pp, ctypes.POINTER(PmgbParams)).contents
            with self.lock:
                if self.live[calc][0] != (p.nx, p.ny, p.nz, p.nlev):
                    self.bad_reconfigure += 1
                    return 0
            return 1

        def run(ctx, calc, natoms, xyz, q, r, energy):
            with self.lock:
                self.running += 1
                self.max_running = max(self.max_running, self.running)
                self.order.append(natoms)
            time.sleep(self.service_s)
            energy[0] = float(sum(q[i] for i in range(natoms))) + natoms
            with self.lock:
                self.running -= 1
            return 1

        def destroy(ctx, calc):
            with self.lock:
                self.live.pop(calc)

        self._cb = (serve.FOOTPRINT(footprint), serve.CREATE(create),
                    serve.RECONFIGURE(reconfigure), serve.RUN(run), serve.DESTROY(destroy))
        self.backend = serve.Backend(None, *self._cb)


def _req(dime, natoms, seed):
    rng = np.random.default_rng(seed)
    mol = synth.Molecule(rng.uniform(-5, 5, (natoms, 3)), rng.choice([-1.0, 0.0, 1.0], natoms),
                         np.full(natoms, 1.5))
    return synth.mg_manual(dime, 0.5, (0.0, 0.0, 0.0)), mol


def test_all_requests_finish_with_their_own_results():
    dev = FakeDevice(0.005)
    with serve.Server(max_inflight=4, hbm_budget_bytes=1 << 30, backend=dev.backend) as srv:
        reqs = [_req(33 if i % 2 else 65, 10 + i, i) for i in range(24)]
        ids = [srv.submit(p, m) for p, m in reqs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for (p, m), r in zip(reqs, res):
        assert r["status"] == 1
        assert r["energy_kT"] == pytest.approx(m.charge.sum() + m.natoms)
        assert r["latency_ms"] >= r["service_ms"] >= 0.0
    assert st["done"] == 24 and st["failed"] == 0
    assert 1 < dev.max_running <= 4          # work overlaps, never beyond the slots
    assert st["inflight_peak"] <= 4
    assert dev.bad_reconfigure == 0
    assert st["reused"] > 0 and st["created"] + st["reused"] == 24
    assert st["p99_ms"] >= st["p50_ms"] > 0.0


def test_admission_keeps_footprint_within_budget_and_order():
    dev = FakeDevice(0.01)
    big = 65 ** 3 * 8
    budget = int(2.5 * big)          # at most two 65^3 calculations resident
    with serve.Server(max_inflight=6, hbm_budget_bytes=budget, pool_per_shape=1,
                      backend=dev.backend) as srv:
        reqs = [_req(65 if i % 3 else 33, 100 + i, i) for i in range(18)]
        ids = [srv.submit(p, m) for p, m in reqs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    assert all(r["status"] == 1 for r in res)
    assert dev.peak_live <= budget
    assert st["bytes_peak"] <= budget
    # requests are admitted in arrival order (the head is never overtaken)
    assert [r["admit_order"] for r in res] == list(range(1, 19))


def test_idle_calculations_released_under_pressure():
    dev = FakeDevice(0.002)
    budget = 97 ** 3 * 8 + 1000      # one 97^3 calculation at a time
    with serve.Server(max_inflight=2, hbm_budget_bytes=budget, backend=dev.backend) as srv:
        ids = [srv.submit(*_req(97 if i % 2 else 65, 5 + i, i)) for i in range(8)]
        for i in ids:
            assert srv.wait(i)["status"] == 1
        st = srv.stats()
    assert st["evicted"] > 0
    assert dev.peak_live <= budget
    assert st["bytes_peak"] <= budget


def test_request_larger_than_budget_is_refused():
    dev = FakeDevice(0.0)
    with serve.Server(max_inflight=1, hbm_budget_bytes=33 ** 3 * 8, backend=dev.backend) as srv:
        with pytest.raises(RuntimeError):
            srv.submit(*_req(65, 5, 0))
        rid = srv.submit(*_req(33, 5, 1))
        assert srv.wait(rid)["status"] == 1


def test_serving_stream_is_seeded():
    a = serve.serving_stream(6, seed=3)
    b = serve.serving_stream(6, seed=3)
    assert [r.t_arrival for r in a] == [r.t_arrival for r in b]
    assert all(r.params.nx in serve.DIMES for r in a)
    assert all(np.array_equal(x.mol.xyz, y.mol.xyz) for x, y in zip(a, b))
    assert all(np.diff([r.t_arrival for r in a]) > 0)


def test_reused_calculation_takes_the_larger_footprint():
    """A pooled calculation reused by a request with more atoms grows to that
    request's footprint (the fill buffers grow with the atom count), and the
    loop counts the growth against the budget."""
    dev = FakeDevice(0.0)
    per_atom = 4096

    def footprint(ctx, pp, precision, natoms):
        p = ctypes.cast(pp, ctypes.POINTER(PmgbParams)).contents
        return p.nx * p.ny * p.nz * 8 + natoms * per_atom

    dev._cb = (serve.FOOTPRINT(footprint),) + dev._cb[1:]
    dev.backend = serve.Backend(None, *dev._cb)
    grid = 33 ** 3 * 8
    with serve.Server(max_inflight=1, hbm_budget_bytes=1 << 30, backend=dev.backend) as srv:
        assert srv.wait(srv.submit(*_req(33, 10, 0)))["status"] == 1
        assert srv.stats()["bytes_in_use"] == grid + 10 * per_atom
        assert srv.wait(srv.submit(*_req(33, 500, 1)))["status"] == 1
        st = srv.stats()
        assert st["reused"] == 1
        assert st["bytes_in_use"] == grid + 500 * per_atom
        # a smaller request keeps the grown calculation's footprint
        assert srv.wait(srv.submit(*_req(33, 20, 2)))["status"] == 1
        st = srv.stats()
        assert st["reused"] == 2 and st["bytes_in_use"] == grid + 500 * per_atom


def test_failed_request_leaves_the_others_alone():
    """A request whose device run fails is reported failed with the others'
    results untouched, and its calculation is not pooled."""
    dev = FakeDevice(0.001)
    bad_natoms = 13
    inner = dev._cb[3]

    def run(ctx, calc, natoms, xyz, q, r, energy):
        if natoms == bad_natoms:
            return 0
        return inner(ctx, calc, natoms, xyz, q, r, energy)

    dev._cb = dev._cb[:3] + (serve.RUN(run),) + dev._cb[4:]
    dev.backend = serve.Backend(None, *dev._cb)
    with serve.Server(max_inflight=3, hbm_budget_bytes=1 << 30, backend=dev.backend) as srv:
        reqs = [_req(33, 10 + i, i) for i in range(10)]
        ids = [srv.submit(p, m) for p, m in reqs]
        res = [srv.wait(i) for i in ids]
        st = srv.stats()
    for (p, m), r in zip(reqs, res):
        if m.natoms == bad_natoms:
            assert r["status"] == -1 and r["error"]
        else:
            assert r["status"] == 1
            assert r["energy_kT"] == pytest.approx(m.charge.sum() + m.natoms)
    assert st["failed"] == 1 and st["done"] == 9
