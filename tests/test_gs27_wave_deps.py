"""Host model of the plane-parallel ordered 27-point Gauss-Seidel's waits
(k_gs27_planes, apbs_b200/csrc/mg_kernels.cu): every plane runs its own
step counter and may start step s once its lower neighbour plane has
finished step s - 1 and its upper neighbour plane step s - LAG + 3, LAG
being the number of wavefronts between successive half-sweeps (and the
residual LAG wavefronts after the last one).

The model runs adversarial interleavings -- random choices among the planes
whose waits are met, the plane furthest ahead first, the one furthest behind
first -- on one shared
array, and checks that the iterates and the residual equal the lockstep
wavefront (every step reads what the earlier steps left) bit for bit, for
several lags, sweep counts and grid shapes; and that steps allowed to run at
the same time touch disjoint points (no step writes what another reads or
writes), so any overlap of them in time gives the same result.  This is the
argument for the
asymmetric waits made executable: a read of an upper neighbour needs that
plane's earlier half-sweep LAG - 3 steps back, a read of a lower neighbour
its current half-sweep one step back, and every anti-dependence (a value a
plane still has to read in its old state) is covered by the neighbour's own
wait on this plane.
"""
import random

import numpy as np
import pytest

OFFS = [(di, dj, dk) for dk in (-1, 0, 1) for dj in (-1, 0, 1) for di in (-1, 0, 1)
        if (di, dj, dk) != (0, 0, 0)]


def schedule(ny, nz, nhalf, do_resid, lag):
    tmin, tmax = 3, (ny - 2) + 2 * (nz - 2)
    resid_lag = lag * nhalf
    last_start = resid_lag if do_resid else lag * (nhalf - 1)
    return tmin, tmax, resid_lag, (tmax - tmin + 1) + last_start


def items(s, k, nx, ny, nhalf, do_resid, first_parity, lag, tmin, tmax, resid_lag):
    hr = (nx - 1) // 2
    out = []
    for ph in range(nhalf + (1 if do_resid else 0)):
        t = tmin + s - (lag * ph if ph < nhalf else resid_lag)
        j = t - 2 * k
        if t < tmin or t > tmax or j < 1 or j > ny - 2:
            continue
        if ph < nhalf:
            parity = (first_parity + ph) & 1
            ii = [1 + (((1 + j + k) & 1) != parity) + 2 * m for m in range(hr)]
            out.append((ph, j, [i for i in ii if i <= nx - 2]))
        else:
            out.append((ph, j, list(range(1, nx - 1))))
    return out


def make(nx, ny, nz, seed):
    rng = np.random.default_rng(seed)
    x0 = rng.normal(size=(nz, ny, nx))
    w = rng.uniform(-0.2, 0.2, size=(len(OFFS), nz, ny, nx))
    d = rng.uniform(4.0, 6.0, size=(nz, ny, nx))
    f = rng.normal(size=(nz, ny, nx))
    return x0, w, d, f


def step(x, r, s, k, prm, w, d, f, snapshot=None):
    nx, ny, nhalf, do_resid, fp, lag, tmin, tmax, resid_lag = prm
    src = snapshot if snapshot is not None else x
    pend = []
    for ph, j, ii in items(s, k, nx, ny, nhalf, do_resid, fp, lag, tmin, tmax, resid_lag):
        for i in ii:
            acc = 0.0
            for q, (di, dj, dk) in enumerate(OFFS):
                acc += w[q, k, j, i] * src[k + dk, j + dj, i + di]
            if ph < nhalf:
                pend.append((k, j, i, (f[k, j, i] + acc) / d[k, j, i]))
            else:
                r[k, j, i] = f[k, j, i] + acc - d[k, j, i] * src[k, j, i]
    # within one plane's step the GS points read no value written in the
    # same step, so applying the writes afterwards is exact
    for k_, j, i, v in pend:
        x[k_, j, i] = v


def lockstep(x0, w, d, f, prm, nz, nsteps):
    x = x0.copy()
    r = np.zeros_like(x0)
    for s in range(nsteps):
        snap = x.copy()
        for k in range(1, nz - 1):
            step(x, r, s, k, prm, w, d, f, snapshot=snap)
    return x, r


def access_sets(s, k, prm):
    """Points read and written by plane k's step s."""
    nx, ny, nhalf, do_resid, fp, lag, tmin, tmax, resid_lag = prm
    rd, wr = set(), set()
    for ph, j, ii in items(s, k, nx, ny, nhalf, do_resid, fp, lag, tmin, tmax, resid_lag):
        for i in ii:
            for di, dj, dk in OFFS + [(0, 0, 0)]:
                rd.add((k + dk, j + dj, i + di))
            if ph < nhalf:
                wr.add((k, j, i))
    return rd, wr


def free_run(x0, w, d, f, prm, nz, nsteps, lag, pick, check_pairs=False):
    x = x0.copy()
    r = np.zeros_like(x0)
    done = {k: 0 for k in range(1, nz - 1)}  # steps finished per plane
    planes = list(range(1, nz - 1))
    while any(done[k] < nsteps for k in planes):
        ready = []
        for k in planes:
            s = done[k]
            if s >= nsteps:
                continue
            # lower neighbour finished step s - 1, upper neighbour step s - LAG + 3
            lo_ok = (k - 1 < 1) or done[k - 1] >= s
            up_ok = (k + 1 > nz - 2) or done[k + 1] >= s - lag + 4
            if lo_ok and up_ok:
                ready.append(k)
        assert ready, "deadlock"
        if check_pairs:
            # steps that may run at the same time touch disjoint data: no step
            # writes a point another ready step reads or writes
            sets = {k: access_sets(done[k], k, prm) for k in ready}
            for a in ready:
                for b in ready:
                    if a != b:
                        assert not (sets[a][1] & (sets[b][0] | sets[b][1])), (a, b)
        k = pick(ready, done)
        step(x, r, done[k], k, prm, w, d, f)
        done[k] += 1
    return x, r


@pytest.mark.parametrize("nx,ny,nz", [(9, 9, 9), (11, 7, 13), (13, 13, 9)])
@pytest.mark.parametrize("nhalf,do_resid", [(2, True), (4, True), (4, False), (1, True)])
@pytest.mark.parametrize("lag", [4, 6, 8])
def test_asymmetric_waits_equal_lockstep(nx, ny, nz, nhalf, do_resid, lag):
    x0, w, d, f = make(nx, ny, nz, seed=nx * 7 + nz + lag)
    tmin, tmax, resid_lag, nsteps = schedule(ny, nz, nhalf, do_resid, lag)
    prm = (nx, ny, nhalf, do_resid, 1, lag, tmin, tmax, resid_lag)
    xt, rt = lockstep(x0, w, d, f, prm, nz, nsteps)
    rng = random.Random(nx + ny + nz + lag + nhalf)
    pickers = [lambda ready, done: rng.choice(ready),
               lambda ready, done: max(ready, key=lambda k: (done[k], k)),
               lambda ready, done: min(ready, key=lambda k: (done[k], -k))]
    for n, pick in enumerate(pickers):
        x, r = free_run(x0, w, d, f, prm, nz, nsteps, lag, pick, check_pairs=(n == 0))
        assert np.array_equal(x, xt)
        assert np.array_equal(r, rt)


def test_lag_changes_nothing():
    # the iterates do not depend on the lag: only the order of independent
    # updates changes
    nx, ny, nz = 11, 9, 11
    x0, w, d, f = make(nx, ny, nz, seed=3)
    ref = None
    for lag in (4, 5, 8):
        tmin, tmax, resid_lag, nsteps = schedule(ny, nz, 4, True, lag)
        x, r = lockstep(x0, w, d, f, (nx, ny, 4, True, 0, lag, tmin, tmax, resid_lag), nz,
                        nsteps)
        if ref is None:
            ref = (x, r)
        assert np.array_equal(x, ref[0]) and np.array_equal(r, ref[1])
