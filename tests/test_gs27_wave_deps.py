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

The second half models the shared-memory variant (k_gs27_mail): every CTA
works on its own copies of planes k-1, k and k+1 and takes its neighbours'
updates from a mailbox at the step that first needs them.  Free-running
interleavings give the lockstep iterates and residual bit for bit, never
deadlock, and no plane is written back before both neighbours loaded it.
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


# --- the shared-memory plane wavefront with a mailbox (k_gs27_mail) --------
# Each plane's CTA holds copies of planes k-1, k, k+1 loaded at its start; an
# update of half-sweep q, row j goes into its own copy and into mailbox slot
# (k, q, j).  At a step, half-sweep q at row j first takes row j+1 of the
# lower plane's half-sweep q and of the upper plane's half-sweep q-1 (and row
# 1 of both when j = 1); a CTA may run the step once every slot it takes
# exists.  At its end a CTA writes its plane back.

def mail_takes(s, k, nz, ny, nhalf, do_resid, lag, tmin, tmax, resid_lag):
    """Mailbox rows (plane, q, row) that plane k's step s takes."""
    out = []
    for ph in range(nhalf + (1 if do_resid else 0)):
        t = tmin + s - (lag * ph if ph < nhalf else resid_lag)
        j = t - 2 * k
        if t < tmin or t > tmax or j < 1 or j > ny - 2:
            continue
        for kn, q in ((k - 1, ph), (k + 1, ph - 1)):
            if kn < 1 or kn > nz - 2 or q < 0 or q >= nhalf:
                continue
            if j + 1 <= ny - 2:
                out.append((kn, q, j + 1))
            if j == 1:
                out.append((kn, q, 1))
    return out


def mail_run(x0, w, d, f, prm, nz, nsteps, pick):
    nx, ny, nhalf, do_resid, fp, lag, tmin, tmax, resid_lag = prm
    xg = x0.copy()  # x in global memory
    r = np.zeros_like(x0)
    planes = list(range(1, nz - 1))
    local = {}  # plane -> its CTA's copy of planes k-1..k+1 (a 3-plane array)
    mail = {}
    done = {k: 0 for k in planes}
    finished = set()
    while len(finished) < len(planes):
        ready = []
        for k in planes:
            s = done[k]
            if k in finished:
                continue
            if s == nsteps or all(key in mail for key in
                                  mail_takes(s, k, nz, ny, nhalf, do_resid, lag, tmin, tmax,
                                             resid_lag)):
                ready.append(k)
        assert ready, "deadlock"
        k = pick(ready, done)
        s = done[k]
        if s == 0 and k not in local:
            local[k] = xg[k - 1:k + 2].copy()
        if s == nsteps:
            # the plane goes back to x only after both neighbours loaded theirs
            for kn in (k - 1, k + 1):
                assert kn < 1 or kn > nz - 2 or kn in local
            xg[k] = local[k][1]
            finished.add(k)
            continue
        L = local[k]
        for kn, q, jj in mail_takes(s, k, nz, ny, nhalf, do_resid, lag, tmin, tmax, resid_lag):
            for i, v in mail[(kn, q, jj)]:
                L[1 + (kn - k), jj, i] = v
        # one plane's step on its copy: the same arithmetic as step()
        pend = []
        for ph, j, ii in items(s, k, nx, ny, nhalf, do_resid, fp, lag, tmin, tmax, resid_lag):
            row = []
            for i in ii:
                acc = 0.0
                for qq, (di, dj, dk) in enumerate(OFFS):
                    acc += w[qq, k, j, i] * L[1 + dk, j + dj, i + di]
                if ph < nhalf:
                    v = (f[k, j, i] + acc) / d[k, j, i]
                    pend.append((j, i, v))
                    row.append((i, v))
                else:
                    r[k, j, i] = f[k, j, i] + acc - d[k, j, i] * L[1, j, i]
            if ph < nhalf:
                mail[(k, ph, j)] = row
        for j, i, v in pend:
            L[1, j, i] = v
        done[k] += 1
    return xg, r


@pytest.mark.parametrize("nx,ny,nz", [(9, 9, 9), (11, 7, 13), (13, 13, 9), (7, 5, 5)])
@pytest.mark.parametrize("nhalf,do_resid", [(2, True), (4, True), (4, False), (2, False)])
@pytest.mark.parametrize("lag", [4, 6, 9])
def test_mailbox_planes_equal_lockstep(nx, ny, nz, nhalf, do_resid, lag):
    x0, w, d, f = make(nx, ny, nz, seed=nx * 5 + nz + lag + nhalf)
    tmin, tmax, resid_lag, nsteps = schedule(ny, nz, nhalf, do_resid, lag)
    prm = (nx, ny, nhalf, do_resid, 0, lag, tmin, tmax, resid_lag)
    xt, rt = lockstep(x0, w, d, f, prm, nz, nsteps)
    rng = random.Random(nx * ny + nz + lag)
    pickers = [lambda ready, done: rng.choice(ready),
               lambda ready, done: max(ready, key=lambda k: (done[k], k)),
               lambda ready, done: min(ready, key=lambda k: (done[k], -k)),
               lambda ready, done: max(ready)]
    for pick in pickers:
        x, r = mail_run(x0, w, d, f, prm, nz, nsteps, pick)
        assert np.array_equal(x, xt)
        if do_resid:
            assert np.array_equal(r, rt)
