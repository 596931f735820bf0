"""Oracle: per-group adaptive Dormand-Prince 5(4) driver (batched_rk45.py).

Test infrastructure only -- see ``oracle/__init__.py``.

``integrate`` restates ``batched_rk45.integrate`` (:55-323) and
``_attempt_step`` (:326-401) for uniform group size E, and additionally
returns a per-group attempt log (h used, error norm, accepted) so tests can
compare acceptance sequences.  ``max_attempts`` (not in the reference) stops
a group after that many attempts, so a bounded slice of a trace can be
compared with the CUDA kernel run for the same number of attempts.
"""

import numpy as np

from .physics import SPEED_OF_LIGHT

# Dormand-Prince 5(4) tableau (batched_rk45.py:30-50).
A = [
    [],
    [1 / 5],
    [3 / 40, 9 / 40],
    [44 / 45, -56 / 15, 32 / 9],
    [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729],
    [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656],
]
B = np.array([35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84])
EE = np.array([71 / 57600, 0.0, -71 / 16695, 71 / 1920, -17253 / 339200, 22 / 525, -1 / 40])


def attempt(accel, pos, vel, t, h, tb, td, gidx, rtol, atol, safety=0.9, fmin=0.2, fmax=10.0):
    """batched_rk45.py:326-401."""
    live = (t[:, None] >= tb) & (t[:, None] < td)
    kp = [None] * 7
    kv = [None] * 7
    for i in range(6):
        ps, vs = pos, vel
        for j, a in enumerate(A[i]):
            if a == 0.0:
                continue
            ps = ps + (h * a)[:, None, None] * kp[j]
            vs = vs + (h * a)[:, None, None] * kv[j]
        kv[i] = accel(ps, vs, live, gidx)
        kp[i] = np.where(live[..., None], vs, 0.0)
    pos_new = pos + h[:, None, None] * sum(B[i] * kp[i] for i in range(6))
    vel_new = vel + h[:, None, None] * sum(B[i] * kv[i] for i in range(6))
    kv[6] = accel(pos_new, vel_new, live, gidx)
    kp[6] = np.where(live[..., None], vel_new, 0.0)
    ep = h[:, None, None] * sum(EE[i] * kp[i] for i in range(7))
    ev = h[:, None, None] * sum(EE[i] * kv[i] for i in range(7))
    sp = atol + rtol * np.maximum(np.abs(pos), np.abs(pos_new))
    sv = SPEED_OF_LIGHT * atol + rtol * np.maximum(np.abs(vel), np.abs(vel_new))
    n = 2 * pos.shape[1] * 3
    sq = np.sum((ep / sp) ** 2, axis=(1, 2)) + np.sum((ev / sv) ** 2, axis=(1, 2))
    err = np.sqrt(sq / n)
    err = np.where(err == 0.0, np.finfo(float).tiny, err)
    ok = err <= 1.0
    fac = np.clip(safety * err ** (-1.0 / 5), fmin, fmax)
    return pos_new, vel_new, t + h, ok, h * fac, err


def integrate(accel, pos0, vel0, t_birth, t_max, rtol, atol, kill=None, on_step=None,
              output_times=None, on_output=None, max_attempts=None, max_steps=10_000_000,
              initial_step_fraction=1e-6):
    """batched_rk45.py:55-323.  Returns (pos, vel, t_death, t, h, log) where
    log[g] = (h_used array, err array, accepted bool array)."""
    G, E, _ = pos0.shape
    pos = pos0.copy()
    vel = vel0.copy()
    td = np.full((G, E), np.inf)
    cps = np.sort(t_birth, axis=1)
    t = cps[:, 0].copy()
    h = (t_max - t) * initial_step_fraction
    have_out = output_times is not None
    if have_out:
        outs = np.sort(output_times)
        n_out = outs.shape[0]
        if on_output is not None:
            last = np.sum(outs[None, :] <= t[:, None], axis=1) - 1
            at0 = (last >= 0) & (outs[np.maximum(last, 0)] == t)
            if np.any(at0):
                ii = np.nonzero(at0)[0]
                ptr = last[ii]
                for p in np.unique(ptr):
                    sel = ii[ptr == p]
                    on_output(int(p), sel, t[sel], pos[sel], vel[sel])
    running = np.ones(G, dtype=bool)
    n_att = np.zeros(G, dtype=np.int64)
    logs = [([], [], []) for _ in range(G)]
    idx = np.nonzero(running)[0]
    for _ in range(max_steps):
        if idx.shape[0] == 0:
            break
        reached = np.sum(cps[idx] <= t[idx][:, None], axis=1)
        cpi = np.minimum(reached, E - 1)
        exhausted = reached >= E
        next_cp = np.where(exhausted, t_max, cps[idx, cpi])
        target = np.minimum(next_cp, t_max)
        if have_out:
            optr = np.sum(outs[None, :] <= t[idx][:, None], axis=1)
            oex = optr >= n_out
            next_out = np.where(oex, t_max, outs[np.minimum(optr, n_out - 1)])
            target = np.minimum(target, next_out)
        hr = np.minimum(h[idx], target - t[idx])
        pn, vn, tn, ok, hn, err = attempt(accel, pos[idx], vel[idx], t[idx], hr, t_birth[idx], td[idx], idx, rtol, atol)
        h[idx] = hn
        n_att[idx] += 1
        for k, g in enumerate(idx):
            logs[g][0].append(hr[k])
            logs[g][1].append(err[k])
            logs[g][2].append(bool(ok[k]))
        if np.any(ok):
            ai = idx[ok]
            t_old, p_old, v_old = t[ai], pos[ai], vel[ai]
            was_live = (t_old[:, None] >= t_birth[ai]) & (t_old[:, None] < td[ai])
            pos[ai] = pn[ok]
            vel[ai] = vn[ok]
            t[ai] = tn[ok]
            tol = 1e-9 * np.maximum(t_max, 1e-30)
            at_cp = (~exhausted[ok]) & (t[ai] >= next_cp[ok] - tol)
            if np.any(at_cp):
                h[ai] = np.where(at_cp, (t_max - t[ai]) * initial_step_fraction, h[ai])
            if kill is not None:
                dead = was_live & kill(pos[ai])
                if np.any(dead):
                    td[ai] = np.where(dead, t[ai][:, None], td[ai])
            if have_out and on_output is not None:
                hit = (~oex[ok]) & (t[ai] >= next_out[ok] - tol)
                if np.any(hit):
                    hl = np.nonzero(hit)[0]
                    ph = optr[ok][hl]
                    for p in np.unique(ph):
                        sg = ai[hl[ph == p]]
                        on_output(int(p), sg, t[sg], pos[sg], vel[sg])
            if on_step is not None:
                on_step(ai, t_old, p_old, v_old, t[ai], pos[ai], vel[ai])
            running[ai] = t[ai] < t_max * (1 - 1e-14)
        if max_attempts is not None:
            running &= n_att < max_attempts
        idx = np.nonzero(running)[0]
    else:
        raise RuntimeError(f"batched RK45 did not converge within {max_steps} steps")
    log = [(np.array(a), np.array(b), np.array(c, dtype=bool)) for a, b, c in logs]
    return pos, vel, td, t, h, log


def integrate_uneven(accel_factory, pos, vel, t_birth, offsets, t_max, rtol, atol, kill=None, max_attempts=None):
    """Uneven group sizes: the reference needs a uniform n_emit
    (emission.py:25-29), so groups are run in bins of equal size, each bin
    through ``integrate``.  ``accel_factory(group_ids)`` returns an accel
    callable over that bin's groups; per-particle arrays are flat with
    ``offsets`` (G+1)."""
    sizes = np.diff(offsets)
    out_pos = pos.copy()
    out_vel = vel.copy()
    out_td = np.full(len(pos), np.inf)
    G = len(sizes)
    t_end = np.zeros(G)
    h_end = np.zeros(G)
    logs = [None] * G
    for E in np.unique(sizes):
        groups = np.nonzero(sizes == E)[0]
        rows = offsets[groups][:, None] + np.arange(E)[None, :]
        p, v, td, t, h, lg = integrate(accel_factory(groups), pos[rows], vel[rows], t_birth[rows], t_max,
                                       rtol, atol, kill=kill, max_attempts=max_attempts)
        out_pos[rows] = p
        out_vel[rows] = v
        out_td[rows] = td
        t_end[groups] = t
        h_end[groups] = h
        for k, g in enumerate(groups):
            logs[g] = lg[k]
    return out_pos, out_vel, out_td, t_end, h_end, logs
