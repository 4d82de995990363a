"""calc_numsol (Nonlinear_solution.f90:33-294) with set_backtr (:386-412), set_eater
(:414-439), run_backtr (:441-631) and check_abserrmax (Check_simulation.f90:37-91),
written out again in Python from the Fortran and driven by the oracle's own make_matvec,
solve_linalg, calc_func and calc_vecjacf (each pinned separately in test_oracle_kat.py):
the oracle's Newton solve must land on the same heads, bit for bit, with the same Newton,
Krylov and backtracking counts.  This pins the Newton controller -- the inexact-Newton
forcing, the step-length cap and the cubic/quadratic line search -- against the source,
including quirk Q2 of the reference AMG mode (the slope reads the preconditioner's last
input, which loop_amg leaves in rhs, Linear_solution.f90:516-529,717-718).
The time loop around it (accept, reject and roll back, dt control, the real(SP) clock) is
restated the same way.
"""
import math

import numpy as np
import pytest

from msg123_b200.config import make_config
from oracle.oracle import Oracle

VARMAX, XMAX = 1.0e3, 1.0e4
MACHI_EPS = float(np.finfo(np.float32).eps)


def _dot(a, b):
    s = 0.0
    for x, y in zip(a.tolist(), b.tolist()):
        s += x * y
    return s


def _maxnum(a, b):
    """MAX of two reals when one may be NaN: the other one (IEEE 754 maxNum, what gfortran's
    MAX and C's fmax return)."""
    if a != a:
        return b
    if b != b:
        return a
    return max(a, b)


def _abserrmax(x_new, x_pre):
    ach = aval = bch = bval = 0.0
    nun = 0
    for i, (a, b) in enumerate(zip(x_new.tolist(), x_pre.tolist())):
        d = a - b
        if abs(d) >= ach:
            bch, ach, nun = d, abs(d), i + 1
        if abs(a) >= aval:
            aval, bval = abs(a), a
    return bch, bval, nun


def _bicgs(o, b, bnorm, errtol, maxit):
    """solve_bicgs from x = 0 (Linear_solution.f90:234-493) with the oracle's matvec and
    preconditioner; returns x, ||r||^2, iterations, convergence flag and the last vector
    handed to the preconditioner (which loop_amg leaves in rhs, quirk Q2)."""
    x, resi, p, v = np.zeros_like(b), b.copy(), np.zeros_like(b), np.zeros_like(b)
    rs = resi.copy()
    sk0, alpha, omega, rnorm, last = np.inf, 0.0, 1.0, 0.0, None
    for it in range(1, maxit + 1):
        sk = _dot(resi, rs)
        p = resi.copy() if it == 1 else resi + ((sk / sk0) * (alpha / omega)) * (p - omega * v)
        last = p
        z = o.precond(p)
        v = o.matvec(z)
        alpha = sk / _dot(v, rs)
        x = x + alpha * z
        resi = resi - alpha * v
        rnorm = _dot(resi, resi)
        if math.sqrt(rnorm / bnorm) <= errtol:
            return x, rnorm, it, 1, last
        last = resi
        z = o.precond(resi)
        t = o.matvec(z)
        omega = _dot(t, resi) / _dot(t, t)
        x = x + omega * z
        resi = resi - omega * t
        rnorm = _dot(resi, resi)
        if math.sqrt(rnorm / bnorm) <= errtol:
            return x, rnorm, it, 1, last
        if it == maxit:
            return x, rnorm, it, 0, last
        sk0 = sk
    raise AssertionError("unreachable")


class _Newton:
    def __init__(self, o, prm):
        self.o, self.prm = o, prm

    def func_l2(self, h):
        f = self.o.calc_func(h)
        return _dot(f, f)

    def run_backtr(self, h_pre, dh, h_new, rhs, l2_pre, l2_jnorm, maxstep):
        o = self.o
        lam, lam2, maxpnorm, lam_length = 1.0, 1.0, 1.0, 1.0
        f = o.calc_func(h_new)
        l2_pnorm = _dot(dh, dh)
        jac = o.vecjacf(h_pre, dh)
        sq = math.sqrt(l2_pnorm)
        if sq > maxstep:
            maxpnorm = maxstep / sq
            dh = dh * maxpnorm
            sq = maxstep
        step_len = sq
        l2_new = _dot(f, f)
        slope = _dot(rhs, jac) * maxpnorm
        for a, b in zip(dh.tolist(), h_new.tolist()):
            if b != 0.0:
                t = abs(a) / abs(b)
                if t > lam_length:
                    lam_length = t
        l2_jnorm = l2_jnorm * maxpnorm * maxpnorm
        lam_min = math.pow(MACHI_EPS, 2.0 / 3.0) / lam_length
        alpha_cond = 0.5 * l2_pre + 1.0e-4 * lam * slope
        back_iter = beta_iter = 0
        l2_new2 = 0.0
        h = h_new
        while not (0.5 * l2_new <= alpha_cond):
            back_iter += 1
            h = h_pre + lam * dh
            l2_new = self.func_l2(h)
            if lam == 1.0:
                tl = -slope / (2.0 * (0.5 * l2_new - 0.5 * l2_pre - slope))
            else:
                r1 = 0.5 * l2_new - 0.5 * l2_pre - lam * slope
                r2 = l2_new2 - 0.5 * l2_pre - lam2 * slope
                li, l2i, dl = 1.0 / (lam ** 2), 1.0 / (lam2 ** 2), 1.0 / (lam - lam2)
                av = (r1 * li - r2 * l2i) * dl
                bv = (-lam2 * r1 * li + lam * r2 * l2i) * dl
                if av == 0:
                    tl = -slope / (2.0 * bv)
                else:
                    root = bv * bv - 3.0 * av * slope
                    if root < 0.0:
                        tl = 0.5 * lam
                    elif bv <= 0.0:
                        tl = (-bv + math.sqrt(root)) / (3.0 * av)
                    else:
                        tl = -slope / (bv + math.sqrt(root))
                    if tl > 0.5 * lam:
                        tl = 0.5 * lam
            lam2, l2_new2 = lam, 0.5 * l2_new
            lam = max(tl, 0.1 * lam)
            if lam < lam_min:
                return h, l2_new, lam, slope, l2_jnorm, 1, back_iter
            alpha_cond = 0.5 * l2_pre + 1.0e-4 * lam * slope
        alpha_cond = 0.5 * l2_pre + 1.0e-4 * lam * slope
        beta_cond = 0.5 * l2_pre + 0.9 * lam * slope
        if 0.5 * l2_new < beta_cond:
            if lam == 1.0 and sq < step_len:
                lam_max = step_len / sq
                while not (0.5 * l2_new > alpha_cond or 0.5 * l2_new >= beta_cond or lam >= lam_max):
                    lam2, l2_new2, lam = lam, 0.5 * l2_new, min(2.0 * lam, lam_max)
                    h = h_pre + lam * dh
                    l2_new = self.func_l2(h)
                    alpha_cond = 0.5 * l2_pre + 1.0e-4 * lam * slope
                    beta_cond = 0.5 * l2_pre + 0.9 * lam * slope
            if lam < 1.0 or (lam > 1.0 and 0.5 * l2_new > alpha_cond):
                lam_base, lam_diff = min(lam, lam2), abs(lam2 - lam)
                while not (0.5 * l2_new <= alpha_cond and (0.5 * l2_new >= beta_cond or lam_diff <= lam_min)):
                    incr = 0.5 * lam_diff
                    lam = lam_base + incr
                    h = h_pre + lam * dh
                    l2_new = self.func_l2(h)
                    alpha_cond = 0.5 * l2_pre + 1.0e-4 * lam * slope
                    beta_cond = 0.5 * l2_pre + 0.9 * lam * slope
                    if 0.5 * l2_new > alpha_cond:
                        lam_diff = incr
                    elif 0.5 * l2_new < beta_cond:
                        lam_base, lam_diff = lam, lam_diff - incr
                    if lam_diff == 0.0:
                        break
                if 0.5 * l2_new < beta_cond:
                    h = h_pre + lam_base * dh
                    l2_new = self.func_l2(h)
                    beta_iter += 1
                if beta_iter == 10:
                    return h, l2_new, lam, slope, l2_jnorm, 1, back_iter
        return h, l2_new, lam, slope, l2_jnorm, 0, back_iter

    def solve(self, h):
        o, prm = self.o, self.prm
        ls = prm["len_scal"]
        maxstep = max(math.sqrt(_dot(h, h)) * VARMAX, 1.0)          # set_backtr
        inner = backs = 0
        status, l2_new, eta = None, 0.0, 0.5
        for out_iter in range(1, prm["maxout_iter"] + 1):
            if out_iter > 1:
                l2_pre = l2_new
            o.set_state(head_new=h)
            _, _, rhs = o.make_matvec()
            if out_iter == 1:
                l2_new = _dot(rhs, rhs)
                l2_pre, eta = l2_new, 0.5
            h_pre = h
            errtol = prm["lin_tol"] if prm["lin_tol"] > 0 else eta
            if prm["precon_type"] == 1 and prm["ref_quirks"]:
                # Q2: loop_amg leaves its last input in rhs, which the line-search slope reads
                dh, l2_jnorm, it, conv, rhs = _bicgs(o, rhs, l2_pre, errtol, prm["maxinn_iter"])
            else:
                dh, l2_jnorm, it, conv = o.solve_linalg(l2_pre, errtol)
            inner += it
            h = h_pre + dh
            maxvar, maxunk, _ = _abserrmax(h, h_pre)
            check, maxunk = abs(maxvar) * ls, abs(maxunk) * ls
            crit = prm["criteria"] * maxunk if prm["criteria_rel"] else prm["criteria"]
            conv_flag, back_flag = conv, 0
            if conv_flag != 0:
                conv_flag = 1 if (check <= crit and maxunk < XMAX) else 0
            if conv_flag != 1:
                h, l2_new, lam, slope, l2_jnorm, back_flag, bi = self.run_backtr(
                    h_pre, dh, h, rhs, l2_pre, l2_jnorm, maxstep)
                backs += bi
                maxvar, maxunk, _ = _abserrmax(h, h_pre)
                check, maxunk = abs(maxvar) * ls, abs(maxunk) * ls
                crit = prm["criteria"] * maxunk if prm["criteria_rel"] else prm["criteria"]
                if check >= VARMAX or maxunk >= XMAX:
                    back_flag = 1
                elif check <= crit and maxunk < XMAX:
                    conv_flag = 1
                if conv_flag != 1 and back_flag != 1:                   # set_eater
                    eta_safe = math.pow(eta, (1.0 + math.sqrt(5.0)) / 2.0)
                    m1 = 1.0 - lam
                    q = m1 * m1 * l2_pre + 2.0 * lam * m1 * slope + lam * lam * l2_jnorm
                    lin = math.sqrt(q) if q >= 0.0 else math.nan      # IEEE sqrt of a negative
                    eta = abs(math.sqrt(l2_new) - lin) / math.sqrt(l2_pre)
                    if eta_safe < 0.1:
                        eta_safe = 0.0
                    eta = min(_maxnum(_maxnum(eta, eta_safe), 1.0e-4), 0.9)
            l2_new = _dot(*(2 * [o.calc_func(h)]))
            if conv_flag == 1:
                status = 0
            elif back_flag == 1:
                status = 3
            elif out_iter == prm["maxout_iter"]:
                status = 1
            elif abs(maxvar * ls) >= VARMAX or maxunk >= XMAX:
                status = 4
            if status is not None:
                return h, status, out_iter, inner, backs, maxvar * ls, l2_new
        raise AssertionError("unreachable")


def _case(name, kw, amp, seed):
    kw = dict(kw)
    kw.setdefault("precon_type", 0)
    p = make_config(name, **kw)
    h0 = p.head0 + amp * np.random.default_rng(seed).standard_normal(p.ncalc) / p.params["len_scal"]
    pair = []
    for _ in range(2):
        o = Oracle(p)
        o.init_state(head=h0)
        pair.append(o)
    return p, pair


@pytest.mark.parametrize("name,kw,amp,seed", [
    ("box", dict(shape=(6, 5, 10)), 0.0, 0),
    ("hetero", dict(shape=(10, 8, 6), seed=3), 0.0, 0),
    ("hetero", dict(shape=(10, 8, 6), seed=3, maxinn_iter=3), 0.3, 1),   # inexact solves, rough start
    ("hetero", dict(shape=(10, 8, 6), seed=3, maxinn_iter=2), 1.0, 2),   # 18 backtracks, Newton cap
    ("hetero", dict(shape=(10, 8, 6), seed=7, maxinn_iter=1), 2.0, 4),   # 24 backtracks, Newton cap
    ("hetero", dict(shape=(10, 8, 6), seed=3, precon_type=1, ref_quirks=1), 0.0, 0),   # quirks Q1, Q2
    ("hetero", dict(shape=(10, 8, 6), seed=3, precon_type=1, ref_quirks=1, maxinn_iter=3), 0.3, 1),
])
def test_newton_controller_restated(name, kw, amp, seed):
    p, (o1, o2) = _case(name, kw, amp, seed)
    rc, st = o1.calc_numsol()
    h1 = o1.get_state()["head_new"]
    h2, status, out_iter, inner, backs, maxvar, l2 = _Newton(o2, p.params).solve(
        o2.get_state()["head_new"].copy())
    assert (rc, st["out_iter"], st["inner_total"], st["back_total"]) == (status, out_iter, inner, backs)
    assert np.array_equal(h1, h2)
    assert st["maxvar"] == maxvar and st["l2_new"] == l2


def _time_loop(o, p, nsteps, rech_until, rech_after):
    """update_tstep / calc_nextst / apply_heuri (Time_module.f90:34-273, :1522-1543) written
    out again around the oracle's calc_numsol: accept -> shift the time levels and grow dt by
    inc_fact or the Newton-count heuristic (capped at max_step); reject -> roll back, step the
    real(SP) clock back and halve dt; the recharge switches at rech_until, where a step is
    cut to land on it (the library's set_delt alignment), and dt below 1e-20 stops."""
    prm = p.params
    f32 = lambda x: float(np.float32(x))
    st = o.get_state()
    hn, ho, so, sh = st["head_new"], st["head_old"], st["srat_old"], st["surf_head"]
    ho2, surf_old = ho.copy(), sh.copy()
    delt, t, nts, d_old1, conv, last_out = prm["ini_step"], 0.0, 0, 0.0, -1, 0
    R = dict(accepted=0, rejected=0, newton_total=0, krylov_total=0, back_total=0)
    incr, decr = int(prm["maxout_iter"] * 0.4), int(prm["maxout_iter"] * 0.8)
    while R["accepted"] < nsteps:
        if conv == 1:
            if nts == 0:
                d_old1 = delt
            nts += 1
            d_old1 = delt
            if prm["sim_type"] == 0:
                delt = delt * prm["inc_fact"]
            else:
                delt = d_old1 * (1.2 if last_out <= incr else (1.0 if last_out <= decr else 0.8))
                if delt > prm["max_step"]:
                    delt = prm["max_step"]
            ho2, ho, so, surf_old = ho, hn, sn, sh
        elif conv == 0:
            t = f32(t - f32(delt))
            delt = delt * 0.5
            hn, sh = ho, surf_old
            R["rejected"] += 1
        if t < rech_until and t + delt > rech_until:
            delt = rech_until - t
        if t + delt > prm["end_time"]:
            delt = prm["end_time"] - t
        if delt < 1.0e-20:
            return 5, R, hn, t, delt
        o.set_recharge(p.rech * (1.0 if t < rech_until else rech_after))
        t = f32(t + f32(delt))
        o.set_state(head_new=hn, head_old=ho, srat_old=so, surf_head=sh, delt=delt)
        rc, s = o.calc_numsol()
        for k in ("newton_total", "krylov_total", "back_total"):
            R[k] += s[{"newton_total": "out_iter", "krylov_total": "inner_total", "back_total": "back_total"}[k]]
        last_out = s["out_iter"]
        conv = 1 if rc == 0 else 0
        g = o.get_state()
        hn, sn, sh = g["head_new"], g["srat_new"], g["surf_head"]
        if conv:
            R["accepted"] += 1
            if t >= prm["end_time"]:
                break
    return 0, R, hn, t, delt


@pytest.mark.parametrize("name,kw,nsteps,rech_until", [
    ("box", dict(shape=(6, 5, 8), maxout_iter=2), 3, 1.0e30),             # Newton cap: rejections, dt halving
    ("hetero", dict(shape=(10, 8, 6), seed=3), 6, 2000.0),                 # heuristic dt, rain stops mid-run
])
def test_time_loop_restated(name, kw, nsteps, rech_until):
    p = make_config(name, precon_type=0, **kw)
    o1, o2 = Oracle(p), Oracle(p)
    for o in (o1, o2):
        o.init_state()
        o.set_recharge(p.rech)
    rc1, r1 = o1.advance(nsteps=nsteps, rech_until=rech_until, rech_after=0.0)
    rc2, r2, h2, t2, d2 = _time_loop(o2, p, nsteps, rech_until, 0.0)
    assert rc1 == rc2 == 0
    for k in ("accepted", "rejected", "newton_total", "krylov_total", "back_total"):
        assert r1[k] == r2[k], k
    assert r1["current_t"] == t2 and r1["delt"] == d2
    assert np.array_equal(o1.get_state()["head_new"], h2)


def test_jv_mode_slope_from_linear_residual():
    """Oracle with jv_mode = 1: the line-search slope comes from the assembled Jacobian
    (rhs - r after BiCGStab) instead of a difference of residuals, so one residual
    evaluation fewer per Newton iteration; the converged heads stay within the Newton
    tolerance of the jv_mode = 0 run."""
    from msg123_b200.config import make_config
    from oracle.oracle import Oracle
    p = make_config("hetero", shape=(12, 10, 8), seed=4)
    ov = dict(precon_type=1, ref_quirks=0, amg_lag=1, sim_type=0, inc_fact=1.0, ini_step=1800.0)
    runs = {}
    for jv in (0, 1):
        o = Oracle(p, jv_mode=jv, **ov)
        o.init_state()
        rc, st = o.advance(nsteps=3)
        assert rc == 0
        runs[jv] = (o.get_state()["head_new"], st, o.counters()["func"])
        o.close()
    h0, s0, f0 = runs[0]
    h1, s1, f1 = runs[1]
    assert np.max(np.abs(h1 - h0)) / np.max(np.abs(h0)) <= 1e-8
    # calc_vecjacf evaluates F once more per Newton iteration with jv_mode = 0
    assert f1 < f0
