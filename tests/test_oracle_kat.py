"""Known-answer tests that pin the CPU oracle (the reference ships no tests or
golden vectors, and no Fortran compiler exists here, so these analytic checks are
what pins the restatement):

* van Genuchten / Mualem closed forms at chosen pressure heads (Calc_parameter.f90:15-77),
  and a second restatement with the C library's pow, bit for bit, in both kr forms;
* hydrostatic equilibrium gives F == 0 exactly (Calc_function.f90:24-101), and the residual
  equals a second term-by-term restatement (storage, upwind flow, recharge, surface, sea,
  free drainage) bit for bit;
* a unit-gradient saturated column between a ponded top and free drainage is steady, and
  an unsaturated column under recharge balances its fluxes term by term;
* make_matrix's dmat and lumat equal a second term-by-term restatement bit for bit;
* the finite-difference Jacobian of make_matrix agrees with a directional derivative of F,
  and calc_vecjacf is the Brown-Saad difference, recomputed bit for bit;
* calc_matvec sums each CSR row in order (recomputed bit for bit);
* BiCGStab + DILU solves the assembled system (Linear_solution.f90:234-493), and its
  iterates equal a second restatement of the Fortran recurrence bit for bit;
* the DILU diagonal and the ILU sweeps equal a second restatement bit for bit;
* the DILU diagonal equals the ILU(0) pivots of a dense LU restricted to the pattern, and the
  reference's AMG preconditioner returns exactly the fine DILU solve (quirk Q1);
* mass balance closes after a time step (Calc_function.f90:103-174), and calc_mass's nine
  volumes equal a second restatement bit for bit;
* the adaptive time step follows apply_heuri's three factors (Time_module.f90:1522-1543);
* the AMG strength filter and smoothed prolongation restated from the Fortran (P bit for
  bit) and the coarse operator equal to P^T A P;
* connectivity layout on a 2x2x3 box written out by hand (Set_condition.f90:1584-2026), and
  every face conductance equal to the distance-weighted harmonic mean of the two cells' K_s.
"""
import numpy as np
import pytest

from msg123_b200.config import make_config, F32
from oracle.oracle import Oracle


def vg_closed_form(psi, alpha, n, thr, ths):
    m = 1.0 - 1.0 / n
    se = (1.0 + abs(alpha * psi) ** n) ** (-m)
    theta = thr + (ths - thr) * se
    kr = np.sqrt(se) * (1.0 - (1.0 - se ** (1.0 / m)) ** m) ** 2
    return theta / ths, kr


def test_vg_closed_forms():
    p = make_config("box", shape=(2, 2, 3))
    o = Oracle(p)
    psi = np.array([-1e-3, -0.1, -1.0, -3.0, -10.0, 0.0, 0.5, -0.02, -0.3, -5.0, 2.0, -7.0])
    h = p.cell_top + psi
    s, kr, ss = o.srat_rperm(h)
    a, n = float(p.reta[0]), float(p.retn[0])
    thr, ths = float(p.resi[0]), float(p.poro[0])
    for k in range(12):
        if psi[k] >= 0:
            assert s[k] == 1.0 and kr[k] == 1.0 and ss[k] == float(p.ss[k])
        else:
            se, kk = vg_closed_form(psi[k], a, n, thr, float(F32(ths - thr)) + thr)
            assert s[k] == pytest.approx(se, rel=1e-12)
            assert kr[k] == pytest.approx(kk, rel=1e-10)
            assert ss[k] == 0.0


def test_vg_form1_closed_form_and_trajectory():
    """vg_form 1 (the library's two-pow kr) against the same closed form, and a time loop
    with it against the reference form: the same Newton and Krylov counts, heads within
    1e-12."""
    p = make_config("box", shape=(2, 2, 3), vg_form=1)
    o = Oracle(p)
    psi = np.array([-1e-3, -0.1, -1.0, -3.0, -10.0, 0.0, 0.5, -0.02, -0.3, -5.0, 2.0, -7.0])
    s, kr, ss = o.srat_rperm(p.cell_top + psi)
    a, n = float(p.reta[0]), float(p.retn[0])
    thr, ths = float(p.resi[0]), float(p.poro[0])
    for k in range(12):
        if psi[k] < 0:
            se, kk = vg_closed_form(psi[k], a, n, thr, float(F32(ths - thr)) + thr)
            assert kr[k] == pytest.approx(kk, rel=1e-10)
    runs = []
    for form in (0, 1):
        q = make_config("hetero", shape=(16, 12, 10), seed=11, vg_form=form)
        o = Oracle(q)
        o.init_state()
        rc, st = o.advance(nsteps=4)
        runs.append((rc, st, o.get_state()["head_new"]))
    (r0, s0, h0), (r1, s1, h1) = runs
    assert r0 == r1 == 0
    assert (s0["newton_total"], s0["krylov_total"]) == (s1["newton_total"], s1["krylov_total"])
    assert np.max(np.abs(h1 - h0)) <= 1e-12 * np.max(np.abs(h0))


def test_hydrostatic_equilibrium_is_exact():
    p = make_config("hetero", shape=(6, 5, 4), rain_mm_h=0.0)
    o = Oracle(p)
    o.init_state()
    f = o.calc_func(p.head0)
    assert np.all(f == 0.0)


def test_unit_gradient_column_is_steady():
    """A saturated box under 1 m of ponding (sea top) with free drainage at the bottom: total
    head falling by exactly the centre-to-centre distance per layer (the sea-face distance at
    the top) is a steady state -- the same flux K_s A enters through the sea face, crosses
    every layer and leaves as free drainage, and nothing moves sideways -- so F vanishes to
    rounding (Calc_function.f90:212-254 flow, :475-513 sea term, plus the free-drainage
    extension) and the time loop keeps it."""
    import dataclasses
    p = make_config("box", shape=(4, 3, 10))
    ls = p.params["len_scal"]
    sea = float(p.sea_head[0]) + 0.95 / ls
    p = dataclasses.replace(p, sea_head=np.full_like(p.sea_head, sea))
    N, nxy = p.ncalc, p.nx * p.ny
    dis = p.dis2face.reshape(6, N)          # face-major: up, north, west, east, south, down
    h = np.empty(N)
    h[:nxy] = sea - dis[0, :nxy]
    for c in range(nxy, N):
        h[c] = h[c - nxy] - (dis[5, c - nxy] + dis[0, c])
    assert np.min(h - p.cell_top) > 0.0     # saturated everywhere (kr = 1)
    o = Oracle(p)
    o.init_state(head=h)
    o.set_state(head_new=h, head_old=h, delt=1800.0)
    flux = float(p.ksz[0]) * float(p.face_area.reshape(6, N)[0, 0])
    assert np.max(np.abs(o.calc_func(h))) <= 1e-14 * flux
    rc, st = o.advance(nsteps=2)
    assert rc == 0 and st["accepted"] == 2
    assert np.max(np.abs(o.get_state()["head_new"] - h)) <= 1e-12 * np.max(np.abs(h))


def test_recharge_column_flux_balance():
    """An unsaturated column (suction 0.7 m at the top) under recharge, with free drainage
    and no sea layer: total head falls by the centre-to-centre distance per layer, so every
    vertical flux is K_s kr_up A (upwind kr from the upper cell, calc_hyd_upwind,
    Calc_parameter.f90:107-125) and F is the recharge (Calc_function.f90:256-275) minus the
    outflow plus the inflow from above, with the free drainage K_s kr A at the bottom."""
    import dataclasses
    p = make_config("box", shape=(3, 2, 4))
    ls = p.params["len_scal"]
    N, nxy = p.ncalc, p.nx * p.ny
    dis, far = p.dis2face.reshape(6, N), p.face_area.reshape(6, N)
    h = np.empty(N)
    h[:nxy] = p.cell_top[:nxy] - 0.7 / ls
    for c in range(nxy, N):
        h[c] = h[c - nxy] - (dis[5, c - nxy] + dis[0, c])
    _, kr, _ = Oracle(dataclasses.replace(p, sea_top=0)).srat_rperm(h)
    assert np.all(kr < 0.01)                 # well inside the unsaturated range
    ks = float(p.ksz[0])
    rech = ks * kr[:nxy] * far[0, :nxy]      # matches the top layer's drainage
    q = dataclasses.replace(p, sea_top=0, rech=rech)
    o = Oracle(q)
    o.init_state(head=h)
    o.set_state(head_new=h, head_old=h, delt=1800.0)
    f = o.calc_func(h)
    pred = np.zeros(N)
    pred[:nxy] += rech
    for c in range(N):
        out = ks * kr[c] * far[5, c]
        pred[c] -= out
        if c + nxy < N:
            pred[c + nxy] += out
    assert np.max(np.abs(f - pred)) <= 1e-15 * ks * far[0, 0]


def test_fd_jacobian_matches_directional_derivative():
    p = make_config("hetero", shape=(8, 7, 6), seed=3)
    o = Oracle(p)
    o.init_state()
    h = p.head0 + 0.002 * np.random.default_rng(1).standard_normal(p.ncalc)
    o.set_state(head_new=h)
    d, lu, r = o.make_matvec()
    v = np.random.default_rng(2).standard_normal(p.ncalc)
    eps = 1e-7
    fd = (o.calc_func(h + eps * v) - o.calc_func(h - eps * v)) / (2 * eps)
    jv = o.matvec(v)
    assert np.linalg.norm(jv - fd) / np.linalg.norm(fd) < 2e-2
    assert np.allclose(r, -o.calc_func(h), rtol=0, atol=0)


def test_bicgs_dilu_solves_system():
    p = make_config("hetero", shape=(10, 9, 8), seed=5)
    o = Oracle(p, maxinn_iter=200)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.01 * np.random.default_rng(0).standard_normal(p.ncalc))
    d, lu, r = o.make_matvec()
    x, last, it, conv = o.solve_linalg(float(r @ r), 1e-12)
    assert conv == 1
    res = r - o.matvec(x)
    assert np.linalg.norm(res) / np.linalg.norm(r) <= 1e-12 * 1.0001


def test_dilu_equals_ilu0_pivots():
    p = make_config("hetero", shape=(4, 3, 3), seed=9)
    o = Oracle(p)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.05 * np.random.default_rng(4).standard_normal(p.ncalc))
    d, lu, r = o.make_matvec()
    c = o.connect()
    n = p.ncalc
    A = np.diag(d)
    rows = np.repeat(np.arange(n), np.diff(c["offind"]))
    A[rows, c["offrow"] - 1] = lu
    pattern = A != 0
    U = A.copy()
    for k in range(n):                         # ILU(0) in natural order
        for i in range(k + 1, n):
            if pattern[i, k]:
                U[i, k] /= U[k, k]
                for j in range(k + 1, n):
                    if pattern[i, j]:
                        U[i, j] -= U[i, k] * U[k, j]
    dd = o.precon_dilu()
    assert np.allclose(dd, np.diag(U), rtol=1e-13, atol=0)


def test_mass_balance_closes():
    p = make_config("hetero", shape=(12, 10, 8), seed=11)
    o = Oracle(p, lin_tol=1e-12, maxinn_iter=200)
    o.init_state()
    rc, st = o.advance(nsteps=2)
    assert rc == 0
    m = o.calc_mass()
    inflow = m[2]
    assert inflow > 0
    assert abs(m[0] + m[1] + m[2] + m[4] + m[7] + m[8]) <= 1e-6 * inflow


def test_connectivity_by_hand():
    p = make_config("box", shape=(2, 2, 3))
    o = Oracle(p)
    c = o.connect()
    # cell 1 (0,0,top): west/north/up absent -> east(2), south(3), down(5)
    assert list(c["offind"][:3]) == [0, 3, 6]
    assert list(c["offrow"][:3]) == [2, 3, 5]
    assert list(c["conn_dir"][:3]) == [4, 5, 6]
    # middle-layer cell index 5 (ix=1, iy=0, iz=1; 1-based 6): up(2), west(5), south(8), down(10)
    k0, k1 = c["offind"][5], c["offind"][6]
    assert list(c["offrow"][k0:k1]) == [2, 5, 8, 10]
    assert list(c["conn_dir"][k0:k1]) == [1, 3, 5, 6]
    assert c["left_off"][c["conn_dir"] <= 3].tolist() == list(range(1, int((c["conn_dir"] <= 3).sum()) + 1))
    # interior faces: x 1*2*3, y 2*1*3, z 2*2*2 -> 6 + 6 + 8 = 20 faces, two entries each
    assert o.nnz == 40
    # sea layer on top: every top cell has one sea face
    from oracle.oracle import lib
    import ctypes
    assert lib().orc_nseal(ctypes.c_void_p(o.h)) == 4


def test_face_conductance_is_harmonic_mean():
    """set_dis_adj + set_sat_hyd (Set_condition.f90:2111-2158): the face conductance between
    cells i and j is the distance-weighted harmonic mean of their K_s, and area_dis is the
    face area over the centre-to-centre distance."""
    p = make_config("hetero", shape=(5, 4, 3), seed=21)
    o = Oracle(p)
    c = o.connect()
    N = p.ncalc
    dis, far = p.dis2face.reshape(6, N), p.face_area.reshape(6, N)
    ks = {1: p.ksz, 2: p.ksy, 3: p.ksx, 4: p.ksx, 5: p.ksy, 6: p.ksz}
    opp = {1: 6, 2: 5, 3: 4, 4: 3, 5: 2, 6: 1}
    for i in range(N):
        for k in range(c["offind"][i], c["offind"][i + 1]):
            j, d = c["offrow"][k] - 1, int(c["conn_dir"][k])
            d1, d2 = dis[d - 1, i], dis[opp[d] - 1, j]
            k1, k2 = float(ks[d][i]), float(ks[d][j])
            harm = k1 * k2 * (d1 + d2) / (d1 * k2 + d2 * k1)
            assert c["hydf"][k] == pytest.approx(harm, rel=1e-14)
            assert c["abyd"][k] == pytest.approx(far[d - 1, i] / (d1 + d2), rel=1e-15)


def test_time_step_heuristic():
    """apply_heuri (Time_module.f90:1522-1543): after an accepted step with n Newton
    iterations the next dt is 1.2, 1 or 0.8 times the last one for n <= int(0.4 maxout),
    n <= int(0.8 maxout) or more, capped at max_step; the simulated time is real(SP)."""
    p = make_config("hetero", shape=(12, 10, 8), seed=3)
    prm = p.params
    o = Oracle(p)
    o.init_state()
    incr, decr = int(prm["maxout_iter"] * 0.4), int(prm["maxout_iter"] * 0.8)
    rc, st = o.advance(nsteps=1)
    seen = set()
    for _ in range(7):
        n, dt, t = st["newton_total"], st["delt"], st["current_t"]
        rc, st = o.advance(nsteps=1)
        assert rc == 0 and st["rejected"] == 0
        factor = 1.2 if n <= incr else (1.0 if n <= decr else 0.8)
        seen.add(factor)
        assert st["delt"] == min(dt * factor, prm["max_step"])
        assert st["current_t"] == float(np.float32(t + st["delt"]))
    assert len(seen) >= 2                     # the sequence exercises more than one branch


def test_reference_amg_preconditioner_is_fine_dilu():
    """Quirk Q1: loop_amg's post-smoother restarts from outx = inrhs (Linear_solution.f90:
    495-740, :820), so with ref_quirks = 1 the reference's AMG preconditioner returns the
    fine-level DILU solve, bit for bit."""
    p = make_config("hetero", shape=(14, 12, 9), seed=4)
    h = p.head0 + 0.003 * np.random.default_rng(2).standard_normal(p.ncalc)
    out = []
    for kw in (dict(precon_type=1, ref_quirks=1), dict(precon_type=0)):
        o = Oracle(p, **kw)
        o.init_state()
        o.set_state(head_new=h, delt=1800.0)
        o.set_system(*o.make_matvec())
        out.append(o.precond(np.random.default_rng(7).standard_normal(p.ncalc)))
    assert np.array_equal(out[0], out[1])


def test_vecjacf_is_brown_saad_difference():
    """calc_vecjacf (Calc_function.f90:515-621): J v = -(F(x + eps v) - F(x)) / eps with
    eps = sign(x.v) sqrt(eps_SP) max(|x.v|, |v|_1) / |v|^2, recomputed here from the
    oracle's own residual with the same sequential sums -- bit for bit."""
    import math
    p = make_config("box", shape=(6, 5, 8))
    o = Oracle(p)
    o.init_state()
    rng = np.random.default_rng(3)
    x = p.head0 + 0.01 * rng.standard_normal(p.ncalc)
    v = rng.standard_normal(p.ncalc)
    l2_v = l2_x = l1_v = 0.0
    for a, b in zip(x.tolist(), v.tolist()):
        l2_v += b * b
        l2_x += a * b
        l1_v += abs(b)
    sign = -1.0 if l2_x < 0.0 else 1.0
    eps = sign * math.sqrt(float(np.finfo(np.float32).eps)) * max(abs(l2_x), l1_v) / l2_v
    f1 = o.calc_func(x)
    f2 = o.calc_func(x + eps * v)
    want = -(f2 - f1) * (1.0 / eps)
    assert np.array_equal(o.vecjacf(x, v), want)


def _seq_dot(a, b):
    s = 0.0
    for x, y in zip(a.tolist(), b.tolist()):
        s += x * y
    return s


def _bicgs(o, b, bnorm, errtol, maxit, x0=None):
    """solve_bicgs (Linear_solution.f90:234-493) written out again from the Fortran, with the
    oracle's own matvec and DILU apply and sequential sums; the first residual is calc_resi
    (Calc_simulation.f90:36-73: b - (d x + the row's entries in order)), i.e. b - A x0."""
    x = np.zeros_like(b) if x0 is None else x0.copy()
    resi = b.copy() if x0 is None else b - o.matvec(x0)
    rs = resi.copy()
    p = np.zeros_like(b)
    v = np.zeros_like(b)
    sk0, alpha, omega, rnorm = np.inf, 0.0, 1.0, 0.0
    for it in range(1, maxit + 1):
        sk = _seq_dot(resi, rs)
        if it == 1:
            p = resi.copy()
        else:
            beta = (sk / sk0) * (alpha / omega)
            p = resi + beta * (p - omega * v)
        z = o.precond(p)
        v = o.matvec(z)
        alpha = sk / _seq_dot(v, rs)
        x = x + alpha * z
        resi = resi - alpha * v
        rnorm = _seq_dot(resi, resi)
        if np.sqrt(rnorm / bnorm) <= errtol:
            return x, rnorm, it
        z = o.precond(resi)
        t = o.matvec(z)
        omega = _seq_dot(t, resi) / _seq_dot(t, t)
        x = x + omega * z
        resi = resi - omega * t
        rnorm = _seq_dot(resi, resi)
        if np.sqrt(rnorm / bnorm) <= errtol or it == maxit:
            return x, rnorm, it
        sk0 = sk
    return x, rnorm, maxit


@pytest.mark.parametrize("maxit,start", [(1, False), (2, False), (4, False), (3, True)])
def test_bicgstab_recurrence_restated_twice(maxit, start):
    """The oracle's BiCGStab against a second restatement of the same Fortran: identical
    iterates, residual norm and iteration count, bit for bit."""
    p = make_config("hetero", shape=(10, 8, 6), seed=5, precon_type=0, maxinn_iter=maxit)
    o = Oracle(p)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.004 * np.random.default_rng(1).standard_normal(p.ncalc), delt=1800.0)
    d, lu, b = o.make_matvec()
    o.set_system(d, lu, b)
    bnorm = _seq_dot(b, b)
    x0 = 0.1 * np.random.default_rng(2).standard_normal(p.ncalc) if start else None
    xo, last, it, _ = o.solve_linalg(bnorm, 1e-30, x0=x0)
    xp, rn, itp = _bicgs(o, b, bnorm, 1e-30, maxit, x0=x0)
    assert it == itp == maxit
    assert np.array_equal(xo, xp) and last == rn


def test_matvec_row_order():
    """calc_matvec (Linear_solution.f90:917-951): y_i = d_i x_i, then + lumat_k x_j over the
    row's CSR entries in order -- recomputed from the exported connectivity, bit for bit."""
    p = make_config("hetero", shape=(7, 6, 5), seed=8, precon_type=0)
    o = Oracle(p)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.004 * np.random.default_rng(4).standard_normal(p.ncalc), delt=1800.0)
    d, lu, b = o.make_matvec()
    o.set_system(d, lu, b)
    c = o.connect()
    x = np.random.default_rng(6).standard_normal(p.ncalc)
    y = np.empty(p.ncalc)
    xl, dl, ll = x.tolist(), d.tolist(), lu.tolist()
    for i in range(p.ncalc):
        t = dl[i] * xl[i]
        for k in range(c["offind"][i], c["offind"][i + 1]):
            t = t + ll[k] * xl[c["offrow"][k] - 1]
        y[i] = t
    assert np.array_equal(o.matvec(x), y)


def test_dilu_and_ilu_solve_restated():
    """precon_dilu and solve_ilu (Linear_solution.f90:742-855) written out again from the
    Fortran (lower = up/north/west faces, conn_dir <= 3): the DILU diagonal, the forward and
    backward sweeps, and the preconditioner apply agree bit for bit."""
    p = make_config("hetero", shape=(9, 7, 6), seed=13, precon_type=0)
    o = Oracle(p)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.004 * np.random.default_rng(5).standard_normal(p.ncalc), delt=1800.0)
    dm, lu, b = o.make_matvec()
    o.set_system(dm, lu, b)
    c = o.connect()
    n = p.ncalc
    off, row, dirs = c["offind"].tolist(), (c["offrow"] - 1).tolist(), c["conn_dir"].tolist()
    lul = lu.tolist()
    d = dm.tolist()
    for i in range(n):
        for k in range(off[i], off[i + 1]):
            r = row[k]
            if dirs[k] <= 3:
                dinv = 1.0 / d[r]
                for j in range(off[r], off[r + 1]):
                    if dirs[j] > 3 and row[j] == i:
                        d[i] = d[i] - lul[k] * dinv * lul[j]
    assert np.array_equal(o.precon_dilu(), np.array(d))
    rhs = np.random.default_rng(9).standard_normal(n)
    x = rhs.tolist()
    for i in range(n):
        t = x[i]
        for k in range(off[i], off[i + 1]):
            if dirs[k] <= 3:
                t = t - lul[k] * x[row[k]]
        x[i] = t / d[i]
    for i in range(n - 1, -1, -1):
        t = 0.0
        for k in range(off[i], off[i + 1]):
            if dirs[k] > 3:
                t = t + lul[k] * x[row[k]]
        x[i] = x[i] - t / d[i]
    assert np.array_equal(o.solve_ilu(np.array(d), rhs), np.array(x))
    assert np.array_equal(o.precond(rhs), np.array(x))


@pytest.mark.parametrize("vg_form", [0, 1])
def test_srat_rperm_restated(vg_form):
    """calc_srat_rperm (Calc_parameter.f90:15-77) written out again with the same operation
    order and the C library's pow (Python's math.pow; numpy's vectorised power differs in
    the last bit), theta_s - theta_r a single-precision difference as the real(SP) parameters
    give it; S and kr agree bit for bit.  vg_form 1 is the library's two-pow form of kr."""
    import math
    p = make_config("hetero", shape=(8, 7, 6), seed=17, vg_form=vg_form)
    o = Oracle(p)
    rng = np.random.default_rng(11)
    h = p.cell_top + rng.uniform(-3.0, 0.3, p.ncalc)
    for pert in (0.0, 1.19e-9):
        s, kr, ss = o.srat_rperm(h, pert)
        for i in range(p.ncalc):
            ph = float(h[i]) - float(p.cell_top[i]) + pert
            if ph >= 0.0:
                assert s[i] == 1.0 and kr[i] == 1.0 and ss[i] == float(p.ss[i])
                continue
            n = float(p.retn[i])
            m = 1.0 - 1.0 / n
            a = abs(ph * float(p.reta[i]))
            beta = math.pow(a, n)
            se = math.pow(1.0 + beta, -m)
            theta = float(p.resi[i]) + float(p.poro[i] - p.resi[i]) * se
            if vg_form == 0:
                t = 1.0 - math.pow(1.0 - math.pow(se, 1.0 / m), m)
            else:
                t = 1.0 - (0.0 if beta == 0.0 or se == 0.0 else se * (beta / a))
            assert s[i] == theta / float(p.poro[i]) and kr[i] == math.sqrt(se) * (t * t) and ss[i] == 0.0


def _vg(p, h, pert=0.0):
    """(S, kr, alp_ss) per cell as calc_srat_rperm computes them (reference kr form)."""
    import math
    S, kr, alp = [], [], []
    for i in range(p.ncalc):
        ph = float(h[i]) - float(p.cell_top[i]) + pert
        if ph < 0.0:
            n = float(p.retn[i])
            m = 1.0 - 1.0 / n
            beta = math.pow(abs(ph * float(p.reta[i])), n)
            se = math.pow(1.0 + beta, -m)
            S.append((float(p.resi[i]) + float(p.poro[i] - p.resi[i]) * se) / float(p.poro[i]))
            t = 1.0 - math.pow(1.0 - math.pow(se, 1.0 / m), m)
            kr.append(math.sqrt(se) * (t * t))
            alp.append(0.0)
        else:
            S.append(1.0)
            kr.append(1.0)
            alp.append(float(p.ss[i]))
    return S, kr, alp


@pytest.mark.parametrize("name,kw", [("box", dict(shape=(5, 4, 6))), ("hetero", dict(shape=(6, 5, 4), seed=23))])
def test_calc_func_restated(name, kw):
    """calc_func (Calc_function.f90:24-101) written out again term by term -- func_stochn
    (:176-210), func_connflow with upwind kr (:212-254, Calc_parameter.f90:107-125),
    func_rechterm (:256-275), func_surfterm (:304-391), func_sealterm (:475-513), summed in the
    reference's order, plus the free-drainage extension last -- on a state with ponded,
    unsaturated and saturated top cells; the oracle's residual agrees bit for bit."""
    import math
    p = make_config(name, **kw)
    N, S = p.ncalc, p.ncals
    rng = np.random.default_rng(31)
    h_old = p.head0 + 0.02 * rng.standard_normal(N)
    h = h_old + 0.01 * rng.standard_normal(N)
    h[: S // 3] = p.surf_top[: S // 3] + 0.003 / p.params["len_scal"]     # some ponded top cells
    sh = p.surf_top + rng.uniform(-0.01, 0.01, S) / p.params["len_scal"]
    o = Oracle(p)
    o.init_state()
    s_old = o.srat_rperm(h_old)[0]
    o.set_state(head_new=h, head_old=h_old, srat_old=s_old, surf_head=sh, delt=1800.0)
    o.set_recharge(p.rech)
    f = o.calc_func(h)

    Sn, kr, alp = _vg(p, h)
    c = o.connect()
    dis, far = p.dis2face.reshape(6, N), p.face_area.reshape(6, N)
    delt_inv = 1.0 / 1800.0
    out = []
    for i in range(N):
        ch1 = alp[i] * float(s_old[i]) * float(h_old[i])
        ch2 = alp[i] * Sn[i] * float(h[i])
        ch = (ch2 - ch1) + float(p.poro[i]) * (Sn[i] - float(s_old[i]))
        stof = -ch * delt_inv * float(p.cell_vol[i])
        conf = 0.0
        for k in range(c["offind"][i], c["offind"][i + 1]):
            j = c["offrow"][k] - 1
            dh = float(h[j]) - float(h[i])
            relat = kr[i] if -dh >= 0.0 else kr[j]
            conf = conf + float(c["hydf"][k]) * relat * float(c["abyd"][k]) * dh
        fs, seaf = 0.0, 0.0
        if i < S:
            x, sh_i = float(h[i]), float(sh[i])
            top, bot, reli, parm = (float(p.surf_top[i]), float(p.surf_bott[i]), float(p.surf_reli[i]),
                                    float(p.surf_parm[i]))
            rati = 1.0
            if x >= top:
                delh = sh_i - x if sh_i > top else top - x
            elif x >= bot:
                delh = sh_i - x if sh_i > bot else bot - x
                if reli != 0.0:
                    rati = math.pow(min((x - bot) / reli, 1.0), parm)
            elif sh_i > bot:
                delh = sh_i - bot
                if reli != 0.0:
                    rati = math.pow(min((sh_i - bot) / reli, 1.0), parm)
            else:
                delh = 0.0
            # a top cell under a sea layer meets the sea through its up face and has no
            # surface face: its surface conductance and area stay zero (set_connect)
            hyd_s, a_s = (0.0, 0.0) if p.sea_top else (float(p.ksz[i]), far[0, i])
            surf = hyd_s * (a_s / dis[0, i]) * delh * kr[i] * rati
            fs = float(p.rech[i]) + surf + 0.0 + 0.0
            if p.sea_top:
                seaf = 0.0 + float(p.ksz[i]) * kr[i] * (far[0, i] / dis[0, i]) * (float(p.sea_head[i]) - x)
        fi = fs + stof + conf + 0.0 + seaf
        if p.free_drainage and i >= N - S:
            fi = fi + (-((float(p.ksz[i]) * far[5, i]) * kr[i]))
        out.append(fi)
    assert np.array_equal(f, np.array(out))


@pytest.mark.parametrize("name,kw", [("box", dict(shape=(5, 4, 6))), ("hetero", dict(shape=(6, 5, 4), seed=23))])
def test_make_matrix_restated(name, kw):
    """make_matrix (Make_linearsystem.f90:70-285, :410-547) written out again: the storage
    derivative (form_stochn), the upwind flow chords with the perturbed kr on either side
    (form_connflow), the surface and sea boundary derivatives, summed in the reference's
    order, plus the free-drainage chord last; dmat and lumat agree bit for bit."""
    p = make_config(name, **kw)
    N, S = p.ncalc, p.ncals
    rng = np.random.default_rng(37)
    h_old = p.head0 + 0.02 * rng.standard_normal(N)
    h = h_old + 0.01 * rng.standard_normal(N)
    h[: S // 3] = p.surf_top[: S // 3] + 0.003 / p.params["len_scal"]
    sh = p.surf_top + rng.uniform(-0.01, 0.01, S) / p.params["len_scal"]
    o = Oracle(p, precon_type=0)
    o.init_state()
    s_old = o.srat_rperm(h_old)[0]
    o.set_state(head_new=h, head_old=h_old, srat_old=s_old, surf_head=sh, delt=1800.0)
    dm, lu, _ = o.make_matvec()

    newper = float(np.finfo(np.float32).eps) * float(np.float32(1.0) / np.float32(p.params["len_scal"]))
    npi = 1.0 / newper
    ps, pk, _ = _vg(p, h, newper)
    sn, kr, alp = _vg(p, h)
    c = o.connect()
    dis, far = p.dis2face.reshape(6, N), p.face_area.reshape(6, N)
    delt_inv = 1.0 / 1800.0
    lu_ref = np.zeros_like(lu)
    d_ref = []
    for i in range(N):
        dsr = (ps[i] - sn[i]) * npi
        dst = alp[i] * dsr * float(h[i])
        stod = -(float(p.poro[i]) * dsr + alp[i] * sn[i] + dst) * delt_inv * float(p.cell_vol[i])
        dc = 0.0
        for k in range(c["offind"][i], c["offind"][i + 1]):
            j = c["offrow"][k] - 1
            dh = float(h[j]) - float(h[i])
            hyd, ab = float(c["hydf"][k]), float(c["abyd"][k])
            rel_hyd = hyd * (kr[i] if -dh >= 0.0 else kr[j])
            h1 = hyd * (pk[i] if (-dh + newper) >= 0.0 else kr[j])
            h2 = hyd * (kr[i] if (-dh - newper) >= 0.0 else pk[j])
            con1 = (h1 - rel_hyd) * npi * dh * ab
            con2 = (h2 - rel_hyd) * npi * dh * ab
            lu_ref[k] = rel_hyd * ab + con2
            dc = dc + (-rel_hyd * ab) + con1
        ds, sead = 0.0, 0.0
        if i < S:
            x, shi = float(h[i]), float(sh[i])
            top, bot = float(p.surf_top[i]), float(p.surf_bott[i])
            if x >= top:
                delh, over = (shi - x if shi > top else top - x), 1.0
            elif x >= bot:
                delh, over = (shi - x if shi > bot else bot - x), 1.0
            elif shi > bot:
                delh, over = shi - bot, 0.0
            else:
                delh, over = 0.0, 1.0
            tran = 0.0 if p.sea_top else float(p.ksz[i]) * (far[0, i] / dis[0, i])
            ds = (-tran * kr[i] + (pk[i] - kr[i]) * npi * delh * tran * over) + 0.0 + 0.0
            if p.sea_top:
                ks, ab = float(p.ksz[i]), far[0, i] / dis[0, i]
                dsea = float(p.sea_head[i]) - x
                sead = 0.0 + (-(kr[i] * ks) * ab) + (pk[i] * ks - kr[i] * ks) * npi * dsea * ab
        di = ds + stod + dc + sead
        if p.free_drainage and i >= N - S:
            di = di + (-((pk[i] - kr[i]) * npi * (float(p.ksz[i]) * far[5, i])))
        d_ref.append(di)
    assert np.array_equal(lu, lu_ref)
    assert np.array_equal(dm, np.array(d_ref))


def test_amg_prolongation_and_galerkin():
    """The AMG built by the oracle, level 1 -> 2, against the reference's formulas:
    make_grapfilt's strength filter (Make_amg_matrix.f90:66-111: a_ij strong when
    a_ij^2 > |d_i d_j theta^2| and d_i d_j a_ij > 0, weak entries lumped into the filtered
    diagonal) and make_prolomat's smoothed prolongation (:224-371: columns in order of first
    appearance among the strong neighbours' aggregates, then the row's own; values
    -sum a_ij * omega / d~_i, plus 1 - omega on the own aggregate), restated from the
    Fortran with the oracle's aggregates -- P bit for bit; and the coarse operator equal
    to P^T A P (scipy) to rounding."""
    import scipy.sparse as sp
    p = make_config("hetero", shape=(12, 10, 8), seed=4, precon_type=1, ref_quirks=0, amg_coarse_max=50)
    o = Oracle(p)
    o.init_state()
    o.set_state(head_new=p.head0 + 0.003 * np.random.default_rng(2).standard_normal(p.ncalc), delt=1800.0)
    o.set_system(*o.make_matvec())
    lv = o.amg_levels()
    assert len(lv) >= 2
    l0, l1 = lv[0], lv[1]
    d, lu, off, col, agg = (l0["dmat"].tolist(), l0["lumat"].tolist(), l0["offind"].tolist(),
                            l0["offrow"].tolist(), l1["agg"].tolist())
    th = float(np.float32(p.params["amg_theta"]))
    th2, om = th * th, float(np.float32(p.params["jac_omega"]))
    pind, pcol, pval = [0], [], []
    for i in range(l0["n"]):
        td, strong = d[i], []
        for k in range(off[i], off[i + 1]):
            dd = d[i] * d[col[k]]
            if lu[k] * lu[k] > abs(dd * th2) and dd * lu[k] > 0.0:
                strong.append(k)
            else:
                td = td + lu[k]
        ags = []
        for k in strong:
            a = agg[col[k]]
            if a >= 0 and a not in ags:
                ags.append(a)
        if agg[i] >= 0 and agg[i] not in ags:
            ags.append(agg[i])
        vals = [0.0] * len(ags)
        for k in strong:
            a = agg[col[k]]
            if a >= 0:
                vals[ags.index(a)] = vals[ags.index(a)] - lu[k]
        vals = [v * om / td for v in vals]
        if agg[i] >= 0:
            q = ags.index(agg[i])
            vals[q] = vals[q] + 1.0 - om
        pcol += ags
        pval += vals
        pind.append(len(pcol))
    assert l1["pindex"].tolist() == pind and l1["poffrow"].tolist() == pcol
    assert np.array_equal(l1["pval"], np.array(pval))
    n0, n1 = l0["n"], l1["n"]
    A = sp.csr_matrix((l0["lumat"], l0["offrow"], l0["offind"]), shape=(n0, n0)) + sp.diags(l0["dmat"])
    P = sp.csr_matrix((l1["pval"], l1["poffrow"], l1["pindex"]), shape=(n0, n1))
    Ac = (P.T @ A @ P).toarray()
    Ao = sp.csr_matrix((l1["lumat"], l1["offrow"], l1["offind"]), shape=(n1, n1)).toarray() + np.diag(l1["dmat"])
    assert np.max(np.abs(Ao - Ac)) <= 1e-12 * np.max(np.abs(Ac))


@pytest.mark.parametrize("name,kw", [("box", dict(shape=(5, 4, 6))), ("hetero", dict(shape=(6, 5, 4), seed=23))])
def test_calc_mass_restated(name, kw):
    """calc_mass (Calc_function.f90:103-174, sfla = 0) written out again: storage change with
    the old level's storage coefficient, upwind flow, recharge, surface (against the surface
    heads of the previous step), sea and the free-drainage extension, each times delt and
    summed over cells in order -- the oracle's nine volumes agree bit for bit."""
    import math
    p = make_config(name, **kw)
    N, S = p.ncalc, p.ncals
    rng = np.random.default_rng(41)
    h_old = p.head0 + 0.02 * rng.standard_normal(N)
    h = h_old + 0.01 * rng.standard_normal(N)
    h[: S // 3] = p.surf_top[: S // 3] + 0.003 / p.params["len_scal"]
    sh = p.surf_top + rng.uniform(-0.01, 0.01, S) / p.params["len_scal"]
    delt = 1800.0
    o = Oracle(p)
    o.init_state()
    s_old = o.srat_rperm(h_old)[0]
    o.set_state(head_new=h, head_old=h_old, srat_old=s_old, surf_head=sh, delt=delt)
    o.set_recharge(p.rech)
    got = o.calc_mass()

    _, _, alp_o = _vg(p, h_old)
    sn, kr, alp_n = _vg(p, h)
    c = o.connect()
    dis, far = p.dis2face.reshape(6, N), p.face_area.reshape(6, N)
    acc = [0.0] * 9
    for i in range(N):
        ch1 = alp_o[i] * float(s_old[i]) * float(h_old[i])
        ch2 = alp_n[i] * sn[i] * float(h[i])
        ch = (ch2 - ch1) + float(p.poro[i]) * (sn[i] - float(s_old[i]))
        acc[0] += -ch * (1.0 / delt) * float(p.cell_vol[i]) * delt
        cf = 0.0
        for k in range(c["offind"][i], c["offind"][i + 1]):
            j = c["offrow"][k] - 1
            dh = float(h[j]) - float(h[i])
            cf = cf + float(c["hydf"][k]) * (kr[i] if -dh >= 0.0 else kr[j]) * float(c["abyd"][k]) * dh
        acc[1] += cf * delt
        if p.free_drainage and i >= N - S:
            acc[8] += -((float(p.ksz[i]) * far[5, i]) * kr[i]) * delt
    for s in range(S):
        x, shs = float(h[s]), float(sh[s])
        top, bot, reli, parm = float(p.surf_top[s]), float(p.surf_bott[s]), float(p.surf_reli[s]), float(p.surf_parm[s])
        rati = 1.0
        if x >= top:
            delh = shs - x if shs > top else top - x
        elif x >= bot:
            delh = shs - x if shs > bot else bot - x
            if reli != 0.0:
                rati = math.pow(min((x - bot) / reli, 1.0), parm)
        elif shs > bot:
            delh = shs - bot
            if reli != 0.0:
                rati = math.pow(min((shs - bot) / reli, 1.0), parm)
        else:
            delh = 0.0
        hyd_s, a_s = (0.0, 0.0) if p.sea_top else (float(p.ksz[s]), far[0, s])
        acc[2] += float(p.rech[s]) * delt
        acc[4] += hyd_s * (a_s / dis[0, s]) * delh * kr[s] * rati * delt
    if p.sea_top:
        for s in range(S):
            dh = float(p.sea_head[s]) - float(h[s])
            acc[7] += float(p.ksz[s]) * kr[s] * (far[0, s] / dis[0, s]) * dh * delt
    assert np.array_equal(got, np.array(acc))


def test_reference_expressible_box():
    """Config 1R (sea-layer top, no-flow bottom, Eisenstat-Walker tolerance, absolute
    criterion): water ponded on the top enters through the sea faces and is all stored --
    no drainage volume, and the step's volumes balance."""
    p = make_config("box1r", shape=(6, 5, 10), nsteps=3)
    assert p.free_drainage == 0 and p.params["lin_tol"] == 0.0 and p.params["criteria_rel"] == 0
    o = Oracle(p)
    o.init_state()
    rc, st = o.advance(nsteps=3)
    assert rc == 0 and st["accepted"] == 3
    m = o.calc_mass()
    assert m[8] == 0.0 and m[7] > 0.0          # no drainage; inflow from the ponded layer
    assert abs(m[0] + m[1] + m[4] + m[7]) <= 1e-10 * m[7]       # measured 2.7e-12


@pytest.mark.parametrize("name,kw", [("box", dict(shape=(5, 4, 7))), ("hetero", dict(shape=(8, 7, 6), seed=3))])
def test_cell_mass_sums_to_calc_mass(name, kw):
    """calc_cell_mas restated per cell: summed over cells in the same order, each array
    gives calc_mass's whole-grid total bit for bit (storage, flow, drainage: cells in order;
    recharge, surface: columns in order), and the sea volume lands in the top cells only."""
    p = make_config(name, **kw)
    o = Oracle(p)
    o.init_state()
    rc, _ = o.advance(nsteps=2)
    assert rc == 0
    cm = o.cell_mass()
    tot = o.calc_mass()
    seq = lambda a: float(np.add.accumulate(a)[-1]) if len(a) else 0.0
    assert seq(cm["sto"]) == tot[0]
    assert seq(cm["con"]) == tot[1]
    assert seq(cm["rec"]) == tot[2]
    assert seq(cm["sur"]) == tot[4]
    assert abs(cm["sea"].sum() - tot[7]) <= 1e-14 * max(abs(tot[7]), 1e-300)
    assert not np.any(cm["sea"][p.ncals:])
    bottom = cm["drn"]
    assert abs(bottom.sum() - tot[8]) <= 1e-13 * max(abs(tot[8]), 1e-300)
    if not p.free_drainage:
        assert not np.any(bottom)


def test_velocity_unit_gradient_column():
    """calc_outvelc on a saturated column under a unit head gradient: every interior face
    carries the saturated conductivity, inward from above and outward below (facev(up) =
    +Ks, facev(down) = -Ks), so the cell-centred vertical velocity is -Ks (downward, the
    half-difference of the opposite-signed pair); the horizontal components are zero and
    the bottom face of the lowest cell carries the free-drainage velocity -Ks."""
    p = make_config("box", shape=(1, 1, 6))
    o = Oracle(p)
    o.init_state()
    dz = p.cell_top[0] - p.cell_top[1]
    h = np.full(p.ncalc, p.cell_top[0] + 0.5)         # equal heads, saturated: no flow between cells
    o.set_state(head_new=h, head_old=h, srat_old=np.ones(p.ncalc), surf_head=h[:1])
    fv, pv = o.velocity()
    assert not np.any(fv[1:5]) and not np.any(fv[0, 1:]) and not np.any(fv[5, :-1])
    h2 = p.cell_top[0] + 0.5 - dz * np.arange(p.ncalc)   # head drops by dz per cell: unit gradient
    o.set_state(head_new=h2, head_old=h2, srat_old=np.ones(p.ncalc), surf_head=h2[:1])
    fv, pv = o.velocity()
    ks = float(p.ksz[0])
    inner = np.arange(1, p.ncalc - 1)
    assert np.allclose(fv[0, inner], ks, rtol=1e-12)
    assert np.allclose(fv[5, inner], -ks, rtol=1e-12)
    assert np.allclose(pv[2, inner], -ks, rtol=1e-12)
    assert not np.any(pv[:2])
    assert fv[5, -1] == -ks                            # free drainage at the bottom, kr = 1


def _boundary_tables(p):
    """A river over three top cells, a lake over one, and two wells of three cells each
    (vertical, one extracting and one injecting), on a heterogeneous block."""
    nx, ny, S = p.nx, p.ny, p.ncals
    top = p.cell_top[:S]
    riv_cells = np.array([2, nx + 3, 2 * nx + 4])            # 1-based surface cells
    rs = riv_cells - 1
    riv = (riv_cells, top[rs] + 0.02, top[rs] - 0.05, np.full(3, 2.5))
    lk = np.array([S - 1])
    lak = (lk, top[lk - 1] - 0.01, top[lk - 1] - 0.2, np.array([1.7]))
    c1 = 1 + (nx // 2) + nx * (ny // 2)                       # a column in the middle
    c2 = 2 + nx * 1
    col = lambda c: np.array([c + k * S for k in (1, 2, 3)])
    wells = (np.array([0, 3, 6]), np.concatenate([col(c1), col(c2)]), np.full(6, 0.8),
             np.array([float(p.cell_top[-1]) - 1.0, float(p.cell_top[-1]) - 1.0]),
             np.array([-2.0e-4, 1.0e-4]))
    return riv, lak, wells


def test_river_lake_terms_added_to_residual_and_diagonal():
    """func_riveterm / func_laketerm enter F on their surface cells only, as
    hydf_surf * abyd * (stage - head) * kr (head above the bed) or * (stage - bed) (only the
    stage above), and set_rivebound / set_lakebound add -tran kr + the kr chord to dmat."""
    p = make_config("hetero", shape=(8, 7, 6), seed=5)
    o = Oracle(p)
    o.init_state()
    rng = np.random.default_rng(2)
    h = p.cell_top + rng.uniform(-0.3, 0.05, p.ncalc)
    o.set_state(head_new=h, delt=600.0)
    f0 = o.calc_func(h)
    d0, lu0, r0 = o.make_matvec()
    riv, lak, _ = _boundary_tables(p)
    o.set_rivers(*riv)
    o.set_lakes(*lak)
    f1 = o.calc_func(h)
    d1, lu1, r1 = o.make_matvec()
    # newper = epsilon(1._SP) * len_scal_inv, the reciprocal in single precision (Prep_calculation.f90:79)
    newper = 1.1920928955078125e-07 * float(np.float32(1.0) / np.float32(p.params["len_scal"]))
    s_, kr, _ = o.srat_rperm(h)
    _, krp, _ = o.srat_rperm(h, newper)
    touched = set()
    for cells, head, bott, abyd in (riv, lak):
        for c, st, bd, ab in zip(cells, head, bott, abyd):
            s = c - 1
            touched.add(s)
            hy = float(p.ksz[s])
            if h[s] >= bd:
                delh, over = st - h[s], 1.0
            elif st > bd:
                delh, over = st - bd, 0.0
            else:
                delh, over = 0.0, 1.0
            term = hy * ab * delh * kr[s]
            assert abs((f1[s] - f0[s]) - term) <= 1e-12 * max(abs(f1[s]), abs(term))
            tran = hy * ab
            dd = -tran * kr[s] + (krp[s] - kr[s]) * (1.0 / newper) * delh * tran * over
            assert abs((d1[s] - d0[s]) - dd) <= 1e-10 * max(abs(d1[s]), abs(dd))
    rest = np.array([i for i in range(p.ncalc) if i not in touched])
    assert np.array_equal(f1[rest], f0[rest]) and np.array_equal(d1[rest], d0[rest])
    assert np.array_equal(lu1, lu0)


def test_well_rates_deliver_the_pumping_rate():
    """set_vwell_head: the virtual well head is set so that the cells' kr*abyd*(whead - h)
    add up to the pumping rate, so over a step the well volumes of calc_mass are the
    rates times delt; the step's volumes balance to the accuracy of the Newton solve (its
    test is on the head change, 1e-8 of max|h|, which leaves ~1e-6 of the volumes here)."""
    p = make_config("hetero", shape=(8, 7, 6), seed=5)
    o = Oracle(p)
    o.init_state()
    _, _, wells = _boundary_tables(p)
    o.set_wells(*wells)
    rc, st = o.advance(nsteps=1)
    assert rc == 0
    m = o.calc_mass()
    delt = st["delt"]
    assert abs(m[3] - wells[4].sum() * delt) <= 1e-12 * abs(wells[4]).sum() * delt
    cm = o.cell_mass()
    assert abs(cm["wel"].sum() - m[3]) <= 1e-14 * abs(m[3]) + 1e-300
    assert np.count_nonzero(cm["wel"]) == 6
    assert abs(float(np.sum(m))) <= 1e-5 * (abs(m[2]) + abs(wells[4]).sum() * delt)
