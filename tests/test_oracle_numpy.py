"""A second, independent restatement of the three right-hand sides (water
only, soil only, two-phase), written in numpy straight from the reference's
Fortran, against the C oracle.

The water-only single_step_for_water (declarations_sph.f90:1439-1526) calls direct_find
(m_particles.f90:938), kernel (:1469, cubic spline), sum_density (:2243), df2
(:1802), delta_sph (:2658), the Tait pressure, df (:1711), art_visc (:2504)
and av_vel (:2761).  Every pair loop here scatters to both ends in pair order
(np.add.at over the pairs' (i, j) ends interleaved), as the Fortran loops do,
and every expression keeps the Fortran's operation order and its
default-real (single-precision) literals.  Integer powers are products, and
the Tait power is the C library's pow.  The two restatements then agree bit
for bit, and the test requires it.
"""
import math

import numpy as np
import pytest

from oracle import Oracle
from sources_b200 import scenes
from sources_b200.abi import SPHG_FP64

F32 = lambda v: float(np.float32(v))   # value of a Fortran default-real literal
PI = F32(3.14159265358979323846)       # real(dp), parameter :: pi = <default-real literal>


def _scatter(n, i, j, vi, vj, init=None):
    """out[i] += vi, out[j] += vj, pair by pair in list order, starting from
    init (zero by default) as the Fortran loops start from the array's value."""
    idx = np.empty(2 * len(i), dtype=np.int64)
    val = np.empty(2 * len(i))
    idx[0::2], idx[1::2] = i, j
    val[0::2], val[1::2] = vi, vj
    out = np.zeros(n) if init is None else np.array(init, dtype=np.float64)
    np.add.at(out, idx, val)
    return out


def _cubic(r, dx, dy, h):
    """kernel, skf = 1, dim = 2 (m_particles.f90:1469-1530).  Integer powers
    are products, as a Fortran compiler expands x**3."""
    q = r / h
    factor = 15.0 / (7.0 * PI * h * h)
    w = np.zeros_like(r)
    gx = np.zeros_like(r)
    gy = np.zeros_like(r)
    a = (q >= 0) & (q <= 1.0)
    qa = q[a]
    w[a] = factor[a] * (F32(2.0 / 3.0) - qa * qa + qa * qa * qa / 2.0)
    s = factor[a] * (-2.0 + 1.5 * qa) / (h[a] * h[a])
    gx[a], gy[a] = s * dx[a], s * dy[a]
    b = (q > 1.0) & (q <= 2)
    u = 2.0 - q[b]
    w[b] = factor[b] * 1.0 / 6.0 * (u * u * u)
    t = -factor[b] * 1.0 / 6.0 * 3.0 * (u * u) / h[b]
    gx[b], gy[b] = t * (dx[b] / r[b]), t * (dy[b] / r[b])
    return w, gx, gy


def _ipow(x, n):
    """x**n for an integer n, as x * x * ... * x from the left (the Fortran
    standard leaves the evaluation of x**n to the compiler)."""
    r = np.ones_like(x)
    for _ in range(n):
        r = r * x
    return r


def _kernel(skf, r, dx, dy, h):
    """kernel (m_particles.f90:1469-1602), dim = 2, every kernel function."""
    if skf == 1:
        return _cubic(r, dx, dy, h)
    q = r / h
    w = np.zeros_like(r)
    s = np.zeros_like(r)       # gradient = s * dx (inner branch) or s * (dx / r)
    inner = np.zeros(r.shape, dtype=bool)
    if skf == 2:
        factor = 1.0 / ((h * h) * math.pow(PI, 2 / 2.0))
        a = (q >= 0) & (q <= 3)
        w[a] = factor[a] * np.array([math.exp(v) for v in -q[a] * q[a]])
        gx = np.where(a, w * (-2.0 * dx / h / h), 0.0)
        gy = np.where(a, w * (-2.0 * dy / h / h), 0.0)
        return w, gx, gy
    if skf == 3:
        factor = 7.0 / (478.0 * PI * h * h)
        a = (q >= 0) & (q <= 1)
        b = (q > 1) & (q <= 2)
        c = (q > 2) & (q <= 3)
        w[a] = factor[a] * (_ipow(3 - q[a], 5) - 6 * _ipow(2 - q[a], 5) + 15 * _ipow(1 - q[a], 5))
        w[b] = factor[b] * (_ipow(3 - q[b], 5) - 6 * _ipow(2 - q[b], 5))
        w[c] = factor[c] * _ipow(3 - q[c], 5)
        gx, gy = np.zeros_like(r), np.zeros_like(r)
        # the reference's q <= 1 branch, kept as written (m_particles.f90:1554)
        ta = (-120 + 120 * q[a] - 50 * _ipow(q[a], 2)) / (h[a] * h[a])
        gx[a], gy[a] = factor[a] * (ta * dx[a]), factor[a] * (ta * dy[a])
        tb = factor[b] * (-5 * _ipow(3 - q[b], 4) + 30 * _ipow(2 - q[b], 4)) / h[b]
        gx[b], gy[b] = tb * (dx[b] / r[b]), tb * (dy[b] / r[b])
        tc = factor[c] * (-5 * _ipow(3 - q[c], 4)) / h[c]
        gx[c], gy[c] = tc * (dx[c] / r[c]), tc * (dy[c] / r[c])
        return w, gx, gy
    factor = 7.0 / (4.0 * PI * h * h)
    a = (q >= 0) & (q <= 2)
    w[a] = factor[a] * (_ipow(1 - q[a] / 2, 4) * (1 + 2 * q[a]))
    t = factor[a] * (-5 + 15 * q[a] / 2 - 15 * _ipow(q[a], 2) / 4 + 5 * _ipow(q[a], 3) / 8) / (h[a] * h[a])
    gx, gy = np.zeros_like(r), np.zeros_like(r)
    gx[a], gy[a] = t * dx[a], t * dy[a]
    return w, gx, gy


def water_rhs(scene):
    prm = scene.params
    P = scene.phases[0]
    n = P.n
    x, vx, m, h = P.x, P.vx, P.mass, P.hsml
    rho, c = P.rho.copy(), P.c.copy()
    # direct_find: i < j in order, sqrt(r^2) < scale_k * (h_i + h_j) / 2
    skf = prm.skf
    scale_k = 3 if skf in (2, 3) else 2
    i, j = np.triu_indices(n, 1)
    dx = x[i, 0] - x[j, 0]
    dy = x[i, 1] - x[j, 1]
    r2 = dx * dx + dy * dy
    mh = (h[i] + h[j]) / 2.0
    keep = np.sqrt(r2) < scale_k * mh
    i, j, dx, dy, r2, mh = i[keep], j[keep], dx[keep], dy[keep], r2[keep], mh[keep]
    w, gx, gy = _kernel(skf, np.sqrt(r2), dx, dy, mh)
    # sum_density: the kernel at r = 0 of each particle's own h
    zero = np.zeros(n)
    self_w = _kernel(skf, zero, zero, zero, h)[0]
    wi = _scatter(n, i, j, m[j] / rho[j] * w, m[i] / rho[i] * w, init=self_w * m / rho)
    rho = _scatter(n, i, j, m[j] * w, m[i] * w, init=self_w * m) / wi
    # drho = -rho * (df2(vx, 'x') + df2(vy, 'y'))
    def df2(f, g):
        fw = (f[j] - f[i]) * g
        return _scatter(n, i, j, m[j] * fw, m[i] * fw) / rho
    drho = -rho * (df2(vx[:, 0], gx) + df2(vx[:, 1], gy))
    # delta_sph(rho, drho)
    if prm.artificial_density:
        rr = 0.0 + dx * dx + dy * dy
        muv = 2.0 * (rho[i] - rho[j]) / rr
        hh = 0.0 + dx * muv * gx + dy * muv * gy
        d = prm.delta
        drho = _scatter(n, i, j, d * h[i] * c[i] * m[j] * hh / rho[j], -(d * h[j] * c[j] * m[i] * hh / rho[i]), init=drho)
    wm = prm.water
    p = P.p.copy()
    pos = rho > 0.0
    # the C library's pow, element by element (numpy's vectorised power may
    # differ from it in the last place)
    p[pos] = wm.b * (np.array([math.pow(r, wm.gamma) for r in rho[pos] / wm.rho0]) - 1)
    # df
    def df(f, g):
        fw = (f[i] + f[j]) * g
        return _scatter(n, i, j, m[j] / rho[j] * fw, -(m[i] / rho[i] * fw))
    c23 = F32(2.0 / 3.0)
    u, v = vx[:, 0], vx[:, 1]
    txx = c23 * (2.0 * df(u, gx) - df(v, gy))
    txy = df(u, gy) + df(v, gx)
    tyy = c23 * (2.0 * df(v, gy) - df(u, gx))
    sxx, syy, sxy = wm.viscosity * txx, wm.viscosity * tyy, wm.viscosity * txy
    ax = -df(p, gx) + df(sxx, gx) + df(sxy, gy)
    ay = -df(p, gy) + df(sxy, gx) + df(syy, gy)
    ax[pos] = ax[pos] / rho[pos]
    ay[pos] = ay[pos] / rho[pos]
    # art_visc
    if prm.visc_artificial:
        dvx, dvy = u[i] - u[j], v[i] - v[j]
        vr = 0.0 + dvx * dx + dvy * dy
        rr = 0.0 + dx * dx + dy * dy
        a = vr < 0.0
        etq = prm.etq
        muv = mh[a] * vr[a] / (rr[a] + mh[a] * mh[a] * etq * etq)
        mc = 0.5 * (c[i[a]] + c[j[a]])
        mrho = 0.5 * (rho[i[a]] + rho[j[a]])
        piv = (prm.beta * muv - prm.alpha * mc) * muv / mrho
        ia, ja = i[a], j[a]
        hx, hy = -piv * gx[a], -piv * gy[a]
        ax = _scatter(n, ia, ja, m[ja] * hx, -(m[ia] * hx), init=ax)
        ay = _scatter(n, ia, ja, m[ja] * hy, -(m[ia] * hy), init=ay)
    ay = ay + prm.gravity
    # av_vel
    av = np.zeros((n, 2))
    if prm.average_velocity:
        mrho = (rho[i] + rho[j]) / 2.0
        for d, comp in enumerate((u, v)):
            dv = comp[i] - comp[j]
            av[:, d] = _scatter(n, i, j, -(m[j] * dv / mrho * w), m[i] * dv / mrho * w)
        av[:P.ntotal] = prm.epsilon * av[:P.ntotal]
    # sxx and txx are one array in the reference (allocate_sph), so the working
    # arrays hold the stresses after newtonian_fluid
    return dict(rho=rho, drho=drho, p=p, dvx=np.stack([ax, ay], axis=1), av=av,
                txx=sxx, tyy=syy, txy=sxy, npairs=len(i))


@pytest.mark.parametrize("seed,skf", [(3, 1), (4, 1), (3, 2), (3, 3), (3, 4)])
def test_numpy_restatement_matches_the_c_oracle(seed, skf):
    s = scenes.jitter(scenes.small("dam_break", precision=SPHG_FP64, skf=skf), 0.0004, seed=seed)
    P = s.phases[0]
    P.vx[:P.ntotal] = np.random.default_rng(seed).normal(0, 0.05, size=(P.ntotal, 2))
    ref = water_rhs(s)
    o = Oracle(s)
    assert o.single_step(1) == 0
    d = o.download(1)
    assert len(o.pairs(0)[0]) == ref["npairs"]
    for f in ("rho", "drho", "p", "dvx", "av", "txx", "tyy", "txy"):
        a, b = np.asarray(getattr(d, f)), ref[f]
        assert np.array_equal(a, b), (f, int((a != b).sum()), float(np.abs(a - b).max()))


def soil_rhs(scene):
    """single_step_for_soil (declarations_sph.f90:1530-1655) with continuity
    density: con_density (m_particles.f90:2402), delta_sph (:2658),
    shear_strain_rate (:2855), velocity_divergence (:1996), pressure (:2133,
    c = soil c), drucker_prager_failure_criterion (:3323), df (:1711),
    plastic_or_not (:3447), plastic_flow_rule3 (:3700), Jaumann_rate (:3047),
    art_visc (:2504), delta_sph on p and the stresses, gravity, av_vel (:2761).
    The soil's spin array wxy is its txy working array (allocate_sph)."""
    prm = scene.params
    P = scene.phases[0]
    sm = prm.soil
    n = P.n
    x, vx, m, h = P.x, P.vx, P.mass, P.hsml
    rho, c = P.rho.copy(), P.c.copy()
    p, sxx, sxy, syy = P.p.copy(), P.sxx.copy(), P.sxy.copy(), P.syy.copy()
    eps_p = P.epsilon_p.copy()
    i, j = np.triu_indices(n, 1)
    dx = x[i, 0] - x[j, 0]
    dy = x[i, 1] - x[j, 1]
    r2 = dx * dx + dy * dy
    mh = (h[i] + h[j]) / 2.0
    keep = np.sqrt(r2) < 2 * mh
    i, j, dx, dy, r2, mh = i[keep], j[keep], dx[keep], dy[keep], r2[keep], mh[keep]
    w, gx, gy = _cubic(np.sqrt(r2), dx, dy, mh)
    u, v = vx[:, 0], vx[:, 1]
    # con_density
    vcc_k = (u[i] - u[j]) * gx + (v[i] - v[j]) * gy
    drho = _scatter(n, i, j, m[j] * vcc_k, m[i] * vcc_k)

    def delta(f, df):
        rr = 0.0 + dx * dx + dy * dy
        muv = 2.0 * (f[i] - f[j]) / rr
        hh = 0.0 + dx * muv * gx + dy * muv * gy
        d = prm.delta
        return _scatter(n, i, j, d * h[i] * c[i] * m[j] * hh / rho[j], -(d * h[j] * c[j] * m[i] * hh / rho[i]), init=df)
    if prm.artificial_density:
        drho = delta(rho, drho)
    # shear_strain_rate, dv = v_j - v_i
    du, dv = u[j] - u[i], v[j] - v[i]
    c23 = F32(2.0 / 3.0)
    hxx = c23 * (2.0 * du * gx - dv * gy)
    hxy = du * gy + dv * gx
    hyy = c23 * (2.0 * dv * gy - du * gx)
    txx = _scatter(n, i, j, m[j] * hxx / rho[j], m[i] * hxx / rho[i])
    txy = _scatter(n, i, j, m[j] * hxy / rho[j], m[i] * hxy / rho[i])
    tyy = _scatter(n, i, j, m[j] * hyy / rho[j], m[i] * hyy / rho[i])
    # velocity_divergence
    hv = du * gx + dv * gy
    vcc = _scatter(n, i, j, m[j] * hv / rho[j], m[i] * hv / rho[i])
    # pressure: c = soil c
    c = np.full(n, sm.c)
    # drucker_prager_failure_criterion
    t = math.tan(sm.phi)
    alpha1 = t / math.sqrt(9.0 + 12.0 * (t * t))
    p = np.where(p < 0.0, 0.0, p)
    I1 = 3.0 * p
    J2 = np.sqrt((sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy)) / 2.0) + 1.0e-6
    fail = J2 > alpha1 * I1
    skale = alpha1 * I1[fail] / J2[fail]
    sxx[fail], sxy[fail], syy[fail] = skale * sxx[fail], skale * sxy[fail], skale * syy[fail]

    def df(f, g):
        fw = (f[i] + f[j]) * g
        return _scatter(n, i, j, m[j] / rho[j] * fw, -(m[i] / rho[i] * fw))
    ax = -df(p, gx) + df(sxx, gx) + df(sxy, gy)
    ay = -df(p, gy) + df(sxy, gx) + df(syy, gy)
    pos = rho > 0.0
    ax[pos] = ax[pos] / rho[pos]
    ay[pos] = ay[pos] / rho[pos]
    dsxx, dsxy, dsyy, dp = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    K, G = sm.k, sm.E / (2.0 * (1 + sm.niu))
    # plastic_or_not, then plastic_flow_rule3 on the failed points
    J2a = np.sqrt((sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy)) / 2.0) + 1.0e-6
    fail = np.abs(J2a - alpha1 * I1) < F32(1.0e-5)
    for a in np.nonzero(fail)[0]:
        exx = txx[a] / 2.0 + vcc[a] / 3.0
        exy = txy[a] / 2.0
        eyy = tyy[a] / 2.0 + vcc[a] / 3.0
        sde = sxx[a] * exx + 2.0 * sxy[a] * exy + syy[a] * eyy
        J2f = (sxx[a] * sxx[a] + 2.0 * (sxy[a] * sxy[a]) + syy[a] * syy[a] + (sxx[a] + syy[a]) * (sxx[a] + syy[a])) / 2.0
        J2f = J2f + 1.0e-10
        dl = (3.0 * alpha1 * K * vcc[a] + G / math.sqrt(J2f) * sde) / (9.0 * (alpha1 * alpha1) * K + G)
        if dl < 0:
            continue
        dsxx[a] = dsxx[a] - dl * (G / math.sqrt(J2f) * sxx[a])
        dsxy[a] = dsxy[a] - dl * (G / math.sqrt(J2f) * sxy[a])
        dsyy[a] = dsyy[a] - dl * (G / math.sqrt(J2f) * syy[a])
        dp[a] = dp[a] + 3.0 * K * alpha1 * dl
        eps_p[a] = eps_p[a] + dl * sxy[a] / (2 * math.sqrt(J2f)) * F32(0.000005)
    # Jaumann_rate: Hooke, pressure rate, spin (into the txy array)
    dsxx, dsxy, dsyy = dsxx + G * txx, dsxy + G * txy, dsyy + G * tyy
    dp = dp - K * vcc
    hw = 0.5 * (du * gy - dv * gx)
    wxy = _scatter(n, i, j, m[j] * hw / rho[j], m[i] * hw / rho[i])
    dsxx = dsxx + 2.0 * sxy * wxy
    dsxy = dsxy - (sxx - syy) * wxy
    dsyy = dsyy - 2.0 * sxy * wxy
    # art_visc
    if prm.visc_artificial:
        ddx, ddy = u[i] - u[j], v[i] - v[j]
        vr = 0.0 + ddx * dx + ddy * dy
        rr = 0.0 + dx * dx + dy * dy
        a = vr < 0.0
        etq = prm.etq
        muv = mh[a] * vr[a] / (rr[a] + mh[a] * mh[a] * etq * etq)
        mc = 0.5 * (c[i[a]] + c[j[a]])
        mrho = 0.5 * (rho[i[a]] + rho[j[a]])
        piv = (prm.beta * muv - prm.alpha * mc) * muv / mrho
        ia, ja = i[a], j[a]
        hx, hy = -piv * gx[a], -piv * gy[a]
        ax = _scatter(n, ia, ja, m[ja] * hx, -(m[ia] * hx), init=ax)
        ay = _scatter(n, ia, ja, m[ja] * hy, -(m[ia] * hy), init=ay)
    if prm.soil_artificial_stress:
        dp, dsxx, dsxy, dsyy = delta(p, dp), delta(sxx, dsxx), delta(sxy, dsxy), delta(syy, dsyy)
    ay = ay + prm.gravity
    av = np.zeros((n, 2))
    if prm.average_velocity:
        mrho = (rho[i] + rho[j]) / 2.0
        for d, comp in enumerate((u, v)):
            dvd = comp[i] - comp[j]
            av[:, d] = _scatter(n, i, j, -(m[j] * dvd / mrho * w), m[i] * dvd / mrho * w)
        av[:P.ntotal] = prm.epsilon * av[:P.ntotal]
    return dict(drho=drho, p=p, sxx=sxx, sxy=sxy, syy=syy, dvx=np.stack([ax, ay], axis=1), av=av,
                dsxx=dsxx, dsxy=dsxy, dsyy=dsyy, dp=dp, epsilon_p=eps_p, fail=fail.astype(np.int32),
                txx=txx, tyy=tyy, txy=wxy, vcc=vcc, c=c, npairs=len(i))


@pytest.mark.parametrize("seed", [5, 6])
def test_numpy_soil_restatement_matches_the_c_oracle(seed):
    s = scenes.jitter(scenes.small("granular_column", precision=SPHG_FP64), 0.0002, seed=seed)
    P = s.phases[0]
    P.vx[:P.ntotal] = np.random.default_rng(seed).normal(0, 0.05, size=(P.ntotal, 2))
    ref = soil_rhs(s)
    o = Oracle(s)
    assert o.single_step(1) == 0
    d = o.download(1)
    assert len(o.pairs(0)[0]) == ref["npairs"]
    assert ref["fail"].sum() > 0                         # the flow rule is exercised
    assert np.array_equal(np.asarray(d.fail) != 0, ref["fail"] != 0)
    for f in ("drho", "p", "sxx", "sxy", "syy", "dvx", "av", "dsxx", "dsxy", "dsyy", "dp", "epsilon_p",
              "txx", "tyy", "txy", "vcc", "c"):
        a, b = np.asarray(getattr(d, f)), ref[f]
        assert np.array_equal(a, b), (f, int((a != b).sum()), float(np.abs(a - b).max()))


def _pairs(xa, ha, xb=None, hb=None):
    """direct_find (same phase, i < j) or direct_find_2 (i of a, j of b), in
    the reference's loop order, with the kernel of each pair."""
    if xb is None:
        i, j = np.triu_indices(len(xa), 1)
        xb, hb = xa, ha
    else:
        i, j = np.divmod(np.arange(len(xa) * len(xb)), len(xb))
    dx = xa[i, 0] - xb[j, 0]
    dy = xa[i, 1] - xb[j, 1]
    r2 = dx * dx + dy * dy
    mh = (ha[i] + hb[j]) / 2.0
    keep = np.sqrt(r2) < 2 * mh
    i, j, dx, dy, r2, mh = i[keep], j[keep], dx[keep], dy[keep], r2[keep], mh[keep]
    w, gx, gy = _cubic(np.sqrt(r2), dx, dy, mh)
    return i, j, dx, dy, mh, w, gx, gy


def two_phase_rhs(scene, itimestep=1):
    """single_step (declarations_sph.f90:1131-1435), water then soil, then the
    water x soil pairs: darcy_law, pore_water_pressure and the volume
    fractions (m_particles.f90:3832-3988).  The shared working arrays (txx,
    tyy, txy and the water stress that aliases them) are not returned."""
    prm = scene.params
    Wp, Sp = scene.phases
    out = {}
    state = {}
    for ph, P in ((1, Wp), (2, Sp)):
        water = ph == 1
        mat = prm.water if water else prm.soil
        n = P.n
        x, vx, m, h = P.x, P.vx, P.mass, P.hsml
        rho, c, vof = P.rho.copy(), P.c.copy(), P.vof.copy()
        p = P.p.copy()
        i, j, dx, dy, mh, w, gx, gy = _pairs(x, h)
        u, v = vx[:, 0], vx[:, 1]
        sc = lambda vi, vj, init=None: _scatter(n, i, j, vi, vj, init)

        def delta(f, df):
            rr = 0.0 + dx * dx + dy * dy
            muv = 2.0 * (f[i] - f[j]) / rr
            hh = 0.0 + dx * muv * gx + dy * muv * gy
            d = prm.delta
            return sc(d * h[i] * c[i] * m[j] * hh / rho[j], -(d * h[j] * c[j] * m[i] * hh / rho[i]), init=df)
        vk = (u[i] - u[j]) * gx + (v[i] - v[j]) * gy
        drho = sc(m[j] * vk, m[i] * vk)
        if prm.artificial_density:
            drho = delta(rho, drho)
        du, dv = u[j] - u[i], v[j] - v[i]
        c23 = F32(2.0 / 3.0)
        hxx = c23 * (2.0 * du * gx - dv * gy)
        hxy = du * gy + dv * gx
        hyy = c23 * (2.0 * dv * gy - du * gx)
        txx = sc(m[j] * hxx / rho[j], m[i] * hxx / rho[i])
        txy = sc(m[j] * hxy / rho[j], m[i] * hxy / rho[i])
        tyy = sc(m[j] * hyy / rho[j], m[i] * hyy / rho[i])
        pos = rho > 0.0
        if water:
            ratio = rho / (mat.rho0 * vof)
            p = mat.b * (np.array([math.pow(r, mat.gamma) for r in ratio]) - 1)
            c = mat.c * np.array([math.pow(r, 3.0) for r in ratio])
            sxx, syy, sxy = mat.viscosity * txx, mat.viscosity * tyy, mat.viscosity * txy

            def df(f, g):
                fw = (f[i] + f[j]) * g
                return sc(m[j] / rho[j] * fw, -(m[i] / rho[i] * fw))
            ax = -(vof * df(p, gx)) + df(vof * sxx, gx) + df(vof * sxy, gy)
            ay = -(vof * df(p, gy)) + df(vof * sxy, gx) + df(vof * syy, gy)
        else:
            hv = du * gx + dv * gy
            vcc = sc(m[j] * hv / rho[j], m[i] * hv / rho[i])
            c = np.full(n, mat.c)
            sxx, sxy, syy = P.sxx.copy(), P.sxy.copy(), P.syy.copy()
            t = math.tan(mat.phi)
            alpha1 = t / math.sqrt(9.0 + 12.0 * (t * t))
            p = np.where(p < 0.0, 0.0, p)
            I1 = 3.0 * p
            J2 = np.sqrt((sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy)) / 2.0) + 1.0e-6
            f1 = J2 > alpha1 * I1
            sk = alpha1 * I1[f1] / J2[f1]
            sxx[f1], sxy[f1], syy[f1] = sk * sxx[f1], sk * sxy[f1], sk * syy[f1]

            def df3(f, g):
                fw = (f[i] / (rho[i] * rho[i]) + f[j] / (rho[j] * rho[j])) * g
                return sc(m[j] * fw, -(m[i] * fw)) * rho
            ax = -df3(vof * p, gx) + df3(vof * sxx, gx) + df3(vof * sxy, gy)
            ay = -df3(vof * p, gy) + df3(vof * sxy, gx) + df3(vof * syy, gy)
        ax[pos] = ax[pos] / rho[pos]
        ay[pos] = ay[pos] / rho[pos]
        if not water:
            K, G = mat.k, mat.E / (2.0 * (1 + mat.niu))
            dsxx, dsxy, dsyy, dp = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
            eps_p = P.epsilon_p.copy()
            J2a = np.sqrt((sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy)) / 2.0) + 1.0e-6
            fail = np.abs(J2a - alpha1 * I1) < F32(1.0e-5)
            for a in np.nonzero(fail)[0]:
                exx = txx[a] / 2.0 + vcc[a] / 3.0
                exy = txy[a] / 2.0
                eyy = tyy[a] / 2.0 + vcc[a] / 3.0
                sde = sxx[a] * exx + 2.0 * sxy[a] * exy + syy[a] * eyy
                J2f = (sxx[a] * sxx[a] + 2.0 * (sxy[a] * sxy[a]) + syy[a] * syy[a]
                       + (sxx[a] + syy[a]) * (sxx[a] + syy[a])) / 2.0 + 1.0e-10
                dl = (3.0 * alpha1 * K * vcc[a] + G / math.sqrt(J2f) * sde) / (9.0 * (alpha1 * alpha1) * K + G)
                if dl < 0:
                    continue
                dsxx[a] = dsxx[a] - dl * (G / math.sqrt(J2f) * sxx[a])
                dsxy[a] = dsxy[a] - dl * (G / math.sqrt(J2f) * sxy[a])
                dsyy[a] = dsyy[a] - dl * (G / math.sqrt(J2f) * syy[a])
                dp[a] = dp[a] + 3.0 * K * alpha1 * dl
                eps_p[a] = eps_p[a] + dl * sxy[a] / (2 * math.sqrt(J2f)) * F32(0.000005)
            dsxx, dsxy, dsyy = dsxx + G * txx, dsxy + G * txy, dsyy + G * tyy
            dp = dp - K * vcc
            hw = 0.5 * (du * gy - dv * gx)
            wxy = sc(m[j] * hw / rho[j], m[i] * hw / rho[i])
            dsxx = dsxx + 2.0 * sxy * wxy
            dsxy = dsxy - (sxx - syy) * wxy
            dsyy = dsyy - 2.0 * sxy * wxy
        if prm.visc_artificial:
            ddx, ddy = u[i] - u[j], v[i] - v[j]
            vr = 0.0 + ddx * dx + ddy * dy
            rr = 0.0 + dx * dx + dy * dy
            a = vr < 0.0
            etq = prm.etq
            muv = mh[a] * vr[a] / (rr[a] + mh[a] * mh[a] * etq * etq)
            mc = 0.5 * (c[i[a]] + c[j[a]])
            mrho = 0.5 * (rho[i[a]] + rho[j[a]])
            piv = (prm.beta * muv - prm.alpha * mc) * muv / mrho
            ia, ja = i[a], j[a]
            hx, hy = -piv * gx[a], -piv * gy[a]
            ax = _scatter(n, ia, ja, m[ja] * hx, -(m[ia] * hx), init=ax)
            ay = _scatter(n, ia, ja, m[ja] * hy, -(m[ia] * hy), init=ay)
        dvof = np.zeros(n)
        if not water and prm.soil_artificial_stress:
            dp, dsxx, dsxy, dsyy = delta(p, dp), delta(sxx, dsxx), delta(sxy, dsxy), delta(syy, dsyy)
        if water and prm.water_artificial_volume:
            dvof = delta(vof, dvof)
        # repulsive_force: real-virtual pairs within dspp, on the real particle
        it = P.itype
        rep = it[i] * it[j] <= 0
        rr = np.sqrt(0.0 + dx * dx + dy * dy)
        rep &= ~(rr > P.dspp)
        for k in np.nonzero(rep)[0]:
            f = (math.pow(P.dspp / rr[k], prm.p1) - math.pow(P.dspp / rr[k], prm.p2)) / (rr[k] * rr[k])
            ii = j[k] if it[i[k]] < 0 else i[k]
            ax[ii] = ax[ii] + prm.dd * dx[k] * f
            ay[ii] = ay[ii] + prm.dd * dy[k] * f
        ay = ay + prm.gravity
        av = np.zeros((n, 2))
        if prm.average_velocity:
            mrho = (rho[i] + rho[j]) / 2.0
            for d, comp in enumerate((u, v)):
                dvd = comp[i] - comp[j]
                av[:, d] = sc(-(m[j] * dvd / mrho * w), m[i] * dvd / mrho * w)
            av[:P.ntotal] = prm.epsilon * av[:P.ntotal]
        res = dict(drho=drho, p=p, c=c, dvx=np.stack([ax, ay], axis=1), av=av, rho=rho, vof=vof)
        if water:
            res["dvof"] = dvof
        else:
            res.update(sxx=sxx, sxy=sxy, syy=syy, dsxx=dsxx, dsxy=dsxy, dsyy=dsyy, dp=dp, epsilon_p=eps_p,
                       vcc=vcc, fail=fail.astype(np.int32))
        out[ph] = res
    # water x soil pairs
    W, S = out[1], out[2]
    i, j, dx, dy, mh, w, gx, gy = _pairs(Wp.x, Wp.hsml, Sp.x, Sp.hsml)
    mw, ms = Wp.mass, Sp.mass
    rw, rs = W["rho"], S["rho"]
    vw, vs = Wp.vx, Sp.vx
    dvw, dvs = W["dvx"].copy(), S["dvx"].copy()
    vofw, vofs = W["vof"], S["vof"]
    ks = prm.soil.permeability
    for k in range(len(i)):           # darcy_law
        a, b = i[k], j[k]
        rrw = w[k] / (rw[a] * rs[b])
        cf = vofw[a] * vofs[b] * rw[a] * (-prm.numeric_gravity) / ks
        for d in range(2):
            sp = cf * (vw[a, d] - vs[b, d]) * rrw
            dvw[a, d] = dvw[a, d] - ms[b] * sp
            dvs[b, d] = dvs[b, d] + mw[a] * sp
    pw = W["p"]
    for k in range(len(i)):           # pore_water_pressure
        a, b = i[k], j[k]
        mprr = mw[a] * pw[a] / (rw[a] * rs[b])
        dvs[b, 0] = dvs[b, 0] + mprr * gx[k] * vofs[b]
        dvs[b, 1] = dvs[b, 1] + mprr * gy[k] * vofs[b]
    W["dvx"], S["dvx"] = dvw, dvs
    if prm.volume_fraction:
        S["vof"] = rs / prm.soil.rho0                                      # volume_fraction_soil
        tmp = (vw[i, 0] - vs[j, 0]) * gx + (vw[i, 1] - vs[j, 1]) * gy      # volume_fraction_water2
        dvof = W["dvof"].copy()
        np.add.at(dvof, i, -(ms[j] * tmp / prm.soil.rho0))
        W["dvof"] = dvof
        vof2 = np.zeros(Wp.n)                                              # volume_fraction_water
        np.add.at(vof2, i, ms[j] * w)
        W["vof2"] = 1.0 - vof2 / prm.soil.rho0
        # the renormalisation every renorm_interval steps (declarations_sph.f90:1414-1421)
        if prm.volume_fraction_renorm and prm.renorm_interval > 0 and itimestep % prm.renorm_interval == 0:
            r = W["rho"] / W["vof"]
            W["vof"] = W["vof2"].copy()
            W["rho"] = r * W["vof"]
    W["npairs_cross"] = len(i)
    return out


@pytest.mark.parametrize("seed,itimestep", [(7, 1), (8, 1), (7, 40)])
def test_numpy_two_phase_restatement_matches_the_c_oracle(seed, itimestep):
    """The two-phase right-hand side, at an ordinary step and at a step that
    renormalises the water volume fraction."""
    s = scenes.jitter(scenes.small("two_phase", precision=SPHG_FP64), 0.0002, seed=seed)
    rng = np.random.default_rng(seed)
    for P in s.phases:
        P.vx[:P.ntotal] = rng.normal(0, 0.03, size=(P.ntotal, 2))
    ref = two_phase_rhs(s, itimestep)
    o = Oracle(s)
    assert o.single_step(itimestep) == 0
    assert len(o.pairs(2)[0]) == ref[1]["npairs_cross"]
    fields = {1: ("drho", "p", "c", "dvx", "av", "rho", "vof", "dvof", "vof2"),
              2: ("drho", "p", "c", "dvx", "av", "rho", "vof", "sxx", "sxy", "syy", "dsxx", "dsxy", "dsyy", "dp",
                  "epsilon_p", "vcc")}
    for ph in (1, 2):
        d = o.download(ph)
        for f in fields[ph]:
            a, b = np.asarray(getattr(d, f)), ref[ph][f]
            assert np.array_equal(a, b), (ph, f, int((a != b).sum()), float(np.abs(a - b).max()))


def _dp_return(p, sxx, sxy, syy, phi):
    """drucker_prager_failure_criterion (m_particles.f90:3323-3381) on arrays."""
    t = math.tan(phi)
    alpha1 = t / math.sqrt(9.0 + 12.0 * (t * t))
    p = np.where(p < 0.0, 0.0, p)
    I1 = 3.0 * p
    J2 = np.sqrt((sxx * sxx + 2.0 * (sxy * sxy) + syy * syy + (sxx + syy) * (sxx + syy)) / 2.0) + 1.0e-6
    f = J2 > alpha1 * I1
    sk = alpha1 * I1[f] / J2[f]
    sxx, sxy, syy = sxx.copy(), sxy.copy(), syy.copy()
    sxx[f], sxy[f], syy[f] = sk * sxx[f], sk * sxy[f], sk * syy[f]
    return p, sxx, sxy, syy


def two_phase_run(scene, steps):
    """time_integration (declarations_sph.f90:525-791) of the two-phase step
    with stress_integration = 1: first_half and Drucker-Prager on the soil
    before the right-hand side (from the second step on), then first_step or
    second_half and Drucker-Prager again.  The right-hand side writes p, c,
    the soil stress, vof and eps_p back into the state, as the reference's
    routines do in place."""
    s = scene.copy()
    prm = s.params
    dt = prm.dt
    rates = {}
    mins = {}
    for it in range(1, steps + 1):
        W, S = s.phases
        if it != 1:
            for ph, P in ((1, W), (2, S)):
                r = rates[ph]
                mins[ph] = dict(rho=P.rho.copy(), v=P.vx.copy())
                P.rho[:] = P.rho + (dt / 2.0) * r["drho"]
                if ph == 1 and prm.volume_fraction:
                    mins[ph]["vof"] = P.vof.copy()
                    P.vof[:] = P.vof + (dt / 2.0) * r["dvof"]
                move = P.itype >= 0
                P.vx[move] = P.vx[move] + (dt / 2.0) * r["dvx"][move]
            S.p[:], S.sxx[:], S.sxy[:], S.syy[:] = _dp_return(S.p, S.sxx, S.sxy, S.syy, prm.soil.phi)
        out = two_phase_rhs(s, it)
        W.p[:], W.c[:] = out[1]["p"], out[1]["c"]
        for f in ("p", "sxx", "sxy", "syy", "c", "vof", "epsilon_p"):
            getattr(S, f)[:] = out[2][f]
        rates = out
        for ph, P in ((1, W), (2, S)):
            r = out[ph]
            if it == 1:
                P.rho[:] = P.rho + (dt / 2.0) * r["drho"]
                if ph == 1 and prm.volume_fraction:
                    P.vof[:] = P.vof + (dt / 2.0) * r["dvof"]
            else:
                P.rho[:] = mins[ph]["rho"] + dt * r["drho"]
                if ph == 1 and prm.volume_fraction:
                    P.vof[:] = mins[ph]["vof"] + dt * r["dvof"]
            if ph == 2:
                P.sxx[:] = P.sxx + dt * r["dsxx"]
                P.sxy[:] = P.sxy + dt * r["dsxy"]
                P.syy[:] = P.syy + dt * r["dsyy"]
                P.p[:] = P.p + dt * r["dp"]
            move = P.itype >= 0
            base = P.vx if it == 1 else mins[ph]["v"]
            hdt = dt / 2.0 if it == 1 else dt
            vnew = base[move] + hdt * r["dvx"][move] + r["av"][move]
            P.vx[move] = vnew
            P.x[move] = P.x[move] + dt * vnew
        S.p[:], S.sxx[:], S.sxy[:], S.syy[:] = _dp_return(S.p, S.sxx, S.sxy, S.syy, prm.soil.phi)
    return s


def test_numpy_two_phase_time_integration_matches_the_c_oracle():
    """Six leapfrog steps (the first step, then predictor / corrector) of the
    two-phase scene, numpy against the C oracle, bit for bit."""
    s = scenes.jitter(scenes.small("two_phase", precision=SPHG_FP64), 0.0002, seed=9)
    ref = two_phase_run(s, 6)
    o = Oracle(s)
    assert o.time_integration(6) == 0
    for ph, fields in ((1, ("x", "vx", "rho", "vof", "p", "c")),
                       (2, ("x", "vx", "rho", "vof", "p", "sxx", "sxy", "syy", "epsilon_p"))):
        d, r = o.download(ph), ref.phases[ph - 1]
        for f in fields:
            a, b = np.asarray(getattr(d, f)), np.asarray(getattr(r, f))
            assert np.array_equal(a, b), (ph, f, int((a != b).sum()), float(np.abs(a - b).max()))


def single_phase_run(scene, steps):
    """time_integration_for_water (declarations_sph.f90:794-886) or
    time_integration_for_soil (:978-1127), with the soil stress integrated by
    full-step Euler (stress_integration = 1) or leapfrog (2).  The right-hand
    side writes back what the reference's routines change in place: the
    summation density and p (water); p, the stresses, c and eps_p (soil)."""
    s = scene.copy()
    prm = s.params
    dt = prm.dt
    P = s.phases[0]
    soil = P.material == 2
    r = None
    leap = soil and prm.stress_integration == 2
    stress = ("sxx", "sxy", "syy", "p")
    rates = {"sxx": "dsxx", "sxy": "dsxy", "syy": "dsyy", "p": "dp"}
    for it in range(1, steps + 1):
        move = P.itype >= 0
        if it != 1:
            rho_min, v_min = P.rho.copy(), P.vx.copy()
            P.rho[:] = P.rho + (dt / 2.0) * r["drho"]
            if leap:
                smin = {f: getattr(P, f).copy() for f in stress}
                for f in stress:
                    getattr(P, f)[:] = getattr(P, f) + (dt / 2.0) * r[rates[f]]
            P.vx[move] = P.vx[move] + (dt / 2.0) * r["dvx"][move]
            if soil:
                P.p[:], P.sxx[:], P.sxy[:], P.syy[:] = _dp_return(P.p, P.sxx, P.sxy, P.syy, prm.soil.phi)
        if soil:
            r = soil_rhs(s)
            for f in ("p", "sxx", "sxy", "syy", "c", "epsilon_p"):
                getattr(P, f)[:] = r[f]
        else:
            r = water_rhs(s)
            P.rho[:], P.p[:] = r["rho"], r["p"]
        if it == 1:
            P.rho[:] = P.rho + (dt / 2.0) * r["drho"]
        else:
            P.rho[:] = rho_min + dt * r["drho"]
        if soil:
            for f in stress:
                if not leap:
                    getattr(P, f)[:] = getattr(P, f) + dt * r[rates[f]]
                elif it == 1:
                    getattr(P, f)[:] = getattr(P, f) + (dt / 2.0) * r[rates[f]]
                else:
                    getattr(P, f)[:] = smin[f] + dt * r[rates[f]]
        base = P.vx if it == 1 else v_min
        hdt = dt / 2.0 if it == 1 else dt
        vnew = base[move] + hdt * r["dvx"][move] + r["av"][move]
        P.vx[move] = vnew
        P.x[move] = P.x[move] + dt * vnew
        if soil:
            P.p[:], P.sxx[:], P.sxy[:], P.syy[:] = _dp_return(P.p, P.sxx, P.sxy, P.syy, prm.soil.phi)
    return s


@pytest.mark.parametrize("name,stress_integration", [("dam_break", 1), ("granular_column", 1),
                                                     ("granular_column", 2)])
def test_numpy_single_phase_time_integration_matches_the_c_oracle(name, stress_integration):
    """Six leapfrog steps of the water-only and the soil-only step (soil
    stress by Euler or by leapfrog), numpy against the C oracle, bit for bit."""
    s = scenes.jitter(scenes.small(name, precision=SPHG_FP64), 0.0002, seed=10)
    s.params.stress_integration = stress_integration
    ref = single_phase_run(s, 6)
    o = Oracle(s)
    assert o.time_integration(6) == 0
    fields = ("x", "vx", "rho", "p") + (("sxx", "sxy", "syy", "epsilon_p") if name == "granular_column" else ())
    d, r = o.download(1), ref.phases[0]
    for f in fields:
        a, b = np.asarray(getattr(d, f)), np.asarray(getattr(r, f))
        assert np.array_equal(a, b), (name, f, int((a != b).sum()), float(np.abs(a - b).max()))
