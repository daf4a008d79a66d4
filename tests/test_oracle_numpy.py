"""A second, independent restatement of the water-only right-hand side,
written in numpy straight from the reference's Fortran, against the C oracle.

single_step_for_water (declarations_sph.f90:1439-1526) calls direct_find
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


def water_rhs(scene):
    prm = scene.params
    P = scene.phases[0]
    n = P.n
    x, vx, m, h = P.x, P.vx, P.mass, P.hsml
    rho, c = P.rho.copy(), P.c.copy()
    # direct_find: i < j in order, sqrt(r^2) < 2 * (h_i + h_j) / 2
    i, j = np.triu_indices(n, 1)
    dx = x[i, 0] - x[j, 0]
    dy = x[i, 1] - x[j, 1]
    r2 = dx * dx + dy * dy
    mh = (h[i] + h[j]) / 2.0
    keep = np.sqrt(r2) < 2 * mh
    i, j, dx, dy, r2, mh = i[keep], j[keep], dx[keep], dy[keep], r2[keep], mh[keep]
    w, gx, gy = _cubic(np.sqrt(r2), dx, dy, mh)
    # sum_density
    self_w = 15.0 / (7.0 * PI * h * h) * F32(2.0 / 3.0)
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


@pytest.mark.parametrize("seed", [3, 4])
def test_numpy_restatement_matches_the_c_oracle(seed):
    s = scenes.jitter(scenes.small("dam_break", precision=SPHG_FP64), 0.0004, seed=seed)
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
