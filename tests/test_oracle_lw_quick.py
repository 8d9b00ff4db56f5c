"""CPU checks of the oracle's lw and QUICK schemes (src/TOOLS/advq_lw.f90,
src/TOOLS/advq_quick.f90), the dispatcher's `case default` and `case ('quick')`
(src/TOOLS/advection.f90:603-614).

The C restatement (oracle/mimica_oracle.c advs_lw_*, advs_quick_*) is checked bit for
bit against an independent pure-Python transcription of the same Fortran on small
pencils, and both against known answers (a linear profile is advected at the exact
rate u * slope / dx by both schemes; the limiter switches fall back to the unlimited
formulas below lim_tol).
"""
import math

import numpy as np
import pytest

from fdd3260_b200 import config
from oracle import oracle as O

EPS = 1.e-18


def _min(a, b):      # the oracle's dmin2 (a < b ? a : b)
    return a if a < b else b


def _max(a, b):
    return a if a > b else b


def _sign1(b):
    return math.copysign(1.0, b)


# ---- advq_lw.f90 transcription ----
def _limiter_lw(lim_tol, x, ffip1, ffip2, ffim1):
    rp1 = rp2 = 1.0
    if abs(ffim1) > lim_tol * abs(x) + EPS:
        rp1 = ffip1 / ffim1
    if abs(ffip2) > lim_tol * abs(x) + EPS:
        rp2 = ffip1 / ffip2
    phil = _max(_min(_min(2. * rp1, 0.5 * (rp1 + 1.)), 2.), 0.)
    phir = _max(_min(_min(2. * rp2, 0.5 * (rp2 + 1.)), 2.), 0.)
    return phir, phil


def _fold(F, i1, i2, dx1, x, u, xa, adv):
    Fold = F[i1 - 1]
    for i in range(i1, i2 + 1):
        xa[i - 1] = xa[i - 1] + (F[i] - Fold) * dx1
        Fold = F[i]
    if adv:
        uold = u[i2]
        for i in range(i2, i1 - 1, -1):
            xa[i - 1] = xa[i - 1] - x[i - 1] * (uold - u[i - 1]) * dx1
            uold = u[i - 1]


def _lw_h(lim_tol, dt0, i1, i2, d, x, u, xa, adv):
    """advsx_lw (advq_lw.f90:57-123); 1-based arrays stored 0-based."""
    X = lambda i: x[i - 1]
    dx1 = 1. / d
    F = {}
    for i in range(i1 - 1, i2 + 1):
        uu, xx = u[i], X(i)
        ffip1 = X(i + 1) - xx
        ffim1 = xx - X(i - 1)
        ffip2 = X(i + 2) - X(i + 1)
        mu = abs(uu) * dt0 * dx1
        if abs(ffim1) > lim_tol * abs(xx) + EPS or abs(ffip2) > lim_tol * abs(xx) + EPS:
            phir, phil = _limiter_lw(lim_tol, xx, ffip1, ffip2, ffim1)
            fl = xx + 0.5 * phil * ffim1 * (1. - mu)
            fr = X(i + 1) - 0.5 * phir * ffip2 * (1. - mu)
        else:
            fl = xx + 0.5 * ffip1 * (1. - mu)
            fr = X(i + 1) - 0.5 * ffip1 * (1. - mu)
        F[i] = 0.5 * uu * (fl * (_sign1(uu) + 1.) - fr * (_sign1(uu) - 1.))
    _fold(F, i1, i2, dx1, x, u, xa, adv)


def _fold_z(F, nz, DW, xa):
    Fold = F[1]
    for k in range(2, nz):
        xa[k - 1] = xa[k - 1] + (F[k] - Fold) * DW(k)
        Fold = F[k]
    xa[0] = xa[0] + (F[1] - 0.) * DW(1)
    xa[nz - 1] = xa[nz - 1] + (0. - F[nz - 1]) * DW(nz)


def _z_faces(face, x, w, dz1):
    """The three face kinds of advsz_lw / advsz_quick: k = 1 (ffim1 = ffip1),
    2..nz-2, k = nz-1 (ffip2 = ffip1), bcl(5) = bcl(6) = 'nnf'."""
    nz = len(x)
    X = lambda k: x[k - 1]
    D1 = lambda k: dz1[k - 1]
    F = {}
    ffip1 = (X(2) - X(1)) * D1(1)
    F[1] = face(1, X(1), X(2), ffip1, ffip1, (X(3) - X(2)) * D1(2), w[1])
    for k in range(2, nz - 1):
        xx = X(k)
        F[k] = face(k, xx, X(k + 1), (xx - X(k - 1)) * D1(k - 1), (X(k + 1) - xx) * D1(k),
                    (X(k + 2) - X(k + 1)) * D1(k + 1), w[k])
    k = nz - 1
    ffip1 = (X(k + 1) - X(k)) * D1(k)
    F[k] = face(k, X(k), X(k + 1), (X(k) - X(k - 1)) * D1(k - 1), ffip1, ffip1, w[nz - 1])
    return F


def _lw_z(lim_tol, dt0, dz, dz1, dz1w, x, w, xa):
    """advsz_lw (advq_lw.f90:209-341), adv = .false."""
    DW = lambda k: dz1w[k - 1]

    def face(k, xx, xp1, ffim1, ffip1, ffip2, ww):
        mu = abs(ww) * dt0 * dz1[k - 1]
        if dz * abs(ffim1) > lim_tol * abs(xx) + EPS or dz * abs(ffip2) > lim_tol * abs(xx) + EPS:
            phir, phil = _limiter_lw(lim_tol, xx, ffip1, ffip2, ffim1)
            fl = xx + 0.5 * phil * ffim1 * (1. - mu) / DW(k)
            fr = xp1 - 0.5 * phir * ffip2 * (1. - mu) / DW(k)
        else:
            fl = xx + 0.5 * ffip1 * (1. - mu) / DW(k)
            fr = xp1 - 0.5 * ffip1 * (1. - mu) / DW(k)
        return 0.5 * ww * (fl * (_sign1(ww) + 1.) - fr * (_sign1(ww) - 1.))

    _fold_z(_z_faces(face, x, w, dz1), len(x), DW, xa)


# ---- advq_quick.f90 transcription ----
def _limiter_quick(lim_tol, phic, ffip1, ffip2, ffim1):
    c1 = 1. / 3.
    rp1 = rp2 = rp11 = rp21 = 1.0
    thr = lim_tol * abs(phic) + EPS
    if abs(ffim1) > thr:
        rp1 = ffip1 / ffim1
    if abs(ffip2) > thr:
        rp2 = ffip1 / ffip2
    if abs(ffip1) > thr:
        rp11 = ffim1 / ffip1
        rp21 = ffip2 / ffip1
    phil = rp1 * (1. - c1 * (1. - rp11))
    phir = rp2 * (1. - c1 * (1. - rp21))
    if abs(ffim1) > thr or abs(ffip2) > thr:
        phil = _max(0., _min(2. * rp1, _min(phil, 2.)))
        phir = _max(0., _min(2. * rp2, _min(phir, 2.)))
    return phil, phir


def _quick_h(lim_tol, i1, i2, d, x, u, xa, adv):
    """advsx_quick (advq_quick.f90:53-115)."""
    X = lambda i: x[i - 1]
    dx1 = 1. / d
    F = {}
    for i in range(i1 - 1, i2 + 1):
        uu, xx = u[i], X(i)
        ffip1 = X(i + 1) - xx
        ffip2 = X(i + 2) - X(i + 1)
        ffim1 = xx - X(i - 1)
        phil, phir = _limiter_quick(lim_tol, xx, ffip1, ffip2, ffim1)
        Fl = xx + 0.5 * phil * ffim1
        Fr = X(i + 1) - 0.5 * phir * ffip2
        F[i] = 0.5 * Fl * (uu + abs(uu)) + 0.5 * Fr * (uu - abs(uu))
    _fold(F, i1, i2, dx1, x, u, xa, adv)


def _quick_z(lim_tol, dz, dz1, dz1w, x, w, xa):
    """advsz_quick (advq_quick.f90:198-309), adv = .false."""
    DW = lambda k: dz1w[k - 1]

    def face(k, xx, xp1, ffim1, ffip1, ffip2, ww):
        phil, phir = _limiter_quick(lim_tol, xx / dz, ffip1, ffip2, ffim1)
        Fl = xx + 0.5 * phil * ffim1 / DW(k)
        Fr = xp1 - 0.5 * phir * ffip2 / DW(k)
        return 0.5 * Fl * (ww + abs(ww)) + 0.5 * Fr * (ww - abs(ww))

    _fold_z(_z_faces(face, x, w, dz1), len(x), DW, xa)


def _pencil(rng, n, flat_from):
    """Random pencil with a flat stretch (so the limiter switch is off there)."""
    x = rng.normal(size=n) * 0.3 + 290.0
    x[flat_from:flat_from + 5] = 290.0
    return x


def _wind(rng, n):
    """Winds of both signs, with exact zeros and a negative zero."""
    u = rng.normal(size=n) * 4.0
    u[::7] = 0.0
    u[3] = -0.0
    return u


@pytest.mark.parametrize("scheme", ["lw", "quick"])
@pytest.mark.parametrize("adv", [0, 1])
def test_horizontal_pencil_bit_exact_vs_transcription(scheme, adv):
    d = config.warm_bubble_domain(16, 16, 12, scheme=scheme, dt0=0.7)
    orc = O.Oracle(d)
    code = {"lw": O.LW, "quick": O.QUICK}[scheme]
    rng = np.random.default_rng(40)
    n, i1 = 28, 4
    i2 = n - 2
    for trial in range(6):
        x = _pencil(rng, n, 6 + trial)
        u = _wind(rng, n)
        xa = rng.normal(size=n)
        got = xa.copy()
        orc.L.mo_advs_h(orc.gp, code, n, i1, i2, d.dx, O.P(x), O.P(u), O.P(got), adv)
        ref = list(xa)
        if scheme == "lw":
            _lw_h(d.lim_tol, d.dt0, i1, i2, d.dx, list(x), list(u), ref, adv)
        else:
            _quick_h(d.lim_tol, i1, i2, d.dx, list(x), list(u), ref, adv)
        assert np.array_equal(got, np.array(ref))


@pytest.mark.parametrize("scheme", ["lw", "quick"])
def test_vertical_pencil_bit_exact_vs_transcription(scheme):
    d = config.cumulus_domain(16, 16, 30, scheme=scheme)   # stretched levels
    orc = O.Oracle(d)
    code = {"lw": O.LW, "quick": O.QUICK}[scheme]
    rng = np.random.default_rng(41)
    nz = d.nz
    for trial in range(6):
        x = _pencil(rng, nz, 3 + 2 * trial)
        w = _wind(rng, nz)
        w[0] = 0.0
        xa = rng.normal(size=nz)
        got = xa.copy()
        orc.L.mo_advs_z(orc.gp, code, O.P(x), O.P(w), O.P(got), 0)
        ref = list(xa)
        if scheme == "lw":
            _lw_z(d.lim_tol, d.dt0, d.dz, list(d.dz1), list(d.dz1w), list(x), list(w), ref)
        else:
            _quick_z(d.lim_tol, d.dz, list(d.dz1), list(d.dz1w), list(x), list(w), ref)
        assert np.array_equal(got, np.array(ref))


@pytest.mark.parametrize("scheme", ["lw", "quick"])
@pytest.mark.parametrize("sgn", [1.0, -1.0])
def test_linear_profile_exact_rate(scheme, sgn):
    """A linear profile x_i = a + b i has r = 1 everywhere: MC gives phi = 1 (the
    Lax-Wendroff face x_i + b (1 - mu) / 2), QUICK phi = 1 (x_i + b / 2); either way the
    flux difference over a cell is u b / dx."""
    d = config.warm_bubble_domain(16, 16, 12, scheme=scheme, dt0=0.5)
    orc = O.Oracle(d)
    code = {"lw": O.LW, "quick": O.QUICK}[scheme]
    n, i1 = 24, 4
    i2 = n - 2
    a, b, u0 = 3.0, 0.25, 2.0 * sgn
    x = a + b * np.arange(1, n + 1, dtype=np.float64)
    u = np.full(n, u0)
    xa = np.zeros(n)
    orc.L.mo_advs_h(orc.gp, code, n, i1, i2, d.dx, O.P(x), O.P(u), O.P(xa), 0)
    np.testing.assert_allclose(xa[i1 - 1:i2], u0 * b / d.dx, rtol=1e-12)


def test_lw_limiter_goes_upwind_at_an_extremum():
    """MC limiter: r < 0 at a local extremum gives phi = 0, so the face takes the upwind
    cell value; a face whose upwind slope is zero keeps phi = 1 (r defaults to 1)."""
    d = config.warm_bubble_domain(16, 16, 12, scheme="lw", dt0=0.5)
    orc = O.Oracle(d)
    n, i1 = 12, 4
    i2 = n - 2
    x = np.array([1., 1., 1., 1., 1., 2., 1., 1., 1., 1., 1., 1.])   # x(6) = 2
    u = np.full(n, 1.0)
    xa = np.zeros(n)
    orc.L.mo_advs_h(orc.gp, O.LW, n, i1, i2, d.dx, O.P(x), O.P(u), O.P(xa), 0)
    # face 5+1/2: ffim1 = 0 -> rp1 = 1, phi_l = 1, fl = x(5) = 1;
    # face 6+1/2: r = (x7 - x6) / (x6 - x5) = -1 -> phi_l = 0, fl = x(6) = 2
    assert xa[5] == (2.0 - 1.0) / d.dx
    # face 4+1/2 has ffim1 = ffip2 = 0: the unlimited branch, fl = x(4) + 0.5 (x5 - x4)(1 - mu) = 1
    assert xa[4] == 0.0
