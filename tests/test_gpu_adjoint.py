"""Tangent linear and adjoint of the WENO scalar advection operator (mg_advection_tl /
mg_advection_ad): dot-product test (adjoint against tangent linear, both from the same
face Jacobians: agreement to round-off, 1e-12 relative) and Taylor test against the FP64
forward operator (the remainder of the first-order expansion falls as h^2)."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config
from fdd3260_b200.autograd import AdvectionFunction, FnContext

pytestmark = pytest.mark.gpu


def _interior(a):
    return a[:, 3:-2, 3:-2]


def _problem(seed):
    d = config.cumulus_domain(32, 32, 24)
    rng = np.random.default_rng(seed)
    st = config.random_state(d, seed=seed)
    x = st.scal[0] * st.dens   # density-weighted field
    mu = st.u * d.den0[:, None, None]
    mv = st.v * d.den0[:, None, None]
    mw = st.w * d.avden0[:, None, None]
    mw[0] = 0.0

    def field(scale):
        a = np.zeros(d.shape)
        a[:, 3:-2, 3:-2] = scale * rng.standard_normal(_interior(a).shape)
        return config.periodic_fill(a)

    return d, x, mu, mv, mw, field


@pytest.mark.parametrize("seed", [3, 4])
def test_dot_product(seed):
    d, x, mu, mv, mw, field = _problem(seed)
    dx, dmu, dmv, dmw = field(1.0), field(0.1), field(0.1), field(0.05)
    dmw[0] = 0.0
    abar = np.zeros(d.shape)
    abar[:, 3:-2, 3:-2] = np.random.default_rng(seed + 100).standard_normal(_interior(abar).shape)
    with Mimica(d, nscal=2) as m:
        ctx = FnContext(m)
        AdvectionFunction.forward(ctx, x, mu, mv, mw)
        tl = AdvectionFunction.jvp(ctx, dx, dmu, dmv, dmw)
        xb, mub, mvb, mwb = AdvectionFunction.backward(ctx, abar)
    lhs = float(np.sum(tl * abar))
    rhs = float(np.sum(dx * xb) + np.sum(dmu * mub) + np.sum(dmv * mvb) + np.sum(dmw * mwb))
    scale = float(np.sum(np.abs(tl * abar)))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)
    # the folded adjoint leaves no weight on ghost cells
    for a in (xb, mub, mvb):
        g = a.copy()
        g[:, 3:-2, 3:-2] = 0.0
        assert not np.any(g)


def _smooth_problem():
    """Smooth periodic fields whose WENO smoothness ratios stay far below the switch
    threshold (20) on every face, so the first-order expansion holds on the whole range
    of h: the switch is discontinuous, and a perturbation that flips a face adds an O(1)
    jump that no expansion captures."""
    d = config.cumulus_domain(32, 32, 24)
    st = config.random_state(d, seed=5)
    nz, ny, nx = d.shape
    i = np.arange(nx)[None, None, :] - 3
    j = np.arange(ny)[None, :, None] - 3
    k = np.arange(nz)[:, None, None]
    rho = d.den0[:, None, None]
    # cell centres symmetric about every extremum: the two faces beside it carry equal
    # differences, the largest ratio of consecutive squared differences is (sin 3pi/32 /
    # sin pi/32)^2 = 8.7
    cx = np.cos(2 * np.pi * i / d.maxx)
    cy = np.cos(2 * np.pi * j / d.maxy)
    x = rho * (300.0 + 0.02 * k + 0.5 * (cx + cy))
    dx = rho * 0.1 * np.cos(2 * np.pi * 2 * i / d.maxx) * np.cos(2 * np.pi * j / d.maxy)
    mu = st.u * d.den0[:, None, None]
    mv = st.v * d.den0[:, None, None]
    mw = st.w * d.avden0[:, None, None]
    mw[0] = 0.0
    rng = np.random.default_rng(6)

    def field(scale):
        a = np.zeros(d.shape)
        a[:, 3:-2, 3:-2] = scale * rng.standard_normal(_interior(a).shape)
        return config.periodic_fill(a)

    return d, config.periodic_fill(x), config.periodic_fill(dx), mu, mv, mw, field


def _max_switch_ratio(x):
    """largest max/min ratio of consecutive squared differences along z, y and x"""
    r = 0.0
    for ax in (0, 1, 2):
        dd = np.diff(x, axis=ax) ** 2 + 1e-15
        a, b = np.take(dd, range(dd.shape[ax] - 1), axis=ax), np.take(dd, range(1, dd.shape[ax]), axis=ax)
        r = max(r, float(np.max(np.maximum(a, b) / np.minimum(a, b))))
    return r


def test_taylor():
    d, x, dx, mu, mv, mw, field = _smooth_problem()
    dmu, dmv, dmw = field(0.1), field(0.1), field(0.05)
    dmw[0] = 0.0
    hs = [1e-2, 1e-3, 1e-4, 1e-5]
    # every face of x and x + h dx keeps its linear weights (ratios far below 20)
    assert max(_max_switch_ratio(x + h * dx) for h in [0.0] + hs) < 10.0
    with Mimica(d, nscal=2) as m:
        ctx = FnContext(m)
        a0 = AdvectionFunction.forward(ctx, x, mu, mv, mw)
        tl = AdvectionFunction.jvp(ctx, dx, dmu, dmv, dmw)
        rem, first = [], []
        for h in hs:
            ah = m.advection_ac(x + h * dx, mu + h * dmu, mv + h * dmv, mw + h * dmw, np.zeros_like(x))
            rem.append(float(np.linalg.norm(_interior(ah - a0 - h * tl))))
            first.append(float(np.linalg.norm(_interior(h * tl))))
    # second-order remainder: each decade of h lowers it by about two decades, and it is
    # small against the first-order term
    ratios = [rem[q] / rem[q + 1] for q in range(len(rem) - 1)]
    assert all(80.0 < rt < 125.0 for rt in ratios), (rem, ratios)
    assert rem[-1] < 1e-6 * first[-1]


@pytest.mark.parametrize("nsubp", [1, 2])
def test_projection_dot_product(nsubp):
    """<P(dm, dp), (mbar, pbar)> = <(dm, dp), P^T(mbar, pbar)> over the interior."""
    from fdd3260_b200.autograd import ProjectionFunction
    d = config.cumulus_domain(32, 32, 24, nsubp=nsubp)
    rng = np.random.default_rng(40 + nsubp)

    def field(scale, bottom_zero=False):
        a = np.zeros(d.shape)
        a[:, 3:-2, 3:-2] = scale * rng.standard_normal(_interior(a).shape)
        if bottom_zero:
            a[0] = 0.0
        return config.periodic_fill(a)

    dm = [field(1.0), field(1.0), field(0.5, bottom_zero=True)]
    dp = field(10.0)
    bars = [field(1.0), field(1.0), field(0.5), field(1.0)]
    for b in bars:   # adjoint inputs live on the interior
        b[:, :3, :] = 0.0; b[:, -2:, :] = 0.0; b[:, :, :3] = 0.0; b[:, :, -2:] = 0.0
    with Mimica(d, nscal=2) as m:
        ctx = FnContext(m)
        out = ProjectionFunction.jvp(ctx, *dm, dp)
        back = ProjectionFunction.backward(ctx, *bars)
    lhs = sum(float(np.sum(_interior(o) * _interior(b))) for o, b in zip(out, bars))
    rhs = sum(float(np.sum(_interior(x) * _interior(y))) for x, y in zip(dm + [dp], back))
    scale = sum(float(np.sum(np.abs(_interior(o) * _interior(b)))) for o, b in zip(out, bars))
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs, scale)
