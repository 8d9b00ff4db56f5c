"""Tangent linear and adjoint of the momentum advection operator qnadv_uvw (mg_qnadv_tl /
mg_qnadv_ad): the per-cell form the adjoint differentiates equals the K2 momentum
advection bit for bit; the tangent linear agrees with central differences of the
forward operator; the adjoint passes the dot-product test to 1e-12."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config

pytestmark = pytest.mark.gpu


def _interior(a):
    return a[:, 3:-2, 3:-2]


def _problem(seed, **kw):
    d = config.cumulus_domain(32, 24, 20, **kw)
    rng = np.random.default_rng(seed)
    st = config.random_state(d, seed=seed)
    mu = config.periodic_fill(st.u * d.den0[:, None, None])
    mv = config.periodic_fill(st.v * d.den0[:, None, None])
    mw = config.periodic_fill(st.w * d.avden0[:, None, None])
    mw[0] = 0.0

    def field(scale):
        a = np.zeros(d.shape)
        a[:, 3:-2, 3:-2] = scale * rng.standard_normal(_interior(a).shape)
        return config.periodic_fill(a)

    return d, mu, mv, mw, field


@pytest.mark.parametrize("ntime", [1, 2])
@pytest.mark.parametrize("mom_ord,lavisc", [(4, 1), (2, 1), (4, 0)])
def test_per_cell_form_equals_k2(ntime, mom_ord, lavisc):
    d, mu, mv, mw, field = _problem(1, mom_ord=mom_ord, lavisc=lavisc)
    with Mimica(d, nscal=1) as m:
        ref = m.qnadv_uvw(mu, mv, mw, ntime)
        (vals, _) = m.qnadv_tl(mu, mv, mw, field(1.0), field(1.0), field(1.0), ntime, values=True)
    for a, b in zip(vals, ref):
        assert np.array_equal(_interior(a), _interior(b))


@pytest.mark.parametrize("ntime", [1, 2])
def test_tangent_linear_central_difference(ntime):
    d, mu, mv, mw, field = _problem(2)
    dmu, dmv, dmw = field(1.0), field(1.0), field(0.5)
    dmw[0] = 0.0
    with Mimica(d, nscal=1) as m:
        tl = m.qnadv_tl(mu, mv, mw, dmu, dmv, dmw, ntime)
        h = 1e-5
        fp = m.qnadv_uvw(mu + h * dmu, mv + h * dmv, mw + h * dmw, ntime)
        fm = m.qnadv_uvw(mu - h * dmu, mv - h * dmv, mw - h * dmw, ntime)
    for t, a, b in zip(tl, fp, fm):
        cd = (_interior(a) - _interior(b)) / (2 * h)
        assert np.abs(_interior(t) - cd).max() <= 1e-6 * np.abs(cd).max()


@pytest.mark.parametrize("ntime", [1, 2])
@pytest.mark.parametrize("mom_ord", [4, 2])
def test_dot_product(ntime, mom_ord):
    d, mu, mv, mw, field = _problem(3 + ntime, mom_ord=mom_ord)
    dmu, dmv, dmw = field(1.0), field(1.0), field(0.5)
    lu, lv, lw = (np.where(np.pad(np.ones_like(_interior(field(1.0))), ((0, 0), (3, 2), (3, 2))) > 0, field(1.0), 0.)
                  for _ in range(3))
    with Mimica(d, nscal=1) as m:
        tl = m.qnadv_tl(mu, mv, mw, dmu, dmv, dmw, ntime)
        ad = m.qnadv_ad(mu, mv, mw, lu, lv, lw, ntime)
    lhs = sum(float(np.sum(_interior(t) * _interior(l))) for t, l in zip(tl, (lu, lv, lw)))
    rhs = sum(float(np.sum(_interior(x) * _interior(a))) for x, a in zip((dmu, dmv, dmw), ad))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))
    for a in ad:   # ghost adjoints are folded onto the interior
        g = a.copy()
        g[:, 3:-2, 3:-2] = 0.0
        assert not g.any()
