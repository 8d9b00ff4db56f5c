"""Parity of the sm_100a CUDA path with the oracle (CPU restatement of the reference).

Tolerance: relative L-inf <= 1e-12 per field (the plain FP64 form).  The advection,
momentum and stage-update kernels are compiled without FMA contraction and are
expected to agree bit for bit; the projection uses a different (but exact-DFT)
transform than the reference's FFTW, so it agrees to round-off.
"""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def rel_linf(a, b, interior=True):
    if interior:
        a, b = a[:, 3:-2, 3:-2], b[:, 3:-2, 3:-2]
    s = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / s


def _mom(d, st):
    return (st.u * d.den0[:, None, None], st.v * d.den0[:, None, None], st.w * d.avden0[:, None, None])


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl", "lw", "quick"])
@pytest.mark.parametrize("limiter", ["minmod", "VL", "MC"])
def test_advection_ac(scheme, limiter):
    if scheme != "muscl" and limiter != "minmod":
        pytest.skip("limiter only selects MUSCL variants")
    d = config.cumulus_domain(64, 32, 24, scheme=scheme)
    d.muscl_limiter = limiter
    st = config.random_state(d, seed=11, nscal=2)
    mu, mv, mw = _mom(d, st)
    x = st.scal[1] * st.dens
    xs0 = np.random.default_rng(3).normal(size=d.shape)
    with Mimica(d, nscal=2) as m:
        got = m.advection_ac(x, mu, mv, mw, xs0)
    ref = O.Oracle(d).advection_ac(x, mu, mv, mw, xs0)
    assert rel_linf(got - xs0, ref - xs0) <= TOL
    assert np.array_equal(got[:, 3:-2, 3:-2], ref[:, 3:-2, 3:-2]), "expected bit-exact"


@pytest.mark.parametrize("ntime", [1, 2])
@pytest.mark.parametrize("mom_ord", [4, 2])
def test_qnadv_uvw(ntime, mom_ord):
    d = config.cumulus_domain(32, 64, 20, mom_ord=mom_ord)
    st = config.random_state(d, seed=12)
    mu, mv, mw = _mom(d, st)
    with Mimica(d, nscal=2) as m:
        got = m.qnadv_uvw(mu, mv, mw, ntime)
    ref = O.Oracle(d).qnadv_uvw(mu, mv, mw, ntime)
    for g, r in zip(got, ref):
        assert rel_linf(g, r) <= TOL
        assert np.array_equal(g[:, 3:-2, 3:-2], r[:, 3:-2, 3:-2]), "expected bit-exact"


def test_fft_solve():
    d = config.cumulus_domain(48, 40, 30)
    rng = np.random.default_rng(13)
    tend = config.periodic_fill(rng.normal(size=d.shape))
    with Mimica(d, nscal=2) as m:
        got = m.fft_solve(tend)
    ref = O.Oracle(d).fft_solve(tend)
    assert rel_linf(got, ref) <= TOL


@pytest.mark.parametrize("nsubp", [1, 2])
def test_anelastic_pressure(nsubp):
    d = config.cumulus_domain(32, 32, 24, nsubp=nsubp)
    st = config.random_state(d, seed=14)
    mu, mv, mw = _mom(d, st)
    mw[0] = 0.0
    wold = mw * 0.9
    with Mimica(d, nscal=2) as m:
        g = m.anelastic_pressure(mu, mv, mw, st.p, wold)
    r = O.Oracle(d).anelastic_pressure(mu, mv, mw, st.p, wold)
    for a, b in zip(g[:4], r[:4]):
        assert rel_linf(a, b) <= TOL
    assert abs(g[4] - r[4]) <= 1e-6 * abs(r[4]) + 1e-16
    assert np.abs(g[5] - r[5]).max() <= 1e-10 * np.abs(r[5]).max() + 1e-16


def _compare_states(g, r, tol=TOL):
    out = {}
    for name, a, b in [("u", g.u, r.u), ("v", g.v, r.v), ("w", g.w, r.w), ("p", g.p, r.p), ("dens", g.dens, r.dens)]:
        out[name] = rel_linf(a, b)
    for s, (a, b) in enumerate(zip(g.scal, r.scal)):
        out[f"s{s}"] = rel_linf(a, b)
    bad = {k: v for k, v in out.items() if not v <= tol}
    assert not bad, (bad, out)
    return out


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl", "lw", "quick"])
def test_step_parity(scheme):
    d = config.warm_bubble_domain(32, 32, 24, scheme=scheme)
    st = config.warm_bubble_state(d, seed=21, centre=(800.0, 800.0, 400.0), radius=400.0)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        m.stepping(3, ntime0=1)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    _compare_states(g, r)


def test_step_parity_moist_stretched():
    d = config.cumulus_domain(32, 32, 40, scheme="weno")
    st = config.cumulus_state(d, seed=1000, n_extra=2)
    with Mimica(d, nscal=len(st.scal), iqt=1) as m:
        m.upload(st)
        m.stepping(2, ntime0=1)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=2, ntime0=1)
    _compare_states(g, r)


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl", "lw", "quick"])
def test_step_parity_six_fields(scheme):
    """Density + 5 scalars, the bench's field count, whose scalar-advection kernels are
    compiled with the field count built in."""
    d = config.cumulus_domain(32, 32, 24, scheme=scheme)
    st = config.cumulus_state(d, seed=1001, n_extra=3)
    assert 1 + len(st.scal) == 6
    with Mimica(d, nscal=len(st.scal), iqt=1) as m:
        m.upload(st)
        m.stepping(2, ntime0=1)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=2, ntime0=1)
    _compare_states(g, r)


def test_warm_bubble_64cubed_10_steps():
    """The CPU-runnable configuration: 64^3 warm bubble, WENO, 10 steps, dt = 0.5 s."""
    d = config.warm_bubble_domain(64, 64, 64, scheme="weno")
    st = config.warm_bubble_state(d, seed=0)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        md, p1 = m.stepping(10, ntime0=1, diagnostics=True)
        g = m.download()
    r, mdr, p1r = O.Oracle(d).stepping(st, nsteps=10, ntime0=1)
    _compare_states(g, r)
    assert abs(md - mdr) <= 1e-6 * abs(mdr) + 1e-15


def test_graph_replay_equals_eager():
    d = config.warm_bubble_domain(32, 32, 16)
    st = config.warm_bubble_state(d, seed=5, centre=(800.0, 800.0, 300.0), radius=300.0)
    outs = []
    for graph in (False, True):
        with Mimica(d, nscal=2) as m:
            m.upload(st)
            m.stepping(5, ntime0=1, graph=graph)
            outs.append(m.download())
    a, b = outs
    for x, y in zip([a.u, a.v, a.w, a.p, a.dens, *a.scal], [b.u, b.v, b.w, b.p, b.dens, *b.scal]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("nsubp", [1, 3])
def test_graph_diagnostics_equal_eager(nsubp):
    """maxdiv after an even number of graph-replayed steps (computed on the final state,
    whose level-n buffers hold velocities) is the divergence of the momentum, as the eager
    step computes it inside the projection: equal to rounding."""
    d = config.cumulus_domain(32, 32, 24, nsubp=nsubp)
    st = config.cumulus_state(d, seed=8, n_extra=1)
    mds = []
    for graph in (False, True):
        with Mimica(d, nscal=len(st.scal), iqt=1) as m:
            m.upload(st)
            md, _ = m.stepping(4, ntime0=1, diagnostics=True, graph=graph)
            mds.append(md)
    a, b = mds
    assert abs(a - b) <= 1e-6 * abs(a) + 1e-14, (a, b)
    if nsubp == 3:
        assert abs(b) <= 1e-10


def test_deterministic_reruns():
    d = config.warm_bubble_domain(32, 32, 16)
    st = config.warm_bubble_state(d, seed=6, centre=(800.0, 800.0, 300.0), radius=300.0)
    res = []
    for _ in range(2):
        with Mimica(d, nscal=2) as m:
            m.upload(st)
            m.stepping(2)
            res.append(m.download())
    for x, y in zip([res[0].u, res[0].p, *res[0].scal], [res[1].u, res[1].p, *res[1].scal]):
        assert np.array_equal(x, y)


def test_step_parity_many_lognormal_tracers():
    """Capacity-run field set at a small size: theta_l, qt and 10 lognormal tracers
    (sigma_log = 1), 13 advected fields with density, on the stretched grid."""
    d = config.cumulus_domain(32, 32, 24, scheme="weno", dt0=0.5)
    st = config.cumulus_state(d, seed=4000, n_extra=10, lognormal_extras=True)
    assert len(st.scal) == 12
    with Mimica(d, nscal=len(st.scal), iqt=1) as m:
        m.upload(st)
        m.stepping(2, ntime0=1)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=2, ntime0=1)
    _compare_states(g, r)
