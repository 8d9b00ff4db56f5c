"""Parity of the SGS turbulence kernels (src/PHYS/subgrid.f90: calc_subgrid, efud, eff0/effs)
with the oracle, through the C-ABI.

The kernels are FP64 without FMA contraction and follow the reference's operation order,
so the unit entries are compared bit for bit; full steps with SGS diffusion on are
compared at the step-parity tolerance (the projection agrees to round-off only).
"""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib, config
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12
MIXED_TOL = 2e-4   # as tests/test_gpu_mixed.py


def _state(d, seed):
    rng = np.random.default_rng(seed)
    sh = d.shape
    z = d.zc()[:, None, None]
    u = config.periodic_fill(-5.0 + 0.01 * z + rng.normal(size=sh))
    v = config.periodic_fill(rng.normal(size=sh))
    w = config.periodic_fill(0.3 * rng.normal(size=sh))
    w[0] = 0.0
    es = config.periodic_fill(300.0 + 0.002 * z + 0.2 * rng.normal(size=sh))
    qt = config.periodic_fill(0.012 - 2e-6 * z + 5e-4 * rng.normal(size=sh))
    dens = config.periodic_fill(d.den0[:, None, None] * (1.0 + 0.01 * rng.normal(size=sh)))
    return u, v, w, es, qt, dens


def _flux(d, seed, scale):
    return np.random.default_rng(seed).normal(size=(d.ny, d.nx)) * scale


@pytest.mark.parametrize("moist", [True, False])
@pytest.mark.parametrize("anis,pran", [(False, 0.4), (True, -0.4)])
def test_calc_subgrid_bit_exact(moist, anis, pran):
    d = config.cumulus_domain(32, 24, 30, sgs=config.Sgs(anis_k=anis, pran=pran, zdec=400.0))
    u, v, w, es, qt, _ = _state(d, 1)
    q = qt if moist else None
    with Mimica(d, nscal=2, iqt=1) as m:
        got = m.calc_subgrid(u, v, w, es, q)
    ref = O.Oracle(d).calc_subgrid(u, v, w, es, q)
    inner = ref[:, 3:-2, 3:-2]
    assert (inner > 0).mean() > 0.2 and (inner == 0).mean() > 0.01, "both Lilly branches exercised"
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("anis,pran,momsf", [(False, 0.4, 0), (True, -0.4, 1), (False, 0.7, 1)])
def test_efud_bit_exact(anis, pran, momsf):
    mflux = None
    d = config.cumulus_domain(32, 24, 30)
    if momsf:
        mflux = _flux(d, 2, 0.05)
    d.sgs = config.Sgs(anis_k=anis, pran=pran, zdec=400.0, momsf=momsf, mflux=mflux, min_w=0.5)
    u, v, w, es, qt, dens = _state(d, 3)
    orc = O.Oracle(d)
    fkv = orc.calc_subgrid(u, v, w, es, qt)
    rng = np.random.default_rng(4)
    acc = [rng.normal(size=d.shape) for _ in range(3)]
    with Mimica(d, nscal=2, iqt=1) as m:
        got = m.efud(u, v, w, dens, fkv, *acc)
    ref = orc.efud(u, v, w, dens, fkv, *acc)
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
        assert not np.array_equal(g, acc[0])


@pytest.mark.parametrize("kind", [1, 2, 3])
@pytest.mark.parametrize("diff", [0.0, 2.5])
def test_eff_bit_exact(kind, diff):
    d = config.cumulus_domain(32, 24, 30)
    esflux, qvflux = _flux(d, 5, 0.1), _flux(d, 6, 1e-4)
    d.sgs = config.Sgs(diff=diff, pran=-0.4, zdec=400.0, anis_k=diff != 0.0, esflux=esflux, qvflux=qvflux,
                       qt0=np.linspace(0.012, 0.004, d.nz))
    u, v, w, es, qt, dens = _state(d, 7)
    orc = O.Oracle(d)
    fkv = orc.calc_subgrid(u, v, w, es, qt)
    x = {1: es, 2: qt, 3: config.periodic_fill(np.random.default_rng(8).lognormal(size=d.shape))}[kind]
    flux_s = {1: -esflux, 2: -qvflux, 3: None}[kind]
    ec0 = np.random.default_rng(9).normal(size=d.shape)
    with Mimica(d, nscal=2, iqt=1) as m:
        got = m.eff(kind, dens, fkv, x, flux_s, ec0)
    ref = orc.eff(kind, dens, fkv, x, ec0)
    assert np.array_equal(got, ref)


def _compare(g, r, tol):
    out = {}
    for name, a, b in [("u", g.u, r.u), ("v", g.v, r.v), ("w", g.w, r.w), ("p", g.p, r.p), ("dens", g.dens, r.dens)]:
        a, b = a[:, 3:-2, 3:-2], b[:, 3:-2, 3:-2]
        out[name] = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    for s, (a, b) in enumerate(zip(g.scal, r.scal)):
        a, b = a[:, 3:-2, 3:-2], b[:, 3:-2, 3:-2]
        out[f"s{s}"] = np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)
    bad = {k: v for k, v in out.items() if not v <= tol}
    assert not bad, (bad, out)
    return out


@pytest.mark.parametrize("scheme", ["weno", "lw"])
def test_step_parity_with_sgs(scheme):
    d = config.warm_bubble_domain(32, 32, 24, scheme=scheme, sgs=config.Sgs(pran=0.4))
    st = config.warm_bubble_state(d, seed=21, centre=(800.0, 800.0, 400.0), radius=400.0)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        m.stepping(3, ntime0=1)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    _compare(g, r, TOL)
    # the diffusion is on: it changes the result
    d.sgs = None
    r0, _, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    assert np.abs(r0.scal[0] - r.scal[0]).max() > 1e-9


def test_step_parity_moist_tracers_surface_fluxes():
    """Moist stretched cumulus with two tracers, damped viscosity (pran < 0), surface heat,
    moisture and momentum fluxes: es/qt take advection + SGS, the tracers start from SGS."""
    d = config.cumulus_domain(32, 32, 40, scheme="weno")
    d.sgs = config.Sgs(pran=-0.4, zdec=600.0, momsf=1, esflux=_flux(d, 11, 0.05) + 0.1,
                       qvflux=_flux(d, 12, 1e-5) + 5e-5, mflux=-np.abs(_flux(d, 13, 0.05)))
    st = config.cumulus_state(d, seed=1000, n_extra=2)
    with Mimica(d, nscal=len(st.scal), iqt=1) as m:
        m.upload(st)
        m.stepping(2, ntime0=1)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=2, ntime0=1)
    _compare(g, r, TOL)


def test_graph_replay_equals_eager_with_sgs():
    d = config.warm_bubble_domain(32, 32, 16, sgs=config.Sgs(pran=0.4))
    st = config.warm_bubble_state(d, seed=5, centre=(800.0, 800.0, 300.0), radius=300.0)
    outs = []
    for graph in (False, True):
        with Mimica(d, nscal=2) as m:
            m.upload(st)
            m.stepping(4, ntime0=1, graph=graph)
            outs.append(m.download())
    a, b = outs
    for x, y in zip([a.u, a.v, a.w, a.p, a.dens, *a.scal], [b.u, b.v, b.w, b.p, b.dens, *b.scal]):
        assert np.array_equal(x, y)


def test_mixed_form_with_sgs():
    d = config.warm_bubble_domain(32, 32, 24, sgs=config.Sgs(pran=0.4))
    st = config.warm_bubble_state(d, seed=21, centre=(800.0, 800.0, 400.0), radius=400.0)
    d.precision = _lib.MG_PREC_MIXED
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        m.stepping(3, ntime0=1)
        g = m.download()
    d.precision = _lib.MG_PREC_FP64
    r, _, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    _compare(g, r, MIXED_TOL)


def test_sgs_params_rejected():
    d = config.warm_bubble_domain(16, 16, 12)
    with Mimica(d, nscal=1) as m:
        for bad in (dict(pran=0.0), dict(zdec=-1.0), dict(min_w=0.0)):
            with pytest.raises(_lib.MimicaError):
                m.set_sgs(config.Sgs(**bad))
