"""CPU checks of the SGS turbulence restatement (src/PHYS/subgrid.f90 with the gradients
of src/TOOLS/gradients.f90) in the oracle, and of the product library's host-side
per-level factors against it.

The reference ships no golden vectors for the SGS path and cannot be built here, so
the restatement is pinned by known answers of the discrete operators: the exact
4th-order gradient of a linear shear and the Smagorinsky viscosity it implies, zero
stress divergence of a uniform stress, zero flux divergence of a linear scalar profile
under constant viscosity, periodic conservation of the horizontal fluxes, and the
Richardson-number cut-off of the Lilly correction.
"""
import ctypes as C

import numpy as np
import pytest

from fdd3260_b200 import _lib, config
from oracle import oracle as O

CS, RIC = 0.23, 0.25


def _uniform(maxx=12, maxy=10, nz=12, dz=40.0, sgs=None, **kw):
    d = config.warm_bubble_domain(maxx, maxy, nz, dz=dz, **kw)
    d.sgs = sgs if sgs is not None else config.Sgs()
    return d


def _rand_state(d, seed, shear=True):
    rng = np.random.default_rng(seed)
    sh = d.shape
    u = config.periodic_fill(rng.normal(size=sh) + (0.01 * d.zc()[:, None, None] if shear else 0.))
    v = config.periodic_fill(rng.normal(size=sh))
    w = config.periodic_fill(rng.normal(size=sh) * 0.3)
    w[0] = 0.0
    es = config.periodic_fill(300.0 + 0.003 * d.zc()[:, None, None] + 0.1 * rng.normal(size=sh))
    qt = config.periodic_fill(0.01 + 0.001 * rng.normal(size=sh))
    dens = config.periodic_fill(d.den0[:, None, None] * (1.0 + 0.01 * rng.normal(size=sh)))
    return u, v, w, es, qt, dens


@pytest.mark.parametrize("anis", [False, True])
@pytest.mark.parametrize("stretched", [False, True])
def test_host_profiles_bit_exact_with_oracle(anis, stretched):
    """The library's per-level SGS factors (pow, exp, sqrt on the host) == the oracle's."""
    sg = config.Sgs(anis_k=anis, pran=-0.4, zdec=300.0, zrough=0.1)
    d = config.cumulus_domain(16, 16, 30, sgs=sg) if stretched else _uniform(sgs=sg)
    prof_o = O.Oracle(d).sgs_profiles()
    p, keep = d.params(2, -1)
    s, keep2 = sg.params(d.nz)
    prof_l = np.zeros(_lib.SGS_NPROF * d.nz)
    _lib.check(_lib.lib().mg_sgs_profiles(C.byref(p), C.byref(s), _lib.ptr(prof_l)), "mg_sgs_profiles")
    assert np.array_equal(prof_o, prof_l)
    np.testing.assert_allclose(prof_o[:d.nz], d.zc(), rtol=1e-14)


def test_linear_shear_gradient_and_viscosity():
    """u = a z on a uniform grid: the 4th-order d/dz is exact, d13 = a/2, S2 = a^2, and in
    a neutral atmosphere (N2 = 0, Ri = 0) the viscosity is (C_s delta)^2 |a|."""
    d = _uniform()
    orc = O.Oracle(d)
    a = 0.02
    z = d.zc()
    u = config.periodic_fill(np.broadcast_to(a * z[:, None, None], d.shape).copy())
    zero = np.zeros(d.shape)
    es = np.full(d.shape, 300.0)
    dij = orc.cal_dij(u, zero, zero)
    inner = (slice(2, d.nz - 2), slice(3, -2), slice(3, -2))
    np.testing.assert_allclose(dij[4][inner], a / 2, rtol=1e-12)
    for q in (0, 1, 2, 3, 5):
        assert np.abs(dij[q][inner]).max() <= 1e-15
    fkv = orc.calc_subgrid(u, zero, zero, es)
    cs2d = orc.sgs_profiles()[d.nz:2 * d.nz]
    np.testing.assert_allclose(fkv[inner], (cs2d[2:d.nz - 2, None, None] * a) * np.ones_like(fkv[inner]), rtol=1e-12)


def test_lilly_cutoff_stable_layer():
    """Ri > Ric switches the viscosity off; Ri < 0 (unstable) raises it above neutral."""
    d = _uniform()
    orc = O.Oracle(d)
    z = d.zc()
    a = 0.01
    u = config.periodic_fill(np.broadcast_to(a * z[:, None, None], d.shape).copy())
    zero = np.zeros(d.shape)
    neutral = orc.calc_subgrid(u, zero, zero, np.full(d.shape, 300.0))
    # N2 = g/theta0 dtheta/dz: Ri = N2/S2 = N2/a^2; strong stability -> Ri >> Ric
    stable = orc.calc_subgrid(u, zero, zero, np.broadcast_to(300.0 + 0.05 * z[:, None, None], d.shape).copy())
    unstable = orc.calc_subgrid(u, zero, zero, np.broadcast_to(300.0 - 0.01 * z[:, None, None], d.shape).copy())
    inner = (slice(2, d.nz - 2), slice(3, -2), slice(3, -2))
    assert np.all(stable[inner] == 0.0)
    assert np.all(unstable[inner] > neutral[inner])


def test_uniform_stress_has_no_divergence():
    """Constant viscosity (diff != 0) and a linear shear: the stress is uniform, so efud
    adds nothing away from the boundaries."""
    d = _uniform(sgs=config.Sgs(diff=5.0))
    orc = O.Oracle(d)
    z = d.zc()
    u = config.periodic_fill(np.broadcast_to(0.02 * z[:, None, None], d.shape).copy())
    zero = np.zeros(d.shape)
    dens = np.ones(d.shape)
    fkv = orc.calc_subgrid(u, zero, zero, np.full(d.shape, 300.0))
    assert np.all(fkv == 5.0)
    su, sv, sw = orc.efud(u, zero, zero, dens, fkv)
    inner = (slice(3, d.nz - 3), slice(3, -2), slice(3, -2))
    for s in (su, sv, sw):
        assert np.abs(s[inner]).max() <= 1e-13


def test_linear_scalar_has_no_flux_divergence():
    d = _uniform(sgs=config.Sgs(diff=5.0))
    orc = O.Oracle(d)
    z = d.zc()
    x = config.periodic_fill(np.broadcast_to(1e-3 * z[:, None, None], d.shape).copy())
    dens = np.ones(d.shape)
    fkv = np.full(d.shape, 5.0)
    ec = orc.eff(3, dens, fkv, x)
    inner = (slice(1, d.nz - 2), slice(3, -2), slice(3, -2))
    assert np.abs(ec[inner]).max() <= 1e-15
    # bottom cell: the flux through the first face enters, nothing leaves below (flux_s = 0)
    k1 = ec[0, 3:-2, 3:-2]
    expect = (0.5 * (5.0 / 0.4 + 5.0 / 0.4) * 1e-3) * d.dz1w[0]
    np.testing.assert_allclose(k1, expect, rtol=1e-12)


@pytest.mark.parametrize("anis", [False, True])
def test_horizontal_fluxes_conserve_per_level(anis):
    """Fields without vertical variation: the horizontal SGS flux divergences sum to zero
    over the periodic plane, for momentum and scalars."""
    d = _uniform(sgs=config.Sgs(anis_k=anis, pran=-0.5, zdec=200.0))
    orc = O.Oracle(d)
    rng = np.random.default_rng(5)
    plane = lambda: np.broadcast_to(rng.normal(size=(1,) + d.shape[1:]), d.shape).copy()
    u, v = config.periodic_fill(plane()), config.periodic_fill(plane())
    zero = np.zeros(d.shape)
    es = np.full(d.shape, 300.0)
    dens = config.periodic_fill(plane() * 0.01 + 1.0)
    fkv = orc.calc_subgrid(u, v, zero, es)
    su, sv, sw = orc.efud(u, v, zero, dens, fkv)
    x = config.periodic_fill(plane())
    ec = orc.eff(3, dens, fkv, x)
    for s, lv in ((su, slice(0, d.nz - 1)), (sv, slice(0, d.nz - 1)), (ec, slice(0, d.nz - 1))):
        tot = s[lv, 3:-2, 3:-2].sum(axis=(1, 2))
        scale = np.abs(s[lv, 3:-2, 3:-2]).sum(axis=(1, 2)) + 1e-300
        assert np.all(np.abs(tot) <= 1e-12 * scale)


def test_surface_flux_enters_bottom_cell():
    """eff0's bottom boundary: ez(1) = (flux(1.5) - flux_s) dz1w(1) with flux_s = -esflux."""
    rng = np.random.default_rng(7)
    d = _uniform()
    esflux = rng.normal(size=(d.ny, d.nx)) * 0.1
    d.sgs = config.Sgs(diff=1.0, esflux=esflux)
    orc = O.Oracle(d)
    dens = np.ones(d.shape)
    fkv = np.ones(d.shape)
    x = np.full(d.shape, 300.0)   # x - pt0(k) is not uniform: compare against no flux
    ec0 = O.Oracle(_uniform(sgs=config.Sgs(diff=1.0))).eff(1, dens, fkv, x)
    ec1 = orc.eff(1, dens, fkv, x)
    diff = (ec1 - ec0)[0, 3:-2, 3:-2]
    np.testing.assert_allclose(diff, esflux[3:-2, 3:-2] * d.dz1w[0], rtol=1e-9, atol=1e-15)
    assert np.array_equal(ec1[1:], ec0[1:])


@pytest.mark.parametrize("scheme", ["weno", "lw"])
def test_oracle_step_with_sgs_is_finite_and_differs(scheme):
    d = config.warm_bubble_domain(16, 16, 12, scheme=scheme)
    st = config.warm_bubble_state(d, seed=1, centre=(400.0, 400.0, 300.0), radius=250.0)
    r0, _, _ = O.Oracle(d).stepping(st, nsteps=2, ntime0=1)
    d.sgs = config.Sgs(pran=0.4)
    r1, _, _ = O.Oracle(d).stepping(st, nsteps=2, ntime0=1)
    for a in [r1.u, r1.v, r1.w, r1.p, r1.dens, *r1.scal]:
        assert np.isfinite(a).all()
    assert not np.array_equal(r0.scal[0], r1.scal[0])
    # density is not diffused
    assert np.abs(r1.dens - r0.dens).max() <= 1e-6 * np.abs(r0.dens).max()
