"""The adjoint workload's gradient check: 128 x 128 x 96 cells at 40 m, FP64, WENO3-switch
scalar advection, FD4 momentum and the projection, 200 integrator steps with a checkpoint
every 25 (the reference's step, src/INTEG/time_step.f90:76-334, as the library runs it
and the oracle restates it).

Initial state: theta' ~ N(0, 0.5 K) smoothed by a 5-cell box filter, winds ~ N(0, 1 m/s)
smoothed likewise and made divergence-free by the library's projection; a seeded target
theta_target of the same kind.  Cost J = 1/2 sum over the interior of rho0 (theta'_T -
theta_target)^2; gradient with respect to the initial theta', u, v and w by the
trajectory adjoint.

* Taylor table over h = 1e-1 .. 1e-8 along one smooth direction: the first-order
  remainder |J(x0 + h d) - J(x0) - h <g, d>| with, per h, the number of WENO switch
  decisions of the initial theta faces that the perturbation flips (the reference's switch
  is discontinuous: a flipped face adds a jump no expansion captures).
* 32 seeded directions: central differences of J (eps = 1e-6) against <g, d>.
* Against the oracle: over 2 steps (the CPU restatement takes seconds per step at this
  size), central differences of the oracle's J along 2 directions against the GPU adjoint.
"""
import json

import numpy as np
import pytest

from fdd3260_b200 import Mimica, config
from oracle import oracle as O

pytestmark = pytest.mark.gpu

NSTEPS, CKPT = 200, 25


def _box5(a):
    """5-cell box filter: periodic in x and y, clamped in z."""
    out = a
    for ax in (1, 2):
        out = sum(np.roll(out, s, axis=ax) for s in range(-2, 3)) / 5.0
    z = np.concatenate([out[:1], out[:1], out, out[-1:], out[-1:]], axis=0)
    return sum(z[2 + s:2 + s + a.shape[0]] for s in range(-2, 3)) / 5.0


def _field3(d, vals):
    a = np.zeros(d.shape)
    a[:, 3:3 + d.maxy, 3:3 + d.maxx] = vals
    return config.periodic_fill(a)


def _smooth_noise(d, rng, sigma):
    """N(0, sigma) smoothed by the box filter, rescaled to standard deviation sigma."""
    x = _box5(rng.standard_normal((d.nz, d.maxy, d.maxx)))
    return sigma * x / x.std()


def _problem():
    d = config.warm_bubble_domain(128, 128, 96, dx=40.0, dy=40.0, dz=40.0, dt0=0.5)
    rng = np.random.default_rng(2002)
    thp = _smooth_noise(d, rng, 0.5)
    u, v, w = (_field3(d, _smooth_noise(d, rng, 1.0)) for _ in range(3))
    w[0] = 0.0
    dens = np.broadcast_to(d.den0[:, None, None], d.shape).copy()
    th = _field3(d, d.pt0[:, None, None] + thp)
    target = _smooth_noise(d, rng, 0.5)
    # divergence-free winds: the library's projection of the momentum
    with Mimica(d, nscal=1) as m:
        mu, mv = u * d.den0[:, None, None], v * d.den0[:, None, None]
        mw = w * d.avden0[:, None, None]
        mu, mv, mw, _, _, _ = m.anelastic_pressure(mu, mv, mw, np.zeros(d.shape), mw)
    u, v = mu / d.den0[:, None, None], mv / d.den0[:, None, None]
    w = mw / d.avden0[:, None, None]
    st = config.State(u, v, w, np.zeros(d.shape), dens, [th], -1)
    return d, st, target


def _cost(d, st, target):
    thp = st.scal[0][:, 3:-2, 3:-2] - d.pt0[:, None, None]
    r = thp - target
    return 0.5 * float(np.sum(d.den0[:, None, None] * r * r))


def _lam(d, st, target):
    """dJ/d(final state): rho0 (theta'_T - theta_target) in theta, zero elsewhere."""
    lam = config.State(*(np.zeros(d.shape) for _ in range(5)), [np.zeros(d.shape)], -1)
    lam.scal[0][:, 3:-2, 3:-2] = d.den0[:, None, None] * (st.scal[0][:, 3:-2, 3:-2] - d.pt0[:, None, None] - target)
    return lam


def _plus(st, dx, h):
    return config.State(st.u + h * dx.u, st.v + h * dx.v, st.w + h * dx.w, st.p, st.dens,
                        [st.scal[0] + h * dx.scal[0]], -1)


def _direction(d, rng):
    z = np.zeros(d.shape)
    du, dv, dw, dth = (_field3(d, _smooth_noise(d, rng, 1.0)) for _ in range(4))
    dw[0] = 0.0
    return config.State(du, dv, dw, z, z.copy(), [dth], -1)


def _inner(g, dx):
    return sum(float(np.sum(a[:, 3:-2, 3:-2] * b[:, 3:-2, 3:-2]))
               for a, b in [(g.u, dx.u), (g.v, dx.v), (g.w, dx.w), (g.scal[0], dx.scal[0])])


def _switch_flags(d, st):
    """The WENO3 switch decisions (either side nonlinear) of the x, y and z faces of the
    initial density-weighted theta, as advq_weno.f90:320-349 decide them."""
    psi = st.scal[0] * d.den0[:, None, None]
    out = []
    for ax in (2, 1, 0):
        a = np.moveaxis(psi, ax, -1)
        d1, d2, d3 = a[..., 1:-2] - a[..., :-3], a[..., 2:-1] - a[..., 1:-2], a[..., 3:] - a[..., 2:-1]
        e1, e2, e3 = d1 * d1, d2 * d2, d3 * d3
        n1 = np.maximum(e1, e2) / (np.minimum(e1, e2) + 1e-15) > 20.0
        n2 = np.maximum(e2, e3) / (np.minimum(e2, e3) + 1e-15) > 20.0
        out.append(np.concatenate([n1.ravel(), n2.ravel()]))
    return np.concatenate(out)


def _run(m, st, nsteps):
    m.upload(st)
    m.stepping(nsteps, ntime0=1, graph=True)
    return m.download()


def test_config2_gradient_check():
    d, st, target = _problem()
    with Mimica(d, nscal=1) as m:
        fin = _run(m, st, NSTEPS)
        J0 = _cost(d, fin, target)
        m.upload(st)
        g = m.traj_adjoint(_lam(d, fin, target), NSTEPS, ntime0=1, ckpt=CKPT)
        rng = np.random.default_rng(77)
        dx = _direction(d, rng)
        gd = _inner(g, dx)
        flags0 = _switch_flags(d, st)
        taylor = []
        for e in range(1, 9):
            h = 10.0 ** (-e)
            p = _plus(st, dx, h)
            Jh = _cost(d, _run(m, p, NSTEPS), target)
            flips = int(np.count_nonzero(_switch_flags(d, p) != flags0))
            taylor.append({"h": h, "dJ": Jh - J0, "h_gd": h * gd, "remainder": abs(Jh - J0 - h * gd), "flips_t0": flips})
        eps = 1e-6
        cds = []
        for q in range(32):
            dq = _direction(d, np.random.default_rng(1000 + q))
            jp = _cost(d, _run(m, _plus(st, dq, eps), NSTEPS), target)
            jm = _cost(d, _run(m, _plus(st, dq, -eps), NSTEPS), target)
            cd, ad = (jp - jm) / (2 * eps), _inner(g, dq)
            cds.append({"cd": cd, "adjoint": ad, "rel": abs(cd - ad) / max(abs(ad), 1e-300)})
    rels = sorted(c["rel"] for c in cds)
    print("GRADCHECK " + json.dumps({"J0": J0, "taylor": taylor, "central_differences": cds,
                                     "rel_median": rels[16], "rel_max": rels[-1]}))
    assert np.isfinite(J0) and gd != 0.0 and all(np.isfinite(t["remainder"]) for t in taylor)
    # the gradient predicts the change of J to 1 % for some step of the table
    assert any(t["remainder"] < 1e-2 * abs(t["h_gd"]) for t in taylor)
    # central differences: most directions agree with the adjoint
    assert rels[16] < 1e-2


def test_config2_gradient_against_the_oracle_short():
    """Over 2 steps: the oracle's central differences against the GPU adjoint gradient."""
    d, st, target = _problem()
    n = 2
    orc = O.Oracle(d, omp=True)
    with Mimica(d, nscal=1) as m:
        fin = _run(m, st, n)
        m.upload(st)
        g = m.traj_adjoint(_lam(d, fin, target), n, ntime0=1, ckpt=1)
    eps = 1e-6
    for q in range(2):
        dq = _direction(d, np.random.default_rng(5000 + q))
        jp = _cost(d, orc.stepping(_plus(st, dq, eps), nsteps=n, ntime0=1)[0], target)
        jm = _cost(d, orc.stepping(_plus(st, dq, -eps), nsteps=n, ntime0=1)[0], target)
        cd, ad = (jp - jm) / (2 * eps), _inner(g, dq)
        print(f"GRADCHECK_ORACLE direction {q}: central difference {cd:.10e}, adjoint {ad:.10e}, "
              f"rel {abs(cd - ad) / abs(ad):.2e}")
        assert abs(cd - ad) <= 1e-5 * abs(ad)
