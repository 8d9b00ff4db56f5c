"""Trajectory tangent linear and adjoint (mg_traj_*): the composition they linearise
reproduces mg_step; the adjoint of nsteps steps passes the dot-product test against the
tangent linear; checkpointing does not change the gradient; and the gradient of a
final-time functional with respect to the initial winds and potential temperature
agrees with finite differences of the forward model: a second-order Taylor check on the
smooth momentum subsystem and central differences inside the smooth piece of the
scalar schemes' switches."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config

pytestmark = pytest.mark.gpu


def _interior(a):
    return a[:, 3:-2, 3:-2]


def _fields(st):
    return [st.u, st.v, st.w, st.p, st.dens, *st.scal]


def _dot(a, b):
    return sum(float(np.sum(_interior(x) * _interior(y))) for x, y in zip(_fields(a), _fields(b)))


def _smooth_state(d, seed=0):
    """Smooth winds and theta (no flat regions, so few WENO switch faces move under small
    perturbations), a passive scalar, hydrostatic density."""
    rng = np.random.default_rng(seed)
    nz, ny, nx = d.shape
    x = (np.arange(nx) - 3 + 0.5) / d.maxx
    y = (np.arange(ny) - 3 + 0.5) / d.maxy
    z = d.zc() / (d.dz * d.nz)
    X, Y = np.meshgrid(x, y)
    two = 2 * np.pi
    u = np.stack([2.0 + 0.8 * np.sin(two * X + 0.3) * np.cos(two * Y) * (1 + 0.2 * zz) for zz in z])
    v = np.stack([-1.0 + 0.6 * np.cos(two * X) * np.sin(two * Y + 0.7) * (1 - 0.2 * zz) for zz in z])
    w = np.stack([0.3 * np.sin(two * X) * np.sin(two * Y) * np.sin(np.pi * zz) for zz in z])
    w[0] = 0.0
    th = np.stack([300.0 + 2.0 * zz + 0.5 * np.sin(two * X + 1.1) * np.cos(two * Y + 0.4) for zz in z])
    sc = np.stack([1.0 + 0.3 * np.cos(two * X) * np.cos(two * Y) + 0.2 * zz for zz in z])
    dens = np.broadcast_to(d.den0[:, None, None], d.shape).copy()
    p = np.zeros(d.shape)
    f = config.periodic_fill
    return config.State(f(u), f(v), f(w), p, dens, [f(th), f(sc)], -1)


def _rand_like(st, rng, scales):
    arrs = []
    for a, s in zip(_fields(st), scales):
        b = np.zeros_like(a)
        _interior(b)[...] = s * rng.standard_normal(_interior(b).shape)
        arrs.append(config.periodic_fill(b))
    arrs[2][0] = 0.0
    return config.State(arrs[0], arrs[1], arrs[2], arrs[3], arrs[4], arrs[5:], st.iqt)


def test_composition_reproduces_step():
    d = config.warm_bubble_domain(32, 32, 16)
    st = config.warm_bubble_state(d, seed=5, centre=(800.0, 800.0, 300.0), radius=300.0)
    outs = []
    for traj in (False, True):
        with Mimica(d, nscal=2) as m:
            m.upload(st)
            if traj:
                m.traj_forward(3, ntime0=1)
            else:
                m.stepping(3, ntime0=1)
            outs.append(m.download())
    a, b = outs
    for x, y in zip(_fields(a), _fields(b)):
        x, y = _interior(x), _interior(y)
        assert np.abs(x - y).max() <= 1e-12 * max(np.abs(y).max(), 1e-300)


@pytest.mark.parametrize("nsteps,ckpt", [(1, 1), (3, 2)])
def test_dot_product(nsteps, ckpt):
    d = config.warm_bubble_domain(24, 24, 12)
    st = config.warm_bubble_state(d, seed=3, centre=(600.0, 600.0, 250.0), radius=300.0)
    rng = np.random.default_rng(7)
    dx0 = _rand_like(st, rng, [0.1, 0.1, 0.05, 1.0, 1e-3, 0.05, 0.01])
    lam = _rand_like(st, rng, [1.0] * 7)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        tl = m.traj_tl(dx0, nsteps)
        ad = m.traj_adjoint(lam, nsteps, ckpt=ckpt)
    lhs, rhs = _dot(tl, lam), _dot(dx0, ad)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_dot_product_single_scalar_larger_grid():
    """theta only (density + one scalar) on 96 x 96 x 48: the adjoint of the momentum
    advection skips the stencil offsets that leave 1..nz at the surface and the lid."""
    d = config.warm_bubble_domain(96, 96, 48, dx=40.0, dy=40.0, dz=40.0)
    st = config.warm_bubble_state(d, seed=9, centre=(1900.0, 1900.0, 700.0), radius=500.0, nscal_passive=0)
    rng = np.random.default_rng(12)
    sc = [0.1, 0.1, 0.05, 1.0, 1e-3, 0.05]
    dx0 = _rand_like(st, rng, sc)
    lam = _rand_like(st, rng, [1.0] * 6)
    with Mimica(d, nscal=1) as m:
        m.upload(st)
        tl = m.traj_tl(dx0, 2)
        ad = m.traj_adjoint(lam, 2, ckpt=1)
    lhs, rhs = _dot(tl, lam), _dot(dx0, ad)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def test_checkpoint_interval_does_not_change_gradient():
    d = config.warm_bubble_domain(24, 24, 12)
    st = config.warm_bubble_state(d, seed=4, centre=(600.0, 600.0, 250.0), radius=300.0)
    lam = _rand_like(st, np.random.default_rng(8), [1.0] * 7)
    res = []
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        for ck in (1, 2, 5, 10):   # 10: one segment longer than the trajectory
            res.append(m.traj_adjoint(lam, 5, ckpt=ck))
        # no stage records kept: every backward step recomputes its stages
        m.traj_record_limit(0)
        res.append(m.traj_adjoint(lam, 5, ckpt=2))
        res.append(m.traj_adjoint(lam, 5, ckpt=5))
        m.traj_record_limit(-1)
    for other in res[1:]:
        for x, y in zip(_fields(res[0]), _fields(other)):
            assert np.abs(x - y).max() <= 1e-12 * max(np.abs(x).max(), 1e-300)


@pytest.mark.parametrize("records", [True, False])
def test_host_checkpoints_give_the_same_gradient(records):
    """Checkpoints kept in page-locked host memory (forced) give the gradient the device
    checkpoints give, bit for bit, with and without the segment's stage records; the
    dot-product test passes with the host checkpoints."""
    from fdd3260_b200 import _lib
    d = config.warm_bubble_domain(24, 24, 12)
    st = config.warm_bubble_state(d, seed=6, centre=(600.0, 600.0, 250.0), radius=300.0)
    rng = np.random.default_rng(10)
    dx0 = _rand_like(st, rng, [0.1, 0.1, 0.05, 1.0, 1e-3, 0.05, 0.01])
    lam = _rand_like(st, rng, [1.0] * 7)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        if not records:
            m.traj_record_limit(0)
        m.traj_checkpoints(_lib.MG_CKPT_DEVICE)
        dev = m.traj_adjoint(lam, 6, ckpt=2)
        m.traj_checkpoints(_lib.MG_CKPT_HOST)
        host = m.traj_adjoint(lam, 6, ckpt=2)
        tl = m.traj_tl(dx0, 6)
    for x, y in zip(_fields(dev), _fields(host)):
        assert np.array_equal(x, y)
    lhs, rhs = _dot(tl, lam), _dot(dx0, host)
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs)), (lhs, rhs)


def _bump_direction(d):
    """A smooth perturbation of u, v, w and theta (w stays 0 on the ground)."""
    nz, ny, nx = d.shape
    X, Y = np.meshgrid(np.arange(nx) / d.maxx, np.arange(ny) / d.maxy)
    bump = np.stack([np.cos(2 * np.pi * (X + 0.1)) * np.sin(2 * np.pi * (Y + 0.2))] * nz)
    f = config.periodic_fill
    return config.State(f(0.5 * bump), f(-0.3 * bump), f(0.1 * bump * (np.arange(nz) > 0)[:, None, None]),
                        np.zeros(d.shape), np.zeros(d.shape), [f(0.2 * bump), np.zeros(d.shape)], -1)


def _functional(d, st, lam, nsteps):
    def J(eps, delta):
        moved = config.State(*[a + eps * b for a, b in zip(_fields(st)[:5], _fields(delta)[:5])],
                             [a + eps * b for a, b in zip(st.scal, delta.scal)], -1)
        with Mimica(d, nscal=2) as m:
            m.upload(moved)
            m.traj_forward(nsteps)
            out = m.download()
        return _dot(out, lam)
    return J


def _gradient(d, st, lam, nsteps):
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        return m.traj_adjoint(lam, nsteps, ckpt=2)


def test_taylor_second_order_momentum():
    """Without buoyancy the winds do not depend on the scalars and the momentum step (FD4
    advection, Heun stages, the linear projection) is smooth: for J = lam . (u, v, w)(T) after
    3 steps the first-order Taylor remainder falls as eps^2 over three decades and the
    central difference matches g . delta."""
    d = config.warm_bubble_domain(32, 32, 16, dt0=1.0, with_buoy=0)
    st = _smooth_state(d)
    nsteps = 3
    lam = _rand_like(st, np.random.default_rng(11), [1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0])
    delta = _bump_direction(d)
    J = _functional(d, st, lam, nsteps)
    gd = _dot(_gradient(d, st, lam, nsteps), delta)
    J0 = J(0.0, delta)
    rems = [abs(J(eps, delta) - J0 - eps * gd) for eps in (1e-2, 1e-3, 1e-4)]
    for a, b in zip(rems, rems[1:]):
        assert 0.005 < b / a < 0.02, rems          # eps^2: a factor 100 per decade
    eps = 1e-4
    cd = (J(eps, delta) - J(-eps, delta)) / (2 * eps)
    assert abs(cd - gd) <= 1e-8 * abs(gd), (cd, gd)


@pytest.mark.parametrize("target", ["winds", "theta"])
def test_central_difference_with_buoyancy_and_scalar_advection(target):
    """With buoyancy on, theta (advected by the WENO-switch scheme) feeds w.  The scheme's
    switch and limiters make J only piecewise smooth: here the nearest branch change lies
    between eps = 1e-6 and 1e-5 along this direction, so the linearisation is checked inside
    the smooth piece, at eps = 1e-6, where the central difference matches g . delta to
    5e-6 relative (its own round-off is about 1e-16 |J| / eps)."""
    d = config.warm_bubble_domain(32, 32, 16, dt0=1.0, with_buoy=1)
    st = _smooth_state(d)
    nsteps = 3
    scales = [1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0] if target == "winds" else [0, 0, 0, 0, 0, 1.0, 0]
    lam = _rand_like(st, np.random.default_rng(11), scales)
    delta = _bump_direction(d)
    J = _functional(d, st, lam, nsteps)
    g = _gradient(d, st, lam, nsteps)
    gd = _dot(g, delta)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        tl = m.traj_tl(delta, nsteps)
    assert abs(_dot(tl, lam) - gd) <= 1e-12 * abs(gd)
    eps = 1e-6
    cd = (J(eps, delta) - J(-eps, delta)) / (2 * eps)
    assert abs(cd - gd) <= 5e-6 * abs(gd), (cd, gd)


def test_time_traj_leaves_state_and_reports():
    d = config.warm_bubble_domain(24, 24, 12)
    st = config.warm_bubble_state(d, seed=6, centre=(600.0, 600.0, 250.0), radius=300.0)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        t = m.time_traj(4, 2)
        out = m.download()
    for x, y in zip(_fields(out), _fields(st)):
        assert np.array_equal(_interior(x), _interior(y))
    assert t["forward_ms"] > 0 and t["tl_ms"] > 0 and t["adjoint_ms"] > t["forward_ms"]
    # checkpoints: 4/2 + 1 states, a segment of 3, adjoint, scratch and the stage records
    assert t["adjoint_device_bytes"] >= (3 + 3 + 2) * 7 * 8 * np.prod(d.shape)


@pytest.mark.parametrize("with_buoy,target,eps,rtol", [(0, "winds", 1e-4, 1e-7), (1, "theta", 1e-6, 1e-5)])
def test_gradient_against_oracle_central_differences(with_buoy, target, eps, rtol):
    """The GPU adjoint's gradient along smooth and single-cell directions of the initial
    winds and theta against central differences of the CPU restatement of the
    reference's step (the oracle), an implementation independent of the GPU code."""
    from oracle import oracle as O
    d = config.warm_bubble_domain(24, 24, 12, dt0=1.0, with_buoy=with_buoy)
    st = _smooth_state(d, seed=2)
    nsteps = 2
    scales = [1.0, 1.0, 1.0, 0, 0, 0, 0] if target == "winds" else [0.3, 0.3, 0.3, 0, 0, 1.0, 0]
    lam = _rand_like(st, np.random.default_rng(21), scales)
    g = _gradient(d, st, lam, nsteps)
    orc = O.Oracle(d)

    def J(e, delta):
        moved = config.State(*[a + e * b for a, b in zip(_fields(st)[:5], _fields(delta)[:5])],
                             [a + e * b for a, b in zip(st.scal, delta.scal)], -1)
        out, _, _ = orc.stepping(moved, nsteps=nsteps, ntime0=1)
        return _dot(out, lam)

    zero = lambda: np.zeros(d.shape)
    directions = [_bump_direction(d)]
    for f, (k, j, i) in [(0, (5, 9, 7)), (2, (6, 12, 15)), (5, (4, 8, 10))]:
        arrs = [zero() for _ in range(7)]
        arrs[f][k, j, i] = 1.0
        config.periodic_fill(arrs[f])
        directions.append(config.State(*arrs[:5], arrs[5:], -1))
    # round-off of the central difference: a few ulps of the largest weighted field per
    # cell, summed with the weights lam, over 2 eps (theta ~ 300 K: ~1e-6 at eps = 1e-6)
    big = max(np.abs(_interior(x)).max() for x, w in zip(_fields(st), scales) if w)
    lam2 = np.sqrt(sum(float(np.sum(_interior(x) ** 2)) for x in _fields(lam)))
    noise = 4 * np.spacing(big) * lam2 / (2 * eps)
    for delta in directions:
        gd = _dot(g, delta)
        cd = (J(eps, delta) - J(-eps, delta)) / (2 * eps)
        assert abs(cd - gd) <= rtol * abs(gd) + noise, (cd, gd, noise)
