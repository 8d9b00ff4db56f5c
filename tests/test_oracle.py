"""CPU tests of the oracle (the CPU restatement used as the checker) and of the
host-side precompute shared with the product library.  No GPU needed.

Parity pins available for this path: the reference ships no golden vectors for
advection or the projection and cannot be compiled here, so these tests pin the
restatement with (a) the reference's own KISS FFT built from its sources, and its
committed golden vectors (tests/golden/kiss_fft.npz, made by
tests/golden/make_kiss_golden.py) where the sources are absent, (b) numpy.fft,
(c) known-answer properties of the discrete operators.
"""
import os

import numpy as np
import pytest

from fdd3260_b200 import config
from oracle import oracle as O


def test_dft_matches_numpy():
    rng = np.random.default_rng(1)
    for ny, nx in [(8, 12), (16, 10), (30, 18), (12, 20)]:
        re, im = rng.normal(size=(ny, nx)), rng.normal(size=(ny, nx))
        r, i = O.fft2d(re, im)
        ref = np.fft.fft2(re + 1j * im)
        assert np.abs(r + 1j * i - ref).max() <= 1e-14 * np.abs(ref).max()
        r, i = O.fft2d(re, im, inverse=True)
        ref = np.fft.ifft2(re + 1j * im) * nx * ny
        assert np.abs(r + 1j * i - ref).max() <= 1e-14 * np.abs(ref).max()


def test_dft_matches_reference_kiss_fft():
    """The reference's own KISS FFT (src/fftmpi/src/kissfft.h, compiled from its sources)."""
    if O.kiss_ref() is None:
        pytest.skip("reference KISS FFT not built (reference tree absent)")
    rng = np.random.default_rng(2)
    for n in [8, 12, 30, 64, 96, 160]:
        x = rng.normal(size=n) + 1j * rng.normal(size=n)
        r, i = O.fft2d(x.real[None, :], x.imag[None, :])
        k = O.kiss_fft(x)
        assert np.abs(k - (r[0] + 1j * i[0])).max() <= 1e-13 * np.abs(k).max()
        r, i = O.fft2d(x.real[None, :], x.imag[None, :], inverse=True)
        k = O.kiss_fft(x, inverse=True)
        assert np.abs(k - (r[0] + 1j * i[0])).max() <= 1e-13 * np.abs(k).max()


GOLDEN_KISS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kiss_fft.npz")


def _kiss_golden_cases():
    """(input, expected, inverse) from tests/golden/kiss_fft.npz: the reference's KISS FFT
    (src/fftmpi/src/kissfft.h) run on seeded inputs by tests/golden/make_kiss_golden.py."""
    g = np.load(GOLDEN_KISS)
    cx = lambda key: g[key + "_re"] + 1j * g[key + "_im"]
    for n in g["n1d"]:
        x = cx(f"1d_{n}_x")[None, :]
        yield x, cx(f"1d_{n}_fwd")[None, :], False
        yield x, cx(f"1d_{n}_bwd")[None, :], True
    for ny, nx in g["n2d"]:
        x = cx(f"2d_{ny}x{nx}_x")
        yield x, cx(f"2d_{ny}x{nx}_fwd"), False
        yield x, cx(f"2d_{ny}x{nx}_bwd"), True


@pytest.mark.parametrize("omp", [False, True], ids=["parity-build", "timed-build"])
def test_dft_matches_kiss_golden(omp):
    """Committed golden vectors of the reference's own FFT: both oracle builds agree to
    2e-15 relative (measured 6e-16) over 1-D lengths 1..256 with radix 2/3/4/5 and prime
    factors, and 2-D row-then-column transforms, forward and unnormalised backward."""
    orc = O.Oracle(config.warm_bubble_domain(16, 16, 8), omp=omp)
    ncase = 0
    for x, ref, inv in _kiss_golden_cases():
        r, i = orc.fft2d(x.real, x.imag, inverse=inv)
        assert r.shape == ref.shape
        assert np.abs(r + 1j * i - ref).max() <= 2e-15 * np.abs(ref).max(), (x.shape, inv)
        ncase += 1
    assert ncase == 2 * (26 + 7)


def test_host_precompute_bit_exact_with_oracle():
    """define_grid / initial / get_wv restatements: product library == oracle, bit for bit."""
    L = O.load()
    d = config.cumulus_domain(16, 24, 40)
    nz = d.nz
    dzw, dz1w, dz1 = (np.zeros(nz) for _ in range(3))
    L.mo_grid_metrics(nz, d.dz, O.P(d.fdz0), O.P(dzw), O.P(dz1w), O.P(dz1))
    assert np.array_equal(dzw, d.dzw) and np.array_equal(dz1w, d.dz1w) and np.array_equal(dz1, d.dz1)
    p0, den0, av, st = (np.zeros(nz) for _ in range(4))
    L.mo_base_state(nz, d.dz, d.psurf, O.P(d.fdz0), O.P(d.dz1), O.P(d.pt0), O.P(d.qv0), O.P(p0), O.P(den0),
                    O.P(av), O.P(st))
    assert np.array_equal(den0, d.den0) and np.array_equal(av, d.avden0) and np.array_equal(st, d.stab0)
    assert np.array_equal(p0, d.p0)
    wv = np.zeros((d.maxy, d.maxx))
    L.mo_get_wv(d.maxx, d.maxy, d.dx, d.dy, O.P(wv))
    assert np.array_equal(wv, d.wv())


def test_base_state_hydrostatic():
    d = config.warm_bubble_domain(8, 8, 40)
    # p0 decreases, density positive and decreasing for an isentropic atmosphere
    assert np.all(np.diff(d.p0) < 0) and np.all(d.den0 > 0) and np.all(np.diff(d.den0) < 0)
    # avden0 is the fdz-weighted face average
    assert np.allclose(d.avden0[1:], 0.5 * (d.den0[1:] + d.den0[:-1]), rtol=1e-14)


def test_wv_uses_reference_pi():
    """get_wv uses the reference's pi = 3.14159265 (src/TYPES/shared_data.f90:147)."""
    d = config.warm_bubble_domain(8, 8, 8)
    wv = d.wv()
    pi = 3.14159265
    l, m = 2, 3
    expect = -4.0 * (np.sin(pi * l / 8) ** 2 / d.dx ** 2 + np.sin(pi * m / 8) ** 2 / d.dy ** 2)
    assert wv[m, l] == pytest.approx(expect, rel=1e-15)
    assert wv[0, 0] == 1.0


def _rand_mom(d, seed):
    st = config.random_state(d, seed=seed, nscal=2)
    mu = st.u * d.den0[:, None, None]
    mv = st.v * d.den0[:, None, None]
    mw = st.w * d.avden0[:, None, None]
    return st, mu, mv, mw


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl", "lw", "quick"])
def test_constant_field_uniform_flow_zero_tendency(scheme):
    d = config.warm_bubble_domain(16, 16, 12, scheme=scheme)
    orc = O.Oracle(d)
    x = np.full(d.shape, 2.5)
    mu = np.full(d.shape, 3.0) * d.den0[:, None, None]
    mv = np.full(d.shape, -1.5) * d.den0[:, None, None]
    mw = np.zeros(d.shape)
    xs = orc.advection_ac(x, mu, mv, mw, np.zeros(d.shape))
    assert np.abs(xs).max() <= 1e-13 * 2.5 * 3.0 / d.dx


@pytest.mark.parametrize("scheme", ["weno", "muscl", "lw", "quick"])
def test_translation_invariance_bit_exact(scheme):
    """WENO, MUSCL, lw and QUICK are translation invariant on the periodic domain (PPM is not:
    it reconstructs the ghost cells 3 and nx-1 with one-sided formulas)."""
    d = config.warm_bubble_domain(16, 16, 10, scheme=scheme)
    orc = O.Oracle(d)
    st, mu, mv, mw = _rand_mom(d, 3)
    x = st.scal[1] * d.den0[:, None, None]
    t0 = orc.advection_ac(x, mu, mv, mw, np.zeros(d.shape))

    def shift(a):
        b = a.copy()
        b[:, 3:-2, 3:-2] = np.roll(a[:, 3:-2, 3:-2], (1, 1), axis=(1, 2))
        return config.periodic_fill(b)

    t1 = orc.advection_ac(shift(x), shift(mu), shift(mv), shift(mw), np.zeros(d.shape))
    assert np.array_equal(shift(t0)[:, 3:-2, 3:-2], t1[:, 3:-2, 3:-2])


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl", "lw", "quick"])
def test_xy_symmetry_bit_exact(scheme):
    d = config.warm_bubble_domain(16, 16, 10, scheme=scheme)
    orc = O.Oracle(d)
    st, mu, mv, mw = _rand_mom(d, 4)
    x = st.scal[1] * d.den0[:, None, None]
    t0 = orc.advection_ac(x, mu, mv, mw, np.zeros(d.shape))
    T = lambda a: np.ascontiguousarray(np.swapaxes(a, 1, 2))
    # u at x-faces becomes v at y-faces: both staggered to the low side, so transposition is exact
    t1 = orc.advection_ac(T(x), T(mv), T(mu), T(mw), np.zeros(d.shape))
    assert np.array_equal(T(t0)[:, 3:-2, 3:-2], t1[:, 3:-2, 3:-2])


def _tridiag_apply(d, y):
    """The reference's per-wavenumber vertical operator (fft_tools.f90:142-173) applied to a
    spectrum y[k, ky, kx] (complex)."""
    nz = d.nz
    dz1, dz1w, stab, fdz = d.dz1, d.dz1w, d.stab0, d.fdz0
    wv = d.wv()
    out = np.zeros_like(y)
    for k in range(nz):
        if 0 < k < nz - 1:
            h = d.dz * (0.5 * fdz[k + 1] + fdz[k] + 0.5 * fdz[k - 1])
            a = dz1[k - 1] * dz1w[k] - stab[k] / h
            c = dz1[k] * dz1w[k] + stab[k] / h
            dd = wv - dz1w[k] * (dz1[k] + dz1[k - 1])
            out[k] = a * y[k - 1] + dd * y[k] + c * y[k + 1]
        elif k == 0:
            c = dz1[0] * dz1w[0] + stab[0] * dz1[0]
            dd = wv - dz1[0] * dz1w[0] - stab[0] * dz1[0]
            out[k] = dd * y[0] + c * y[1]
        else:
            a = dz1w[-1] * dz1[-2] - stab[-1] * dz1[-2]
            dd = wv - dz1w[-1] * dz1[-2] + stab[-1] * dz1[-2]
            out[k] = a * y[k - 1] + dd * y[k]
    return out


@pytest.mark.parametrize("maxx,maxy,nz", [(16, 12, 20), (20, 30, 12), (10, 18, 9), (8, 50, 15)])
def test_fft_solve_manufactured_solution(maxx, maxy, nz):
    """fft_solve inverts the reference's spectral operator: build rhs from a known solution.
    Grids with radix 2, 3 and 5 factors (the sizes the product accepts), non-square, odd nz."""
    d = config.cumulus_domain(maxx, maxy, nz)
    orc = O.Oracle(d)
    rng = np.random.default_rng(5)
    sol = rng.normal(size=(d.nz, d.maxy, d.maxx))
    sol -= sol.mean(axis=(1, 2), keepdims=True)          # no (0,0) content
    Y = np.fft.fft2(sol)
    B = _tridiag_apply(d, Y)
    rhs_int = np.fft.ifft2(B).real
    tend = np.zeros(d.shape)
    tend[:, 3:3 + d.maxy, 3:3 + d.maxx] = rhs_int
    out = orc.fft_solve(tend)
    got = out[:, 3:3 + d.maxy, 3:3 + d.maxx] / (d.maxx * d.maxy)
    got -= got.mean(axis=(1, 2), keepdims=True)
    assert np.abs(got - sol).max() <= 1e-10 * np.abs(sol).max()


def test_projection_reduces_divergence():
    d = config.warm_bubble_domain(16, 16, 16)
    orc = O.Oracle(d)
    st, mu, mv, mw = _rand_mom(d, 6)
    mw[0] = 0.0

    def maxdiv(mu, mv, mw):
        div = np.zeros(d.shape)
        L = orc.L
        L.mo_caldiv(orc.gp, O.P(mu.copy()), O.P(mv.copy()), O.P(mw.copy()), O.P(div))
        return np.abs(div[1:-1, 3:-2, 3:-2]).max()

    d0 = maxdiv(mu, mv, mw)
    mu2, mv2, mw2, p2, md, p1 = orc.anelastic_pressure(mu, mv, mw, np.zeros(d.shape), mw)
    d1 = maxdiv(mu2, mv2, mw2)
    assert d1 < 1e-5 * d0
    assert abs(md) <= d1 + 1e-30


def test_nsubp_iterations_converge():
    """Each extra sub-iteration (nsubp, pressure_solver.f90:100-111) shrinks the residual."""
    res = []
    for nsubp in (1, 2, 3):
        d = config.cumulus_domain(16, 16, 24, nsubp=nsubp)
        orc = O.Oracle(d)
        st, mu, mv, mw = _rand_mom(d, 8)
        mw[0] = 0.0
        _, _, _, _, md, _ = orc.anelastic_pressure(mu, mv, mw, np.zeros(d.shape), mw)
        res.append(abs(md))
    assert res[1] < res[0] and res[2] < res[1]


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl", "lw", "quick"])
def test_oracle_step_finite_and_conservative(scheme):
    d = config.warm_bubble_domain(16, 16, 12, scheme=scheme)
    st = config.warm_bubble_state(d, seed=1, centre=(400.0, 400.0, 300.0), radius=250.0)
    orc = O.Oracle(d)
    st1, md, p1 = orc.stepping(st, nsteps=2, ntime0=1)
    for a in [st1.u, st1.v, st1.w, st1.p, st1.dens, *st1.scal]:
        assert np.isfinite(a).all()
    # flux form with rigid lid conserves the domain total of the density-weighted scalar
    # up to the non-periodic PPM ghost-cell reconstruction
    tot0 = (st.scal[1] * st.dens)[:, 3:-2, 3:-2].sum(axis=(1, 2)) @ d.dzw
    tot1 = (st1.scal[1] * st1.dens)[:, 3:-2, 3:-2].sum(axis=(1, 2)) @ d.dzw
    tol = 1e-12 if scheme != "ppm" else 1e-4
    assert abs(tot1 - tot0) <= tol * abs(tot0)


def test_timed_build_agrees_with_parity_build():
    """The OpenMP build (the timed CPU baseline) runs the same restatement with a tabulated
    twiddle FFT and thread-parallel loops: its transforms agree with the parity build to
    1e-14 relative, and one full step agrees to 1e-10 relative per field."""
    rng = np.random.default_rng(7)
    d = config.warm_bubble_domain(24, 20, 16)
    par, omp = O.Oracle(d), O.Oracle(d, omp=True)
    for ny, nx in [(64, 64), (59, 61), (18, 12), (5, 7), (9, 1), (49, 121)]:
        re, im = rng.normal(size=(ny, nx)), rng.normal(size=(ny, nx))
        for inv in (False, True):
            a = par.fft2d(re, im, inverse=inv)
            b = omp.fft2d(re, im, inverse=inv)
            sc = max(np.abs(a[0]).max(), np.abs(a[1]).max())
            assert np.abs(a[0] - b[0]).max() <= 1e-14 * sc and np.abs(a[1] - b[1]).max() <= 1e-14 * sc
    st = config.warm_bubble_state(d, seed=3, centre=(300.0, 250.0, 300.0), radius=200.0)
    s1, md1, _ = par.stepping(st, nsteps=1, ntime0=1)
    s2, md2, _ = omp.stepping(st, nsteps=1, ntime0=1)
    for a, b in zip([s1.u, s1.v, s1.w, s1.p, s1.dens, *s1.scal], [s2.u, s2.v, s2.w, s2.p, s2.dens, *s2.scal]):
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1e-300)
