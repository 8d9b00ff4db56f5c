"""The compressible model's acoustic sub-steps on the GPU (mg_prognostic_pressure)
against the oracle's restatement of prognostic_pressure.f90, through the C-ABI.

Every operation is the oracle's, in its order, compiled without FMA contraction, except
two: the equation of state's power (CUDA's pow against the C library's, which may
differ in the last bit) and the order of the level sums of the sound speed.  So the
fields agree to a relative 1e-11 after the sub-steps, not bit for bit."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib, acoustic, config
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-11


def _interior(d):
    return (slice(None), slice(3, 3 + d.maxy), slice(3, 3 + d.maxx))


def _run(d, inp, st):
    with Mimica(d, nscal=1) as m:
        return m.prognostic_pressure(inp, st)


def _check(d, gpu, ref):
    I = _interior(d)
    for f in acoustic.AcousticState.FIELDS:
        a, b = getattr(gpu, f)[I], getattr(ref, f)[I]
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= TOL * scale, (f, np.abs(a - b).max() / scale)
    for a, b in zip(gpu.scal + gpu.tscal, ref.scal + ref.tscal):
        assert np.abs(a[I] - b[I]).max() <= TOL * max(np.abs(b[I]).max(), 1e-300)
    # the state's ghost cells are periodic images
    for f in ("dens", "p", "u", "v", "w", "es", "qt"):
        x = getattr(gpu, f)
        np.testing.assert_array_equal(x, config.periodic_fill(x.copy()))


@pytest.mark.parametrize("im,ntau,cst_cp,nscal", [(1, 8, 1, 1), (2, 8, 1, 1), (1, 3, 0, 0), (2, 5, 0, 2)])
def test_acoustic_substeps_match_the_oracle(im, ntau, cst_cp, nscal):
    d = config.warm_bubble_domain(40, 32, 24, dz=40.0, dt0=0.5, scheme="weno")
    inp, st = acoustic.acoustic_case(d, seed=20 + im + ntau, im=im, ntau=ntau, nscal=nscal, cst_cp=cst_cp)
    ref = O.Oracle(d).prognostic_pressure(inp, st)
    _check(d, _run(d, inp, st), ref)


def test_every_limited_scheme_uses_the_lax_wendroff_faces():
    """advection.f90:582-592: without the limiter, every scheme but quick takes lw_nl."""
    base = config.warm_bubble_domain(32, 24, 16, dz=40.0, dt0=0.5, scheme="weno")
    inp, st = acoustic.acoustic_case(base, seed=3)
    ref = O.Oracle(base).prognostic_pressure(inp, st)
    for scheme in ("ppm", "muscl", "lw"):
        d = config.warm_bubble_domain(32, 24, 16, dz=40.0, dt0=0.5, scheme=scheme)
        _check(d, _run(d, inp, st), ref)


@pytest.mark.parametrize("im", [1, 2])
def test_quick_faces_match_the_oracle(im):
    """quick takes advq_quick_nolim's faces (advection.f90:586-587)."""
    d = config.warm_bubble_domain(40, 32, 24, dz=40.0, dt0=0.5, scheme="quick")
    inp, st = acoustic.acoustic_case(d, seed=40 + im, im=im, ntau=5, nscal=1)
    ref = O.Oracle(d).prognostic_pressure(inp, st)
    _check(d, _run(d, inp, st), ref)


def test_quick_needs_six_levels():
    """A quick context of 5 levels is refused (by mg_create, which needs more levels for
    the anelastic step, or by the acoustic entry, whose bottom face reads x(nz-5))."""
    d = config.warm_bubble_domain(16, 16, 5, scheme="quick")
    inp, st = acoustic.acoustic_case(d, seed=1, ntau=2)
    with pytest.raises(_lib.MimicaError) as ex:
        with Mimica(d, nscal=1) as m:
            m.prognostic_pressure(inp, st)
    assert ex.value.code == _lib.MG_ERR_PARAM


def test_mass_conservation_at_size():
    """At 192 x 192 x 64 (no oracle at this size): stage 1 changes the domain's mass by
    the slow tendency's share only, and the pressure obeys the equation of state."""
    d = config.warm_bubble_domain(192, 192, 64, dz=40.0, dt0=0.5, scheme="weno")
    inp, st = acoustic.acoustic_case(d, seed=9, im=1, ntau=8)
    out = _run(d, inp, st)
    I = _interior(d)
    vol = d.dzw[:, None, None]
    m0, m1 = (st.dens[I] * vol).sum(), (out.dens[I] * vol).sum()
    slow = (inp.sdens[I] * vol).sum() * d.dt0
    assert abs((m1 - m0) - slow) <= 1e-12 * m0
    R = 1004.0 - 716.0
    th = out.es[I] / out.dens[I]
    pfull = out.dens[I] * R * th * (out.dens[I] * R * th / 1e5) ** (R / 716.0)
    np.testing.assert_allclose(out.p[I] + d.p0[:, None, None], pfull, rtol=1e-12)


def test_timed_entry_runs_the_same_calls():
    """mg_time_prognostic_pressure: the first call, `warmup` and `reps` more on the
    resident fields give what as many separate calls give, bit for bit."""
    d = config.warm_bubble_domain(32, 24, 16, dz=40.0, dt0=0.5, scheme="weno")
    inp, st = acoustic.acoustic_case(d, seed=4, ntau=4)
    with Mimica(d, nscal=1) as m:
        timed, ms = m.prognostic_pressure(inp, st, reps=2, warmup=1)
        seq = st
        for _ in range(4):
            seq = m.prognostic_pressure(inp, seq)
    assert ms > 0
    I = _interior(d)
    for f in ("dens", "p", "u", "v", "w", "es", "qt", "tu", "tw", "tdens", "cs2"):
        np.testing.assert_array_equal(getattr(timed, f)[I], getattr(seq, f)[I])
