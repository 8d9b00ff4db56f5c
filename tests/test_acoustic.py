"""The compressible model's acoustic sub-steps (prognostic_pressure.f90) in the oracle:
the flux-form faces conserve mass, so over ntau sub-steps of stage 1 the domain's mass
changes by exactly the slow tendency's share; quick takes its own faces."""
import numpy as np
import pytest

from fdd3260_b200 import acoustic, config
from oracle import oracle as O


def _interior(d):
    return (slice(None), slice(3, 3 + d.maxy), slice(3, 3 + d.maxx))


@pytest.mark.parametrize("scheme", ["weno", "muscl", "quick"])
def test_stage1_mass_changes_by_the_slow_tendency_only(scheme):
    d = config.warm_bubble_domain(24, 20, 16, dz=40.0, dt0=0.5, scheme=scheme)
    inp, st = acoustic.acoustic_case(d, seed=11, im=1, ntau=8)
    out = O.Oracle(d).prognostic_pressure(inp, st)
    I = _interior(d)
    vol = d.dzw[:, None, None]
    m0, m1 = (st.dens[I] * vol).sum(), (out.dens[I] * vol).sum()
    slow = (inp.sdens[I] * vol).sum() * d.dt0
    assert abs((m1 - m0) - slow) <= 1e-12 * m0
    # es is advected in flux form as well: its integral changes by its slow tendency only
    e0, e1 = (st.es[I] * vol).sum(), (out.es[I] * vol).sum()
    eslow = (inp.ses[I] * vol).sum() * d.dt0
    # the equation of state's es/rho*rho round trip perturbs es by rounding only
    assert abs((e1 - e0) - eslow) <= 1e-12 * e0
    for f in acoustic.AcousticState.FIELDS:
        assert np.isfinite(getattr(out, f)[I]).all()
    # the pressure is the equation of state's: p + p0 = rho R theta Pi
    R = 1004.0 - 716.0
    th = out.es[I] / out.dens[I]
    pfull = out.dens[I] * R * th * (out.dens[I] * R * th / 1e5) ** (R / 716.0)
    np.testing.assert_allclose(out.p[I] + d.p0[:, None, None], pfull, rtol=1e-12)


def test_quick_needs_six_levels():
    """advsz_quick_nl's bottom face reads x(nz-5) (advq_quick_nolim.f90:233)."""
    d = config.warm_bubble_domain(16, 16, 5, scheme="quick")
    inp, st = acoustic.acoustic_case(d, seed=1, ntau=2)
    with pytest.raises(RuntimeError):
        O.Oracle(d).prognostic_pressure(inp, st)


def test_quick_and_lax_wendroff_faces_differ():
    """Without the limiter, quick takes its own faces and every other scheme the
    Lax-Wendroff ones (advection.f90:582-592)."""
    out = {}
    for scheme in ("quick", "weno", "ppm"):
        d = config.warm_bubble_domain(24, 20, 16, dz=40.0, dt0=0.5, scheme=scheme)
        inp, st = acoustic.acoustic_case(d, seed=2, ntau=2)
        out[scheme] = O.Oracle(d).prognostic_pressure(inp, st)
    assert np.array_equal(out["weno"].dens, out["ppm"].dens)
    assert not np.array_equal(out["weno"].dens, out["quick"].dens)
