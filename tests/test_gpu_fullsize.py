"""Size-independent properties of the integrator at the bench's full size, the shallow
cumulus 512 x 512 x 256 (density + 5 scalars, WENO3 switch, FD4), where the CPU
restatement would take hours:

- translation invariance: one step commutes with a periodic shift of the domain by one
  cell in x (stage 1 is shift-invariant bit for bit; the FFT projection adds round-off);
- conservation: with flux-form advection, periodic sides and a rigid lid, the domain
  total of every density-weighted field, sum of psi / dz1w(k), is unchanged by a step.
"""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def problem():
    d = config.cumulus_domain(512, 512, 256)
    st = config.cumulus_state(d, seed=1000, n_extra=3)
    return d, st


def _interior(a):
    return a[:, 3:-2, 3:-2]


def _totals(d, st):
    """domain totals of the density and of every density-weighted scalar"""
    w = (1.0 / d.dz1w)[:, None, None]
    dens = _interior(st.dens)
    out = [float(np.sum(dens * w))]
    for s in st.scal:
        out.append(float(np.sum(_interior(s) * dens * w)))
    return np.array(out)


def test_translation_invariance_one_step(problem):
    d, st = problem

    def roll(a):
        b = a.copy()
        _interior(b)[...] = np.roll(_interior(a), 1, axis=2)
        return config.periodic_fill(b)

    shifted = config.State(roll(st.u), roll(st.v), roll(st.w), roll(st.p), roll(st.dens), [roll(s) for s in st.scal],
                           st.iqt)
    outs = []
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        for s0 in (st, shifted):
            m.upload(s0)
            m.stepping(1, ntime0=1)
            outs.append(m.download())
    a, b = outs
    for x, y in zip([a.u, a.v, a.w, a.p, a.dens, *a.scal], [b.u, b.v, b.w, b.p, b.dens, *b.scal]):
        ref = np.roll(_interior(x), 1, axis=2)
        scale = max(np.abs(ref).max(), 1e-300)
        assert np.abs(_interior(y) - ref).max() <= 1e-12 * scale
    # the scalars of stage 1 do not see the projection: density is shift-invariant to rounding
    assert np.abs(_interior(b.dens) - np.roll(_interior(a.dens), 1, axis=2)).max() <= 1e-14 * np.abs(a.dens).max()


def test_conservation_two_steps(problem):
    d, st = problem
    t0 = _totals(d, st)
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        m.upload(st)
        m.stepping(2, ntime0=1, graph=True)
        out = m.download()
    t1 = _totals(d, out)
    rel = np.abs(t1 - t0) / np.abs(t0)
    assert np.all(rel <= 1e-11), rel
    # the step did move the fields
    assert np.abs(_interior(out.scal[0]) - _interior(st.scal[0])).max() > 1e-6
