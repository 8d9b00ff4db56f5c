"""Failure detection on the GPU, in forms that fault, trap or hang nothing.

* A zero pivot of the vertical tridiagonal system (the reference's TRIDAG2 CODE 1,
  src/PRESSURE/fft_tools.f90:214-227, which the reference ignores) is reported by
  mg_create as MG_ERR_PIVOT; the oracle's Thomas elimination flags the same system.
* A bounded mbarrier wait that runs out (mg_selftest_wait: bytes armed that no copy
  delivers, a limit of a few thousand cycles) returns MG_ERR_TIMEOUT, and the same
  context then steps normally, equal to the oracle.
* A non-finite value in the resident state is found by checkall with its first location
  (MG_ERR_NAN); a clean state uploaded afterwards checks normally.
"""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib, config
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pivot_domain():
    """A grid whose bottom row has a zero pivot for the horizontal mode (kx, ky) = (1, 0):
    with dz1(1) = 1 and dz1w(1) = 0 the first diagonal is wv(1,0) - stab0(1), and stab0(1)
    is set to that eigenvalue, so the difference is exactly zero."""
    d = config.warm_bubble_domain(16, 16, 8)
    wv = d.wv()
    d.dz1 = d.dz1.copy()
    d.dz1w = d.dz1w.copy()
    d.stab0 = d.stab0.copy()
    d.dz1[0], d.dz1w[0], d.stab0[0] = 1.0, 0.0, wv[0, 1]
    return d


def test_zero_pivot_reported_at_create():
    d = _pivot_domain()
    with pytest.raises(_lib.MimicaError) as ei:
        Mimica(d, nscal=2)
    assert ei.value.code == _lib.MG_ERR_PIVOT
    # the oracle's elimination meets the same zero pivot (TRIDAG2 CODE 1)
    rng = np.random.default_rng(5)
    tend = config.periodic_fill(rng.normal(size=d.shape))
    with pytest.raises(RuntimeError):
        O.Oracle(d).fft_solve(tend)
    # a well-posed context on the same device is unaffected
    g = config.warm_bubble_domain(16, 16, 8)
    st = config.warm_bubble_state(g, seed=2, centre=(400.0, 400.0, 200.0), radius=200.0)
    with Mimica(g, nscal=2) as m:
        m.upload(st)
        m.stepping(1, ntime0=1)


def test_bounded_wait_timeout_then_recovery():
    d = config.warm_bubble_domain(32, 32, 16)
    st = config.warm_bubble_state(d, seed=3, centre=(800.0, 800.0, 300.0), radius=300.0)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        # a limit of 4000 cycles (about 2 microseconds): the wait runs out
        assert m._L.mg_selftest_wait(m._h, 4000) == _lib.MG_ERR_TIMEOUT
        # the flag was cleared: a second self-test times out again (not stuck), and the
        # context's next step succeeds and equals the oracle's
        assert m._L.mg_selftest_wait(m._h, 4000) == _lib.MG_ERR_TIMEOUT
        assert m._L.mg_selftest_wait(m._h, -1) == _lib.MG_ERR_PARAM
        m.stepping(1, ntime0=1)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=1, ntime0=1)
    for a, b in [(g.u, r.u), (g.w, r.w), (g.p, r.p), *zip(g.scal, r.scal)]:
        a, b = a[:, 3:-2, 3:-2], b[:, 3:-2, 3:-2]
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("field,bad", [("w", np.nan), ("es", np.inf), ("u", -np.inf)])
def test_nonfinite_state_found_by_checkall(field, bad):
    d = config.cumulus_domain(32, 24, 20)
    st = config.cumulus_state(d, seed=9, n_extra=0)
    clean = st.copy()
    arr = st.scal[0] if field == "es" else getattr(st, field)
    # two bad cells; the first in the reference's loop order (k outermost, i fastest) is reported
    k1, j1, i1 = 7, 5, 9       # 0-based array indices: (k, j, i) = (8, 6, 10) 1-based
    arr[k1, j1, i1] = bad
    arr[12, 3, 4] = bad
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        m.upload(st)
        with pytest.raises(_lib.MimicaError) as ei:
            m.checkall(apply=False)
        assert ei.value.code == _lib.MG_ERR_NAN
        assert ei.value.ijk == (i1 + 1, j1 + 1, k1 + 1)
        m.upload(clean)
        r = m.checkall(apply=False)
        assert r["nonfinite"] == 0 and r["stop"] == _lib.MG_STOP_NONE
