"""checkall on the GPU (src/IO/check.f90) against the oracle: the max CFL and the es/qt
bounds with their first-occurrence locations, and an adaptive-time-step run whose dt
sequence and fields follow the oracle's."""
import ctypes as C

import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib, config
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.mark.parametrize("moist", [True, False])
def test_checkall_matches_oracle(moist):
    d = config.cumulus_domain(32, 24, 30, dt0=1.0)
    st = config.cumulus_state(d, seed=1000, n_extra=1)
    rng = np.random.default_rng(3)
    st.u = config.periodic_fill(st.u + rng.normal(size=d.shape))
    st.w = config.periodic_fill(rng.normal(size=d.shape))
    st.w[0] = 0.0
    if not moist:
        st = config.State(st.u, st.v, st.w, st.p, st.dens, [st.scal[0], st.scal[2]], -1)
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        m.upload(st)
        r = m.checkall(apply=False)
    orc = O.Oracle(d)
    mx, loc = orc.checkwind(st.u, st.v, st.w)
    assert r["maxcfl"] == mx and r["cfl_ijk"] == loc
    mn, mxe, lmin, lmax = orc.checkx(st.scal[0])
    assert (r["es_min"], r["es_max"], r["es_min_ijk"], r["es_max_ijk"]) == (mn, mxe, lmin, lmax)
    if moist:
        mn, mxq, lmin, lmax = orc.checkx(st.scal[1])
        assert (r["qt_min"], r["qt_max"], r["qt_min_ijk"], r["qt_max_ijk"]) == (mn, mxq, lmin, lmax)
    assert r["stop"] == _lib.MG_STOP_NONE


def test_checkall_ties_and_stop_reasons():
    d = config.warm_bubble_domain(32, 32, 16, dt0=1.0)
    st = config.warm_bubble_state(d, seed=2)
    # uniform |u| everywhere: every cell ties, the first interior cell is reported
    st.u[...] = 3.0
    st.v[...] = 0.0
    st.w[...] = 0.0
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        r = m.checkall(apply=False)
        assert r["cfl_ijk"] == (4, 4, 1) and r["maxcfl"] == 1.0 * 3.0 / d.dx
        bad = config.State(st.u, st.v, st.w, st.p, st.dens, [st.scal[0] * 0 + 150.0, st.scal[1]], -1)
        m.upload(bad)
        assert m.checkall(apply=False)["stop"] == _lib.MG_STOP_ES
        still = config.State(st.u * 0, st.v, st.w, st.p, st.dens, st.scal, -1)
        m.upload(still)
        assert m.checkall(apply=False)["stop"] == _lib.MG_STOP_CFL   # maxcfl < 1e-7 stops the reference too


def test_adaptive_time_step_run_matches_oracle():
    """ldtfix = 0: after every step pair checkall adapts dt0 (cfl_max 0.5, cfl_min 0.4); the
    GPU run (graphs re-recorded at each change) follows the oracle's dt decisions (to
    1e-12: the states agree to round-off) and fields."""
    d = config.warm_bubble_domain(32, 32, 24, dt0=4.0)
    st = config.warm_bubble_state(d, seed=21, centre=(800.0, 800.0, 400.0), radius=400.0, amp=3.0)
    st.u = config.periodic_fill(st.u + 8.0)   # CFL 0.64 at dt0 = 4 s: the first check shrinks dt0
    ch = config.Checks()
    nsteps = 6
    dts_g, dts_o = [], []
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        for s in range(nsteps):
            m.stepping(2, ntime0=1 + 2 * s, graph=True)
            r = m.checkall(ch, apply=True)
            dts_g.append(r["dt0_new"])
            assert r["stop"] == 0
        g = m.download()
    orc = O.Oracle(d)
    p = ch.params(d.dt0)
    cur = st
    for s in range(nsteps):
        cur, _, _ = orc.stepping(cur, nsteps=2, ntime0=1 + 2 * s)
        mx, _ = orc.checkwind(cur.u, cur.v, cur.w)
        new, stop = C.c_double(0.0), C.c_int(0)
        _lib.lib().mg_cfl_dt(C.byref(p), mx, orc.g.dt0, C.byref(new), C.byref(stop))
        dts_o.append(new.value)
        # the states agree to round-off (the projection is not bit-exact), so the maximum
        # CFL and the new step may differ in the last bits: the oracle continues with
        # the GPU's step to stay in lockstep
        orc.g.dt0 = dts_g[s]
    np.testing.assert_allclose(dts_o, dts_g, rtol=1e-12, atol=0)
    assert dts_g[0] < d.dt0, "the run should change dt"
    for a, b in zip([g.u, g.v, g.w, g.p, g.dens, *g.scal], [cur.u, cur.v, cur.w, cur.p, cur.dens, *cur.scal]):
        a, b = a[:, 3:-2, 3:-2], b[:, 3:-2, 3:-2]
        assert np.abs(a - b).max() <= TOL * max(np.abs(b).max(), 1e-300)
