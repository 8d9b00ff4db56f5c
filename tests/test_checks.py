"""CPU checks of the per-step checks (src/IO/check.f90): the library's time-step rule
(mg_cfl_dt, host code) against a transcription of checkwind's advective branch, and the
oracle's CFL / bounds reductions against known answers."""
import ctypes as C

import numpy as np
import pytest

from fdd3260_b200 import _lib, config
from oracle import oracle as O


def _rule(p, maxcfl, dt0):
    """checkwind :191-264 (advective part, ldtmic off): (dt0_new, stop)."""
    if maxcfl > 2. or maxcfl < 1.e-7:
        return dt0, _lib.MG_STOP_CFL
    new, stop = dt0, 0
    dtref = dt0
    if maxcfl >= p.cfl_max and p.ldtfix == 0:
        new = 0.95 * p.cfl_max / (maxcfl / dtref)
        if p.limit_ts > 1. and new <= p.dt0_i / max(1., p.limit_ts):
            stop = _lib.MG_STOP_DT
    if maxcfl <= p.cfl_min and maxcfl > 0. and p.ldtfix == 0:
        new = min(1.15 * p.cfl_min / (maxcfl / dtref), 2. * p.dt0_i)
    return new, stop


@pytest.mark.parametrize("ldtfix", [0, 1])
def test_time_step_rule_bit_exact(ldtfix):
    L = _lib.lib()
    ch = config.Checks(ldtfix=ldtfix)
    p = ch.params(dt0_i=1.0)
    rng = np.random.default_rng(1)
    cases = [2.5, 2.0, 1e-8, 1e-7, 0.5, 0.4, 0.45, 0.7, 1.999, 0.01, 0.3] + list(rng.uniform(1e-6, 2.0, 200))
    for maxcfl in cases:
        for dt0 in (1.0, 0.3, 0.051, 0.049, 1.7):
            new = C.c_double(0.0)
            stop = C.c_int(-1)
            _lib.check(L.mg_cfl_dt(C.byref(p), maxcfl, dt0, C.byref(new), C.byref(stop)), "mg_cfl_dt")
            want = _rule(p, maxcfl, dt0)
            assert (new.value, stop.value) == want, (maxcfl, dt0)


def test_time_step_rule_known_answers():
    L = _lib.lib()
    p = config.Checks().params(dt0_i=2.0)
    def run(m, dt):
        new, stop = C.c_double(0.0), C.c_int(-1)
        L.mg_cfl_dt(C.byref(p), m, dt, C.byref(new), C.byref(stop))
        return new.value, stop.value
    # CFL 1.0 at dt 2 -> the step that gives 0.95 cfl_max
    assert run(1.0, 2.0) == (pytest.approx(0.95 * 0.5 * 2.0), 0)
    # small CFL -> grows by 1.15 cfl_min / cfl, capped at 2 dt0_i
    assert run(0.2, 2.0)[0] == pytest.approx(min(1.15 * 0.4 / 0.1, 4.0))
    assert run(0.01, 2.0)[0] == 4.0
    # between the bounds: unchanged
    assert run(0.45, 2.0) == (2.0, 0)
    # too small a step -> stop
    assert run(1.9, 0.1)[1] == _lib.MG_STOP_DT
    assert run(2.1, 1.0)[1] == _lib.MG_STOP_CFL and run(0.0, 1.0)[1] == _lib.MG_STOP_CFL


def test_oracle_checkwind_first_occurrence():
    d = config.warm_bubble_domain(12, 10, 8, dt0=1.0)
    orc = O.Oracle(d)
    u, v, w = (np.zeros(d.shape) for _ in range(3))
    m, loc = orc.checkwind(u, v, w)
    assert m == 0.0 and loc == (0, 0, 0)
    # two cells with the same maximum: the first in (k, j, i) order wins
    u[3, 5, 7] = 10.0      # (i, j, k) = (8, 6, 4)
    v[3, 5, 6] = 10.0 * d.dy / d.dx   # same CFL, smaller i in the same row
    m, loc = orc.checkwind(u, v, w)
    assert m == pytest.approx(10.0 * d.dt0 / d.dx) and loc == (7, 6, 4)
    mn, mx, lmin, lmax = orc.checkx(u)
    assert (mn, mx, lmax, lmin) == (0.0, 10.0, (8, 6, 4), (4, 4, 1))
