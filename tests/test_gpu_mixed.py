"""Mixed form (FP32 stencil and flux arithmetic, FP64 state) against the FP64 oracle.

The error of each field is measured relative to the change the oracle makes to
that field over the run, in the L2 norm over the interior:

    err(f) = ||f_gpu - f_oracle||_2 / ||f_oracle - f_initial||_2

(for the pressure, whose initial value is zero, that is the relative L2 error).
Scalars and velocities carry large base values, so an error relative to the value
itself would say nothing about the FP32 arithmetic; the change over the run is what
the FP32 fluxes compute.  Tolerance: MIXED_TOL = 2e-4 per field.
"""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config
from fdd3260_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu
MIXED_TOL = 2e-4


def _interior(a):
    return a[:, 3:-2, 3:-2]


def field_errors(g, r, s0):
    out = {}
    pairs = [("u", g.u, r.u, s0.u), ("v", g.v, r.v, s0.v), ("w", g.w, r.w, s0.w), ("p", g.p, r.p, s0.p),
             ("dens", g.dens, r.dens, s0.dens)]
    pairs += [(f"s{i}", a, b, c) for i, (a, b, c) in enumerate(zip(g.scal, r.scal, s0.scal))]
    for name, a, b, c in pairs:
        a, b, c = _interior(a), _interior(b), _interior(c)
        den = np.linalg.norm(b - c)
        if den == 0.0:
            den = max(np.linalg.norm(b), 1e-300)
        out[name] = float(np.linalg.norm(a - b) / den)
    return out


def _run_mixed(d, st, nsteps, nscal, iqt=-1):
    d.precision = _lib.MG_PREC_MIXED
    with Mimica(d, nscal=nscal, iqt=iqt) as m:
        m.upload(st)
        m.stepping(nsteps, ntime0=1)
        g = m.download()
    d.precision = _lib.MG_PREC_FP64
    r, _, _ = O.Oracle(d).stepping(st, nsteps=nsteps, ntime0=1)
    return field_errors(g, r, st)


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl"])
def test_mixed_warm_bubble(scheme):
    d = config.warm_bubble_domain(32, 32, 24, scheme=scheme)
    st = config.warm_bubble_state(d, seed=21, centre=(800.0, 800.0, 400.0), radius=400.0)
    err = _run_mixed(d, st, 4, nscal=2)
    print(scheme, err)
    bad = {k: v for k, v in err.items() if not v <= MIXED_TOL}
    assert not bad, (bad, err)


def test_mixed_cumulus_moist():
    d = config.cumulus_domain(32, 32, 40, scheme="weno")
    st = config.cumulus_state(d, seed=1000, n_extra=2)
    err = _run_mixed(d, st, 4, nscal=len(st.scal), iqt=1)
    print("cumulus", err)
    bad = {k: v for k, v in err.items() if not v <= MIXED_TOL}
    assert not bad, (bad, err)
