"""Mixed form (FP32 stencil and flux arithmetic, FP64 state) against the FP64 oracle.

The error of each field is measured relative to the change the oracle makes to
that field over the run, in the L2 norm over the interior:

    err(f) = ||f_gpu - f_oracle||_2 / ||f_oracle - f_initial||_2

(for the pressure, whose initial value is zero, that is the relative L2 error).
Scalars and velocities carry large base values, so an error relative to the value
itself would say nothing about the FP32 arithmetic; the change over the run is what
the FP32 fluxes compute.  Tolerances per field, about five times the measured errors:
- warm bubble 32 x 32 x 24, 4 steps, every scheme: winds and density 2.5e-10 measured,
  pressure 3.4e-8, scalars 4.7e-7;
- moist cumulus 32 x 32 x 40, 4 steps: winds 5.8e-7, pressure 2.4e-6, density 6.8e-8,
  scalars 1.2e-7 to 7.9e-6.
"""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config
from fdd3260_b200 import _lib
from oracle import oracle as O

pytestmark = pytest.mark.gpu
BUBBLE_TOL = {"u": 2e-9, "v": 2e-9, "w": 2e-9, "p": 2e-7, "dens": 2e-9, "scalars": 3e-6}
CUMULUS_TOL = {"u": 3e-6, "v": 3e-6, "w": 3e-6, "p": 1.5e-5, "dens": 4e-7, "scalars": 4e-5}


def _over(err, tol):
    return {k: v for k, v in err.items() if not v <= tol.get(k, tol["scalars"])}


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


@pytest.mark.parametrize("scheme", ["weno", "ppm", "muscl", "lw", "quick"])
def test_mixed_warm_bubble(scheme):
    d = config.warm_bubble_domain(32, 32, 24, scheme=scheme)
    st = config.warm_bubble_state(d, seed=21, centre=(800.0, 800.0, 400.0), radius=400.0)
    err = _run_mixed(d, st, 4, nscal=2)
    print(scheme, err)
    bad = _over(err, BUBBLE_TOL)
    assert not bad, (bad, err)


def test_mixed_cumulus_moist():
    d = config.cumulus_domain(32, 32, 40, scheme="weno")
    st = config.cumulus_state(d, seed=1000, n_extra=2)
    err = _run_mixed(d, st, 4, nscal=len(st.scal), iqt=1)
    print("cumulus", err)
    bad = _over(err, CUMULUS_TOL)
    assert not bad, (bad, err)


def _rel_l2(g, r):
    """||f_gpu - f_oracle||_2 / ||f_oracle||_2 over the interior, per field."""
    out = {}
    for name in ("u", "v", "w", "p", "dens"):
        a, b = _interior(getattr(g, name)), _interior(getattr(r, name))
        out[name] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    for i, (a, b) in enumerate(zip(g.scal, r.scal)):
        a, b = _interior(a), _interior(b)
        out[f"s{i}"] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
    return out


def _mixed_run(d, st, nsteps, nscal, iqt, refine_iters, refine_tol):
    d.precision = _lib.MG_PREC_MIXED
    d.refine_iters, d.refine_tol = refine_iters, refine_tol
    try:
        with Mimica(d, nscal=nscal, iqt=iqt) as m:
            m.upload(st)
            md, _ = m.stepping(nsteps, ntime0=1, diagnostics=True)
            return m.download(), md
    finally:
        d.precision = _lib.MG_PREC_FP64


def test_mixed_refinement_skips_when_converged():
    """Refinement passes whose starting residual is below refine_tol change nothing."""
    d = config.warm_bubble_domain(32, 32, 24)
    st = config.warm_bubble_state(d, seed=3, centre=(800.0, 800.0, 400.0), radius=400.0)
    a, _ = _mixed_run(d, st, 2, 2, -1, refine_iters=0, refine_tol=0.0)
    b, _ = _mixed_run(d, st, 2, 2, -1, refine_iters=3, refine_tol=1e30)
    for x, y in zip([a.u, a.v, a.w, a.p, *a.scal], [b.u, b.v, b.w, b.p, *b.scal]):
        assert np.array_equal(x, y)


def test_mixed_refinement_reaches_fp64_divergence():
    """FP32 transforms with FP64-residual refinement: fields within 1e-6 relative L2 of
    the FP64 oracle and the post-projection divergence at the FP64 path's level (the
    reference's single pass leaves a discretisation residual of its own, which the
    refined mixed solve reproduces rather than removes)."""
    d = config.cumulus_domain(32, 32, 40, scheme="weno")
    st = config.cumulus_state(d, seed=1000, n_extra=2)
    nscal = len(st.scal)
    g0, md0 = _mixed_run(d, st, 3, nscal, 1, refine_iters=0, refine_tol=0.0)
    g, md = _mixed_run(d, st, 3, nscal, 1, refine_iters=3, refine_tol=1e-13)
    with Mimica(d, nscal=nscal, iqt=1) as m:
        m.upload(st)
        md64, _ = m.stepping(3, ntime0=1, diagnostics=True)
    r, mdr, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    e = _rel_l2(g, r)
    e0 = _rel_l2(g0, r)
    print("refined", e, "md", md, "| unrefined", e0, "md", md0, "| fp64 md", md64, "oracle md", mdr)
    # every field within 1e-6 relative L2 of the FP64 oracle, except the pressure, which
    # integrates the FP32 rounding of the momentum stencils: 1.2e-6 measured, 3e-6 allowed
    tol = {k: (3e-6 if k == "p" else 1e-6) for k in e}
    bad = {k: v for k, v in e.items() if not v <= tol[k]}
    assert not bad, (bad, e)
    # the refined projection leaves the FP64 path's post-projection divergence
    assert abs(md - md64) <= 1e-3 * abs(md64) + 1e-13, (md, md64)


def test_mixed_projection_unit_refinement():
    """anelastic_pressure in the mixed form: FP32 transforms alone agree with the FP64
    oracle to ~2e-7; one refinement pass on the FP64 Poisson residual brings every
    output to 1e-8 (measured ~1e-9 for the winds, ~4e-9 for p)."""
    d = config.cumulus_domain(32, 32, 24)
    st = config.random_state(d, seed=14)
    mu, mv, mw = (st.u * d.den0[:, None, None], st.v * d.den0[:, None, None], st.w * d.avden0[:, None, None])
    mw[0] = 0.0
    wold = mw * 0.9
    r = O.Oracle(d).anelastic_pressure(mu, mv, mw, st.p, wold)
    errs = {}
    for iters in (0, 1):
        d.precision, d.refine_iters, d.refine_tol = _lib.MG_PREC_MIXED, iters, 0.0
        try:
            with Mimica(d, nscal=2) as m:
                g = m.anelastic_pressure(mu, mv, mw, st.p, wold)
        finally:
            d.precision = _lib.MG_PREC_FP64
        errs[iters] = [float(np.linalg.norm(_interior(a) - _interior(b)) / np.linalg.norm(_interior(b)))
                       for a, b in zip(g[:4], r[:4])]
    assert max(errs[0]) <= 1e-6, errs
    assert max(errs[1]) <= 1e-8, errs


def test_exact_projection_reaches_fp64_divergence():
    """The exact projection: three passes of the reference's nsubp loop, each solving for
    the physical divergence (caldiv) of the corrected momentum.  The plain FP64 form
    matches the oracle's nsubp = 3 step to 1e-12; in the mixed form each pass is an FP32
    solve against the FP64 divergence (no refinement against the Poisson operator), and
    the post-projection divergence falls below 1e-10 1/s (the one-pass residual is about
    1e-5 on this grid).  Density + 5 scalars: the kernels with the field count built in."""
    d = config.cumulus_domain(32, 32, 40, scheme="weno", nsubp=3)
    st = config.cumulus_state(d, seed=1003, n_extra=3)
    nscal = len(st.scal)
    with Mimica(d, nscal=nscal, iqt=1) as m:
        m.upload(st)
        md64, _ = m.stepping(3, ntime0=1, diagnostics=True)
        g64 = m.download()
    r, mdr, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    e64 = _rel_l2(g64, r)
    assert max(e64.values()) <= 1e-12, e64
    g, md = _mixed_run(d, st, 3, nscal, 1, refine_iters=0, refine_tol=0.0)
    e = _rel_l2(g, r)
    d.nsubp = 1
    r1, md1, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    dep = _rel_l2(r, r1)
    print("exact: fp64 md", md64, "oracle md", mdr, "mixed md", md, "one-pass md", md1, "| mixed vs fp64 exact", e,
          "| exact vs one-pass", dep)
    assert abs(md) <= 1e-10 and abs(mdr) <= 1e-10 and abs(md1) > 1e-8
    # the mixed exact form stays close to the FP64 exact form (measured in the print above)
    bad = {k: v for k, v in e.items() if not v <= 1e-5}
    assert not bad, (bad, e)


@pytest.mark.parametrize("maxy", [64, 128, 256])
def test_mixed_fft_solve_with_the_shuffle_y_transform(maxy):
    """FP32 spectra whose y length is 64..512 take the warp-shuffle y transform: the
    mixed fft_solve stays within FP32 rounding of the oracle's FP64 solve."""
    d = config.warm_bubble_domain(48, maxy, 12)
    d.precision = _lib.MG_PREC_MIXED
    rng = np.random.default_rng(maxy)
    tend = rng.standard_normal(d.shape)
    with Mimica(d, nscal=1) as m:
        got = m.fft_solve(tend)
    d.precision = _lib.MG_PREC_FP64
    ref = O.Oracle(d).fft_solve(tend)
    a, b = _interior(got), _interior(ref)
    rel = np.linalg.norm(a - b) / np.linalg.norm(b)
    print(f"maxy {maxy}: mixed fft_solve relative L2 {rel:.2e}")
    assert rel <= 1e-4


def test_mixed_step_with_the_shuffle_y_transform():
    """Four mixed steps of a 64 x 64 bubble (the shuffle y transform in every projection
    pass) within the warm bubble's tolerances of the FP64 oracle."""
    d = config.warm_bubble_domain(64, 64, 24)
    st = config.warm_bubble_state(d, seed=12, centre=(1600.0, 1600.0, 400.0), radius=500.0)
    err = _run_mixed(d, st, 4, len(st.scal))
    assert not _over(err, BUBBLE_TOL), err
