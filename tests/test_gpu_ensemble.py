"""Batched ensemble stepping (mg_ensemble_step: one graph per step pair) gives, bit for
bit, what stepping every member alone gives, in both recording modes: grouped launches
over the blocks of all members, and every member's own launches forked to its stream."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib
from fdd3260_b200 import ensemble as E

pytestmark = pytest.mark.gpu

SPECS = [E.MemberSpec(0, 32, 16, 11, 2.0, (800.0, 800.0, 200.0)),
         E.MemberSpec(1, 48, 24, 12, 1.5, (1200.0, 1000.0, 300.0)),
         E.MemberSpec(2, 40, 20, 13, 3.0, (1000.0, 900.0, 250.0))]


def _alone(probs, nsteps, plans=None):
    out = []
    for q, (d, st) in enumerate(probs):
        with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
            if plans and plans[q]:
                m.tune_set({**m.tune_get(), **plans[q]})
            m.upload(st)
            m.stepping(nsteps, ntime0=1)
            out.append(m.download())
    return out


def _batched(probs, nsteps, mode, plans=None):
    members = [Mimica(d, nscal=len(st.scal), iqt=st.iqt) for d, st in probs]
    try:
        for q, (m, (d, st)) in enumerate(zip(members, probs)):
            if plans and plans[q]:
                m.tune_set({**m.tune_get(), **plans[q]})
            m.upload(st)
        with E.Ensemble(members, mode=mode) as ens:
            assert ens.mode == mode
            ens.step(nsteps, ntime0=1)   # graph pairs, and one eager step when nsteps is odd
            launches = ens.launches_per_step
        return [m.download() for m in members], launches
    finally:
        for m in members:
            m.close()


def _same(alone, batched):
    for a, b in zip(alone, batched):
        for x, y in zip([a.u, a.v, a.w, a.p, a.dens, *a.scal], [b.u, b.v, b.w, b.p, b.dens, *b.scal]):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("mode", ["grouped", "streams"])
@pytest.mark.parametrize("precision", [_lib.MG_PREC_FP64, _lib.MG_PREC_MIXED])
def test_ensemble_equals_members_stepped_alone(precision, mode):
    probs = [E.member_problem(s, precision=precision) for s in SPECS]
    batched, launches = _batched(probs, 5, mode)
    assert launches > 0
    _same(_alone(probs, 5), batched)


@pytest.mark.parametrize("precision", [_lib.MG_PREC_FP64, _lib.MG_PREC_MIXED])
def test_grouped_launch_count_does_not_grow_with_members(precision):
    """Grouped recording: one launch per kernel of a stage over all members, so two and
    three members take the same launches per step (the streams mode takes one set per
    member)."""
    probs = [E.member_problem(s, precision=precision) for s in SPECS]
    _, l3 = _batched(probs, 2, "grouped")
    _, l2 = _batched(probs[:2], 2, "grouped")
    _, s3 = _batched(probs, 2, "streams")
    assert l2 == l3 and l3 < s3
    # per stage: K1, 2 halos, K2, residual reset, x/y/tridiagonal/y/x-inverse per pass,
    # correction, cal_p1 (2); the mixed form adds one refinement pass (5)
    per_stage = 14 + (5 if precision == _lib.MG_PREC_MIXED else 0)
    assert l3 == 2 * per_stage


def test_grouped_members_with_different_transform_plans():
    """Members whose x transforms use different threads per row pair are launched in one
    x-transform launch per plan; the results are still those of the members alone (the
    refined form's block sums follow each member's own thread layout)."""
    probs = [E.member_problem(s, precision=_lib.MG_PREC_MIXED) for s in SPECS]
    plans = [{"x_threads": 16}, None, {"x_threads": 64, "y_threads": 64, "tri_block": 256}]
    batched, launches = _batched(probs, 4, "grouped", plans)
    _same(_alone(probs, 4, plans), batched)
    _, base = _batched(probs, 2, "grouped")
    assert launches > base   # extra x-transform launches for the other plans


def test_grouped_mode_refuses_mixed_forms():
    probs = [E.member_problem(SPECS[0], precision=_lib.MG_PREC_FP64),
             E.member_problem(SPECS[1], precision=_lib.MG_PREC_MIXED)]
    members = [Mimica(d, nscal=len(st.scal), iqt=st.iqt) for d, st in probs]
    try:
        for m, (d, st) in zip(members, probs):
            m.upload(st)
        with E.Ensemble(members) as ens:
            assert ens.mode == "streams"
            with pytest.raises(_lib.MimicaError):
                ens.mode = "grouped"
    finally:
        for m in members:
            m.close()


@pytest.mark.parametrize("scheme", ["ppm", "muscl", "quick"])
def test_grouped_other_schemes_equal_members_stepped_alone(scheme):
    """The grouped K1 instantiates every scheme (PPM keeps whole columns, as here)."""
    specs = [E.MemberSpec(0, 24, 16, 21, 2.0, (600.0, 600.0, 200.0)),
             E.MemberSpec(1, 32, 12, 22, 1.5, (800.0, 700.0, 150.0))]
    probs = []
    for s in specs:
        d, st = E.member_problem(s, precision=_lib.MG_PREC_FP64)
        d.scal_adv = scheme
        probs.append((d, st))
    batched, _ = _batched(probs, 4, "grouped")
    _same(_alone(probs, 4), batched)


def test_grouped_more_members_than_one_momentum_launch_holds():
    """K2's grouped arguments are a kernel parameter of at most 64 members: 70 members
    take two K2 launches per stage, with the same results."""
    rng = np.random.default_rng(7)
    specs = [E.MemberSpec(q, int(rng.choice([16, 24])), 12, 100 + q, 1.0 + q % 3, (300.0, 300.0, 150.0))
             for q in range(70)]
    probs = [E.member_problem(s, precision=_lib.MG_PREC_FP64) for s in specs]
    batched, launches = _batched(probs, 2, "grouped")
    _same(_alone(probs, 2), batched)
    assert launches == 2 * (14 + 1)   # one more K2 launch per stage
