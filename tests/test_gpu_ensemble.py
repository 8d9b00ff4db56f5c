"""Batched ensemble stepping (mg_ensemble_step: one graph per step pair, forked to the
members' streams) gives, bit for bit, what stepping every member alone gives."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib
from fdd3260_b200 import ensemble as E

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [_lib.MG_PREC_FP64, _lib.MG_PREC_MIXED])
def test_ensemble_equals_members_stepped_alone(precision):
    specs = [E.MemberSpec(0, 32, 16, 11, 2.0, (800.0, 800.0, 200.0)),
             E.MemberSpec(1, 48, 24, 12, 1.5, (1200.0, 1000.0, 300.0)),
             E.MemberSpec(2, 40, 20, 13, 3.0, (1000.0, 900.0, 250.0))]
    probs = [E.member_problem(s, precision=precision) for s in specs]
    alone = []
    for d, st in probs:
        with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
            m.upload(st)
            m.stepping(5, ntime0=1)
            alone.append(m.download())
    members = [Mimica(d, nscal=len(st.scal), iqt=st.iqt) for d, st in probs]
    try:
        for m, (d, st) in zip(members, probs):
            m.upload(st)
        with E.Ensemble(members) as ens:
            ens.step(5, ntime0=1)   # two graph pairs and one eager step
            assert ens.launches_per_step > 0
        batched = [m.download() for m in members]
    finally:
        for m in members:
            m.close()
    for a, b in zip(alone, batched):
        for x, y in zip([a.u, a.v, a.w, a.p, a.dens, *a.scal], [b.u, b.v, b.w, b.p, b.dens, *b.scal]):
            assert np.array_equal(x, y)
