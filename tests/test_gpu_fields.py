"""Field-at-a-time transfers (mg_upload_field / mg_download_field) on the GPU: a state
uploaded one field at a time steps exactly as the same state uploaded whole, a partial
upload holds no state, and single-field downloads equal the whole-state download."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib, config

pytestmark = pytest.mark.gpu


def _fields(st):
    return [st.u, st.v, st.w, st.p, st.dens, *st.scal]


def test_field_upload_steps_like_state_upload():
    d = config.cumulus_domain(32, 24, 20)
    st = config.cumulus_state(d, seed=17, n_extra=2)
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as whole:
        whole.upload(st)
        whole.stepping(2, ntime0=1)
        ref = whole.download()
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        arrs = _fields(st)
        for f, a in enumerate(arrs[:-1]):
            m.upload_field(f, a)
        # not every field yet: no state to step
        with pytest.raises(_lib.MimicaError) as ei:
            m.stepping(1, ntime0=1)
        assert ei.value.code == _lib.MG_ERR_STATE
        m.upload_field(len(arrs) - 1, arrs[-1])
        m.stepping(2, ntime0=1)
        got = m.download()
        for a, b in zip(_fields(got), _fields(ref)):
            assert np.array_equal(a, b)
        for f, b in enumerate(_fields(got)):
            assert np.array_equal(m.download_field(f), b)
        # replacing one field between steps: the same as a whole upload of the changed state
        th = got.scal[0].copy()
        th[:, 3:-2, 3:-2] += 0.5
        m.upload_field(_lib.MG_FIELD_SCAL, th)
        m.stepping(1, ntime0=3)
        one = m.download()
    got.scal[0] = th
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as whole:
        whole.upload(got)
        whole.stepping(1, ntime0=3)
        two = whole.download()
    for a, b in zip(_fields(one), _fields(two)):
        assert np.array_equal(a, b)
