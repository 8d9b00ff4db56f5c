"""Restart files written from and read into the GPU context (the reference's savedata /
readdata format): a run restarted from a file continues bit for bit, and turbu%ksgs
written with SGS diffusion on matches the oracle's viscosity."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, config, restart
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _domain():
    return config.cumulus_domain(32, 32, 30, scheme="weno", sgs=config.Sgs(pran=-0.4, zdec=500.0))


def test_restart_continues_bit_for_bit(tmp_path):
    d = _domain()
    st = config.cumulus_state(d, seed=1000, n_extra=2)
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        m.upload(st)
        m.stepping(4, ntime0=1)
        a = m.download()
    path = str(tmp_path / "restart.dat")
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        m.upload(st)
        m.stepping(2, ntime0=1)
        m.save_restart(path, time=2 * d.dt0, ntime=2)
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        h = m.load_restart(path)
        assert h["ntime"] == 2 and h["nscal"] == len(st.scal) - 2
        m.stepping(2, ntime0=h["ntime"] + 1)
        b = m.download()
    for x, y in zip([a.u, a.v, a.w, a.p, a.dens, *a.scal], [b.u, b.v, b.w, b.p, b.dens, *b.scal]):
        assert np.array_equal(x, y)
    r = restart.read(path, with_dif=True)
    assert r.ksgs is not None and np.isfinite(r.ksgs).all()


def test_ksgs_matches_oracle(tmp_path):
    d = _domain()
    st = config.cumulus_state(d, seed=7, n_extra=1)
    rng = np.random.default_rng(2)
    st.u = config.periodic_fill(st.u + 0.5 * rng.normal(size=d.shape))
    with Mimica(d, nscal=len(st.scal), iqt=st.iqt) as m:
        m.upload(st)
        m.stepping(1, ntime0=1)
        ks = m.ksgs()
    orc = O.Oracle(d)
    fkv = orc.calc_subgrid(st.u, st.v, st.w, st.scal[0], st.scal[st.iqt])
    delta = orc.sgs_profiles()[10 * d.nz:11 * d.nz]
    t = fkv / (0.12 * delta)[:, None, None]
    assert np.array_equal(ks, t * t)
