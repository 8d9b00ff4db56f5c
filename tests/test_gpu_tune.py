"""The projection's plan and its autotuner (mg_autotune, mg_tune_get/set) on the GPU:
every candidate plan gives the default plan's projection to round-off, a step with a
tuned plan keeps step parity with the oracle, the autotuner leaves the state as it was,
invalid plans are rejected, and a wisdom file replays a plan without timing."""
import numpy as np
import pytest

from fdd3260_b200 import Mimica, _lib, config, tune
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _fields(st):
    return [st.u, st.v, st.w, st.p, st.dens, *st.scal]


def _momentum(d, seed):
    rng = np.random.default_rng(seed)
    mu, mv, mw = (config.periodic_fill(rng.normal(size=d.shape)) for _ in range(3))
    mw[0] = 0.0
    return mu, mv, mw


def _project(m, d, mom):
    mu, mv, mw = (a.copy() for a in mom)
    p = np.zeros(d.shape)
    out = m.anelastic_pressure(mu, mv, mw, p, mw.copy())
    return out[:4]


def test_every_candidate_plan_projects_alike():
    d = config.cumulus_domain(96, 160, 24)   # radix 3 and 5 in the transforms
    mom = _momentum(d, 1)
    with Mimica(d, nscal=2, iqt=1) as m:
        base_plan = m.tune_get()
        assert base_plan["x_radix"] == [8, 4, 3] and base_plan["y_radix"] == [8, 4, 5]
        ref = _project(m, d, mom)
        plans = [dict(base_plan, x_radix=xr) for xr in tune.radix_candidates(96)]
        plans += [dict(base_plan, y_radix=yr) for yr in tune.radix_candidates(160)]
        plans += [dict(base_plan, x_threads=xt, y_threads=yt, tri_block=tb)
                  for xt, yt, tb in [(8, 16, 64), (16, 128, 256), (64, 32, 128)]]
        for plan in plans:
            m.tune_set(plan)
            assert m.tune_get() == plan
            got = _project(m, d, mom)
            for g, r in zip(got, ref):
                scale = max(np.abs(r[:, 3:-2, 3:-2]).max(), 1e-300)
                assert np.abs(g[:, 3:-2, 3:-2] - r[:, 3:-2, 3:-2]).max() <= 1e-13 * scale, plan


def test_autotune_keeps_state_and_step_parity():
    d = config.warm_bubble_domain(48, 40, 20)
    st = config.warm_bubble_state(d, seed=3, centre=(1200.0, 1000.0, 400.0), radius=300.0)
    with Mimica(d, nscal=2) as m:
        m.upload(st)
        res = m.autotune(reps=2)
        assert res["source"] == "measured" and res["candidates"] > 5
        assert res["ms_tuned"] > 0 and res["ms_default"] > 0
        plan = m.tune_get()
        assert plan == {k: res[k] for k in tune.FIELDS}
        back = m.download()
        for x, y in zip(_fields(back), _fields(st)):
            assert np.array_equal(x[:, 3:-2, 3:-2], y[:, 3:-2, 3:-2])
        # a non-default plan (the scalar advection and the momentum in two k segments of
        # 10 levels each), then
        # a few steps against the oracle
        m.tune_set(dict(plan, x_radix=[2, 8, 3], y_radix=[5, 8], x_threads=16, y_threads=16, tri_block=64,
                        k1_segments=2, k2_segments=2))
        m.stepping(3, ntime0=1, graph=True)
        g = m.download()
    r, _, _ = O.Oracle(d).stepping(st, nsteps=3, ntime0=1)
    for a, b in zip(_fields(g), _fields(r)):
        a, b = a[:, 3:-2, 3:-2], b[:, 3:-2, 3:-2]
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300)


def test_invalid_plans_rejected():
    d = config.warm_bubble_domain(32, 24, 12)
    with Mimica(d, nscal=1) as m:
        base = m.tune_get()
        for bad in (dict(base, x_radix=[8, 8]), dict(base, y_radix=[7, 3]), dict(base, x_threads=128),
                    dict(base, y_threads=256), dict(base, x_threads=12), dict(base, tri_block=96),
                    dict(base, x_radix=[6, 4]),
                    dict(base, k1_segments=-1), dict(base, k1_segments=13), dict(base, k2_segments=-1),
                    dict(base, k2_segments=13)):
            with pytest.raises(_lib.MimicaError):
                m.tune_set(bad)
        assert m.tune_get() == base


def test_default_plan_round_trips_on_a_384_wide_grid():
    """A grid whose maxx/8 and maxy/8 are not powers of two gets 48 threads per row of the
    transforms by default; mg_tune_set takes that plan back (the bench's end-to-end leg
    copies a plan from one context to another), and a step with it set again equals the
    step before, bit for bit."""
    d = config.warm_bubble_domain(384, 384, 8)
    st = config.warm_bubble_state(d, seed=3, centre=(9600.0, 9600.0, 200.0), radius=150.0)
    with Mimica(d, nscal=len(st.scal)) as m:
        plan = m.tune_get()
        assert plan["x_threads"] == 48 and plan["y_threads"] == 48
        m.upload(st)
        m.stepping(1, ntime0=1)
        a = m.download()
        m.tune_set(plan)
        assert m.tune_get() == plan
        m.upload(st)
        m.stepping(1, ntime0=1)
        b = m.download()
    for x, y in zip(_fields(a), _fields(b)):
        assert np.array_equal(x, y)


def test_wisdom_replays_a_plan(tmp_path):
    path = str(tmp_path / "wisdom.json")
    d = config.warm_bubble_domain(64, 48, 16)
    with Mimica(d, nscal=1) as m:
        first = m.autotune(reps=2, wisdom=path)
    assert first["source"] == "measured"
    stored = tune.load(path)[tune.key(64, 48, 16, _lib.MG_PREC_FP64, 1)]
    with Mimica(d, nscal=1) as m:
        second = m.autotune(wisdom=path)
        assert second["source"] == "wisdom"
        assert m.tune_get() == stored
