"""CPU test of bench.py's timing schedule with a stand-in model (no GPU, no library).

The contract: exactly --warmup W untimed steps, then exactly K timed steps.  The step
graphs cover pairs of steps keyed by the parity of their first step (the momentum
direction order alternates with the step counter), so the last warm-up pair must run at
the timed region's parity: the graph the timed steps replay is then recorded before
timing, never inside it.
"""
import argparse
import ctypes as C
import os
import sys
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402

KERNELS = ("k1_scalar_advection", "halo_scalars", "k2_momentum", "halo_momentum", "fft_x_fwd_div",
           "fft_y_tridiag_fft_y_fft_x_inv", "correction_halo", "cal_p1")


class FakeLib:
    def __init__(self, log):
        self.log = log

    def mg_time_steps(self, h, nsteps, ntime0, use_graph, ms_ref):
        self.log.append(("timed", nsteps, ntime0, bool(use_graph)))
        ms_ref._obj.value = 10.0 * nsteps
        return 0

    def mg_profile_enable(self, h, on):
        self.log.append(("profile", on))
        return 0

    def mg_profile_report(self, h, buf, n):
        buf.value = "\n".join(f"{k} 2 {1.0 + i}" for i, k in enumerate(KERNELS)).encode()
        return 0


class FakeModel:
    def __init__(self):
        self.log = []
        self._L = FakeLib(self.log)
        self._h = object()
        self.launches_per_call = 8

    def autotune(self, reps=3):
        self.log.append(("autotune",))
        return {"source": "tuned"}

    def tune_get(self):
        return {}

    def stepping(self, nsteps=1, ntime0=1, diagnostics=False, graph=False):
        self.log.append(("step", nsteps, ntime0, graph))

    def synchronize(self):
        pass


@pytest.mark.parametrize("warmup", [3, 4, 5, 8])
@pytest.mark.parametrize("steps", [1, 2, 20])
def test_warmup_is_exact_and_records_the_timed_graph(warmup, steps):
    args = argparse.Namespace(steps=steps, warmup=warmup, scheme="weno", autotune="on")
    d = types.SimpleNamespace(cells=64 * 64 * 32, nsubp=1, sgs=None)
    st = types.SimpleNamespace(scal=[None] * 5)
    m = FakeModel()
    out = bench.time_form(args, m, d, st, True, 1, 0)

    timed = [e for e in m.log if e[0] == "timed"]
    assert len(timed) == 1
    _, k, t0, graph = timed[0]
    assert k == steps and graph and t0 == warmup + 1
    i_timed = m.log.index(timed[0])
    warm = [e for e in m.log[:i_timed] if e[0] == "step"]
    # exactly W warm-up steps, numbered 1..W without gaps
    assert sum(e[1] for e in warm) == warmup
    n = 1
    for e in warm:
        assert e[2] == n
        n += e[1]
    # the last warm-up call is a graph pair at the timed region's parity
    last = warm[-1]
    assert last[1] == 2 and last[3] and (last[2] & 1) == (t0 & 1)
    # the profiled pass comes after the timed steps
    after = [e for e in m.log[i_timed:] if e[0] == "step"]
    assert after and after[0][2] == warmup + steps + 1
    assert out["gpu_launches"] == 8 * steps
    assert out["ms_per_step"] == pytest.approx(10.0)
