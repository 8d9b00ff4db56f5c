"""Ensembles of independent domains: batched stepping on one GPU, sharding across GPUs.

An ensemble member is a domain of its own (sizes, seed, parameters).  On one GPU the
members are advanced together by ``mg_ensemble_step`` (one CUDA graph per step pair
that forks to every member's stream).  Across GPUs the members are independent units:
``partition`` assigns them to ranks by a greedy cell-count balance (largest first, to
the least-loaded rank), with no collective on the data path -- each rank steps its own
members, and only the timing/metrics are gathered on the host.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib, config
from .model import Mimica

NX_CHOICES = (96, 128, 160, 192, 256)
NZ_CHOICES = (64, 96, 128)


@dataclass
class MemberSpec:
    """One member of the batched warm-bubble ensemble."""
    index: int
    nxy: int
    nz: int
    seed: int
    amp: float
    centre: tuple

    @property
    def cells(self) -> int:
        return self.nxy * self.nxy * self.nz


def ensemble_specs(n: int = 64, seed: int = 3000, dx: float = 50.0, dz: float = 40.0,
                   nx_choices=NX_CHOICES, nz_choices=NZ_CHOICES) -> list[MemberSpec]:
    """Seeded uneven sizes: nx = ny in {96,...,256}, nz in {64, 96, 128} (or the given
    sets); warm bubble of amplitude U[1,3] K centred at a random point in the lower third
    of the domain."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n):
        nxy = int(rng.choice(nx_choices))
        nz = int(rng.choice(nz_choices))
        amp = float(rng.uniform(1.0, 3.0))
        lx, lz = nxy * dx, nz * dz
        centre = (float(rng.uniform(0.2, 0.8) * lx), float(rng.uniform(0.2, 0.8) * lx),
                  float(rng.uniform(0.1, 1.0 / 3.0) * lz))
        out.append(MemberSpec(i, nxy, nz, seed + 1 + i, amp, centre))
    return out


def partition(cells: list[int], nranks: int) -> list[list[int]]:
    """Greedy balance of member indices over ranks by cell count (largest first to the
    least-loaded rank; ties by rank number), deterministic for equal inputs."""
    if nranks < 1:
        raise ValueError("nranks >= 1")
    load = [0] * nranks
    parts: list[list[int]] = [[] for _ in range(nranks)]
    for i in sorted(range(len(cells)), key=lambda q: (-cells[q], q)):
        r = min(range(nranks), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += cells[i]
    return [sorted(p) for p in parts]


def shard_and_time(specs: list[MemberSpec], rank: int, world: int, build, warmup: int, steps: int,
                   barrier=lambda: None, reduce_max=lambda x: x, reduce_sum=lambda x: x, timed_region=None) -> dict:
    """The per-rank path of a sharded ensemble run.  The members are partitioned over the
    ranks by cell count; ``build(my_specs)`` returns this rank's stepper (an object with
    ``step(n, ntime0)`` and ``time_steps(n, ntime0) -> ms``, e.g. an ``Ensemble``).  It runs
    exactly ``warmup`` untimed steps, the last two at the timed steps' parity (the momentum
    direction order alternates with the step's parity, so that pair is what the timed steps
    repeat), then ``steps`` timed steps after a barrier.  Only scalars cross ranks: the max
    of the timed milliseconds and the sum of the cells stepped.  ``timed_region`` is an
    optional context manager around the timed steps (clock sampling)."""
    if warmup < 3:
        raise ValueError("warmup >= 3")
    parts = partition([s.cells for s in specs], world)
    mine = [specs[i] for i in parts[rank]]
    stepper = build(mine)
    stepper.step(warmup - 2, ntime0=1)
    stepper.step(2, ntime0=warmup - 1)
    barrier()
    if timed_region is None:
        t_ms = stepper.time_steps(steps, ntime0=1 + warmup)
    else:
        with timed_region:
            t_ms = stepper.time_steps(steps, ntime0=1 + warmup)
    t_max = reduce_max(t_ms)
    cells = reduce_sum(sum(s.cells for s in mine))
    return {"t_ms": t_max, "rank_ms": t_ms, "cells": cells, "members": parts[rank], "parts": parts,
            "stepper": stepper, "value": cells * steps / (t_max / 1e3) / 1e6}


def member_problem(spec: MemberSpec, precision: int = _lib.MG_PREC_FP64, dx: float = 50.0, dz: float = 40.0,
                   dt0: float = 0.5, init=None):
    """(Domain, State) of a member: dry warm bubble, WENO, FD4 momentum.  ``init``: see
    config.Domain.finish."""
    d = config.warm_bubble_domain(spec.nxy, spec.nxy, spec.nz, dx=dx, dy=dx, dz=dz, dt0=dt0, scheme="weno",
                                  init=init)
    d.precision = precision
    st = config.warm_bubble_state(d, seed=spec.seed, amp=spec.amp, radius=min(500.0, 0.25 * spec.nz * dz),
                                  centre=spec.centre)
    return d, st


MODES = {"grouped": _lib.MG_ENS_GROUPED, "streams": _lib.MG_ENS_STREAMS}


class Ensemble:
    """Members on one device advanced together (``mg_ensemble_*``).

    ``mode`` "grouped" (the default when the members allow it) launches each kernel of a
    stage once over the blocks of all members; "streams" forks every member's own
    launches onto its stream.  Both give the same results."""

    def __init__(self, members: list[Mimica], mode: str | None = None):
        if not members:
            raise ValueError("an ensemble needs at least one member")
        self.members = members
        L = _lib.lib()
        arr = (C.c_void_p * len(members))(*[m._h.value for m in members])
        h = C.c_void_p()
        _lib.check(L.mg_ensemble_create(arr, len(members), C.byref(h)), "mg_ensemble_create")
        self._h = h
        self._L = L
        if mode is not None:
            self.mode = mode

    @property
    def mode(self) -> str:
        m = self._L.mg_ensemble_get_mode(self._h)
        return {v: k for k, v in MODES.items()}[m]

    @mode.setter
    def mode(self, mode: str) -> None:
        if mode not in MODES:
            raise ValueError(f"unknown ensemble mode {mode!r}")
        _lib.check(self._L.mg_ensemble_set_mode(self._h, MODES[mode]), "mg_ensemble_set_mode")

    def step(self, nsteps: int, ntime0: int = 1) -> None:
        _lib.check(self._L.mg_ensemble_step(self._h, nsteps, ntime0), "mg_ensemble_step")

    def time_steps(self, nsteps: int, ntime0: int = 1) -> float:
        ms = C.c_double(0.0)
        _lib.check(self._L.mg_ensemble_time_steps(self._h, nsteps, ntime0, C.byref(ms)), "mg_ensemble_time_steps")
        return ms.value

    def autotune(self, reps: int = 3, wisdom: str | None = None) -> dict:
        """The projection's plan of every member (``Mimica.autotune``): each distinct grid
        is timed once and its plan applied to the members of the same size.  Returns the
        plans by grid key."""
        from . import tune
        plans = {}
        for m in self.members:
            d = m.domain
            k = tune.key(d.maxx, d.maxy, d.nz, d.precision, m.nscal)
            if k in plans:
                m.tune_set({f: plans[k][f] for f in tune.FIELDS})
            else:
                plans[k] = m.autotune(reps=reps, wisdom=wisdom)
        return plans

    @property
    def launches_per_step(self) -> int:
        return self._L.mg_ensemble_launch_count(self._h)

    @property
    def cells(self) -> int:
        return sum(m.domain.cells for m in self.members)

    def close(self) -> None:
        if getattr(self, "_h", None) is not None and self._h.value:
            self._L.mg_ensemble_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
