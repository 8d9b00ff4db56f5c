"""The tuned plan as a dictionary -- radix sequences of the horizontal transforms, launch
shapes of the transforms and of the vertical tridiagonal solve, and the scalar
advection's k segments per column tile (0: chosen per launch) -- and a wisdom file that
keeps the plans ``mg_autotune`` chose, keyed by grid, precision and scalar count, so that
a later run on the same problem applies them without timing again (as FFTW's wisdom does
for the reference's transforms).  The file is JSON: {key: plan}."""
from __future__ import annotations

import ctypes as C
import json
import os

from . import _lib

FIELDS = ("x_radix", "y_radix", "x_threads", "y_threads", "tri_block", "k1_segments", "k2_segments")


def to_dict(t: _lib.MgTune) -> dict:
    return {"x_radix": list(t.x_radix)[:t.x_nstage], "y_radix": list(t.y_radix)[:t.y_nstage],
            "x_threads": t.x_threads, "y_threads": t.y_threads, "tri_block": t.tri_block, "k1_segments": t.k1_segments,
            "k2_segments": t.k2_segments}


def from_dict(d: dict) -> _lib.MgTune:
    t = _lib.MgTune()
    xr, yr = list(d["x_radix"]), list(d["y_radix"])
    if not (1 <= len(xr) <= 16 and 1 <= len(yr) <= 16):
        raise ValueError("a radix sequence has 1 to 16 stages")
    t.x_nstage, t.y_nstage = len(xr), len(yr)
    for q, r in enumerate(xr):
        t.x_radix[q] = int(r)
    for q, r in enumerate(yr):
        t.y_radix[q] = int(r)
    t.x_threads, t.y_threads, t.tri_block = int(d["x_threads"]), int(d["y_threads"]), int(d["tri_block"])
    t.k1_segments = int(d.get("k1_segments", 0))
    t.k2_segments = int(d.get("k2_segments", 0))
    return t


def key(maxx: int, maxy: int, nz: int, precision: int, nscal: int) -> str:
    """grid, precision and scalar count (the scalar advection's shared memory, and so its
    CTAs per SM, depends on the number of fields)"""
    return f"{maxx}x{maxy}x{nz}/{'mixed' if precision == _lib.MG_PREC_MIXED else 'fp64'}/{nscal}"


def load(path: str) -> dict:
    """The wisdom file's plans; a missing or unreadable file is an empty cache."""
    if not path or not os.path.exists(path):
        return {}
    try:
        with open(path) as f:
            w = json.load(f)
    except (OSError, ValueError):
        return {}
    return w if isinstance(w, dict) else {}


def store(path: str, k: str, plan: dict) -> None:
    """Add one plan. The file is replaced atomically through a temporary file of this
    process, so concurrent writers (ranks tuning their own grids) never leave a partial
    file; one writer's entry can be lost to another's, and is then tuned again."""
    w = load(path)
    # the segment counts default to the wave model's choice (0)
    w[k] = {f: plan.get(f, 0) if f.endswith("_segments") else plan[f] for f in FIELDS}
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(w, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def radix_candidates(n: int, maxc: int = 16) -> list[list[int]]:
    """The radix sequences mg_autotune tries for a transform of length n (host only)."""
    radix = (C.c_int * (16 * maxc))()
    nst = (C.c_int * maxc)()
    nc = _lib.lib().mg_radix_candidates(n, radix, nst, maxc)
    if nc < 0:
        _lib.check(nc, "mg_radix_candidates")
    return [list(radix[16 * q:16 * q + nst[q]]) for q in range(nc)]
