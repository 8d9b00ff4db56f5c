"""CPU checks of the projection's plan space: the radix sequences the autotuner tries
(host code of the library, no device needed) and the wisdom file."""
import json
import math
import os

import pytest

from fdd3260_b200 import _lib, tune


@pytest.mark.parametrize("n", [8, 24, 30, 64, 96, 128, 160, 192, 250, 256, 512, 1024, 4096])
def test_radix_candidates_factor_n(n):
    cands = tune.radix_candidates(n)
    assert cands, n
    seen = set()
    for c in cands:
        assert math.prod(c) == n
        assert set(c) <= {2, 3, 4, 5, 8}
        assert 1 <= len(c) <= 16
        seen.add(tuple(c))
    assert len(seen) == len(cands), "distinct sequences"


def test_radix_candidates_start_with_the_default_plan():
    # the plan at context creation: radix 8 first, then 4 or 2, then 3 and 5
    assert tune.radix_candidates(512)[0] == [8, 8, 8]
    assert tune.radix_candidates(96)[0] == [8, 4, 3]
    assert tune.radix_candidates(160)[0] == [8, 4, 5]


def test_radix_candidates_reject_other_primes():
    assert tune.radix_candidates(14) == []
    assert tune.radix_candidates(2 * 7 * 3) == []


def test_wisdom_round_trip(tmp_path):
    plan = {"x_radix": [4, 4, 4, 4, 2], "y_radix": [3, 8, 4], "x_threads": 16, "y_threads": 64, "tri_block": 256,
            "k1_segments": 2, "k2_segments": 3}
    t = tune.from_dict(plan)
    assert tune.to_dict(t) == plan
    # a plan stored before K2's segments were a coordinate replays with the wave model's choice
    old = {f: v for f, v in plan.items() if f != "k2_segments"}
    assert tune.to_dict(tune.from_dict(old)) == dict(old, k2_segments=0)
    path = str(tmp_path / "wisdom.json")
    k = tune.key(512, 96, 64, _lib.MG_PREC_FP64, 5)
    tune.store(path, k, dict(plan, ms_tuned=1.0))
    tune.store(path, tune.key(64, 64, 32, _lib.MG_PREC_MIXED, 2), plan)
    w = tune.load(path)
    assert w[k] == plan and len(w) == 2
    assert tune.load(str(tmp_path / "absent.json")) == {}
    assert tune.key(512, 96, 64, _lib.MG_PREC_FP64, 5) != tune.key(512, 96, 64, _lib.MG_PREC_FP64, 2)
    with pytest.raises(ValueError):
        tune.from_dict(dict(plan, x_radix=[]))


def _store_many(path, wid, n):
    from fdd3260_b200 import tune as T
    plan = {"x_radix": [4, 4, 2], "y_radix": [8, 4], "x_threads": 16, "y_threads": 64, "tri_block": 128,
            "k1_segments": wid}
    for i in range(n):
        T.store(path, f"writer{wid}-{i}", plan)


def test_wisdom_concurrent_writers_leave_a_valid_file(tmp_path):
    """Ranks that tune at the same time write the same wisdom file: every replacement is
    a complete file (entries may be lost to another writer, never half-written)."""
    import multiprocessing as mp
    path = str(tmp_path / "wisdom.json")
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_store_many, args=(path, w, 25)) for w in range(4)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    with open(path) as f:
        w = json.load(f)
    assert w and all(k.startswith("writer") for k in w)
    assert not [f for f in os.listdir(tmp_path) if f.endswith(".tmp")]


def test_wisdom_unreadable_file_is_an_empty_cache(tmp_path):
    path = tmp_path / "wisdom.json"
    path.write_text('{"truncated": ')
    assert tune.load(str(path)) == {}
    path.write_text("[1, 2]")
    assert tune.load(str(path)) == {}
