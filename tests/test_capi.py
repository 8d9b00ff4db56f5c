"""The C-ABI library loads and exports every symbol include/mimica_gpu.h declares.
No compute call is made (CPU only)."""
import ctypes as C
import os
import re

import numpy as np

from fdd3260_b200 import _lib, config

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = []
    for h in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if h.endswith(".h"):
            src = open(os.path.join(ROOT, "include", h)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names += re.findall(r"\b(mg_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_error_strings():
    L = _lib.lib()
    for code in range(8):
        s = L.mg_error_string(code).decode()
        assert s and s != "unknown error"


def test_invalid_params_rejected_without_device():
    d = config.warm_bubble_domain(16, 16, 8)
    L = _lib.lib()
    for bad in [dict(mom_ord=3), dict(nsubp=0), dict(scal_adv="weno", maxx=14)]:
        dd = config.warm_bubble_domain(**{**dict(maxx=16, maxy=16, nz=8), **{k: v for k, v in bad.items()
                                                                            if k in ("maxx",)}})
        if "mom_ord" in bad:
            dd.mom_ord = 3
        if "nsubp" in bad:
            dd.nsubp = 0
        p, keep = dd.params(2, -1)
        h = C.c_void_p()
        rc = L.mg_create(C.byref(p), 0, C.byref(h))
        assert rc == _lib.MG_ERR_PARAM
    # iqt must not alias es
    p, keep = d.params(2, 0)
    h = C.c_void_p()
    assert L.mg_create(C.byref(p), 0, C.byref(h)) == _lib.MG_ERR_PARAM


def test_null_pointers_rejected():
    L = _lib.lib()
    assert L.mg_destroy(None) == _lib.MG_ERR_PARAM
    assert L.mg_step(None, 1, 1, None, None) == _lib.MG_ERR_PARAM
    assert L.mg_grid_metrics(1, 1.0, None, None, None, None) == _lib.MG_ERR_PARAM
    # trajectory, autotuner and timing entries: a null context is rejected before any
    # device work
    assert L.mg_traj_forward(None, 1, 1) == _lib.MG_ERR_PARAM
    assert L.mg_traj_tl(None, 1, 1, None, None) == _lib.MG_ERR_PARAM
    assert L.mg_traj_adjoint(None, 1, 1, 1, None, None) == _lib.MG_ERR_PARAM
    assert L.mg_traj_record_limit(None, 0.0) == _lib.MG_ERR_PARAM
    assert L.mg_traj_checkpoints(None, 1) == _lib.MG_ERR_PARAM
    assert L.mg_time_traj(None, 1, 1, 1, None) == _lib.MG_ERR_PARAM
    assert L.mg_autotune(None, 3, None) == _lib.MG_ERR_PARAM
    assert L.mg_tune_get(None, None) == _lib.MG_ERR_PARAM
    assert L.mg_tune_set(None, None) == _lib.MG_ERR_PARAM
    assert L.mg_radix_candidates(0, None, None, 4) == _lib.MG_ERR_PARAM
    assert L.mg_qnadv_ad(None, 1, *([None] * 9)) == _lib.MG_ERR_PARAM
    assert L.mg_selftest_wait(None, 1000) == _lib.MG_ERR_PARAM
    assert L.mg_upload_field(None, 0, None) == _lib.MG_ERR_PARAM
    assert L.mg_download_field(None, 0, None) == _lib.MG_ERR_PARAM


def test_host_precompute_matches_formulas():
    d = config.cumulus_domain(8, 8, 30)
    assert np.allclose(d.dzw, d.dz * d.fdz0, rtol=0, atol=0)
    assert np.allclose(d.dz1w, 1.0 / (d.dz * d.fdz0), rtol=1e-15)
    assert np.allclose(d.dz1[:-1], 1.0 / (d.dz * 0.5 * (d.fdz0[:-1] + d.fdz0[1:])), rtol=1e-15)
    assert d.dz1[-1] == d.dz1[-2]
