"""mg_maxdiv_noalloc: the allocation-free residual entry, checked through the C-ABI
against the context path (mg_anelastic_pressure's maxdiv) on the same momentum, on two
calls in a row that share the library's fixed scratch.  Collected last on purpose: it
must pass alone and after every other test in the session."""
import ctypes as C

import numpy as np
import pytest

from fdd3260_b200 import Mimica, config, _lib


def _fn():
    L = _lib.lib()
    f = L.mg_maxdiv_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_void_p]
    return f


def test_noalloc_rejects_sizes_beyond_its_limits():
    f = _fn()
    for (mx, my, nz) in [(4097, 8, 8), (8, 4097, 8), (8, 8, 4097), (8, 8, 2), (0, 8, 8)]:
        assert f(mx, my, nz, 1.0, 1.0, 1, 1, 1, 1, 1, None) == _lib.MG_ERR_PARAM


@pytest.mark.gpu
def test_noalloc_maxdiv_matches_context_path_twice():
    import torch
    d = config.cumulus_domain(32, 32, 24)
    st = config.random_state(d, seed=14)
    mu = st.u * d.den0[:, None, None]
    mv = st.v * d.den0[:, None, None]
    mw = st.w * d.avden0[:, None, None]
    mw[0] = 0.0
    wold = mw * 0.9
    with Mimica(d, nscal=2) as m:
        gu, gv, gw, gp, md, p1 = m.anelastic_pressure(mu, mv, mw, st.p, wold)
    dev = torch.device("cuda", 0)
    tu = torch.from_numpy(np.ascontiguousarray(gu)).to(dev)
    tv = torch.from_numpy(np.ascontiguousarray(gv)).to(dev)
    tw = torch.from_numpy(np.ascontiguousarray(gw)).to(dev)
    tz = torch.from_numpy(np.ascontiguousarray(d.dz1w)).to(dev)
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    f = _fn()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        rc = f(d.maxx, d.maxy, d.nz, d.dx, d.dy, tz.data_ptr(), tu.data_ptr(), tv.data_ptr(), tw.data_ptr(),
               out.data_ptr() + 8 * call, stream)
        assert rc == 0, _lib.error_string(rc) if hasattr(_lib, "error_string") else rc
    torch.cuda.synchronize(dev)
    a, b = out.cpu().numpy()
    assert a == b
    assert a == md, (a, md)
