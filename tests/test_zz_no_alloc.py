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


def _numpy_maxdiv(d, mu, mv, mw):
    """maxval of caldiv over the interior and k = 2..nz-1, with the kernel's operation order."""
    sl = (slice(1, d.nz - 1), slice(3, 3 + d.maxy), slice(3, 3 + d.maxx))
    c = mu[sl]
    du = mu[1:d.nz - 1, 3:3 + d.maxy, 4:4 + d.maxx] - c
    dv = mv[1:d.nz - 1, 4:4 + d.maxy, 3:3 + d.maxx] - mv[sl]
    dw = mw[2:d.nz, 3:3 + d.maxy, 3:3 + d.maxx] - mw[sl]
    dd = ((0.0 + du * (1.0 / d.dx)) + dv * (1.0 / d.dy)) + dw * d.dz1w[1:d.nz - 1][:, None, None]
    return float(dd.max())


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["grid_stride", "all_negative"])
def test_noalloc_maxdiv_matches_numpy(case):
    """128 x 128 x 24 has 360,448 cells in the residual range, more than the 1024 blocks x
    256 threads of the scratch: every block folds several cells.  all_negative has a
    strictly converging vertical flow, so the signed maximum is negative."""
    import torch
    d = config.cumulus_domain(128, 128, 24)
    rng = np.random.default_rng(21)
    if case == "grid_stride":
        mu, mv, mw = (config.periodic_fill(rng.normal(size=d.shape)) for _ in range(3))
    else:
        mu, mv = np.zeros(d.shape), np.zeros(d.shape)
        mw = -np.broadcast_to(np.arange(d.nz, dtype=np.float64)[:, None, None], d.shape).copy()
        mw += 1e-3 * config.periodic_fill(rng.uniform(0.0, 1.0, size=d.shape))
    want = _numpy_maxdiv(d, mu, mv, mw)
    if case == "all_negative":
        assert want < 0.0
    dev = torch.device("cuda", 0)
    t = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (d.dz1w, mu, mv, mw)]
    out = torch.full((2,), float("nan"), dtype=torch.float64, device=dev)
    f = _fn()
    stream = torch.cuda.current_stream(dev).cuda_stream
    for call in range(2):
        rc = f(d.maxx, d.maxy, d.nz, d.dx, d.dy, *[x.data_ptr() for x in t], out.data_ptr() + 8 * call, stream)
        assert rc == 0, rc
    torch.cuda.synchronize(dev)
    a, b = out.cpu().numpy()
    assert a == b == want, (a, b, want)
