"""ctypes wrapper of the CPU restatement (oracle/mimica_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  Never part of the product path.

Parity status: the Fortran reference cannot be compiled here and ships no golden
vectors for this path, so the restatement is "parity unpinned" against a
reference binary; its FFT is pinned against the reference's own KISS FFT
(oracle/_ref/libkissref.so, built from src/fftmpi/src/kissfft.h when the
reference tree is present; its outputs are committed in tests/golden/kiss_fft.npz)
and numpy.fft.

Oracle(d) loads the parity build (libmimica_oracle.so); Oracle(d, omp=True) loads the
timed OpenMP build (libmimica_oracle_omp.so) that bench.py's CPU legs time.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = C.POINTER(C.c_double)

WENO, PPM, MUSCL, LW, QUICK = 0, 1, 2, 3, 4
LIM = {"minmod": 0, "VL": 1, "MC": 2, "default": 3}


class MoSgs(C.Structure):
    _fields_ = [
        ("with_dif", C.c_int), ("anis_k", C.c_int), ("momsf", C.c_int), ("pad", C.c_int),
        ("diff", C.c_double), ("pran", C.c_double), ("zdec", C.c_double), ("zrough", C.c_double),
        ("min_w", C.c_double), ("qt0", _dp), ("esflux", _dp), ("qvflux", _dp), ("mflux", _dp),
    ]


SGS_NPROF = 11


class MoGrid(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("scal_adv", C.c_int), ("muscl_limiter", C.c_int), ("mom_ord", C.c_int), ("lavisc", C.c_int),
        ("nsubp", C.c_int), ("with_buoy", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double), ("dt0", C.c_double),
        ("lim_tol", C.c_double), ("u0shift", C.c_double), ("v0shift", C.c_double),
        ("fdz0", _dp), ("dzw", _dp), ("dz1w", _dp), ("dz1", _dp), ("den0", _dp), ("avden0", _dp),
        ("stab0", _dp), ("pt0", _dp), ("qv0", _dp), ("wv", _dp), ("sgs", C.POINTER(MoSgs)),
    ]


class MoAcoustic(C.Structure):
    _fields_ = [
        ("im", C.c_int), ("ntau", C.c_int), ("cst_cp", C.c_int), ("nscal", C.c_int), ("p0", _dp),
        ("su", _dp), ("sv", _dp), ("sw", _dp), ("sdens", _dp), ("ses", _dp), ("sqt", _dp),
        ("sscal", C.POINTER(_dp)), ("uadv", _dp), ("vadv", _dp), ("wadv", _dp),
    ]


class MoAcousticState(C.Structure):
    _fields_ = [
        ("dens", _dp), ("p", _dp), ("u", _dp), ("v", _dp), ("w", _dp), ("es", _dp), ("qt", _dp),
        ("scal", C.POINTER(_dp)), ("tu", _dp), ("tv", _dp), ("tw", _dp), ("tdens", _dp), ("tes", _dp),
        ("tqt", _dp), ("tscal", C.POINTER(_dp)), ("cs2", _dp),
    ]


_libs = {}


def load(omp: bool = False) -> C.CDLL:
    name = "libmimica_oracle_omp.so" if omp else "libmimica_oracle.so"
    if name not in _libs:
        path = os.path.join(HERE, name)
        if not os.path.exists(path):
            raise RuntimeError(f"{path} missing: build with `python fdd3260_b200/build.py`")
        L = C.CDLL(path)
        g = C.POINTER(MoGrid)
        L.mo_advection_ac.argtypes = [g, _dp, _dp, _dp, _dp, _dp, C.c_int]
        L.mo_advection_dir.argtypes = [g, C.c_int, _dp, _dp, _dp, C.c_int]
        L.mo_advs_h.argtypes = [g, C.c_int, C.c_int, C.c_int, C.c_int, C.c_double, _dp, _dp, _dp, C.c_int]
        L.mo_advs_z.argtypes = [g, C.c_int, _dp, _dp, _dp, C.c_int]
        L.mo_get_advective.argtypes = [g, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mo_qnadv_uvw.argtypes = [g, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mo_caldiv.argtypes = [g, _dp, _dp, _dp, _dp]
        L.mo_gradp.argtypes = [g, _dp, _dp, _dp, _dp, _dp]
        L.mo_buoyancy.argtypes = [g, _dp, _dp, _dp, _dp]
        L.mo_fft2d.argtypes = [C.c_int, C.c_int, _dp, _dp, C.c_int]
        L.mo_fft_solve.argtypes = [g, _dp, _dp]
        L.mo_fft_solve.restype = C.c_int
        L.mo_tridiag.argtypes = [g, C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, C.c_size_t, C.c_size_t]
        L.mo_tridiag.restype = C.c_int
        L.mo_rescale_pressure.argtypes = [g, _dp]
        L.mo_horav.argtypes = [g, _dp, _dp]
        L.mo_anelastic_pressure.argtypes = [g, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mo_anelastic_pressure.restype = C.c_int
        L.mo_step.argtypes = [g, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int, C.POINTER(_dp), C.c_int, _dp, _dp]
        L.mo_step.restype = C.c_int
        L.mo_statebc.argtypes = [g, _dp]
        L.mo_grid_metrics.argtypes = [C.c_int, C.c_double, _dp, _dp, _dp, _dp]
        L.mo_base_state.argtypes = [C.c_int, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mo_get_wv.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _dp]
        L.mo_checkwind.argtypes = [g, _dp, _dp, _dp, _dp, C.POINTER(C.c_int)]
        L.mo_checkx.argtypes = [g, _dp, _dp, _dp, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.mo_sgs_profiles.argtypes = [g, _dp]
        L.mo_cal_dij.argtypes = [g, _dp, _dp, _dp, C.POINTER(_dp)]
        L.mo_calc_subgrid.argtypes = [g, _dp, _dp, _dp, _dp, _dp, _dp]
        L.mo_efud.argtypes = [g] + [_dp] * 8
        L.mo_eff.argtypes = [g, C.c_int, _dp, _dp, _dp, _dp]
        _libs[name] = L
    return _libs[name]


def P(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


class Init:
    """The oracle's restatement of the reference's init routines, in the form
    config.Domain.finish(init=...) takes: grid metrics (define_grid.f90:179-187) and the
    anelastic base state (initial.f90:473-558).  Used where a domain must be built without
    loading the CUDA library (bench.py's CPU reference arm)."""

    def __init__(self, omp: bool = False):
        self.L = load(omp)

    def grid_metrics(self, nz, dz, fdz0, dzw, dz1w, dz1):
        self.L.mo_grid_metrics(nz, dz, P(fdz0), P(dzw), P(dz1w), P(dz1))

    def base_state(self, nz, dz, psurf, fdz0, dz1, pt0, qv0, p0, den0, avden0, stab0):
        self.L.mo_base_state(nz, dz, psurf, P(fdz0), P(dz1), P(pt0), P(qv0), P(p0), P(den0), P(avden0), P(stab0))


class Oracle:
    """Oracle bound to one domain (config.Domain)."""

    def __init__(self, d, omp: bool = False):
        self.d = d
        self.L = load(omp)
        self._keep = [np.ascontiguousarray(a, dtype=np.float64) for a in
                      (d.fdz0, d.dzw, d.dz1w, d.dz1, d.den0, d.avden0, d.stab0, d.pt0, d.qv0)]
        self.wv = np.zeros((d.maxy, d.maxx))
        self.L.mo_get_wv(d.maxx, d.maxy, d.dx, d.dy, P(self.wv))
        g = MoGrid()
        g.nx, g.ny, g.nz = d.nx, d.ny, d.nz
        g.scal_adv = {"weno": WENO, "ppm": PPM, "muscl": MUSCL, "lw": LW, "quick": QUICK}[d.scal_adv]
        g.muscl_limiter = LIM[d.muscl_limiter]
        g.mom_ord, g.lavisc, g.nsubp, g.with_buoy = d.mom_ord, d.lavisc, d.nsubp, d.with_buoy
        g.dx, g.dy, g.dz, g.dt0 = d.dx, d.dy, d.dz, d.dt0
        g.lim_tol, g.u0shift, g.v0shift = d.lim_tol, d.u0shift, d.v0shift
        (g.fdz0, g.dzw, g.dz1w, g.dz1, g.den0, g.avden0, g.stab0, g.pt0, g.qv0) = [P(a) for a in self._keep]
        g.wv = P(self.wv)
        sg = getattr(d, "sgs", None)
        if sg is not None:
            ms = MoSgs()
            ms.with_dif, ms.anis_k, ms.momsf, ms.pad = 1, int(sg.anis_k), int(sg.momsf), 0
            ms.diff, ms.pran, ms.zdec, ms.zrough, ms.min_w = sg.diff, sg.pran, sg.zdec, sg.zrough, sg.min_w
            for name in ("qt0", "esflux", "qvflux", "mflux"):
                a = getattr(sg, name)
                if a is not None:
                    a = np.ascontiguousarray(a, dtype=np.float64)
                    self._keep.append(a)
                    setattr(ms, name, P(a))
            self._sgs = ms
            g.sgs = C.pointer(ms)
        self.g = g
        self.gp = C.byref(g)

    def advection_ac(self, x, mu, mv, mw, xs):
        ua, va, wa = self.get_advective(mu, mv, mw)
        xs = np.array(xs, dtype=np.float64, copy=True)
        self.L.mo_advection_ac(self.gp, P(np.ascontiguousarray(x)), P(ua), P(va), P(wa), P(xs), 0)
        return xs

    # ---- per-step checks (check.f90) ----
    def checkwind(self, u, v, w):
        mx = C.c_double(0.0)
        loc = (C.c_int * 3)()
        self.L.mo_checkwind(self.gp, *[P(np.ascontiguousarray(a)) for a in (u, v, w)], C.byref(mx), loc)
        return mx.value, tuple(loc)

    def checkx(self, x):
        mn, mx = C.c_double(0.0), C.c_double(0.0)
        lmin, lmax = (C.c_int * 3)(), (C.c_int * 3)()
        self.L.mo_checkx(self.gp, P(np.ascontiguousarray(x)), C.byref(mn), C.byref(mx), lmin, lmax)
        return mn.value, mx.value, tuple(lmin), tuple(lmax)

    # ---- SGS turbulence (subgrid.f90) ----
    def sgs_profiles(self) -> np.ndarray:
        prof = np.zeros(SGS_NPROF * self.d.nz)
        self.L.mo_sgs_profiles(self.gp, P(prof))
        return prof

    def cal_dij(self, u, v, w):
        d = [np.zeros(self.d.shape) for _ in range(6)]
        arr = (_dp * 6)(*[P(a) for a in d])
        self.L.mo_cal_dij(self.gp, *[P(np.ascontiguousarray(a)) for a in (u, v, w)], arr)
        return d

    def calc_subgrid(self, u, v, w, es, qt=None):
        fkv = np.zeros(self.d.shape)
        c = [None if a is None else np.ascontiguousarray(a) for a in (u, v, w, es, qt)]
        self.L.mo_calc_subgrid(self.gp, *[P(a) for a in c], P(fkv))
        return fkv

    def efud(self, u, v, w, dens, fkv, su=None, sv=None, sw=None):
        outs = [np.zeros(self.d.shape) if a is None else np.array(a, dtype=np.float64, copy=True) for a in (su, sv, sw)]
        c = [np.ascontiguousarray(a) for a in (u, v, w, dens, fkv)]
        self.L.mo_efud(self.gp, *[P(a) for a in c], *[P(a) for a in outs])
        return tuple(outs)

    def eff(self, kind, dens, fkv, x, ec=None):
        out = np.zeros(self.d.shape) if ec is None else np.array(ec, dtype=np.float64, copy=True)
        c = [np.ascontiguousarray(a) for a in (dens, fkv, x)]
        self.L.mo_eff(self.gp, kind, *[P(a) for a in c], P(out))
        return out

    def get_advective(self, mu, mv, mw):
        ua, va, wa = (np.zeros(self.d.shape) for _ in range(3))
        self.L.mo_get_advective(self.gp, P(mu), P(mv), P(mw), P(ua), P(va), P(wa))
        return ua, va, wa

    def qnadv_uvw(self, mu, mv, mw, ntime=1):
        ua, va, wa = self.get_advective(mu, mv, mw)
        au, av, aw = (np.zeros(self.d.shape) for _ in range(3))
        self.L.mo_qnadv_uvw(self.gp, ntime, P(mu), P(mv), P(mw), P(ua), P(va), P(wa), P(au), P(av), P(aw))
        return au, av, aw

    def fft_solve(self, tend, out=None):
        out = np.zeros(self.d.shape) if out is None else np.array(out, dtype=np.float64, copy=True)
        rc = self.L.mo_fft_solve(self.gp, P(np.ascontiguousarray(tend)), P(out))
        if rc:
            raise RuntimeError(f"oracle tridiagonal pivot error {rc}")
        return out

    def anelastic_pressure(self, mu, mv, mw, p, wold):
        mu, mv, mw, p = (np.array(a, dtype=np.float64, copy=True) for a in (mu, mv, mw, p))
        md = C.c_double(0.0)
        p1 = np.zeros(self.d.nz)
        rc = self.L.mo_anelastic_pressure(self.gp, P(mu), P(mv), P(mw), P(p), P(np.ascontiguousarray(wold)),
                                          C.byref(md), P(p1))
        if rc:
            raise RuntimeError(f"oracle tridiagonal pivot error {rc}")
        return mu, mv, mw, p, md.value, p1

    def stepping(self, st, nsteps=1, ntime0=1):
        """Advance a config.State (copied) by nsteps; returns (state, maxdiv, p1)."""
        st = st.copy()
        scal = [np.ascontiguousarray(s) for s in st.scal]
        sp = (_dp * len(scal))(*[P(s) for s in scal])
        md = C.c_double(0.0)
        p1 = np.zeros(self.d.nz)
        for s in range(nsteps):
            rc = self.L.mo_step(self.gp, ntime0 + s, P(st.u), P(st.v), P(st.w), P(st.p), P(st.dens), len(scal), sp,
                                st.iqt, C.byref(md), P(p1))
            if rc:
                raise RuntimeError(f"oracle tridiagonal pivot error {rc}")
        st.scal = scal
        return st, md.value, p1

    def prognostic_pressure(self, inp, st):
        """The acoustic sub-steps (prognostic_pressure.f90) on copies of an
        acoustic.AcousticState; returns the updated copy."""
        st = st.copy()
        c = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        keep = [c(a) for a in (inp.p0, inp.su, inp.sv, inp.sw, inp.sdens, inp.ses, inp.sqt, inp.uadv, inp.vadv,
                               inp.wadv)]
        sscal = [c(a) for a in inp.sscal]
        a = MoAcoustic()
        a.im, a.ntau, a.cst_cp, a.nscal = inp.im, inp.ntau, inp.cst_cp, len(st.scal)
        (a.p0, a.su, a.sv, a.sw, a.sdens, a.ses, a.sqt, a.uadv, a.vadv, a.wadv) = [P(x) for x in keep]
        sp = (_dp * max(1, len(sscal)))(*[P(x) for x in sscal])
        a.sscal = C.cast(sp, C.POINTER(_dp))
        s = MoAcousticState()
        for f in ("dens", "p", "u", "v", "w", "es", "qt", "tu", "tv", "tw", "tdens", "tes", "tqt", "cs2"):
            setattr(st, f, c(getattr(st, f)))
            setattr(s, f, P(getattr(st, f)))
        st.scal = [c(x) for x in st.scal]
        st.tscal = [c(x) for x in st.tscal]
        scp = (_dp * max(1, len(st.scal)))(*[P(x) for x in st.scal])
        tsp = (_dp * max(1, len(st.tscal)))(*[P(x) for x in st.tscal])
        s.scal, s.tscal = C.cast(scp, C.POINTER(_dp)), C.cast(tsp, C.POINTER(_dp))
        rc = self.L.mo_prognostic_pressure(self.gp, C.byref(a), C.byref(s))
        if rc:
            raise RuntimeError("the oracle's acoustic sub-steps need nz >= 6 with scal_adv = quick")
        return st

    def buoyancy(self, dens, es, qt=None):
        out = np.zeros(self.d.shape)
        self.L.mo_buoyancy(self.gp, P(dens), P(es), P(qt) if qt is not None else None, P(out))
        return out

    def statebc(self, x):
        x = np.array(x, dtype=np.float64, copy=True)
        self.L.mo_statebc(self.gp, P(x))
        return x

    def fft2d(self, re, im, inverse=False):
        re = np.array(re, dtype=np.float64, copy=True)
        im = np.array(im, dtype=np.float64, copy=True)
        ny, nx = re.shape
        self.L.mo_fft2d(nx, ny, P(re), P(im), 1 if inverse else 0)
        return re, im


def fft2d(re, im, inverse=False):
    L = load()
    re = np.array(re, dtype=np.float64, copy=True)
    im = np.array(im, dtype=np.float64, copy=True)
    ny, nx = re.shape
    L.mo_fft2d(nx, ny, P(re), P(im), 1 if inverse else 0)
    return re, im


def kiss_ref():
    """The reference's own KISS FFT (built from its sources), or None if not built."""
    path = os.path.join(HERE, "_ref", "libkissref.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    L.ref_kiss_fft.argtypes = [C.c_int, C.c_int, _dp, _dp]
    L.ref_kiss_fft.restype = C.c_int
    return L


def kiss_fft(x: np.ndarray, inverse=False):
    L = kiss_ref()
    if L is None:
        return None
    x = np.ascontiguousarray(x, dtype=np.complex128)
    inter = np.empty(2 * x.size)
    inter[0::2], inter[1::2] = x.real, x.imag
    out = np.empty_like(inter)
    L.ref_kiss_fft(x.size, 1 if inverse else 0, P(inter), P(out))
    return out[0::2] + 1j * out[1::2]
