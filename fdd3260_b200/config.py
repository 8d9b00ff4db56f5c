"""Domains, base states and seeded initial fields of the benchmark configurations.

Fields use the reference's array layout: ``x(1:nx,1:ny,1:nz)`` in Fortran order,
i.e. numpy arrays of shape ``(nz, ny, nx)`` (C order, x fastest) with
``nx = MAXX+5``, ``ny = MAXY+5`` (three ghost cells low, two high).

The grid metrics and the base state are computed by the library's restatement of
the reference's init routines (src/TOOLS/define_grid.f90:179-187,
src/IO/initial.f90:473-558); no public dataset is involved: every field is drawn
from ``numpy.random.Generator(PCG64(seed))`` with the shapes, sizes and value
ranges the benchmark configurations state.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib


@dataclass
class Sgs:
    """SGS turbulence switches (the reference's with_dif, diff, pran, zdec, anis_k, momsf,
    zrough, min_w; src/TYPES/shared_data.f90, defaults of INCLUDE/default.h) and the
    surface fluxes surf%esflux, surf%qvflux, surf%mflux ((ny, nx) arrays or None)."""
    diff: float = 0.0
    pran: float = 0.4
    zdec: float = 2000.0
    anis_k: bool = False
    momsf: int = 0
    zrough: float = 0.01
    min_w: float = 0.1
    qt0: np.ndarray | None = None
    esflux: np.ndarray | None = None
    qvflux: np.ndarray | None = None
    mflux: np.ndarray | None = None

    def params(self, nz: int, with_dif: bool = True) -> tuple[_lib.MgSgsParams, list]:
        keep = []
        p = _lib.MgSgsParams()
        p.with_dif, p.anis_k, p.momsf, p.reserved = int(with_dif), int(self.anis_k), int(self.momsf), 0
        p.diff, p.pran, p.zdec, p.zrough, p.min_w = self.diff, self.pran, self.zdec, self.zrough, self.min_w
        if self.qt0 is not None:
            q = np.ascontiguousarray(self.qt0, dtype=np.float64)
            assert q.shape == (nz,)
            keep.append(q)
            p.qt0 = _lib.ptr(q)
        return p, keep


@dataclass
class Checks:
    """Switches of checkall (src/IO/check.f90) and the time-step control (namelist cm_num /
    cm_run: cfl_max, cfl_min, limit_ts, ldtfix; checkx bounds of es and qt)."""
    cfl_max: float = 0.5
    cfl_min: float = 0.4
    limit_ts: float = 20.0
    ldtfix: int = 0
    es_min: float = 200.0
    es_max: float = 4000.0
    qt_min: float = 1e-15
    qt_max: float = 1.0

    def params(self, dt0_i: float, apply: bool = True) -> _lib.MgCheckParams:
        p = _lib.MgCheckParams()
        p.cfl_max, p.cfl_min, p.dt0_i, p.limit_ts = self.cfl_max, self.cfl_min, dt0_i, self.limit_ts
        p.es_min, p.es_max, p.qt_min, p.qt_max = self.es_min, self.es_max, self.qt_min, self.qt_max
        p.ldtfix, p.apply = int(self.ldtfix), int(apply)
        return p


@dataclass
class Domain:
    maxx: int
    maxy: int
    nz: int
    dx: float
    dy: float
    dz: float
    dt0: float
    fdz0: np.ndarray
    pt0: np.ndarray
    qv0: np.ndarray
    psurf: float = 101600.0
    scal_adv: str = "weno"
    muscl_limiter: str = "minmod"
    mom_ord: int = 4
    lavisc: int = 1
    nsubp: int = 1
    with_buoy: int = 1
    lim_tol: float = 1e-9
    u0shift: float = 0.0
    v0shift: float = 0.0
    precision: int = _lib.MG_PREC_FP64
    refine_iters: int = 1
    refine_tol: float = 1e-13
    sgs: Sgs | None = None        # SGS turbulence diffusion (with_dif) when set
    # derived (filled by finish())
    dzw: np.ndarray = field(default=None, repr=False)
    dz1w: np.ndarray = field(default=None, repr=False)
    dz1: np.ndarray = field(default=None, repr=False)
    p0: np.ndarray = field(default=None, repr=False)
    den0: np.ndarray = field(default=None, repr=False)
    avden0: np.ndarray = field(default=None, repr=False)
    stab0: np.ndarray = field(default=None, repr=False)

    @property
    def nx(self) -> int:
        return self.maxx + 5

    @property
    def ny(self) -> int:
        return self.maxy + 5

    @property
    def shape(self) -> tuple[int, int, int]:
        return (self.nz, self.ny, self.nx)

    @property
    def cells(self) -> int:
        return self.maxx * self.maxy * self.nz

    def finish(self, init=None) -> "Domain":
        """Fill the grid metrics and the base state.

        ``init`` is None for the library's own init routines (mg_grid_metrics,
        mg_base_state), or an object with ``grid_metrics(nz, dz, fdz0, dzw, dz1w, dz1)``
        and ``base_state(nz, dz, psurf, fdz0, dz1, pt0, qv0, p0, den0, avden0, stab0)``
        methods taking numpy arrays, for a caller that must not load the CUDA library
        (a CPU-only timing of another implementation)."""
        nz = self.nz
        self.fdz0 = np.ascontiguousarray(self.fdz0, dtype=np.float64)
        self.pt0 = np.ascontiguousarray(self.pt0, dtype=np.float64)
        self.qv0 = np.ascontiguousarray(self.qv0, dtype=np.float64)
        self.dzw, self.dz1w, self.dz1 = (np.zeros(nz) for _ in range(3))
        self.p0, self.den0, self.avden0, self.stab0 = (np.zeros(nz) for _ in range(4))
        if init is not None:
            init.grid_metrics(nz, self.dz, self.fdz0, self.dzw, self.dz1w, self.dz1)
            init.base_state(nz, self.dz, self.psurf, self.fdz0, self.dz1, self.pt0, self.qv0, self.p0, self.den0,
                            self.avden0, self.stab0)
            return self
        L = _lib.lib()
        _lib.check(L.mg_grid_metrics(nz, self.dz, _lib.ptr(self.fdz0), _lib.ptr(self.dzw), _lib.ptr(self.dz1w),
                                     _lib.ptr(self.dz1)), "mg_grid_metrics")
        _lib.check(L.mg_base_state(nz, self.dz, self.psurf, _lib.ptr(self.fdz0), _lib.ptr(self.dz1),
                                   _lib.ptr(self.pt0), _lib.ptr(self.qv0), _lib.ptr(self.p0), _lib.ptr(self.den0),
                                   _lib.ptr(self.avden0), _lib.ptr(self.stab0)), "mg_base_state")
        return self

    def wv(self) -> np.ndarray:
        out = np.zeros((self.maxy, self.maxx))
        _lib.check(_lib.lib().mg_get_wv(self.maxx, self.maxy, self.dx, self.dy, _lib.ptr(out)), "mg_get_wv")
        return out

    def zc(self) -> np.ndarray:
        """cell-centre heights (define_grid.f90:132-136)"""
        z = np.zeros(self.nz)
        z[0] = 0.5 * self.dz * self.fdz0[0]
        for k in range(1, self.nz):
            z[k] = z[k - 1] + 0.5 * self.dz * (self.fdz0[k - 1] + self.fdz0[k])
        return z

    def params(self, nscal: int, iqt: int) -> tuple[_lib.MgParams, list]:
        keep = []

        def dp(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return _lib.ptr(a)

        p = _lib.MgParams()
        p.maxx, p.maxy, p.nz = self.maxx, self.maxy, self.nz
        p.nscal, p.iqt = nscal, iqt
        p.scal_adv = _lib.SCHEMES[self.scal_adv]
        p.muscl_limiter = _lib.LIMITERS[self.muscl_limiter]
        p.mom_ord, p.lavisc, p.nsubp, p.with_buoy = self.mom_ord, self.lavisc, self.nsubp, self.with_buoy
        p.precision, p.refine_iters = self.precision, self.refine_iters
        p.dx, p.dy, p.dz, p.dt0 = self.dx, self.dy, self.dz, self.dt0
        p.lim_tol, p.u0shift, p.v0shift, p.refine_tol = self.lim_tol, self.u0shift, self.v0shift, self.refine_tol
        p.fdz0, p.dzw, p.dz1w, p.dz1 = dp(self.fdz0), dp(self.dzw), dp(self.dz1w), dp(self.dz1)
        p.den0, p.avden0, p.stab0 = dp(self.den0), dp(self.avden0), dp(self.stab0)
        p.pt0, p.qv0 = dp(self.pt0), dp(self.qv0)
        return p, keep


@dataclass
class State:
    """Natural variables at time level n (the reference's wind2/pressure2/state2)."""
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    p: np.ndarray
    dens: np.ndarray
    scal: list          # es (potential temperature) first, then qt (if iqt >= 0), passive scalars
    iqt: int = -1

    def copy(self) -> "State":
        return State(self.u.copy(), self.v.copy(), self.w.copy(), self.p.copy(), self.dens.copy(),
                     [s.copy() for s in self.scal], self.iqt)


def periodic_fill(x: np.ndarray) -> np.ndarray:
    """Ghost cells := periodic images (src/TOOLS/bc.f90 qnbc_p4, serial branch)."""
    nz, ny, nx = x.shape
    mx, my = nx - 5, ny - 5
    x[:, :, 0:3] = x[:, :, mx:mx + 3]
    x[:, :, nx - 2:nx] = x[:, :, 3:5]
    x[:, 0:3, :] = x[:, my:my + 3, :]
    x[:, ny - 2:ny, :] = x[:, 3:5, :]
    return x


def _interior_xy(d: Domain):
    xc = (np.arange(d.maxx) + 0.5) * d.dx
    yc = (np.arange(d.maxy) + 0.5) * d.dy
    return xc, yc


def _new(d: Domain) -> np.ndarray:
    return np.zeros(d.shape)


def warm_bubble_domain(maxx=64, maxy=64, nz=64, dx=50.0, dy=50.0, dz=50.0, dt0=0.5, scheme="weno", init=None,
                       **kw) -> Domain:
    """Dry warm bubble: doubly periodic box, rigid lid, theta0 = 300 K.  ``init``: see Domain.finish."""
    d = Domain(maxx=maxx, maxy=maxy, nz=nz, dx=dx, dy=dy, dz=dz, dt0=dt0, fdz0=np.ones(nz),
               pt0=np.full(nz, 300.0), qv0=np.zeros(nz), scal_adv=scheme, **kw)
    return d.finish(init)


def warm_bubble_state(d: Domain, seed: int = 0, amp: float = 2.0, radius: float = 500.0,
                      centre=(1600.0, 1600.0, 500.0), nscal_passive: int = 1) -> State:
    """theta' = amp*cos^2(pi r/2R) (r < R) + U(+-0.01) K; u,v,w ~ U(+-0.1) m/s; w(1) = 0;
    passive scalars U[0,1]; dens = rho0(z); p = 0."""
    rng = np.random.Generator(np.random.PCG64(seed))
    xc, yc = _interior_xy(d)
    zc = d.zc()
    Z, Y, X = np.meshgrid(zc, yc, xc, indexing="ij")
    r = np.sqrt((X - centre[0]) ** 2 + (Y - centre[1]) ** 2 + (Z - centre[2]) ** 2)
    thp = np.where(r < radius, amp * np.cos(np.pi * r / (2 * radius)) ** 2, 0.0)
    thp = thp + rng.uniform(-0.01, 0.01, thp.shape)
    th = _new(d)
    th[:, 3:3 + d.maxy, 3:3 + d.maxx] = d.pt0[:, None, None] + thp
    u, v, w = _new(d), _new(d), _new(d)
    for a in (u, v, w):
        a[:, 3:3 + d.maxy, 3:3 + d.maxx] = rng.uniform(-0.1, 0.1, (d.nz, d.maxy, d.maxx))
    w[0] = 0.0
    scal = [th]
    for _ in range(nscal_passive):
        s = _new(d)
        s[:, 3:3 + d.maxy, 3:3 + d.maxx] = rng.uniform(0.0, 1.0, (d.nz, d.maxy, d.maxx))
        scal.append(s)
    dens = np.broadcast_to(d.den0[:, None, None], d.shape).copy()
    st = State(u, v, w, _new(d), dens, scal, iqt=-1)
    for a in [st.u, st.v, st.w, st.p, st.dens, *st.scal]:
        periodic_fill(a)
    return st


def tanh_levels(nz: int, dz_bottom: float, dz_top: float, width: float = 0.18) -> np.ndarray:
    """cell thickness profile: tanh transition from dz_bottom at the surface to dz_top aloft"""
    s = (np.arange(nz) + 0.5) / nz
    return dz_bottom + (dz_top - dz_bottom) * 0.5 * (1.0 + np.tanh((s - 0.5) / width))


def cumulus_domain(maxx=512, maxy=512, nz=256, dx=25.0, dy=25.0, dt0=1.0, scheme="weno", init=None, **kw) -> Domain:
    """Shallow-cumulus-like domain: stretched grid, 10 m at the surface to 100 m at the top.
    Thicknesses enter through fdz = thickness/dz as the grid-file path
    (src/TOOLS/define_grid.f90:143-172) would produce them.  ``init``: see Domain.finish."""
    dz = 10.0
    thick = tanh_levels(nz, 10.0, 100.0)
    fdz = thick / dz
    zc = np.cumsum(thick) - 0.5 * thick
    zt = zc[-1]
    pt0 = 298.0 + (310.0 - 298.0) * zc / zt
    qt = np.interp(zc, [0.0, 500.0, 1500.0, zt], [17e-3, 16e-3, 8e-3, 4e-3])
    d = Domain(maxx=maxx, maxy=maxy, nz=nz, dx=dx, dy=dy, dz=dz, dt0=dt0, fdz0=fdz, pt0=pt0, qv0=qt,
               scal_adv=scheme, **kw)
    return d.finish(init)


def cumulus_state(d: Domain, seed: int = 1000, n_extra: int = 3, lognormal_extras: bool = False) -> State:
    """theta_l, qt from the base profiles plus N(0,0.1 K / 0.1 g/kg) below 500 m; u = -8 + N(0,0.5);
    v = N(0,0.5); w = 0.  Extra scalars (qr, nr, aerosol number): smooth positive profiles
    decreasing with height with 1 % seeded Gaussian perturbations below 500 m, or, with
    lognormal_extras, independent lognormal values (sigma_log = 1) in every cell."""
    rng = np.random.Generator(np.random.PCG64(seed))
    zc = d.zc()
    sh = (d.nz, d.maxy, d.maxx)
    low = (zc < 500.0)[:, None, None]

    def field3(vals):
        a = _new(d)
        a[:, 3:3 + d.maxy, 3:3 + d.maxx] = vals
        return periodic_fill(a)

    th = field3(d.pt0[:, None, None] + np.where(low, rng.normal(0, 0.1, sh), 0.0))
    qt = field3(np.maximum(d.qv0[:, None, None] + np.where(low, rng.normal(0, 1e-4, sh), 0.0), 1e-6))
    u = field3(-8.0 + rng.normal(0, 0.5, sh))
    v = field3(rng.normal(0, 0.5, sh))
    w = _new(d)
    scal = [th, qt]
    scales = [1e-4, 1e5, 1e8]
    prof = np.exp(-zc / 1500.0)[:, None, None]
    for e in range(n_extra):
        if lognormal_extras:
            scal.append(field3(scales[e % 3] * np.exp(rng.normal(0.0, 1.0, sh))))
        else:
            scal.append(field3(scales[e % 3] * prof * (1.0 + np.where(low, rng.normal(0, 0.01, sh), 0.0))))
    dens = np.broadcast_to(d.den0[:, None, None], d.shape).copy()
    return State(u, v, w, _new(d), dens, scal, iqt=1)


def cumulus_field(d: Domain, field: int, seed: int = 1000, lognormal_extras: bool = True) -> np.ndarray:
    """One field of a cumulus-like state, for states too large to hold on the host at once
    (fields are uploaded one at a time).  ``field`` is _lib.MG_FIELD_U .. _DENS or
    MG_FIELD_SCAL + s: s = 0 theta_l, 1 qt, 2.. extra tracers.  Each field draws from its
    own PCG64 stream (seed * 100 + field), with the distributions of cumulus_state: theta_l
    and qt from the base profiles plus N(0, 0.1 K / 0.1 g/kg) below 500 m, u = -8 + N(0, 0.5),
    v = N(0, 0.5), w = 0, p = 0, dens = rho0(z), extra tracers lognormal (sigma_log = 1)
    with magnitudes 1e-4, 1e5, 1e8 in turn, or smooth profiles when not lognormal_extras."""
    rng = np.random.Generator(np.random.PCG64(seed * 100 + field))
    sh = (d.nz, d.maxy, d.maxx)
    zc = d.zc()
    low = (zc < 500.0)[:, None, None]

    def field3(vals):
        a = _new(d)
        a[:, 3:3 + d.maxy, 3:3 + d.maxx] = vals
        return periodic_fill(a)

    if field == _lib.MG_FIELD_U:
        return field3(-8.0 + rng.normal(0, 0.5, sh))
    if field == _lib.MG_FIELD_V:
        return field3(rng.normal(0, 0.5, sh))
    if field in (_lib.MG_FIELD_W, _lib.MG_FIELD_P):
        return _new(d)
    if field == _lib.MG_FIELD_DENS:
        return np.broadcast_to(d.den0[:, None, None], d.shape).copy()
    s = field - _lib.MG_FIELD_SCAL
    if s == 0:
        return field3(d.pt0[:, None, None] + np.where(low, rng.normal(0, 0.1, sh), 0.0))
    if s == 1:
        return field3(np.maximum(d.qv0[:, None, None] + np.where(low, rng.normal(0, 1e-4, sh), 0.0), 1e-6))
    scale = (1e-4, 1e5, 1e8)[(s - 2) % 3]
    if lognormal_extras:
        return field3(scale * np.exp(rng.normal(0.0, 1.0, sh)))
    prof = np.exp(-zc / 1500.0)[:, None, None]
    return field3(scale * prof * (1.0 + np.where(low, rng.normal(0, 0.01, sh), 0.0)))


def random_state(d: Domain, seed: int = 7, nscal: int = 2) -> State:
    """Generic smooth-ish random state for unit tests (positive scalars)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sh = (d.nz, d.maxy, d.maxx)

    def field3(vals):
        a = _new(d)
        a[:, 3:3 + d.maxy, 3:3 + d.maxx] = vals
        return periodic_fill(a)

    u, v = field3(rng.normal(0, 1.0, sh)), field3(rng.normal(0, 1.0, sh))
    w = field3(rng.normal(0, 0.5, sh))
    w[0] = 0.0
    scal = [field3(300.0 + rng.normal(0, 0.5, sh))]
    for _ in range(nscal - 1):
        scal.append(field3(rng.uniform(0.0, 1.0, sh)))
    dens = np.broadcast_to(d.den0[:, None, None], d.shape).copy()
    p = field3(rng.normal(0, 1.0, sh))
    return State(u, v, w, p, dens, scal, iqt=-1)
