"""Host-side interface of the GPU path, named after the reference routines it replaces.

``Mimica`` owns one device context (``mg_create``): the fields of one domain stay
resident on the GPU across both integrator stages of every step; host arrays in
the reference's layout cross the boundary only in ``upload``/``download`` and in
the unit-level entry points used by the parity tests.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .config import Domain, State


class Mimica:
    def __init__(self, domain: Domain, nscal: int, iqt: int = -1, device: int = 0):
        self.domain = domain
        self.nscal = nscal
        self.iqt = iqt
        self.device = device
        L = _lib.lib()
        params, self._keep = domain.params(nscal, iqt)
        h = C.c_void_p()
        _lib.check(L.mg_create(C.byref(params), device, C.byref(h)), "mg_create")
        self._h = h
        self._L = L
        self.dt0 = domain.dt0          # current time step (checkall / set_dt may change it)
        self._sgs_on = False
        if domain.sgs is not None:
            self.set_sgs(domain.sgs)

    # ---- lifetime ----
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._L.mg_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def device_bytes(self) -> int:
        return int(self._L.mg_device_bytes(self._h))

    @property
    def launches_per_call(self) -> int:
        return int(self._L.mg_last_launch_count(self._h))

    # ---- per-step checks and time-step control (check.f90) ----
    def checkall(self, checks=None, apply: bool = True) -> dict:
        """checkall on the resident state: max CFL (with location), es/qt bounds, and the
        reference's advective time-step rule; with apply, a new dt0 is used from the next
        step on."""
        from .config import Checks
        ch = checks if checks is not None else Checks()
        p = ch.params(self.domain.dt0, apply)
        r = _lib.MgCheckResult()
        rc = self._L.mg_checkall(self._h, C.byref(p), C.byref(r))
        if rc == _lib.MG_ERR_NAN:
            err = _lib.MimicaError(rc, f"mg_checkall: non-finite value at (i, j, k) = {tuple(r.nonfinite_ijk)}")
            err.ijk = tuple(r.nonfinite_ijk)
            raise err
        _lib.check(rc, "mg_checkall")
        if apply and r.stop == _lib.MG_STOP_NONE:
            self.dt0 = r.dt0_new
        out = {f: getattr(r, f) for f, _ in r._fields_}
        for f, _ in r._fields_:
            if f.endswith("_ijk"):
                out[f] = tuple(out[f])
        return out

    # ---- the projection's plan and its autotuner ----
    def tune_get(self) -> dict:
        from . import tune
        t = _lib.MgTune()
        _lib.check(self._L.mg_tune_get(self._h, C.byref(t)), "mg_tune_get")
        return tune.to_dict(t)

    def tune_set(self, plan: dict) -> None:
        from . import tune
        t = tune.from_dict(plan)
        _lib.check(self._L.mg_tune_set(self._h, C.byref(t)), "mg_tune_set")

    def autotune(self, reps: int = 5, wisdom: str | None = None) -> dict:
        """Pick the projection's plan for this grid: from the wisdom file when it holds one
        for this grid and precision, else by timing candidates (mg_autotune), which is
        then stored there.  Returns the plan, with the timings when it was measured."""
        from . import tune
        d = self.domain
        k = tune.key(d.maxx, d.maxy, d.nz, d.precision, self.nscal)
        known = tune.load(wisdom).get(k) if wisdom else None
        if known is not None:
            self.tune_set(known)
            return dict(known, source="wisdom")
        t = _lib.MgTune()
        _lib.check(self._L.mg_autotune(self._h, int(reps), C.byref(t)), "mg_autotune")
        plan = tune.to_dict(t)
        if wisdom:
            tune.store(wisdom, k, plan)
        return dict(plan, source="measured", candidates=t.candidates, ms_default=t.ms_default, ms_tuned=t.ms_tuned,
                    k1_ms_default=t.k1_ms_default, k1_ms_tuned=t.k1_ms_tuned, k2_ms_default=t.k2_ms_default,
                    k2_ms_tuned=t.k2_ms_tuned)

    def set_dt(self, dt0: float) -> None:
        _lib.check(self._L.mg_set_dt(self._h, float(dt0)), "mg_set_dt")
        self.dt0 = float(dt0)

    # ---- restart files (restarting.f90 savedata / readdata) ----
    def ksgs(self) -> np.ndarray:
        """turbu%ksgs of the last step's level n (SGS diffusion on)."""
        out = np.zeros(self.domain.shape)
        _lib.check(self._L.mg_download_ksgs(self._h, _lib.ptr(out)), "mg_download_ksgs")
        return out

    def save_restart(self, path: str, time: float = 0.0, ntime: int = 0, ntau: int = 1, profiles: dict | None = None,
                     xn_ccn0: float = 0.0, xn_in0: float = 0.0) -> None:
        """Write the resident state as the reference's savedata does ('V04').  Profiles
        not given are taken from the domain (p0, den0, avden0, stab0, pt0, qv0) or zero."""
        from . import restart
        d = self.domain
        st = self.download()
        qt = st.scal[st.iqt] if st.iqt >= 0 else np.zeros(d.shape)
        passive = [a for q, a in enumerate(st.scal) if q != 0 and q != st.iqt]
        prof = {"p0": d.p0, "den0": d.den0, "avden0": d.avden0, "stab0": d.stab0, "pt0": d.pt0, "qv0": d.qv0}
        prof.update(profiles or {})
        hdr = {"time": float(time), "ntime": int(ntime), "dt": float(self.dt0), "ntau": int(ntau), "nx": d.nx,
               "ny": d.ny, "nz": d.nz, "dx": d.dx, "dy": d.dy, "dz": d.dz, "nscal": len(passive), "nparc": 0,
               "xn_ccn0": float(xn_ccn0), "xn_in0": float(xn_in0)}
        r = restart.Restart(hdr, prof, {"u": st.u, "v": st.v, "w": st.w, "p": st.p, "es": st.scal[0], "qt": qt,
                                        "dens": st.dens}, passive, ksgs=self.ksgs() if self._sgs_on else None)
        restart.write(path, r)

    def load_restart(self, path: str) -> dict:
        """Read a restart file of this domain, upload its state and take its time step;
        returns the header (time, ntime, ...)."""
        from . import restart
        from .config import State
        d = self.domain
        r = restart.read(path, with_dif=self._sgs_on)
        h = r.header
        if (h["nx"], h["ny"], h["nz"]) != (d.nx, d.ny, d.nz):
            raise ValueError("restart file of another grid (the reference interpolates; not supported here)")
        npass = self.nscal - 1 - (1 if self.iqt >= 0 else 0)
        if h["nscal"] != npass:
            raise ValueError(f"restart file holds {h['nscal']} passive scalars, the context {npass}")
        scal = [r.fields["es"]]
        it = iter(r.scal)
        for q in range(1, self.nscal):
            scal.append(r.fields["qt"] if q == self.iqt else next(it))
        self.upload(State(r.fields["u"], r.fields["v"], r.fields["w"], r.fields["p"], r.fields["dens"], scal, self.iqt))
        if h["dt"] != self.dt0:
            self.set_dt(h["dt"])
        return h

    # ---- SGS turbulence diffusion (subgrid.f90) ----
    def set_sgs(self, sgs, with_dif: bool = True) -> None:
        """Switch SGS diffusion on (or off) for the following steps; uploads the surface
        fluxes of ``sgs`` (``None`` = zero)."""
        p, keep = sgs.params(self.domain.nz, with_dif)
        _lib.check(self._L.mg_set_sgs(self._h, C.byref(p)), "mg_set_sgs")
        self._sgs_on = bool(with_dif)
        self.set_surface_fluxes(sgs.esflux, sgs.qvflux, sgs.mflux)

    def set_surface_fluxes(self, esflux=None, qvflux=None, mflux=None) -> None:
        d = self.domain
        arrs = [None if a is None else np.ascontiguousarray(a, dtype=np.float64) for a in (esflux, qvflux, mflux)]
        for a in arrs:
            if a is not None and a.shape != (d.ny, d.nx):
                raise ValueError(f"surface flux arrays are (ny, nx) = {(d.ny, d.nx)}")
        _lib.check(self._L.mg_set_surface_fluxes(self._h, *[_lib.ptr(a) for a in arrs]), "mg_set_surface_fluxes")

    def calc_subgrid(self, u, v, w, es, qt=None) -> np.ndarray:
        fkv = np.zeros(self.domain.shape)
        c = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None for a in (u, v, w, es, qt)]
        _lib.check(self._L.mg_calc_subgrid(self._h, *[_lib.ptr(a) for a in c], _lib.ptr(fkv)), "mg_calc_subgrid")
        return fkv

    def efud(self, u, v, w, dens, fkv, su=None, sv=None, sw=None):
        d = self.domain
        outs = [np.zeros(d.shape) if a is None else np.array(a, dtype=np.float64, copy=True) for a in (su, sv, sw)]
        c = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, v, w, dens, fkv)]
        _lib.check(self._L.mg_efud(self._h, *[_lib.ptr(a) for a in c], *[_lib.ptr(a) for a in outs]), "mg_efud")
        return tuple(outs)

    def eff(self, kind: int, dens, fkv, x, flux_s=None, ec=None) -> np.ndarray:
        out = np.zeros(self.domain.shape) if ec is None else np.array(ec, dtype=np.float64, copy=True)
        c = [np.ascontiguousarray(a, dtype=np.float64) for a in (dens, fkv, x)]
        fs = None if flux_s is None else np.ascontiguousarray(flux_s, dtype=np.float64)
        _lib.check(self._L.mg_eff(self._h, kind, *[_lib.ptr(a) for a in c], _lib.ptr(fs), _lib.ptr(out)), "mg_eff")
        return out

    # ---- resident state ----
    def upload(self, st: State) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in st.scal]
        sp = (_lib._dp * len(arrs))(*[_lib.ptr(a) for a in arrs])
        _lib.check(self._L.mg_upload_state(self._h, _lib.ptr(st.u), _lib.ptr(st.v), _lib.ptr(st.w), _lib.ptr(st.p),
                                           _lib.ptr(st.dens), sp), "mg_upload_state")

    def download(self, out: State | None = None) -> State:
        """The resident state in natural variables.  out: arrays to fill (C-contiguous
        float64 of the domain's shape, e.g. page-locked buffers reused across steps)."""
        d = self.domain
        if out is None:
            u, v, w, p, dens = (np.zeros(d.shape) for _ in range(5))
            scal = [np.zeros(d.shape) for _ in range(self.nscal)]
        else:
            u, v, w, p, dens, scal = out.u, out.v, out.w, out.p, out.dens, list(out.scal)
            if len(scal) != self.nscal:
                raise ValueError(f"out has {len(scal)} scalars, the context {self.nscal}")
            for a in (u, v, w, p, dens, *scal):
                if a.shape != d.shape or a.dtype != np.float64 or not a.flags.c_contiguous or not a.flags.writeable:
                    raise ValueError("out arrays must be writeable C-contiguous float64 of the domain's shape")
        sp = (_lib._dp * len(scal))(*[_lib.ptr(a) for a in scal])
        _lib.check(self._L.mg_download_state(self._h, _lib.ptr(u), _lib.ptr(v), _lib.ptr(w), _lib.ptr(p),
                                             _lib.ptr(dens), sp), "mg_download_state")
        if out is not None:
            return out
        return State(u, v, w, p, dens, scal, self.iqt)

    def upload_field(self, field: int, a: np.ndarray) -> None:
        """One field of the level-n state (``_lib.MG_FIELD_*``; ``MG_FIELD_SCAL + s`` for
        scalar s), natural values of the domain's shape."""
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != self.domain.shape:
            raise ValueError("field shape differs from the domain's")
        _lib.check(self._L.mg_upload_field(self._h, int(field), _lib.ptr(a)), "mg_upload_field")

    def download_field(self, field: int, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.zeros(self.domain.shape)
        elif out.shape != self.domain.shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be C-contiguous float64 of the domain's shape")
        _lib.check(self._L.mg_download_field(self._h, int(field), _lib.ptr(out)), "mg_download_field")
        return out

    def upload_device(self, ptrs: dict) -> None:
        """Upload from device pointers (ints), same layout as the host path."""
        sp = (C.c_void_p * self.nscal)(*ptrs["scal"])
        _lib.check(self._L.mg_upload_state_device(self._h, ptrs["u"], ptrs["v"], ptrs["w"], ptrs["p"], ptrs["dens"],
                                                  sp), "mg_upload_state_device")

    def download_device(self, ptrs: dict) -> None:
        sp = (C.c_void_p * self.nscal)(*ptrs["scal"])
        _lib.check(self._L.mg_download_state_device(self._h, ptrs["u"], ptrs["v"], ptrs["w"], ptrs["p"],
                                                    ptrs["dens"], sp), "mg_download_state_device")

    # ---- stepping (src/INTEG/time_step.f90:76) ----
    def stepping(self, nsteps: int = 1, ntime0: int = 1, diagnostics: bool = False, graph: bool = False):
        md = C.c_double(0.0)
        p1 = np.zeros(self.domain.nz) if diagnostics else None
        fn = self._L.mg_step_graph if graph else self._L.mg_step
        _lib.check(fn(self._h, nsteps, ntime0, C.byref(md) if diagnostics else None, _lib.ptr(p1)), "mg_step")
        if diagnostics:
            return md.value, p1
        return None

    def synchronize(self) -> None:
        _lib.check(self._L.mg_synchronize(self._h), "mg_synchronize")

    # ---- unit-level entry points ----
    def advection_ac(self, x, mu, mv, mw, xs) -> np.ndarray:
        """src/TOOLS/advection.f90:801 advection_ac; returns the updated xs."""
        xs = np.array(xs, dtype=np.float64, copy=True)
        _lib.check(self._L.mg_advection_ac(self._h, _lib.ptr(np.ascontiguousarray(x)), _lib.ptr(mu), _lib.ptr(mv),
                                           _lib.ptr(mw), _lib.ptr(xs)), "mg_advection_ac")
        return xs

    def advection_tl(self, x, mu, mv, mw, dx, dmu, dmv, dmw) -> np.ndarray:
        """Tangent linear of the advective tendency A(x, m) = -(Tx+Ty+Tz) (WENO)."""
        out = np.zeros(self.domain.shape)
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, mu, mv, mw, dx, dmu, dmv, dmw)]
        _lib.check(self._L.mg_advection_tl(self._h, *[_lib.ptr(a) for a in args], _lib.ptr(out)), "mg_advection_tl")
        return out

    def advection_ad(self, x, mu, mv, mw, abar):
        """Adjoint of the advective tendency: returns (xbar, mubar, mvbar, mwbar)."""
        outs = [np.zeros(self.domain.shape) for _ in range(4)]
        args = [np.ascontiguousarray(a, dtype=np.float64) for a in (x, mu, mv, mw, abar)]
        _lib.check(self._L.mg_advection_ad(self._h, *[_lib.ptr(a) for a in args], *[_lib.ptr(o) for o in outs]),
                   "mg_advection_ad")
        return tuple(outs)

    def qnadv_tl(self, mu, mv, mw, dmu, dmv, dmw, ntime: int = 1, values: bool = False):
        """Tangent linear of qnadv_uvw at (mu, mv, mw) along (dmu, dmv, dmw); with values,
        also the operator itself (the per-cell form the adjoint differentiates)."""
        d = self.domain
        c = [np.ascontiguousarray(a, dtype=np.float64) for a in (mu, mv, mw, dmu, dmv, dmw)]
        outs = [np.zeros(d.shape) for _ in range(6)]
        vals = outs[:3] if values else [None] * 3
        _lib.check(self._L.mg_qnadv_tl(self._h, ntime, *[_lib.ptr(a) for a in c], *[_lib.ptr(a) for a in vals],
                                       *[_lib.ptr(a) for a in outs[3:]]), "mg_qnadv_tl")
        return (tuple(outs[:3]), tuple(outs[3:])) if values else tuple(outs[3:])

    def qnadv_ad(self, mu, mv, mw, aub, avb, awb, ntime: int = 1):
        d = self.domain
        c = [np.ascontiguousarray(a, dtype=np.float64) for a in (mu, mv, mw, aub, avb, awb)]
        outs = [np.zeros(d.shape) for _ in range(3)]
        _lib.check(self._L.mg_qnadv_ad(self._h, ntime, *[_lib.ptr(a) for a in c], *[_lib.ptr(a) for a in outs]),
                   "mg_qnadv_ad")
        return tuple(outs)

    # ---- trajectory tangent linear and adjoint (FP64, WENO, SGS off) ----
    def _fields(self, st) -> list:
        return [np.ascontiguousarray(a, dtype=np.float64) for a in (st.u, st.v, st.w, st.p, st.dens, *st.scal)]

    def _parr(self, arrs):
        return (_lib._dp * len(arrs))(*[_lib.ptr(a) for a in arrs])

    def _state_of(self, arrs):
        from .config import State
        return State(arrs[0], arrs[1], arrs[2], arrs[3], arrs[4], list(arrs[5:]), self.iqt)

    def traj_forward(self, nsteps: int, ntime0: int = 1) -> None:
        """Advance the resident state through the composition the trajectory adjoint
        linearises (unit-mode K1/K2, stage kernels, projection)."""
        _lib.check(self._L.mg_traj_forward(self._h, nsteps, ntime0), "mg_traj_forward")

    def traj_tl(self, dx0, nsteps: int, ntime0: int = 1):
        """Tangent linear of nsteps steps from the resident state along dx0 (a State)."""
        din = self._fields(dx0)
        out = [np.zeros(self.domain.shape) for _ in din]
        _lib.check(self._L.mg_traj_tl(self._h, nsteps, ntime0, self._parr(din), self._parr(out)), "mg_traj_tl")
        return self._state_of(out)

    def traj_adjoint(self, lam, nsteps: int, ntime0: int = 1, ckpt: int = 4):
        """Adjoint of nsteps steps from the resident state: the gradient, with respect to
        the initial state, of J = sum over the interior of lam . x(final)."""
        lin = self._fields(lam)
        out = [np.zeros(self.domain.shape) for _ in lin]
        _lib.check(self._L.mg_traj_adjoint(self._h, nsteps, ntime0, ckpt, self._parr(lin), self._parr(out)),
                   "mg_traj_adjoint")
        return self._state_of(out)

    def traj_record_limit(self, nbytes: float) -> None:
        """Cap the device bytes the trajectory adjoint may keep as stage records (< 0: half
        the free memory; 0: recompute every backward step's stages)."""
        _lib.check(self._L.mg_traj_record_limit(self._h, float(nbytes)), "mg_traj_record_limit")

    def traj_checkpoints(self, where: int) -> None:
        """Where the trajectory adjoint keeps its checkpoints: _lib.MG_CKPT_DEVICE,
        MG_CKPT_HOST (page-locked host memory) or MG_CKPT_AUTO (the default)."""
        _lib.check(self._L.mg_traj_checkpoints(self._h, int(where)), "mg_traj_checkpoints")

    def time_traj(self, nsteps: int, ckpt: int, ntime0: int = 1) -> dict:
        """Device times of nsteps of the trajectory composition, its tangent linear and its
        checkpointed adjoint from the resident state (left unchanged)."""
        out = np.zeros(4)
        _lib.check(self._L.mg_time_traj(self._h, nsteps, ntime0, ckpt, _lib.ptr(out)), "mg_time_traj")
        return {"forward_ms": out[0], "tl_ms": out[1], "adjoint_ms": out[2], "adjoint_device_bytes": int(out[3])}

    def anelastic_pressure_ad(self, mub, mvb, mwb, pb):
        """Adjoint of anelastic_pressure (the momentum/pressure map): returns (mub, mvb, mwb, pb)."""
        io = [np.array(a, dtype=np.float64, copy=True) for a in (mub, mvb, mwb, pb)]
        _lib.check(self._L.mg_anelastic_pressure_ad(self._h, *[_lib.ptr(a) for a in io]), "mg_anelastic_pressure_ad")
        return tuple(io)

    def qnadv_uvw(self, mu, mv, mw, ntime: int = 1):
        """src/INTEG/windadv.f90:46 qnadv_uvw; returns (au, av, aw)."""
        d = self.domain
        au, av, aw = (np.zeros(d.shape) for _ in range(3))
        _lib.check(self._L.mg_qnadv_uvw(self._h, ntime, _lib.ptr(mu), _lib.ptr(mv), _lib.ptr(mw), _lib.ptr(au),
                                        _lib.ptr(av), _lib.ptr(aw)), "mg_qnadv_uvw")
        return au, av, aw

    def fft_solve(self, tend, out=None) -> np.ndarray:
        """src/PRESSURE/pressure_solver.f90:462 fft_solve (unnormalised solution)."""
        out = np.zeros(self.domain.shape) if out is None else np.array(out, dtype=np.float64, copy=True)
        _lib.check(self._L.mg_fft_solve(self._h, _lib.ptr(np.ascontiguousarray(tend)), _lib.ptr(out)), "mg_fft_solve")
        return out

    def prognostic_pressure(self, inp, st, reps: int = 0, warmup: int = 0):
        """src/INTEG/prognostic_pressure.f90:64 (the compressible model's acoustic
        sub-steps) on copies of an acoustic.AcousticState with acoustic.AcousticInput;
        returns the updated copy.  reps >= 1: after the call, `warmup` untimed and `reps`
        timed calls run on the uploaded fields (mg_time_prognostic_pressure), and
        (state, device ms per call) is returned."""
        st = st.copy()
        c = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        keep = [c(x) for x in (inp.p0, inp.su, inp.sv, inp.sw, inp.sdens, inp.ses, inp.sqt, inp.uadv, inp.vadv,
                               inp.wadv)]
        sscal = [c(x) for x in inp.sscal]
        a = _lib.MgAcoustic()
        a.im, a.ntau, a.cst_cp, a.nscal = inp.im, inp.ntau, inp.cst_cp, len(st.scal)
        (a.p0, a.su, a.sv, a.sw, a.sdens, a.ses, a.sqt, a.uadv, a.vadv, a.wadv) = [_lib.ptr(x) for x in keep]
        for f in st.FIELDS:
            setattr(st, f, c(getattr(st, f)))
            setattr(a, f, _lib.ptr(getattr(st, f)))
        st.scal = [c(x) for x in st.scal]
        st.tscal = [c(x) for x in st.tscal]
        arr = lambda xs: (C.POINTER(C.c_double) * max(1, len(xs)))(*[_lib.ptr(x) for x in xs])  # noqa: E731
        ps, pc, pt = arr(sscal), arr(st.scal), arr(st.tscal)
        a.sscal = C.cast(ps, C.POINTER(C.POINTER(C.c_double)))
        a.scal = C.cast(pc, C.POINTER(C.POINTER(C.c_double)))
        a.tscal = C.cast(pt, C.POINTER(C.POINTER(C.c_double)))
        if reps >= 1:
            ms = C.c_double(0.0)
            _lib.check(self._L.mg_time_prognostic_pressure(self._h, C.byref(a), warmup, reps, C.byref(ms)),
                       "mg_time_prognostic_pressure")
            return st, ms.value
        _lib.check(self._L.mg_prognostic_pressure(self._h, C.byref(a)), "mg_prognostic_pressure")
        return st

    def anelastic_pressure(self, mu, mv, mw, p, wold):
        """src/PRESSURE/pressure_solver.f90:73 anelastic_pressure; returns (mu, mv, mw, p, maxdiv, p1)."""
        mu, mv, mw, p = (np.array(a, dtype=np.float64, copy=True) for a in (mu, mv, mw, p))
        md = C.c_double(0.0)
        p1 = np.zeros(self.domain.nz)
        _lib.check(self._L.mg_anelastic_pressure(self._h, _lib.ptr(mu), _lib.ptr(mv), _lib.ptr(mw), _lib.ptr(p),
                                                 _lib.ptr(np.ascontiguousarray(wold)), C.byref(md), _lib.ptr(p1)),
                   "mg_anelastic_pressure")
        return mu, mv, mw, p, md.value, p1
