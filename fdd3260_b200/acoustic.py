"""The compressible model's acoustic sub-steps (``prognostic_pressure``): data and cases.

In the reference's compressible build (no ``ANELASTIC``), ``integrate_all`` replaces
the anelastic projection by ``prognostic_pressure`` (src/INTEG/prognostic_pressure.f90:64):
``ntau`` acoustic sub-steps of ``dtau = dt0 / ntau`` per integrator stage ``im``.  Each
sub-step advects density and es with the unlimited Lax-Wendroff faces
(src/TOOLS/advq_lw_nolim.f90) on the step's advective velocities, integrates every
scalar with the step's slow tendencies (integ_scal), evaluates the equation of state
for the pressure and the sound speed (src/TOOLS/thermodynamics.f90:74-294), and
integrates the momentum with the pressure gradient, the density buoyancy and a
divergence damping of ``adiv * dtau * <cs2>_k * grad(div m)`` (integ_mom).  The
integrator's tendency accumulators (integpack ``tend``) carry across the sub-steps.

The build covered is the dry ISENTROPIC CONSERVATIVE one: es is density-weighted
potential temperature, ``div_pressure`` is compiled out, there are no hydrometeors,
the time scheme is the two-stage one (sorder = 2) and the sponge is off.

``AcousticInput`` holds what the sub-steps only read, ``AcousticState`` what they
update; every 3-D array has the halo'd (nz, ny, nx) layout of ``config.State``.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import config


@dataclass
class AcousticInput:
    im: int                      # integrator stage (1: a = 1, b = 0; 2: a = 1/2, b = 1)
    ntau: int                    # acoustic sub-steps per dt0
    p0: np.ndarray               # base-state pressure (nz)
    su: np.ndarray               # winds: the step's slow momentum tendencies
    sv: np.ndarray
    sw: np.ndarray
    sdens: np.ndarray            # pressures%dens
    ses: np.ndarray              # states%es
    sqt: np.ndarray              # states%qt
    uadv: np.ndarray             # wind_adv
    vadv: np.ndarray
    wadv: np.ndarray
    sscal: list = field(default_factory=list)   # states%scal
    cst_cp: int = 1              # 1: cp_a, cv_a; 0: cp, cv of moist air from qt


@dataclass
class AcousticState:
    dens: np.ndarray             # pressure%dens
    p: np.ndarray                # pressure%p (perturbation from p0)
    u: np.ndarray                # wind: momentum
    v: np.ndarray
    w: np.ndarray
    es: np.ndarray               # state%es, density-weighted
    qt: np.ndarray               # state%qt, density-weighted
    tu: np.ndarray               # integpack tend accumulators
    tv: np.ndarray
    tw: np.ndarray
    tdens: np.ndarray
    tes: np.ndarray
    tqt: np.ndarray
    cs2: np.ndarray              # thermo_prop%cs2 (written)
    scal: list = field(default_factory=list)
    tscal: list = field(default_factory=list)

    FIELDS = ("dens", "p", "u", "v", "w", "es", "qt", "tu", "tv", "tw", "tdens", "tes", "tqt", "cs2")

    def copy(self) -> "AcousticState":
        return AcousticState(*[getattr(self, f).copy() for f in self.FIELDS], [s.copy() for s in self.scal],
                             [s.copy() for s in self.tscal])


def acoustic_case(d: config.Domain, seed: int = 5, im: int = 1, ntau: int = 8, nscal: int = 1,
                  cst_cp: int = 1) -> tuple[AcousticInput, AcousticState]:
    """Seeded synthetic inputs of a compressible state near the domain's base state:
    density rho0(z) (1 + 1e-4 N(0,1)), theta = theta0(z) + 0.05 N(0,1) K, qt = 2e-3 (1 + 0.1 N)
    kg/kg, momentum of velocities N(0, 0.5) m/s (w: N(0, 0.2), 0 at the surface), advective
    velocities (1, -0.5, 0) m/s + N(0, 0.02) (nearly non-divergent: a divergent advective
    field would compress the density steadily), slow tendencies of the size a step's
    advection gives, and, for stage 2, non-zero tendency accumulators of stage 1.
    Every array has periodic ghost cells.  The default of 8 sub-steps keeps the acoustic
    Courant number of a 0.5 s step on a 50 m grid below 1/sqrt(3)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    sh = d.shape
    nrm = lambda s=1.0: rng.standard_normal(sh) * s  # noqa: E731
    rho0 = d.den0[:, None, None]
    dens = rho0 * (1.0 + 1e-4 * nrm())
    th = d.pt0[:, None, None] + nrm(0.05)
    qt = 2e-3 * (1.0 + 0.1 * nrm())
    U, V, W = nrm(0.5), nrm(0.5), nrm(0.2)
    W[0] = 0.0

    def fill(a):
        return config.periodic_fill(np.ascontiguousarray(a, dtype=np.float64))

    scal = [fill(dens * rng.uniform(0.0, 1.0, sh)) for _ in range(nscal)]
    sw = nrm(1e-3) * rho0
    sw[0] = 0.0
    inp = AcousticInput(
        im=im, ntau=ntau, p0=np.ascontiguousarray(d.p0, dtype=np.float64),
        su=fill(nrm(1e-3) * rho0), sv=fill(nrm(1e-3) * rho0), sw=fill(sw),
        sdens=fill(nrm(1e-6)), ses=fill(nrm(1e-3) * rho0), sqt=fill(nrm(1e-8)),
        uadv=fill(1.0 + nrm(0.02)), vadv=fill(-0.5 + nrm(0.02)),
        wadv=fill(np.where(np.arange(d.nz)[:, None, None] == 0, 0.0, nrm(0.01))),
        sscal=[fill(nrm(1e-5)) for _ in range(nscal)], cst_cp=cst_cp)
    z = np.zeros(sh)
    st = AcousticState(
        dens=fill(dens), p=fill(z.copy()), u=fill(dens * U), v=fill(dens * V), w=fill(dens * W),
        es=fill(dens * th), qt=fill(dens * qt),
        tu=fill(nrm(1e-3) if im == 2 else z.copy()), tv=fill(nrm(1e-3) if im == 2 else z.copy()),
        tw=fill(nrm(1e-3) if im == 2 else z.copy()), tdens=fill(nrm(1e-6) if im == 2 else z.copy()),
        tes=fill(nrm(1e-3) if im == 2 else z.copy()), tqt=fill(nrm(1e-8) if im == 2 else z.copy()),
        cs2=z.copy(), scal=scal, tscal=[fill(nrm(1e-5) if im == 2 else z.copy()) for _ in range(nscal)])
    return inp, st
