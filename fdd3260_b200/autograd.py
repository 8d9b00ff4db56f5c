"""Forward/backward pairs shaped like an autograd Function, over the C-ABI.

``AdvectionFunction.forward(ctx, x, mu, mv, mw)`` returns the advective tendency
A(x, m) = -(Tx + Ty + Tz) of one density-weighted field (WENO, the plain FP64 form) and
saves its inputs; ``backward(ctx, abar)`` returns the vector-Jacobian products
(xbar, mubar, mvbar, mwbar).  ``jvp`` gives the tangent-linear product.  Arrays are host
float64 arrays in the reference layout with periodic ghosts filled.
"""
from __future__ import annotations

import numpy as np

from .model import Mimica


class FnContext:
    """Holds what forward saves for backward (the role of autograd's ctx)."""

    def __init__(self, model: Mimica):
        self.model = model
        self.saved: tuple = ()

    def save_for_backward(self, *arrays):
        self.saved = arrays


class AdvectionFunction:
    @staticmethod
    def forward(ctx: FnContext, x, mu, mv, mw) -> np.ndarray:
        ctx.save_for_backward(x, mu, mv, mw)
        return ctx.model.advection_ac(x, mu, mv, mw, np.zeros_like(x))

    @staticmethod
    def backward(ctx: FnContext, abar):
        x, mu, mv, mw = ctx.saved
        return ctx.model.advection_ad(x, mu, mv, mw, abar)

    @staticmethod
    def jvp(ctx: FnContext, dx, dmu, dmv, dmw) -> np.ndarray:
        x, mu, mv, mw = ctx.saved
        return ctx.model.advection_tl(x, mu, mv, mw, dx, dmu, dmv, dmw)


class ProjectionFunction:
    """anelastic_pressure as a map of (mu, mv, mw, p): affine, linear in the momentum."""

    @staticmethod
    def forward(ctx: FnContext, mu, mv, mw, p):
        ctx.save_for_backward()
        z = np.zeros_like(mw)
        out = ctx.model.anelastic_pressure(mu, mv, mw, p, z)
        return out[:4]

    @staticmethod
    def backward(ctx: FnContext, mub, mvb, mwb, pb):
        return ctx.model.anelastic_pressure_ad(mub, mvb, mwb, pb)

    @staticmethod
    def jvp(ctx: FnContext, dmu, dmv, dmw, dp):
        z = np.zeros_like(dmw)
        return ctx.model.anelastic_pressure(dmu, dmv, dmw, dp, z)[:4]
