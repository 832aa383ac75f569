"""Fluid properties: density and a constant or Carreau-Yasuda viscosity.

Mirrors ``zvcfd.fv.reference.Fluid`` (``zvcfd/fv/reference.py:176-182``) and
``zvcfd.rheology.CarreauYasuda`` (``zvcfd/rheology.py:37-62``); the device
kernels evaluate ``mu_inf + (mu_0 - mu_inf) (1 + (lam g)^a)^((n - 1)/a)`` at
every flux point, without the optional shear-rate clips (as the reference's
GPU path does, ``zvcfd/fv/solver.py:135-136``).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class CarreauYasuda:
    mu_0: float = 0.056
    mu_inf: float = 0.00345
    lam: float = 3.313
    a: float = 2.0
    n: float = 0.3568

    def __call__(self, gamma):
        g = np.asarray(gamma, float)
        return self.mu_inf + (self.mu_0 - self.mu_inf) * (1.0 + (self.lam * g) ** self.a) ** (
            (self.n - 1.0) / self.a)


@dataclass
class Fluid:
    """Density (kg/m^3) and viscosity: a constant ``mu`` (Pa s), or ``viscosity(gamma_dot)``."""

    rho: float = 1.0
    mu: float = 1.0
    viscosity: CarreauYasuda | None = None


__all__ = ["CarreauYasuda", "Fluid"]
