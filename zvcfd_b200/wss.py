"""Time statistics of wall shear stress (TAWSS, OSI, RRT), accumulated where the samples live.

The reference's ``WallShearStats`` (``zvcfd/fv/wss.py:21-48``) integrates, per wall node and
by the trapezoidal rule over the committed time steps, ``∫ τ dt`` and ``∫ |τ| dt``; then

    TAWSS = ∫ |τ| dt / T,   OSI = ½ (1 − |∫ τ dt| / ∫ |τ| dt),   RRT = 1 / ((1 − 2 OSI) TAWSS)

(He & Ku 1996 for OSI; Himburg et al. 2004 for RRT). Here the running integrals are tensors on
the device of the samples, so a transient solve that samples ``wall_shear`` every step adds
two small elementwise updates per step and no host transfer until :meth:`results`.
"""

from __future__ import annotations

import numpy as np
import torch


class WallShearStats:
    """Accumulates ``∫ τ dt`` and ``∫ |τ| dt`` for ``n`` wall nodes (trapezoidal rule).

    Args:
        n: number of wall nodes.
        device: where the integrals live; by default that of the first tensor sample (the CPU
            for NumPy samples).
    """

    def __init__(self, n: int, device=None):
        self.n = int(n)
        self.device = torch.device(device) if device is not None else None
        self.int_tau = self.int_mag = None
        self.T = 0.0
        self._last = None

    def _tensor(self, tau):
        if self.device is None:
            self.device = tau.device if isinstance(tau, torch.Tensor) else torch.device("cpu")
        tau = torch.as_tensor(tau, dtype=torch.float64, device=self.device)
        if tau.shape != (self.n, 3):
            raise ValueError(f"wall shear sample of shape {tuple(tau.shape)}, expected "
                             f"({self.n}, 3)")
        return tau

    def add(self, t: float, tau) -> None:
        """One sample ``tau`` ``(n, 3)`` at time ``t`` (a tensor or an array)."""
        tau = self._tensor(tau)
        mag = torch.linalg.vector_norm(tau, dim=1)
        if self.int_tau is None:
            self.int_tau = torch.zeros((self.n, 3), dtype=torch.float64, device=self.device)
            self.int_mag = torch.zeros(self.n, dtype=torch.float64, device=self.device)
        if self._last is not None:
            t0, tau0, mag0 = self._last
            h = float(t) - t0
            self.int_tau += 0.5 * h * (tau0 + tau)
            self.int_mag += 0.5 * h * (mag0 + mag)
            self.T += h
        self._last = (float(t), tau.clone(), mag)

    def results(self) -> dict:
        """``{"tawss", "osi", "rrt"}``, each ``(n,)`` on the host."""
        if self.T <= 0:
            raise ValueError("need at least two samples")
        tawss = self.int_mag / self.T
        osi = 0.5 * (1 - torch.linalg.vector_norm(self.int_tau, dim=1)
                     / torch.clamp(self.int_mag, min=1e-300))
        rrt = 1.0 / torch.clamp((1 - 2 * osi) * tawss, min=1e-300)
        return {k: v.cpu().numpy() for k, v in (("tawss", tawss), ("osi", osi), ("rrt", rrt))}


__all__ = ["WallShearStats"]
