"""Modified Broyden density mixing for the ground-state SCF loop.

Restates SALMON's ``broyden`` (common/broyden.f90:21-176) as called from the
periodic ground-state loop without a communicator (control/ground_state.f90:138,
``call broyden(rho,rho_in,rho_out,nl,iter,iter,nscf)``), with the defaults of
io/inputoutput.f90:649-650 (alpha_mb = 0.75, nmemory_mb = 8) and the constants
iter_mb = 0, omega0 = 0.01 of broyden.f90:35-36.  The history lives on the host:
it holds NL doubles per iteration, tiny next to the orbitals.
"""
from __future__ import annotations

import numpy as np


class Broyden:
    """rho_in(:, iter) / rho_out(:, iter) history and the mixing step.

    ``start(rho0)`` sets rho_in(:, 1); ``mix(rho_out)`` at iteration ``iter``
    (1, 2, ...) stores rho_out(:, iter) and returns rho_in(:, iter+1)."""

    def __init__(self, alpha: float = 0.75, nmemory: int = 8, omega0: float = 0.01):
        self.alpha = float(alpha)
        self.nmemory = int(nmemory)
        self.omega0 = float(omega0)
        self.rho_in: dict[int, np.ndarray] = {}
        self.rho_out: dict[int, np.ndarray] = {}
        self.iter = 0

    def start(self, rho0):
        self.rho_in = {1: np.array(rho0, dtype=np.float64)}
        self.rho_out = {}
        self.iter = 0

    def residual(self, it: int) -> np.ndarray:
        return self.rho_out[it] - self.rho_in[it]

    def mix(self, rho_out) -> np.ndarray:
        self.iter += 1
        it = self.iter
        a = self.alpha
        self.rho_out[it] = np.array(rho_out, dtype=np.float64)
        f_it = self.residual(it)
        if it <= 1:                                          # iter <= iter_mb + 1
            self.rho_in[it + 1] = self.rho_in[it] + a * f_it
        else:
            it_s = max(1, it - self.nmemory)
            it_e = it - 1
            rng = range(it_s, it_e + 1)
            dx, df = [], []
            for i in rng:
                d_x = self.rho_in[i + 1] - self.rho_in[i]
                d_f = self.residual(i + 1) - self.residual(i)
                ss = float(np.sum(d_f * d_f))                # squared norm (the branch without icomm)
                dx.append(d_x / ss)
                df.append(d_f / ss)
            n = len(df)
            aa = np.empty((n, n))
            for i in range(n):
                for j in range(n):
                    aa[i, j] = float(np.sum(df[i] * df[j]))
                aa[i, i] += self.omega0 ** 2
            beta = np.linalg.inv(aa)
            proj = np.array([float(np.sum(df[i] * f_it)) for i in range(n)])
            tmp = np.zeros_like(f_it)
            for i in range(n):
                for j in range(n):
                    tmp += beta[i, j] * proj[i] * (a * df[j] + dx[j])
            new = self.rho_in[it] + a * f_it - tmp
            if np.any(new < 0.0):                            # fall back to linear mixing
                new = self.rho_in[it] + a * f_it
            self.rho_in[it + 1] = new
            for k in [k for k in self.rho_in if k < it - self.nmemory]:
                del self.rho_in[k]
            for k in [k for k in self.rho_out if k < it - self.nmemory]:
                del self.rho_out[k]
        return self.rho_in[it + 1].copy()
