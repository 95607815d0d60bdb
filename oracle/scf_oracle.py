"""CPU oracle (numpy) for the self-consistent local potential.

TEST INFRASTRUCTURE ONLY: tests compare salmon_b200/csrc/k_xc.cu against it.

  hartree   common/Hartree.f90:20-130: rho(G) = sum_r rho e^{-iG.r} / NL with
            G = 2 pi m / aL, m in [-N/2, N/2) (init.f90:52-70), Vh(G) = 4 pi rho(G) / G^2,
            Vh(0) = 0, Vh(r) = sum_G Vh(G) e^{iG.r}; the separable DFT of the
            reference evaluated with numpy's FFT (the same sums).
  pz        xc/builtin_pz.f90:23-80 (exc_cor_pz / PZxc): the Perdew-Zunger 1981
            LDA, unpolarised, for the total density rho.
  vloc      RT/dt_evolve.f90:201-207: Vloc = Vh + Vpsl + Vexc.
"""
from __future__ import annotations

import numpy as np

PZ = dict(gammaU=-0.1423, beta1U=1.0529, beta2U=0.3334, AU=0.0311, BU=-0.048, CU=0.002, DU=-0.0116)


def hartree(rho, shape, aL):
    NLx, NLy, NLz = shape
    R = np.fft.fftn(rho.reshape(shape)) / rho.size
    ms = [np.where(np.arange(n) < n - n // 2, np.arange(n), np.arange(n) - n) for n in shape]
    g = [2 * np.pi * m / a for m, a in zip(ms, aL)]
    G2 = g[0][:, None, None] ** 2 + g[1][None, :, None] ** 2 + g[2][None, None, :] ** 2
    G2[0, 0, 0] = 1.0
    V = 4 * np.pi * R / G2
    V[0, 0, 0] = 0.0
    return np.real(np.fft.ifftn(V) * rho.size).ravel()


def pz(rho):
    """(exc, vxc) per point for the total density rho (PZxc with trho = rho)."""
    p = PZ
    ttrho = rho + 1e-10
    rs = (3.0 / (4 * np.pi * ttrho)) ** (1.0 / 3.0)
    const = 0.75 * (3.0 / (2.0 * np.pi)) ** (2.0 / 3.0)
    exc = -const / rs
    dexc = exc / (3 * ttrho)
    hi = rs > 1.0
    sq = np.sqrt(rs)
    den = 1.0 + p["beta1U"] * sq + p["beta2U"] * rs
    lnr = np.log(rs)
    exc_hi = exc + p["gammaU"] / den
    dexc_hi = dexc + p["gammaU"] * (0.5 * p["beta1U"] * sq + p["beta2U"] * rs) / (3 * ttrho) / den ** 2
    exc_lo = exc + p["AU"] * lnr + p["BU"] + p["CU"] * rs * lnr + p["DU"] * rs
    dexc_lo = dexc - rs / (3 * ttrho) * (p["AU"] / rs + p["CU"] * (lnr + 1) + p["DU"])
    e = np.where(hi, exc_hi, exc_lo)
    d = np.where(hi, dexc_hi, dexc_lo)
    return e, e + rho * d


def vloc(rho, vpsl, shape, aL, Hxyz):
    """Vloc and (Eh, Exc) = (1/2 sum Vh rho Hxyz, sum exc rho Hxyz)."""
    vh = hartree(rho, shape, aL)
    exc, vxc = pz(rho)
    return vh + vpsl + vxc, (0.5 * float(np.dot(vh, rho)) * Hxyz, float(np.dot(exc, rho)) * Hxyz)
