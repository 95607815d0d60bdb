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


def gs_exact(sysm, kAc0, vpsl, hpsi_columns, n_iter: int = 20, mixer=None):
    """Ground-state SCF by exact diagonalisation, the checker of the device's
    CG-based loop (control/ground_state.f90:100-175 with CG + subspace diag
    replaced by a full eigendecomposition of H(k) on the grid).

    hpsi_columns(ik, vloc) -> H(k) as an (NL, NL) matrix whose column j is H
    applied to the j-th grid delta; the static part (H - diag(Vloc)) is built
    once.  The density of the lowest NBoccmax bands (occ of the system) is mixed
    by ``mixer`` (a salmon_b200.broyden.Broyden-like object with start/mix);
    Vloc = Vh + Vpsl + Vexc.  Returns (esp (NK, NB), ddns history)."""
    from scipy.linalg import eigh
    NL, NK, NB, nocc = sysm.NL, sysm.NK, sysm.NB, sysm.NBoccmax
    shape = (sysm.NLx, sysm.NLy, sysm.NLz)
    nelec = float(np.sum(sysm.occ))
    h0 = [hpsi_columns(ik, vpsl) - np.diag(vpsl) for ik in range(NK)]
    rho = np.full(NL, nelec / sysm.aLxyz)
    mixer.start(rho)
    v, _ = vloc(rho, vpsl, shape, sysm.aL, sysm.Hxyz)
    hist = []
    esp = np.zeros((NK, NB))
    for _ in range(n_iter):
        rho_out = np.zeros(NL)
        for ik in range(NK):
            w, vec = eigh(h0[ik] + np.diag(v), subset_by_index=[0, NB - 1])
            esp[ik] = w
            psi = vec[:, :nocc] / np.sqrt(sysm.Hxyz)
            rho_out += (np.abs(psi) ** 2) @ sysm.occ[ik, :nocc]
        hist.append(float(np.abs(rho_out - mixer.rho_in[mixer.iter + 1]).sum() * sysm.Hxyz / nelec))
        rho = mixer.mix(rho_out)
        v, _ = vloc(rho, vpsl, shape, sysm.aL, sysm.Hxyz)
    return esp, hist
