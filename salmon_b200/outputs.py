"""SALMON's periodic-run output files and the Fourier-transform spectra, in the
reference's column layout and number format (atomic units, unit_system = 'au'),
so that scripts reading a SALMON run's `<sysname>_*.data` files read these.

Reference routines restated here (paths relative to the SALMON source tree):
  write_k_data        ARTED/GS/write_GS_data.f90:324-354   <sysname>_k.data
  write_eigen_data    ARTED/GS/write_GS_data.f90:358-386   <sysname>_eigen.data
  write_rt_data       ARTED/control/control_sc.f90:487-545 <sysname>_rt.data
  rt energy rows      ARTED/control/control_sc.f90:549-607 <sysname>_rt_energy.data
  Fourier_tr          ARTED/RT/Fourier_tr.f90:17-160        <sysname>_lr.data (spectra)
"""
from __future__ import annotations

import math

import numpy as np


def fortran_e(v: float, width: int = 23, digits: int = 15, expdigits: int = 3) -> str:
    """A real in Fortran's E<width>.<digits>E<expdigits> edit descriptor: a
    mantissa in [0.1, 1) with a leading '0.', e.g. ' -0.250620000000000E-001'."""
    v = float(v)
    if v == 0.0 or not math.isfinite(v):
        body = "0." + "0" * digits + "E+" + "0" * expdigits if v == 0.0 else repr(v)
        return body.rjust(width)
    sign = "-" if v < 0 else ""
    a = abs(v)
    e = math.floor(math.log10(a)) + 1
    m = round(a / 10.0 ** e, digits)
    if m >= 1.0:                      # rounding carried into the next decade
        m /= 10.0
        e += 1
    if m < 0.1:                       # log10 rounding at an exact power of ten
        m *= 10.0
        e -= 1
    mant = f"{m:.{digits}f}"          # '0.ddd...'
    es = "+" if e >= 0 else "-"
    return f"{sign}{mant}E{es}{abs(e):0{expdigits}d}".rjust(width)


def fortran_f(v: float, width: int = 16, digits: int = 8) -> str:
    """F<width>.<digits>."""
    return f"{float(v):{width}.{digits}f}"


def _row(first: str, values) -> str:
    return first + "".join(" " + fortran_e(x) for x in values)


def write_k_data(path: str, kAc0, bl, wk=None):
    """ik, k in reduced coordinates (kAc0 / bL), weight.  kAc0: (3, NK)."""
    kAc0 = np.asarray(kAc0)
    nk = kAc0.shape[1]
    wk = np.ones(nk) if wk is None else np.asarray(wk)
    with open(path, "w") as f:
        f.write("# k-point distribution\n# ik: k-point index\n# kx,ky,kz: Reduced coordinate of k-points\n"
                "# wk: Weight of k-point\n# 1:ik[none] 2:kx[none] 3:ky[none] 4:kz[none] 5:wk[none]\n")
        for ik in range(nk):
            f.write(_row(f"{ik + 1:6d}", [kAc0[0, ik] / bl[0], kAc0[1, ik] / bl[1], kAc0[2, ik] / bl[2], wk[ik]])
                    + "\n")


def write_eigen_data(path: str, esp, occ, nkxyz: int, wk=None):
    """ik, ib, eigenenergy, occupation occ / wk * NKxyz.  esp, occ: (NK, NB)."""
    esp = np.asarray(esp)
    occ = np.asarray(occ)
    nk, nb = esp.shape
    wk = np.ones(nk) if wk is None else np.asarray(wk)
    with open(path, "w") as f:
        f.write("# Ground state eigenenergies\n# ik: k-point index\n# ib: Band index\n# energy: Eigenenergy\n"
                "# occup: Occupation\n# 1:ik[none] 2:ib[none] 3:energy[a.u.] 4:occup[none]\n")
        for ik in range(nk):
            for ib in range(nb):
                f.write(_row(f"{ik + 1:6d} {ib + 1:6d}", [esp[ik, ib], occ[ik, ib] / wk[ik] * nkxyz]) + "\n")


def fields_from_Ac(Ac, dt: float):
    """E(iter) = -(A(iter+1) - A(iter-1)) / (2 dt) (control_sc.f90:218-220) for
    iter = 0..len(Ac)-3, with Ac rows holding iter = -1, 0, 1, ... (init_Ac)."""
    Ac = np.asarray(Ac)
    return -(Ac[2:] - Ac[:-2]) / (2 * dt)


def write_rt_data(path: str, dt: float, Ac_ext, E_ext, Ac_tot, E_tot, javt, niter: int):
    """Rows iter = 0..niter: time, Ac_ext, E_ext, Ac_tot, E_tot, Jm (3 each).
    Ac_* indexed by iter (row iter of the arrays), E_* and javt likewise."""
    with open(path, "w") as f:
        f.write("# Real time calculation\n# Ac_ext: External vector potential field\n"
                "# E_ext: External electric field\n# Ac_tot: Total vector potential field\n"
                "# E_tot: Total electric field\n# Jm: Matter current density\n")
        cols = ["Time", "Ac_ext_x", "Ac_ext_y", "Ac_ext_z", "E_ext_x", "E_ext_y", "E_ext_z", "Ac_tot_x", "Ac_tot_y",
                "Ac_tot_z", "E_tot_x", "E_tot_y", "E_tot_z", "Jm_x", "Jm_y", "Jm_z"]
        f.write("#" + "".join(f" {i + 1}:{c}[a.u.]" for i, c in enumerate(cols)) + "\n")
        for it in range(niter + 1):
            vals = list(Ac_ext[it]) + list(E_ext[it]) + list(Ac_tot[it]) + list(E_tot[it]) + list(javt[it])
            f.write(_row(fortran_f(it * dt), vals) + "\n")


def write_rt_energy_data(path: str, dt: float, Eall_t, Eall0: float, niter: int, nstep_energy_calc: int = 10):
    """Rows every nstep_energy_calc steps: time, Eall, Eall - Eall0.  Eall_t maps
    iter -> Eall (the energy after step iter, field energy included)."""
    with open(path, "w") as f:
        f.write("# Real time calculation\n# Eall: Total energy\n# Eall0: Initial energy\n"
                "# 1:Time[a.u.] 2:Eall[a.u.] 3:Eall-Eall0[a.u.]\n")
        for it in range(0, niter + 1, nstep_energy_calc):
            f.write(_row(fortran_f(it * dt), [Eall_t[it], Eall_t[it] - Eall0]) + "\n")


def smoothing_t(tt, Nt: int, dt: float):
    """1 - 3 (t/T)^2 + 2 (t/T)^3, T = Nt dt (Fourier_tr.f90:142-150)."""
    x = np.asarray(tt) / (Nt * dt)
    return 1.0 - 3.0 * x ** 2 + 2.0 * x ** 3


def fourier_tr(javt, E_ext, E_tot, dt: float, Nt: int, nomega: int, domega: float, ae_shape: str = "impulse",
               trans_longi: str = "tr", dAc: float = 1e-3, epdir=(1.0, 0.0, 0.0), insulator: bool = True):
    """The spectra of Fourier_tr.f90:64-102 for hw = domega, 2 domega, ...,
    nomega domega: smoothed transforms of J(t) - J_dc, E_ext(t), E_tot(t) over
    iter = 0..Nt (J_dc = the smoothed time average when the system is an
    insulator, KbTev < 0), then for an impulse: sigma = J(w)/dAc and
    eps = epdir + 4 pi i sigma / hw ('tr'), or eps = 1/(1 - E_tot(w)/dAc) ('lo').
    Returns a dict of (nomega, 3) complex arrays and hw."""
    javt = np.asarray(javt)[:Nt + 1]
    E_ext = np.asarray(E_ext)[:Nt + 1]
    E_tot = np.asarray(E_tot)[:Nt + 1]
    tt = np.arange(Nt + 1) * dt
    sm = smoothing_t(tt, Nt, dt)
    jav_d = (javt * sm[:, None]).sum(axis=0) / sm.sum() if insulator else np.zeros(3)
    hw = np.arange(1, nomega + 1) * domega
    ph = np.exp(1j * np.outer(hw, tt)) * sm[None, :]          # (nomega, Nt+1)
    jw = ph @ (javt - jav_d) * dt
    ew = ph @ E_ext * dt
    tw = ph @ E_tot * dt
    out = {"hw": hw, "jav_w": jw, "E_ext_w": ew, "E_tot_w": tw}
    if ae_shape == "impulse":
        if trans_longi == "lo":
            out["eps"] = 1.0 / (1.0 - tw / dAc)
        else:
            sigma = jw / dAc
            out["sigma"] = sigma
            out["eps"] = np.asarray(epdir)[None, :] + 1j * 4.0 * np.pi * sigma / hw[:, None]
    return out


def write_lr_data(path: str, spec: dict, ae_shape: str = "impulse", trans_longi: str = "tr"):
    """<sysname>_lr.data rows as Fourier_tr writes them."""
    hw = spec["hw"]
    with open(path, "w") as f:
        f.write("# Fourier-transform spectra\n")
        for i, w in enumerate(hw):
            if ae_shape == "impulse" and trans_longi == "lo":
                vals = list(spec["eps"][i].real) + list(spec["eps"][i].imag)
            elif ae_shape == "impulse":
                vals = (list(spec["sigma"][i].real) + list(spec["sigma"][i].imag) + list(spec["eps"][i].real)
                        + list(spec["eps"][i].imag))
            else:
                vals = []
                for key in ("jav_w", "E_ext_w", "E_tot_w"):
                    vals += list(spec[key][i].real) + list(spec[key][i].imag)
            f.write(_row(fortran_f(w), vals) + "\n")
