"""Ground-state and real-time drivers over the C ABI.

These follow the control flow of SALMON's ARTED drivers, either with the
local potential held fixed or updated self-consistently (Hartree + PZ LDA on
the device, sgpu_update_vloc):

  init_Ac          RT/init_Ac.f90:17-100      A_ext(t) of 'impulse' and 'Acos<n>' pulses
  ground_state     control/ground_state.f90:100-150  Gram-Schmidt, subspace diag,
                                              Gram-Schmidt, CG, Gram-Schmidt per iteration
  rt_propagate     control/control_sc.f90:150-230 with dt_evolve_omp_KB
                   'middlepoint' (RT/dt_evolve.f90:45-49, 176-207): k+A at the
                   midpoint for the Taylor step, then rho -> Vh + Vexc -> Vloc
                   (scf=True), k+A(t+dt) for the current; or 'etrs'
                   (dt_evolve_etrs_omp_KB, RT/dt_evolve.f90:218-348): two half steps
                   around the extrapolated potential
  ground_state_scf the ground-state loop with the density mixed linearly between
                   iterations
  gs_scf           the reference's SCF loop: Broyden mixing (common/broyden.f90) and
                   the 'rho_dne' convergence test (control/ground_state.f90:43-180)
"""
from __future__ import annotations

import numpy as np

F0_PER_SQRT_WCM2 = 5.338e-9  # electric field in a.u. per sqrt(W/cm^2) (init_Ac.f90:34)


def init_Ac(Nt: int, dt: float, shape: str = "impulse", epdir=(1.0, 0.0, 0.0), e_impulse: float = 1e-3,
            rlaser_int_wcm2: float = 1e12, omega: float = 0.05696144984638035, pulse_tw: float = 110.0,
            phi_cep: float = 0.0, t_delay: float = 0.0):
    """Ac_ext(iter) for iter = -1..Nt+1 as an array of shape (Nt+3, 3); row
    iter+1 holds time iter*dt (RT/init_Ac.f90:44-84)."""
    ep = np.asarray(epdir, dtype=np.float64)
    Ac = np.zeros((Nt + 3, 3))
    if shape == "impulse":
        Ac[:, :] = ep * e_impulse
        return Ac
    if not shape.startswith("Acos"):
        raise ValueError(f"unsupported pulse shape {shape!r}")
    npower = int(shape[4:])
    f0 = F0_PER_SQRT_WCM2 * np.sqrt(rlaser_int_wcm2)
    for it in range(-1, Nt + 2):
        tt = it * dt - 0.5 * pulse_tw - t_delay
        if abs(tt) < 0.5 * pulse_tw:
            Ac[it + 1] = -f0 / omega * np.cos(np.pi * tt / pulse_tw) ** npower * np.imag(
                ep * np.exp(1j * (omega * tt + phi_cep * 2 * np.pi)))
    return Ac


def ground_state(g, n_iter: int = 4, ncg: int = 4):
    """Iterations of the ground-state sequence at fixed potential on the device
    ground-state orbitals; returns (esp (nkl,NB), esp_var (nkl,NB), history)
    with history[i] = (sum of esp, max of esp_var) after iteration i."""
    esp = esp_var = None
    history = []
    for _ in range(n_iter):
        g.gram_schmidt()
        esp = g.subspace_diag()
        g.gram_schmidt()
        esp_var, _ = g.cg(ncg)
        g.gram_schmidt()
        history.append((float(esp.sum()), float(esp_var.max())))
    esp = g.subspace_diag()
    return esp, esp_var, history


def ground_state_scf(g, n_iter: int = 40, ncg: int = 4, mix: float = 0.3):
    """Ground-state iterations with a self-consistent Vloc = Vh + Vpsl + Vexc
    (the caller has set Vpsl and an initial Vloc).  After each iteration the
    occupied bands' density rho_out is mixed into rho_in <- (1-mix) rho_in + mix
    rho_out and the potential is rebuilt from rho_in.  Returns (esp, history)
    with history[i] = (sum of esp, max esp_var, |rho_out - rho_in| Hxyz)."""
    history = []
    rho_in = None
    esp = None
    for _ in range(n_iter):
        g.gram_schmidt()
        esp = g.subspace_diag()
        g.gram_schmidt()
        esp_var, _ = g.cg(ncg)
        g.gram_schmidt()
        g.gs_to_rt()
        rho_out = g.psi_rho_RT()
        if rho_in is None:
            rho_in = rho_out
        drho = float(np.abs(rho_out - rho_in).sum() * g.sysm.Hxyz)
        rho_in = (1 - mix) * rho_in + mix * rho_out
        g.update_vloc(rho_in)
        history.append((float(esp.sum()), float(esp_var.max()), drho))
    esp = g.subspace_diag()
    return esp, history


def gs_scf(g, sysm, kAc0, vpsl, nscf: int = 100, ncg: int = 5, threshold: float = 1e-9, mixer=None):
    """The periodic ground-state SCF loop of control/ground_state.f90:43-175 on
    the device orbitals (the caller loads the initial guess with gs_set_state):
    Gram-Schmidt, rho_in(1) = rho(psi0), Vloc = Vh + Vpsl + Vexc; then per
    iteration Gram-Schmidt, subspace diag, Gram-Schmidt, CG(ncg), Gram-Schmidt,
    rho_out, Broyden mixing (common/broyden.f90) and the new Vloc, until
    ddns_abs_1e = sum|rho_out - rho_in| Hxyz / Nelec < threshold (the 'rho_dne'
    criterion, ground_state.f90:180).  A final subspace diag gives the
    eigenvalues.  Returns (esp (nkl,NB), history) with history[i] =
    (ddns_abs_1e, max esp_var) of iteration i+1."""
    from .broyden import Broyden
    mixer = mixer if mixer is not None else Broyden()
    nelec = float(np.sum(sysm.occ))
    g.update_projector(np.ascontiguousarray(kAc0, dtype=np.float64))
    g.set_vpsl(vpsl)
    g.gram_schmidt()
    g.gs_to_rt()
    rho = g.psi_rho_RT()
    mixer.start(rho)
    g.update_vloc(rho)
    history = []
    for _ in range(nscf):
        g.gram_schmidt()
        g.subspace_diag()
        g.gram_schmidt()
        esp_var, _ = g.cg(ncg)
        g.gram_schmidt()
        g.gs_to_rt()
        rho_out = g.psi_rho_RT()
        rho_in = mixer.rho_in[mixer.iter + 1]
        ddns = float(np.abs(rho_out - rho_in).sum() * sysm.Hxyz / nelec)
        rho_new = mixer.mix(rho_out)
        g.update_vloc(rho_new)
        history.append((ddns, float(esp_var[:, :sysm.NBoccmax].max())))
        if ddns < threshold:
            break
    esp = g.subspace_diag()
    g.gram_schmidt()
    g.gs_to_rt()
    return esp, history


def band_energy(g, sysm, kAc, vloc):
    """Ekin + Enl + sum_i Vloc_i rho_i Hxyz of the resident orbitals (FP64)."""
    ek, en = g.energy_terms(kAc)
    rho = g.psi_rho_RT()
    return ek + en + float(np.dot(vloc, rho)) * sysm.Hxyz


def total_energy(g, sysm, kAc, vpsl, eion: float = 0.0):
    """Ekin + Enl + sum Vpsl rho Hxyz + Eh + Exc + eion of the resident orbitals
    (FP64; eion is the ion-ion energy, a constant for fixed ions:
    pseudo.ewald_energy); also rebuilds Vloc from their density, as the
    reference's step does."""
    ek, en = g.energy_terms(kAc)
    rho = g.psi_rho_RT()
    eh, exc = g.update_vloc(rho)
    return ek + en + float(np.dot(vpsl, rho)) * sysm.Hxyz + eh + exc + eion


def rt_propagate(g, sysm, kAc0, vloc, Ac, dt: float, Nt: int, energy_every: int = 0, scf: bool = False,
                 eion: float = 0.0, propagator: str = "middlepoint"):
    """Nt Taylor-propagator steps of the resident orbitals; returns
    (javt (Nt+1,3) with javt[0] the current before the first step,
     energies {step: energy} every `energy_every` steps).
    scf=False: vloc is the fixed local potential (energies: band energy).
    scf=True: vloc is Vpsl; Vloc = Vh + Vpsl + Vexc is rebuilt from the density
    after every step on the device (energies: total_energy).
    propagator (dt_evolve_KB, RT/dt_evolve.f90:28-63):
      'middlepoint'  one Taylor step of dt at k + (A(t) + A(t+dt))/2
                     (dt_evolve_omp_KB, :104-207);
      'etrs'         a half step dt/2 at k + A(t), the potential extrapolated to
                     t + dt from its history (3 V - 3 V1 + V2), a half step dt/2 at
                     k + A(t+dt) (dt_evolve_etrs_omp_KB, :218-348; LDA functionals)."""
    if propagator not in ("middlepoint", "etrs"):
        raise ValueError(f"invalid propagator {propagator!r}")
    kAc0 = np.ascontiguousarray(kAc0, dtype=np.float64)
    if scf:
        g.set_vpsl(vloc)
        g.update_vloc()
    else:
        g.set_vloc(vloc)
    if propagator == "etrs":
        g.vloc_history_reset()   # Vloc_old(:,1) = Vloc_old(:,2) = Vloc (control_sc.f90:82)
    energy = (lambda k: total_energy(g, sysm, k, vloc, eion)) if scf else (lambda k: band_energy(g, sysm, k, vloc))
    javt = np.zeros((Nt + 1, 3))
    javt[0] = g.current_RT(kAc0 + Ac[1][:, None])
    energies = {}
    if energy_every:
        energies[0] = energy(kAc0 + Ac[1][:, None])
    for it in range(Nt):
        if propagator == "middlepoint":
            kmid = kAc0 + 0.5 * (Ac[it + 1] + Ac[it + 2])[:, None]   # kAc0 + (Ac(it)+Ac(it+1))/2
            g.update_projector(kmid)
            g.hamiltonian(dt, flag_current=True)
        else:
            g.update_projector(kAc0 + Ac[it + 1][:, None])            # kAc = kAc0 + Ac_tot(iter)
            g.hamiltonian(0.5 * dt)
            g.vloc_extrapolate()                                      # dt_evolve.f90:248-252
            g.update_projector(kAc0 + Ac[it + 2][:, None])            # kAc = kAc_new
            g.hamiltonian(0.5 * dt, flag_current=True)
        if scf:
            g.update_vloc()       # psi_rho_RT, Hartree, Exc_Cor, Vloc (dt_evolve.f90:190-207)
        knew = kAc0 + Ac[it + 2][:, None]
        javt[it + 1] = g.current_RT(knew)
        if energy_every and (it + 1) % energy_every == 0:
            energies[it + 1] = energy(knew)
    return javt, energies


def j_error(j_ref, j_test):
    """max_t |J_test(t) - J_ref(t)| / max_t |J_ref(t)|, per component maximum."""
    j_ref = np.asarray(j_ref)
    j_test = np.asarray(j_test)
    return float(np.abs(j_test - j_ref).max() / np.abs(j_ref).max())


def j_error_dynamic(j_ref, j_test):
    """The same error relative to the time-dependent part of J (J(t) - J(0))."""
    d_ref = np.asarray(j_ref) - np.asarray(j_ref)[0]
    d_test = np.asarray(j_test) - np.asarray(j_test)[0]
    return float(np.abs(d_test - d_ref).max() / max(np.abs(d_ref).max(), 1e-300))
