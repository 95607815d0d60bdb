"""Ground-state CG preconditioners: training data from plain CG, training of the
learned network on the GPU (the library's own BF16 kernels), and the CG
convergence driver used to compare plain CG, TPA and the learned network.

The ground-state sequence is that of control/ground_state.f90:100-150
(Gram-Schmidt, subspace diagonalisation, Gram-Schmidt, CG, Gram-Schmidt) at a
fixed potential.
"""
from __future__ import annotations

import numpy as np

from . import system as S


def displaced_system(base_args: dict, sigma: float, seed: int):
    """A Si supercell (``system.si_supercell_system`` arguments) with every atom
    displaced by N(0, sigma^2) bohr per axis; returns (system, kAc, Vloc, zu)."""
    rng = np.random.default_rng(seed)
    sysm, kAc, vloc, zu = S.si_supercell_system(**base_args)
    R = sysm.Rion + sigma * rng.standard_normal(sysm.Rion.shape)
    NLx, NLy, NLz = sysm.NLx, sysm.NLy, sysm.NLz
    Mps, Jxyz, Jxx, Jyy, Jzz, dist = S.calc_jxyz(NLx, NLy, NLz, sysm.aL, R, sysm.Rps)
    uV, iuV, a_tbl = S.gaussian_projectors(Mps, dist, sysm.Hxyz)
    vloc = S.periodic_gaussian_vloc(NLx, NLy, NLz, sysm.aL, R, sysm.extra["depth"], sysm.extra["width"])
    sysm2 = S.System(NLx=NLx, NLy=NLy, NLz=NLz, aL=sysm.aL, kAc0=sysm.kAc0, NB=sysm.NB, NBoccmax=sysm.NBoccmax,
                     occ=sysm.occ, Rion=R, Rps=sysm.Rps, Mps=Mps, Jxyz=Jxyz, Jxx=Jxx, Jyy=Jyy, Jzz=Jzz, uV=uV,
                     iuV=iuV, a_tbl=a_tbl)
    sysm2.extra.update(sysm.extra)
    return sysm2, kAc, vloc, zu


def gs_iteration(g, ncg, nconv=None):
    """One ground-state iteration; returns (esp, CG iterations summed over bands
    and k-points, max residual norm of the lowest nconv bands (all if None))."""
    g.gram_schmidt()
    esp = g.subspace_diag()
    g.gram_schmidt()
    _, its = g.cg(ncg)
    g.gram_schmidt()
    return esp, int(its.sum()), float(g.cg_residuals()[:, :nconv].max())


def solve_to(g, tol=1e-8, ncg=4, max_outer=400, nconv=None):
    """Ground-state iterations until the residual of each of the lowest nconv
    bands (all bands if None; the rest are buffer bands, like the empty bands
    of a ground-state run) is below tol.
    Returns dict(outer, cg_iterations, residual, esp, converged)."""
    total, res, esp = 0, np.inf, None
    for it in range(1, max_outer + 1):
        esp, n, res = gs_iteration(g, ncg, nconv)
        total += n
        if res < tol:
            return {"outer": it, "cg_iterations": total, "residual": res, "esp": g.subspace_diag(), "converged": True}
    return {"outer": max_outer, "cg_iterations": total, "residual": res, "esp": esp, "converged": False}


def _shifted_solve(g, ik, r, shift, iters, tol=1e-10):
    """t = (H - shift)^{-1} r by CG (H - shift is positive definite here)."""
    t = np.zeros_like(r)
    res = r.copy()
    p = res.copy()
    rr = float(np.vdot(res, res).real)
    r0 = rr
    for _ in range(iters):
        hp, _ = g.hpsi_omp_KB_GS(ik, p)
        ap = hp - shift * p
        a = rr / float(np.vdot(p, ap).real)
        t += a * p
        res -= a * ap
        rn = float(np.vdot(res, res).real)
        if rn < tol * tol * r0:
            break
        p = res + (rn / rr) * p
        rr = rn
    return t


def correction_pairs(g, sysm, snaps, nconv, emin, margin=1.0, iters=80, bands=None):
    """Residual/correction pairs from snapshots of plain CG.  For each of the
    lowest nconv bands psi of every snapshot: the gradient
    r = H psi - <psi|H|psi> psi, and the correction t that solves the shifted
    correction equation (H - eps + sigma) t = r, sigma = eps - eps_min + margin
    (eps_min the lowest eigenvalue at that k-point; H - eps + sigma is then
    positive definite; emin (nkl,) are converged lowest eigenvalues), by CG.
    This is the update an ideal preconditioner
    would return; the kinetic-energy (TPA) factor approximates it with T in
    place of H.  A margin near the band kinetic energy (1 Ha here) keeps the
    target flat over the occupied spectrum, as TPA is; a small margin
    over-weights the lowest states and a large one flattens the high-energy
    fall-off (both measured to slow CG down).  Returns complex arrays (n, NL) of r and t, and per pair the
    local k-point index and the band's kinetic energy <psi|T|psi> (for TPA).
    `bands` restricts the pairs to those bands (default: all nconv)."""
    Hxyz = sysm.Hxyz
    R, E, K, TB = [], [], [], []
    for Z in snaps:
        for kl in range(sysm.nk_local):
            ik = sysm.NK_s + kl
            for b in (range(nconv) if bands is None else bands):
                psi = Z[kl, b]
                hpsi, tpsi = g.hpsi_omp_KB_GS(ik, psi)
                eps = float(np.vdot(psi, hpsi).real * Hxyz)
                r = hpsi - eps * psi
                if np.vdot(r, r).real * Hxyz < 1e-20:
                    continue
                sigma = eps - emin[kl] + margin
                R.append(r)
                E.append(_shifted_solve(g, ik, r, eps - sigma, iters))
                K.append(kl)
                TB.append(float(np.vdot(psi, tpsi).real * Hxyz))
    return np.array(R), np.array(E), np.array(K, np.int32), np.array(TB)


def cg_training_pairs(g, sysm, nconv, snap_at=(10, 20, 40, 60, 80), ncg=4, margin=1.0, bands=None):
    """Runs the reference's plain CG from the loaded ground-state orbitals and
    keeps snapshots of the bands at the iterations in snap_at; the lowest
    eigenvalue of each k-point (for the shift) comes from converging further
    with TPA.  Returns the residual/correction pairs of the snapshots
    (``correction_pairs``)."""
    g.set_cg_preconditioner("plain")
    snaps = []
    for it in range(1, max(snap_at) + 1):
        gs_iteration(g, ncg, nconv)
        if it in snap_at:
            snaps.append(g.gs_get_state())
    g.set_cg_preconditioner("tpa")
    emin = solve_to(g, tol=1e-6, ncg=ncg, max_outer=200, nconv=1)["esp"][:, 0]
    g.set_cg_preconditioner("plain")
    return correction_pairs(g, sysm, snaps, nconv, emin, margin=margin, bands=bands)


def tpa_inputs(g, R, kidx, tband):
    """The network's inputs: the TPA-preconditioned gradients (device tensor)."""
    import torch
    Rd = torch.from_numpy(np.ascontiguousarray(R)).cuda()
    out = torch.empty_like(Rd)
    torch.cuda.synchronize()
    g.tpa_apply(Rd.data_ptr(), out.data_ptr(), R.shape[0], tband, kidx)
    return out


def train(g, X, E, steps=300, batch=16, lr=2e-3, seed=0, log_every=0):
    """Adam training of the loaded network on inputs X (device tensor or complex
    array (n, NL), normally ``tpa_inputs``) and targets E, with the library's
    kernels on the GPU.  Returns the loss history."""
    import torch
    rng = np.random.default_rng(seed)
    R = X
    Rd = X if torch.is_tensor(X) else torch.from_numpy(np.ascontiguousarray(X)).cuda()
    Ed = torch.from_numpy(np.ascontiguousarray(E)).cuda()
    n = Rd.shape[0]
    gb = torch.empty((batch,) + tuple(Rd.shape[1:]), dtype=torch.complex128, device="cuda")
    tb = torch.empty_like(gb)
    hist = []
    for step in range(steps):
        idx = torch.from_numpy(rng.choice(n, size=min(batch, n), replace=False)).cuda()
        m = idx.numel()
        gb[:m] = Rd[idx]
        tb[:m] = Ed[idx]
        torch.cuda.synchronize()
        loss = g.net_train_step(gb.data_ptr(), tb.data_ptr(), m, lr)
        hist.append(loss)
        if log_every and step % log_every == 0:
            print("step", step, "loss", loss, flush=True)
    return hist


def identity_weights(noise: float = 0.0, seed: int = 0):
    """Network weights of the identity map (centre taps: the input feeds channel
    0 of layer 1, layer 2 passes each channel through, layer 3 reads channel 0),
    so the learned refinement starts as TPA itself; optional N(0, noise^2) on
    every weight.  Layout: sgpu_net_weight_count() floats, layer by layer, each
    [co][ci][tap], tap = (dx+1)*9 + (dy+1)*3 + (dz+1)."""
    from .rt import GpuSystem
    C, NTAP = 8, 27
    W1, W2, W3 = (np.zeros(x) for x in ((C, 1, NTAP), (C, C, NTAP), (1, C, NTAP)))
    W1[0, 0, 13] = 1.0
    W3[0, 0, 13] = 1.0
    for c in range(C):
        W2[c, c, 13] = 1.0
    w = np.concatenate([W1.ravel(), W2.ravel(), W3.ravel()])
    if noise:
        w = w + noise * np.random.default_rng(seed).standard_normal(w.size)
    assert w.size == GpuSystem.net_weight_count()
    return w.astype(np.float32)


def cg_cost(g, zu0, weights, tol=1e-8, ncg=4, max_outer=60, nconv=None):
    """The real objective of a preconditioner on one configuration: the CG
    iterations (summed over bands and k-points) that the ground-state sequence
    from the orbitals zu0 needs to bring the lowest nconv bands below the
    residual tol, with the learned preconditioner carrying `weights` (None: TPA
    alone); a run that does not converge in max_outer iterations costs
    twice its iterations."""
    g.gs_set_state(zu0)
    if weights is None:
        g.set_cg_preconditioner("tpa")
    else:
        g.net_set_weights(weights)
        g.set_cg_preconditioner("learned")
    r = solve_to(g, tol=tol, ncg=ncg, max_outer=max_outer, nconv=nconv)
    return r["cg_iterations"] * (1 if r["converged"] else 2)


def train_and_select(g, X, E, variants, validate, seed=0):
    """Trains one network per variant (dict name -> train() keyword arguments)
    from the identity on the inputs X and targets E, and scores each with
    validate(weights) (lower is better; validate(None) scores TPA alone), which
    should run CG on a configuration held out from the training data
    (cg_cost).  The best network is kept only if it scores below TPA; otherwise
    the identity weights are returned, so the learned preconditioner falls back
    to TPA and is not worse than it on the validation configuration.
    Returns (weights, report {name: (final loss, score)}, chosen name)."""
    report = {"tpa": (None, validate(None))}
    report["identity"] = report["tpa"]  # the identity network is TPA alone
    best_name, best_w, best_score = "identity", identity_weights(), report["tpa"][1]
    for name, kw in variants.items():
        g.net_set_weights(identity_weights(noise=1e-2, seed=seed))
        hist = train(g, X, E, seed=seed, **kw)
        w = g.net_get_weights()
        score = validate(w)
        report[name] = (float(np.mean(hist[-20:])), score)
        if score < best_score:
            best_name, best_w, best_score = name, w, score
    return best_w, report, best_name


DEFAULT_VARIANTS = {"short": dict(steps=100, lr=5e-4, batch=16), "mid": dict(steps=200, lr=1e-3, batch=16),
                    "long": dict(steps=400, lr=2e-3, batch=16)}
