"""Unfolding unit-cell Bloch states onto a supercell (system.folded_kpoints,
system.unfold_to_supercell), the construction of the Si216 workload's starting
state.  For a perfect crystal the unit-cell eigenstate at k_u = k_s + m b_s,
tiled and multiplied by exp(i m b_s . r), is an eigenstate of the supercell
Hamiltonian at k_s in the continuum.  On the grid it is exact for m = 0; for
m != 0 it is exact only to the finite-difference error of SALMON's k+A
treatment (hpsi.f90:120-124 adds k through -i k.nab and |k|^2/2, which is not
the grid conjugation of the k = 0 stencil by exp(i q r)): O((q h)^2), so the
residual falls with the grid spacing.  Checked with the CPU oracle's hpsi on
the physical Si pseudopotential."""
import os

import numpy as np

from _helpers import GOLDEN
from oracle import oracle as O
from salmon_b200 import pseudo as P, system as S


def _unfold_case(g):
    import torch
    tabs = P.prepare(P.from_npz(os.path.join(GOLDEN, "si_rps_ky.npz"), lloc=2))
    ncell = (2, 1, 1)
    big, kS, vpsl_b, _ = S.si_pp_system(tabs, ncell=ncell, grid=(2 * g, g, g), nkgrid=(1, 1, 1), NB=2, Nocc=2,
                                        with_orbitals=False)
    kU, ms = S.folded_kpoints(kS, ncell, big.aL)
    assert kU.shape[1] == 2 and np.allclose(kU[:, 1] - kU[:, 0], [2 * np.pi / big.aL[0], 0, 0])
    cell, _, vpsl_c, _ = S.si_pp_system(tabs, grid=(g, g, g), NB=1, Nocc=1, kpoints=kU, with_orbitals=False)
    _, zp_c = O.update_projector(cell, kU)
    NL = cell.NL
    eye = np.eye(NL, dtype=np.complex128)
    zu = np.zeros((2, 1, NL), np.complex128)
    eps = np.zeros(2)
    for ik in range(2):  # the exact lowest eigenpair of the unit-cell H(k_u) on the grid
        Hm = np.array([O.hpsi(cell, kU, vpsl_c, zp_c, ik + 1, eye[j]) for j in range(NL)]).T
        w, v = np.linalg.eigh(0.5 * (Hm + Hm.conj().T))
        eps[ik] = w[0]
        zu[ik, 0] = v[:, 0] / np.sqrt(cell.Hxyz)
    zs = S.unfold_to_supercell(torch.from_numpy(zu), ncell, ms, 1, (g, g, g)).numpy()[0]
    _, zp_b = O.update_projector(big, kS)
    res = []
    for j in range(2):
        u = zs[j]
        assert abs(np.vdot(u, u).real * big.Hxyz - 1.0) < 1e-12          # normalised on the supercell
        hu = O.hpsi(big, kS, vpsl_b, zp_b, 1, u)
        res.append(np.abs(hu - eps[j] * u).max() / np.abs(u).max())
    assert abs(np.vdot(zs[0], zs[1]) * big.Hxyz) < 1e-12                # different k_u: orthogonal
    return res


def test_unfolded_states_are_supercell_eigenstates_to_the_grid_error():
    r8 = _unfold_case(8)
    r12 = _unfold_case(12)
    assert r8[0] < 1e-12 and r12[0] < 1e-12           # m = 0: exact
    assert r12[1] < 0.3 * r8[1] and r12[1] < 1e-2     # m != 0: the FD k+A error, falling with h
