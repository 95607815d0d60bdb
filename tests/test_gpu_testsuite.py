"""SALMON's bulk-Si testsuites end to end on the GPU, against the reference's own
verification tables (testsuites/001_bulk_gs/verification, 002_bulk_rt/verification,
stored in tests/golden/testsuite_si.json).

001_bulk_gs: diamond Si, 8 atoms, a = 10.26 bohr, 8^3 grid, 4^3 k-points, 32 bands
(16 occupied), the KY pseudopotential testsuites/pseudo/Si_rps.dat with lloc = 2, PZ
LDA, ncg = 5, Broyden mixing, nscf = 100 iterations.  Checked: eigenvalues of
bands 15-18 at ik = 1 and 64 (tolerance 1e-3 Ha, the reference's).
002_bulk_rt: from that ground state, 1200 middle-point Taylor steps of dt = 0.1 under
an Acos2 pulse (1e12 W/cm^2, 110.3 au, omega 0.05696 Ha, z polarised) with the
self-consistent Hartree + PZ potential rebuilt every step.  Checked: Jm_z at t = 60 and
120 au and the excitation energy Eall - Eall0 at t = 60 and 120 au (tolerances of the
reference's table), for complex(8) orbitals and for complex(4) orbitals with FP64
reductions.
"""
import json
import os

import numpy as np
import pytest

from _helpers import GOLDEN
from salmon_b200 import drive, outputs as OUT, pseudo as P, system as S

pytestmark = pytest.mark.gpu


def _suite():
    with open(os.path.join(GOLDEN, "testsuite_si.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def ground_state(cuda_lib):
    from salmon_b200.rt import GpuSystem
    suite = _suite()
    inp = suite["inputs"]
    tabs = P.prepare(P.from_npz(os.path.join(GOLDEN, "si_rps_ky.npz"), lloc=inp["lloc_ps"]))
    sysm, kAc0, vpsl, zu0 = S.si_pp_system(tabs, grid=tuple(inp["num_rgrid"]), nkgrid=tuple(inp["num_kgrid"]),
                                           NB=inp["nstate"], Nocc=inp["nelec"] // 2)
    with GpuSystem(sysm, "c128") as g:
        g.gs_set_state(zu0)
        esp, hist = drive.gs_scf(g, sysm, kAc0, vpsl, nscf=inp["nscf"], ncg=inp["ncg"],
                                 threshold=inp["threshold"])
        zu_gs = g.gs_get_state()
    return suite, sysm, kAc0, vpsl, esp, hist, zu_gs


def _check_table(table, folder, tag=""):
    """The reference's verification rule on the files a run wrote: np.loadtxt of
    each file, the value at (row, col) within the tolerance."""
    data = {}
    for r in table:
        if r["file"] not in data:
            data[r["file"]] = np.loadtxt(os.path.join(folder, r["file"]))
        got = data[r["file"]][r["row"], r["col"]]
        print(f"{tag}{r['label']}: {got:+.6e} (ref {r['value']:+.4e}, tol {r['tol']:.0e})")
        assert abs(got - r["value"]) <= r["tol"], (tag, r["label"], got)


def test_gs_eigenvalues_match_001(ground_state, tmp_path):
    suite, sysm, kAc0, vpsl, esp, hist, zu = ground_state
    # Bands 16 (occupied) and 17 (empty) lie within 1e-3 Ha of each other at several
    # k-points, so with occupations fixed by band index the density keeps swapping
    # between them and ddns stalls near 1e-2 (the CPU oracle's exact-diagonalisation
    # SCF does the same); the reference's table checks the eigenvalues after its
    # nscf = 100 iterations, and so does this test.
    print("SCF iterations", len(hist), "ddns of the last five", [f"{h[0]:.2e}" for h in hist[-5:]])
    bl = 2 * np.pi / sysm.aL
    OUT.write_k_data(str(tmp_path / "Si_k.data"), kAc0, bl)
    OUT.write_eigen_data(str(tmp_path / "Si_eigen.data"), np.sort(esp, axis=1), sysm.occ, sysm.NK)
    _check_table(suite["001_bulk_gs"], str(tmp_path))


@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_rt_current_and_energy_match_002(ground_state, precision, tmp_path):
    """002_bulk_rt starts from the orbital files 001 wrote: the ground state goes
    through gs_wfn_k/ (SALMON's unformatted layout) and is read back."""
    _run_002(ground_state, precision, tmp_path, "middlepoint")


def test_rt_etrs_matches_002(ground_state, tmp_path):
    """The same run with propagator = 'etrs' (RT/dt_evolve.f90:218-348) in place
    of the input's middle point: the table's rows hold within its tolerances."""
    _run_002(ground_state, "c128", tmp_path, "etrs")


def _run_002(ground_state, precision, tmp_path, propagator):
    from salmon_b200 import wfn_io
    from salmon_b200.rt import GpuSystem
    suite, sysm, kAc0, vpsl, esp, hist, zu_gs = ground_state
    wfn_io.write_gs_wfn_k(str(tmp_path), zu_gs, sysm.occ)
    zu_read, occ = wfn_io.read_gs_wfn_k(str(tmp_path), sysm.NK, sysm.NB, sysm.NL)
    assert np.array_equal(occ, sysm.occ)
    zu = np.ascontiguousarray(zu_read[:, :sysm.NBoccmax])   # zu_t = zu_GS(:,1:NBoccmax,:) (io_gs_wfn_k.f90:67)
    eion = P.ewald_energy(sysm.Rion, sysm.extra["zps"], sysm.aL, (sysm.NLx, sysm.NLy, sysm.NLz))
    inp = suite["inputs"]
    dt, nt = inp["dt"], inp["nt"]
    # one step past nt: the energy row of step it is taken after that step (control_sc.f90:203-231)
    Ac = drive.init_Ac(nt + 1, dt, "Acos2", epdir=inp["epdir_re1"], rlaser_int_wcm2=inp["rlaser_int_wcm2_1"],
                       omega=inp["omega1"], pulse_tw=inp["pulse_tw1"])
    with GpuSystem(sysm, precision) as g:
        g.set_state(zu)
        javt, energies = drive.rt_propagate(g, sysm, kAc0, vpsl, Ac, dt, nt + 1, energy_every=1, scf=True,
                                            eion=eion, propagator=propagator)
    # the rows as control_sc.f90 writes them: A and E = -dA/dt at step iter (transverse
    # geometry: total = external), J after step iter-1, and Eall_t(iter) = the energy
    # after step iter plus the field energy aLxyz |E|^2 / (8 pi)
    E = OUT.fields_from_Ac(Ac, dt)
    A = Ac[1:]
    eall_t = {it: energies[it + 1] + sysm.aLxyz * float(E[it] @ E[it]) / (8 * np.pi) for it in range(nt + 1)}
    OUT.write_rt_data(str(tmp_path / "Si_rt.data"), dt, A, E, A, E, javt, nt)
    OUT.write_rt_energy_data(str(tmp_path / "Si_rt_energy.data"), dt, eall_t, energies[0], nt)
    _check_table(suite["002_bulk_rt"], str(tmp_path), tag=f"{precision} {propagator} ")
