"""Output files in the reference's layout (salmon_b200/outputs.py) and the
Fourier-transform spectra, on the CPU."""
import json
import os

import numpy as np

from _helpers import GOLDEN
from salmon_b200 import drive, outputs as W, system as S


def test_fortran_edit_descriptors():
    assert W.fortran_e(-0.025062) == " -0.250620000000000E-001"[1:].rjust(23)
    assert W.fortran_e(1.0) == "  0.100000000000000E+001"[1:].rjust(23)
    assert W.fortran_e(0.0) == "0.000000000000000E+000".rjust(23)
    assert W.fortran_e(0.5) == "0.500000000000000E+000".rjust(23)
    assert W.fortran_e(9.9999999999999999e-3).strip() == "0.100000000000000E-001"
    assert W.fortran_e(123.456) == "0.123456000000000E+003".rjust(23)
    assert W.fortran_f(60.0) == "     60.00000000"
    for v in (3.3138e-2, -4.6521e-4, 1.7546e-4, 2.0, -36.92215):
        assert float(W.fortran_e(v)) == float(f"{v:.15e}")


def test_k_and_eigen_files_match_001_layout(tmp_path):
    with open(os.path.join(GOLDEN, "testsuite_si.json")) as f:
        suite = json.load(f)
    bl = 2 * np.pi / np.asarray(suite["inputs"]["al"])
    k = S.uniform_k_grid(4, 4, 4, bl)
    W.write_k_data(str(tmp_path / "Si_k.data"), k, bl)
    occ = np.zeros((64, 32))
    occ[:, :16] = 2.0 / 64
    esp = np.tile(np.linspace(-0.2, 0.4, 32), (64, 1))
    W.write_eigen_data(str(tmp_path / "Si_eigen.data"), esp, occ, 64)
    data = {name: np.loadtxt(str(tmp_path / name)) for name in ("Si_k.data", "Si_eigen.data")}
    assert data["Si_eigen.data"].shape == (64 * 32, 4)
    for r in suite["001_bulk_gs"]:
        if r["file"] == "Si_eigen.data" and r["col"] == 2:
            continue                                     # eigenvalues: the GPU test
        got = data[r["file"]][r["row"], r["col"]]
        assert abs(got - r["value"]) <= r["tol"], r["label"]


def test_rt_files_and_pulse_rows(tmp_path):
    with open(os.path.join(GOLDEN, "testsuite_si.json")) as f:
        suite = json.load(f)
    inp = suite["inputs"]
    dt, nt = inp["dt"], inp["nt"]
    Ac = drive.init_Ac(nt + 1, dt, "Acos2", epdir=inp["epdir_re1"], rlaser_int_wcm2=inp["rlaser_int_wcm2_1"],
                       omega=inp["omega1"], pulse_tw=inp["pulse_tw1"])
    E = W.fields_from_Ac(Ac, dt)                         # E(iter), iter = 0..nt+1
    A = Ac[1:]                                           # A(iter), iter = 0..nt+2
    javt = np.zeros((nt + 1, 3))
    W.write_rt_data(str(tmp_path / "Si_rt.data"), dt, A, E, A, E, javt, nt)
    W.write_rt_energy_data(str(tmp_path / "Si_rt_energy.data"), dt, {i: 0.01 * i for i in range(nt + 1)}, 0.0, nt)
    d = np.loadtxt(str(tmp_path / "Si_rt.data"))
    assert d.shape == (nt + 1, 16) and abs(d[600, 0] - 60.0) < 1e-12
    for r in suite["002_bulk_rt"]:
        if r["file"] == "Si_rt.data" and r["col"] in (9, 12):   # Ac_tot_z, E_tot_z
            assert abs(d[r["row"], r["col"]] - r["value"]) <= r["tol"], r["label"]
    e = np.loadtxt(str(tmp_path / "Si_rt_energy.data"))
    assert e.shape == (nt // 10 + 1, 3) and abs(e[60, 0] - 60.0) < 1e-12 and abs(e[60, 2] - 6.0) < 1e-12


def test_fourier_tr_of_a_damped_oscillation():
    """sigma(w) of an impulse response J(t) = dAc s0 g e^{-g t} cos(w0 t) (a Drude-
    like line at w0): Re sigma peaks at w0; the vectorised transform equals the
    reference's loop form; eps = 1 + 4 pi i sigma / w."""
    dt, nt, w0, g, dAc = 0.08, 2000, 0.3, 0.02, 1e-3
    tt = np.arange(nt + 1) * dt
    j = np.zeros((nt + 1, 3))
    j[:, 0] = dAc * 0.05 * np.exp(-g * tt) * np.cos(w0 * tt)
    zero = np.zeros((nt + 1, 3))
    spec = W.fourier_tr(j, zero, zero, dt, nt, 200, 0.005, dAc=dAc, insulator=False)
    hw = spec["hw"]
    assert abs(hw[np.argmax(spec["sigma"][:, 0].real)] - w0) <= 0.005
    # loop form (Fourier_tr.f90:78-83) at three frequencies
    for i in (10, 59, 150):
        acc = 0j
        for it in range(nt + 1):
            acc += j[it, 0] * np.exp(1j * hw[i] * it * dt) * W.smoothing_t(it * dt, nt, dt)
        assert abs(acc * dt / dAc - spec["sigma"][i, 0]) <= 1e-12 * abs(acc * dt / dAc)
    assert np.allclose(spec["eps"][:, 0], 1 + 4j * np.pi * spec["sigma"][:, 0] / hw)
    lo = W.fourier_tr(j, zero, j, dt, nt, 5, 0.1, trans_longi="lo", dAc=dAc, insulator=False)
    assert np.allclose(lo["eps"], 1.0 / (1.0 - lo["E_tot_w"] / dAc))
