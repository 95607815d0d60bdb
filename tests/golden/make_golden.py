"""Generates the golden fixtures of tests/golden from SALMON's own code.

Run where the reference tree is present (it builds oracle/_ref from the
reference's AVX sources with oracle/Makefile):

    python tests/golden/make_golden.py

Outputs (small .npz files, committed):
  ref_stencil_<NLx>x<NLy>x<NLz>.npz   hpsi1_rt_stencil_ (stencil/C/AVX/hpsi.c) on seeded inputs
  ref_current_stencil.npz             current_stencil_ (stencil/C/AVX/current.c)
  ref_total_energy_stencil.npz        total_energy_stencil_ (stencil/C/AVX/total_energy.c)
  ref_taylor_step.npz                 one hamiltonian() Taylor step driven by the AVX stencil
                                      (oracle/ref_driver.c), with every input array stored
Inputs are stored next to the outputs so the fixtures do not depend on the
random generator of a later numpy.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from salmon_b200 import system as S  # noqa: E402


def coefs(sysm, k):
    ln = sysm.lap_nab()
    lapt = np.concatenate([ln["lapx"][1:], ln["lapy"][1:], ln["lapz"][1:]])
    nab = np.concatenate([ln["nabx"][1:], ln["naby"][1:], ln["nabz"][1:]])
    nabt = np.concatenate([k[0] * ln["nabx"][1:], k[1] * ln["naby"][1:], k[2] * ln["nabz"][1:]])
    A = (k @ k - (ln["lapx"][0] + ln["lapy"][0] + ln["lapz"][0])) * 0.5
    lap0_2 = -(ln["lapx"][0] + ln["lapy"][0] + ln["lapz"][0]) * 0.5
    return lapt, nab, nabt, A, lap0_2


def system_arrays(sysm):
    return dict(NL=np.array([sysm.NLx, sysm.NLy, sysm.NLz]), aL=sysm.aL, kAc0=sysm.kAc0, occ=sysm.occ,
                Mps=sysm.Mps, Jxyz=sysm.Jxyz, Jxx=sysm.Jxx, Jyy=sysm.Jyy, Jzz=sysm.Jzz, uV=sysm.uV, iuV=sysm.iuV,
                a_tbl=sysm.a_tbl, Rion=sysm.Rion, Rps=np.array(sysm.Rps), NB=np.array([sysm.NB, sysm.NBoccmax]))


def main():
    O.build()
    if not O.ref_available():
        raise SystemExit("oracle/_ref was not built: the reference tree is needed")
    for shape, seed in (((8, 10, 12), 11), ((16, 16, 16), 12)):
        sysm, kAc, vloc, zu = S.small_system(*shape, nk=2, nb=2, seed=seed)
        lapt, nab, nabt, A, _ = coefs(sysm, kAc[:, 1])
        E = zu[1, 1]
        F = O.ref_stencil(sysm, A, vloc, lapt, nabt, E)
        np.savez_compressed(os.path.join(HERE, "ref_stencil_%dx%dx%d.npz" % shape), shape=np.array(shape), A=A,
                            B=vloc, C=lapt, D=nabt, E=E, F=F)
    sysm, kAc, vloc, zu = S.small_system(8, 10, 12, nk=2, nb=2, seed=13)
    lapt, nab, nabt, A, lap0_2 = coefs(sysm, kAc[:, 0])
    E = zu[0, 1]
    fgh = O.ref_current_stencil(sysm, nab, E)
    np.savez_compressed(os.path.join(HERE, "ref_current_stencil.npz"), shape=np.array([8, 10, 12]), C=nab, E=E,
                        FGH=fgh)
    tp = O.ref_total_energy_stencil(sysm, lap0_2, lapt, nabt, E)
    np.savez_compressed(os.path.join(HERE, "ref_total_energy_stencil.npz"), shape=np.array([8, 10, 12]), A=lap0_2,
                        C=lapt, D=nabt, E=E, F=np.array([tp]))
    sysm, kAc, vloc, zu = S.small_system(8, 10, 12, nk=2, nb=3, seed=14)
    _, zproj = O.update_projector(sysm, kAc)
    dt = 0.05
    za = O.aligned_state(zu)
    O.ref_hamiltonian(sysm, kAc, vloc, zproj, dt, za)
    np.savez_compressed(os.path.join(HERE, "ref_taylor_step.npz"), kAc=kAc, vloc=vloc, zu=zu, dt=dt, zu_next=np.array(za),
                        **system_arrays(sysm))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
