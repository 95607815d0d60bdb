"""The step tuner (sgpu_autotune_step) and the launch-shape table
(salmon_b200/tune.py): tuning leaves the resident orbitals untouched, the chosen
launch shapes give the same Taylor step as the oracle (1e-12 complex(8),
2e-6 complex(4)), and a second handle of the same shape takes its choice from
the table without tuning."""
import numpy as np
import pytest

from _helpers import rel
from oracle import oracle as O
from salmon_b200 import system as S, tune

pytestmark = pytest.mark.gpu
TOL = {"c128": 1e-12, "c64": 2e-6}


@pytest.mark.parametrize("shape", ["16", "20x32"])
@pytest.mark.parametrize("precision", ["c128", "c64"])
def test_step_tuner_and_table(cuda_lib, tmp_path, precision, shape):
    from salmon_b200.rt import GpuSystem
    if shape == "16":
        sysm, kAc, vloc, zu = S.si_supercell_system((1, 1, 1), (16, 16, 16), (2, 2, 1), 8, A=(1e-2, 0.0, 0.0))
    else:
        sysm, kAc, vloc, zu = S.microbench_system(20, nk_limit=2, Nb=32)
    path = str(tmp_path / "table.json")
    _, zproj = O.update_projector(sysm, kAc)
    z_in = zu if precision == "c128" else zu.astype(np.complex64).astype(np.complex128)
    z_ref = O.hamiltonian(sysm, kAc, vloc, zproj, 0.08, z_in)
    chosen = None
    for attempt in ("tuned", "table"):
        with GpuSystem(sysm, precision) as g:
            g.set_state(zu)
            g.set_vloc(vloc)
            g.update_projector(kAc)
            entry, source = tune.apply(g, sysm, precision, path=path, reps=2)
            assert source == attempt
            if chosen is None:
                chosen = entry["params"]
                assert entry["ms_per_step"] > 0
                np.testing.assert_array_equal(g.get_state(), z_in)   # tuning ran on a copy
            for p, v in chosen.items():
                assert g.get_param(p) == v
            g.hamiltonian(0.08)
            assert rel(g.get_state(), z_ref) < TOL[precision]
