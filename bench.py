#!/usr/bin/env python
"""RT orbital-updates/s of SALMON's 4th-order Taylor step on B200.

Workload: the hpsi/Taylor operator microbench (cubic Si-like cell a=10.26 bohr,
grid 32^3 by default, 4x4x4 = 64 k-points, 32 bands, 8 atoms x {s,p} Gaussian
Kleinman-Bylander projectors, seeded synthetic orbitals and V_loc).  A step is
one Taylor step of every orbital (4 H applications, each with its stage update).  Both orbital
precisions run: complex(8) (FP64) and complex(4) orbitals with FP64
reductions.  The headline `value` is the complex(4) path; the FP64 path is
reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--grid 32] [--impl reference]

Under torchrun (N>1) every rank propagates its own k-block of the same shape
(weak scaling: fixed work per GPU, no collective in the timed Taylor loop; the
end-to-end leg allreduces rho and J over NCCL like the reference's
comm_summation).  Times are CUDA events on the library's stream, max over ranks.
Inputs are larger than L2 (126 MB) at every pass, so no L2 flush is inserted.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RT orbital-updates/s: FP32+FP64-reduce vs FP64 GPU at ΔJ<1e-5; hpsi %HBM peak"
DT = 0.08
# ncu dram__bytes_read.sum + dram__bytes_write.sum of one Taylor-stage launch, per
# orbital, from the capture in profiles/k_hpsi_pass_stage_c64_32cubed_864orb.md
# (864 orbitals; traffic grows with the orbital count).
NCU_TRAFFIC_BYTES_PER_ORBITAL = {("taylor_stage", "c64", 32): 534.936064e6 / 864}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--grid", type=int, default=32)
    p.add_argument("--nkgrid", type=int, default=4)
    p.add_argument("--nb", type=int, default=32)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--only", choices=["c128", "c64"], help="run one precision (profiling)")
    p.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling)")
    p.add_argument("--no-precision", action="store_true", help="skip the FP32-vs-FP64 J(t) run")
    p.add_argument("--no-batched", action="store_true", help="skip the batched-systems run")
    p.add_argument("--batched-steps", type=int, default=1000)
    p.add_argument("--no-large", action="store_true", help="skip the Si216 48^3 run")
    p.add_argument("--precond", action="store_true", help="also run the Si64 CG preconditioner comparison (minutes)")
    p.add_argument("--no-precond", action="store_true", help="skip the Si8 CG preconditioner comparison")
    p.add_argument("--pass-fixed", type=int, default=1, choices=[0, 1],
                   help="stencil pass of the main leg: 1 compile-time plane shapes where they apply, 0 the generic kernel")
    p.add_argument("--profile-current", action="store_true",
                   help="profiling: one complex(4) Taylor step of the workload, then two sgpu_current calls, and exit")
    p.add_argument("--taylor-kernel", type=int, default=0, choices=[0, 1, 2],
                   help="Taylor step of the main leg: 0 by grid, 1 stencil passes, 2 shared-memory resident")
    p.add_argument("--no-si8", action="store_true", help="skip the Si8 16^3 resident-vs-passes leg")
    p.add_argument("--config5-check", type=int, default=0, metavar="STEPS",
                   help="steps of the complex(8) run the config-5 J(t) is checked against (default: all)")
    p.add_argument("--config5", type=int, default=0, metavar="STEPS",
                   help="also run the Si216 pulsed RT workload for STEPS steps (minutes; 5000 as configured)")
    p.add_argument("--kb-kernel", type=int, default=0, choices=[0, 1, 2, 3],
                   help="KB term kernel of the main leg: 0 by grid size, 1 band-group tile, 2 band-quad, "
                        "3 split projections + point-parallel field (profiling)")
    return p.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get("hbm_gbs", 6650.0), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def make_workload(args, rank, world=1):
    """The microbench system on a k-grid of nkgrid x nkgrid x (nkgrid * world)
    points, sharded over the ranks by the reference's k partition (each rank
    gets nkgrid^3 k-points: weak scaling); the orbitals of the rank's block only."""
    from salmon_b200 import dist as D, system as S
    nk = args.nkgrid
    sysm, kAc, vloc, _ = S.microbench_system(args.grid, nkgrid=(nk, nk, nk * world), Nb=args.nb, with_orbitals=False)
    loc = D.local_system(sysm, rank, world)
    rng = np.random.default_rng(S.SEED + rank)
    shape = (loc.nk_local, args.nb, loc.NL)
    zu = S.orthonormalise(rng.standard_normal(shape) + 1j * rng.standard_normal(shape), loc.Hxyz)
    return loc, kAc, vloc, zu


def cpu_baseline(sysm, kAc, vloc, zu, seconds):
    """SALMON's own AVX stencil (compiled from the reference tree into oracle/_ref)
    driving the Taylor step like RT/hamiltonian.f90, on all host cores, over a
    bounded sample of the workload's orbitals."""
    from oracle import oracle as O
    if not O.ref_available():
        return None
    _, zproj = O.update_projector(sysm, kAc)
    nthreads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    chunk = max(nthreads * 4, 16)
    # sample: the orbitals of the first k-points (at least `chunk` of them), propagated repeatedly
    from salmon_b200 import system as S
    sub = S.System(**{**{k: getattr(sysm, k) for k in ("NLx", "NLy", "NLz", "aL", "kAc0", "NB", "NBoccmax", "occ",
                                                       "Rion", "Rps", "Mps", "Jxyz", "Jxx", "Jyy", "Jzz", "uV",
                                                       "iuV", "a_tbl")}})
    nkl = max(1, chunk // sysm.NBoccmax)
    sub.NK_s, sub.NK_e = 1, nkl
    za = O.aligned_state(zu[:nkl])
    _, zp = O.update_projector(sub, kAc)
    O.ref_hamiltonian(sub, kAc, vloc, zp, DT, za, nthreads=nthreads)  # warm-up
    n = 0
    t0 = time.perf_counter()
    while True:
        O.ref_hamiltonian(sub, kAc, vloc, zp, DT, za, nthreads=nthreads)
        n += nkl * sysm.NBoccmax
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return {"value": n / el, "unit": "orbital-updates/s", "cores": nthreads, "kind": "reference",
            "sample": f"{nkl * sysm.NBoccmax} orbitals of the {sysm.NLx}^3 workload x {n // (nkl * sysm.NBoccmax)} "
                      f"Taylor steps ({el:.1f} s); SALMON AVX hpsi1_rt_stencil_ + restated pseudo_pt/update, "
                      f"OpenMP over orbitals, complex(8)"}


def precision_check(nsteps=500):
    """J(t) of the complex(4) path against the complex(8) path on the Si8 RT
    shape: 16^3 grid, 4x4x4 k, 16 occupied bands (+4 empty in the ground
    state), self-consistent LDA potential (Hartree + PZ on the device).  Ground
    state by SCF with TPA-preconditioned CG, then an impulsive kick A_x = 1e-3
    and `nsteps` middle-point Taylor steps of dt = 0.08 with Vloc rebuilt from
    the density after every step; J after each step (FP64 reductions)."""
    from salmon_b200 import drive, system as S
    from salmon_b200.rt import GpuSystem
    sysm, _, vpsl, zu = S.si_supercell_system((1, 1, 1), (16, 16, 16), (4, 4, 4), Nb=20, Nocc=16)
    kAc0 = np.ascontiguousarray(sysm.kAc0)
    with GpuSystem(sysm) as g:
        g.set_vpsl(vpsl)
        g.set_vloc(vpsl)
        g.update_projector(kAc0)
        g.gs_set_state(zu)
        g.set_state(zu[:, :sysm.NBoccmax])
        g.update_vloc()
        g.set_cg_preconditioner("tpa")
        _, hist = drive.ground_state_scf(g, n_iter=60, ncg=4, mix=0.2)
        zgs = g.gs_get_state()
    Ac = drive.init_Ac(nsteps, DT, "impulse", epdir=(1.0, 0.0, 0.0), e_impulse=1e-3)
    out = {}
    for prec in ("c128", "c64"):
        with GpuSystem(sysm, "c128") as g:
            g.set_vloc(vpsl)
            g.update_projector(kAc0)
            g.gs_set_state(zgs)
            g.gs_to_rt()
            if prec == "c64":
                g.set_precision("c64")
            out[prec] = drive.rt_propagate(g, sysm, kAc0, vpsl, Ac, DT, nsteps, energy_every=50, scf=True)
    (j64, e64), (j32, e32) = out["c128"], out["c64"]
    de = max(abs((e32[t] - e32[0]) - (e64[t] - e64[0])) for t in e64)
    return {"j_rel_err": drive.j_error(j64, j32), "j_dyn_rel_err": drive.j_error_dynamic(j64, j32),
            "max_abs_j_fp64": float(np.abs(j64).max()), "energy_change_abs_diff_ha": de,
            "energy_drift_fp64_ha": float(e64[nsteps] - e64[0]), "gs_scf_drho": hist[-1][2],
            "gs_max_residual": hist[-1][1],
            "workload": f"Si8 16^3, 64 k x 16 occupied bands, LDA (PZ) + Hartree self-consistent, impulse "
                        f"A_x=1e-3, dt={DT}, {nsteps} steps, J every step (FP64 reductions)", "target": 1e-5}


def batched_bench(nsteps=1000, per_replay=10):
    """Si8 (16^3, 64 k x 16 b), Si16 (16x16x32, 32 k x 32 b) and Si64 (32^3, 8 k x
    128 b) in complex(4), launch shapes autotuned per system, advanced together by
    graph replays of `per_replay` Taylor steps; beside it the same systems stepped
    one sgpu_hamiltonian call at a time."""
    import torch
    from salmon_b200 import system as S, tune
    from salmon_b200.rt import GpuBatch, GpuSystem
    gs, tuned, norb = [], {}, 0
    for name, (cells, grid, nkg, nb) in S.BATCHED_SYSTEMS.items():
        sysm, kAc, vloc, zu = S.si_supercell_system(cells, grid, nkg, nb, A=(1e-2, 0.0, 0.0))
        g = GpuSystem(sysm, "c64")
        g.set_state(zu)
        g.set_vloc(vloc)
        g.update_projector(kAc)
        entry, source = tune.apply(g, sysm, "c64", write=False)  # the launch-shape table (tuned if absent)
        tuned[name] = {"params": entry["params"], "from": source, "norb": sysm.nk_local * nb, "grid": list(grid)}
        norb += sysm.nk_local * nb
        gs.append(g)
    dts = [DT] * len(gs)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with GpuBatch(gs) as b:
        st = torch.cuda.ExternalStream(b.stream)
        for _ in range(3):
            b.step(dts, per_replay)
        for g in gs:
            g.synchronize()
        torch.cuda.synchronize()
        reps = max(1, nsteps // per_replay)
        e0.record(st)
        for _ in range(reps):
            b.step(dts, per_replay)
        e1.record(st)
        e1.synchronize()
        ms_graph = e0.elapsed_time(e1) / (reps * per_replay)
    # one call at a time, same systems and shapes (host wall clock after a sync)
    nseq = max(10, nsteps // 10)
    for g in gs:
        g.synchronize()
    t0 = time.perf_counter()
    for _ in range(nseq):
        for g in gs:
            g.hamiltonian(DT)
    for g in gs:
        g.synchronize()
    ms_seq = (time.perf_counter() - t0) * 1e3 / nseq
    for g in gs:
        g.close()
    return {"value": norb / (ms_graph * 1e-3), "unit": "orbital-updates/s", "ms_per_step": ms_graph,
            "steps": reps * per_replay, "steps_per_graph_replay": per_replay,
            "sequential_ms_per_step": ms_seq, "graph_speedup": ms_seq / ms_graph, "systems": tuned,
            "workload": "Si8 16^3 64k x16b + Si16 16x16x32 32k x32b + Si64 32^3 8k x128b, complex(4), "
                        "synthetic Gaussian projectors / V_loc"}


def large_bench(nsteps=10):
    """The Si216 RT shape: 3x3x3 diamond supercell, 48^3 grid (planes split into
    y-blocks), 2x2x1 = 4 k-points, 432 bands (1728 orbitals); seeded random
    orbitals made on the device; Taylor-step throughput in complex(4) (launch
    shapes autotuned) and complex(8)."""
    import torch
    from salmon_b200 import system as S, tune
    from salmon_b200.rt import GpuSystem
    sysm, kAc, vloc, _ = S.si_supercell_system((3, 3, 3), (48, 48, 48), (2, 2, 1), 432, with_orbitals=False)
    norb = sysm.nk_local * sysm.NBoccmax
    gen = torch.Generator(device="cuda").manual_seed(S.SEED)
    z = torch.randn((norb, sysm.NL), dtype=torch.complex128, device="cuda", generator=gen) / np.sqrt(sysm.NL * sysm.Hxyz)
    out = {"workload": "Si216 48^3, 4 k x 432 bands (1728 orbitals), synthetic Gaussian projectors / V_loc"}
    for prec in ("c64", "c128"):
        g = GpuSystem(sysm, prec)
        torch.cuda.synchronize()
        g.set_state_dev(z.data_ptr())
        g.set_vloc(vloc)
        g.update_projector(kAc)
        tuned = tune.apply(g, sysm, prec, write=False)
        st = torch.cuda.ExternalStream(g.stream)
        for _ in range(2):
            g.hamiltonian(DT)
        g.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(nsteps):
            g.hamiltonian(DT)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / nsteps
        out[prec] = {"ms_per_step": ms, "orbital_updates_per_s": norb / (ms * 1e-3),
                     "stencil_pass_ms": g.time_kernel("stencil_pass", reps=3)}
        out[prec]["tuned"] = {"params": tuned[0]["params"], "from": tuned[1]}
        g.close()
    del z
    out["fp32_over_fp64"] = out["c64"]["orbital_updates_per_s"] / out["c128"]["orbital_updates_per_s"]
    return out


PRECOND_SHAPES = {
    # the configured Si64 ground state: 2x2x2 diamond supercell, 32^3 grid, 2x2x2
    # k-points, 128 occupied + 16 empty bands (minutes: bench.py --precond)
    "Si64": dict(base=dict(ncell=(2, 2, 2), grid=(32, 32, 32), nkgrid=(2, 2, 2), Nb=144, Nocc=128), nconv=128,
                 seeds=(101, 303, 202), pairs=dict(snap_at=(10, 20, 40), bands=(0, 31, 63, 95, 127)), max_outer=60),
    # the same comparison on the Si8 cell (16^3, 2 k-points, 8 + 4 bands): seconds,
    # in every bench run
    "Si8": dict(base=dict(ncell=(1, 1, 1), grid=(16, 16, 16), nkgrid=(2, 1, 1), Nb=12), nconv=8,
                seeds=(11, 13, 12), pairs=dict(), max_outer=100),
}


def precond_bench(shape="Si64"):
    """CG to a 1e-8 residual on a ground-state shape (PRECOND_SHAPES, fixed V_loc,
    FP64): the learned preconditioner, trained on residual/correction pairs from
    plain CG on one displaced configuration (sigma = 0.05 bohr) and selected by
    CG cost on a second (held out; TPA alone is the fallback), evaluated on a third
    against TPA alone and plain CG (each capped at the shape's outer iterations)."""
    from salmon_b200 import precond as P
    from salmon_b200.rt import GpuSystem
    cfg = PRECOND_SHAPES[shape]
    base, nconv, max_outer = cfg["base"], cfg["nconv"], cfg["max_outer"]
    s_train, s_val, s_eval = cfg["seeds"]

    def gpu(seed):
        sysm, kAc, vloc, zu = P.displaced_system(base, 0.05, seed=seed)
        g = GpuSystem(sysm, "c128")
        g.set_vloc(vloc)
        g.update_projector(kAc)
        g.gs_set_state(zu)
        g.set_cg_delta(1e-24)
        return sysm, g

    t0 = time.perf_counter()
    sysm, g = gpu(s_train)
    R, E, kidx, tb = P.cg_training_pairs(g, sysm, nconv, **cfg["pairs"])
    vsys, gv = gpu(s_val)  # held-out validation configuration
    zv = gv.gs_get_state()
    w, report, chosen = P.train_and_select(g, P.tpa_inputs(g, R, kidx, tb), E, P.DEFAULT_VARIANTS,
                                           lambda wt: P.cg_cost(gv, zv, wt, max_outer=max_outer, nconv=nconv))
    gv.close()
    g.close()
    t_train = time.perf_counter() - t0
    runs = {}
    for kind in ("learned", "tpa", "plain"):
        sysm, g = gpu(s_eval)
        if kind == "learned":
            g.net_set_weights(w)
        g.set_cg_preconditioner(kind)
        t1 = time.perf_counter()
        r = P.solve_to(g, tol=1e-8, ncg=4, max_outer=max_outer, nconv=nconv)
        runs[kind] = {"outer": r["outer"], "cg_iterations": r["cg_iterations"], "residual": r["residual"],
                      "converged": r["converged"], "seconds": time.perf_counter() - t1, "esp": r["esp"][:, :nconv]}
        g.close()
    de = float(np.abs(runs["learned"]["esp"] - runs["tpa"]["esp"]).max())
    for r in runs.values():
        r.pop("esp")
    nk = int(np.prod(base["nkgrid"]))
    return {"runs": runs, "learned_vs_plain_iterations": runs["learned"]["cg_iterations"] / runs["plain"]["cg_iterations"],
            "learned_vs_tpa_iterations": runs["learned"]["cg_iterations"] / runs["tpa"]["cg_iterations"],
            "eigenvalue_max_abs_diff_learned_vs_tpa": de, "training_pairs": int(R.shape[0]),
            "selection": {k: list(v) for k, v in report.items()}, "chosen": chosen, "training_seconds": t_train,
            "workload": f"{shape} {base['grid'][0]}x{base['grid'][1]}x{base['grid'][2]}, {nk} k x {base['Nb']} bands "
                        f"({nconv} converged), fixed V_loc, CG to residual 1e-8 (each run capped at {max_outer} "
                        "outer iterations)"}


def config5_bench(nsteps=5000, nscf=60, check_steps=500, npolish=3):
    """The large pulsed RT run: Si216 (3x3x3 diamond supercell, a = 10.26 bohr),
    48^3 grid, 2x2x1 = 4 k-points, 432 occupied bands, the physical Si
    pseudopotential (KY, lloc = 2, the testsuites' Si_rps.dat as parsed into
    tests/golden/si_rps_ky.npz), PZ LDA.  Ground state: the perfect crystal's
    supercell state is the unit cell's unfolded, so the reference's SCF loop
    (Broyden, TPA-preconditioned CG, FP64) runs on Si8 (16^3, the same spacing) at
    the 108 unit-cell k-points that fold onto the supercell's four, its 16
    occupied bands per k-point are unfolded onto the 48^3 grid on the device
    (system.unfold_to_supercell) and `npolish` supercell ground-state iterations
    remove the grid error of the unfolding.  Then `nsteps` middle-point Taylor steps of
    dt = 0.08 in complex(4) with FP64 reductions under a cos^2-envelope pulse
    (hbar omega = 1.55 eV, 1e12 W/cm^2, 20 fs), the Hartree + PZ potential
    rebuilt every step on the device, J every step; the first `check_steps` steps
    again in complex(8) for the J(t) error."""
    import torch
    from salmon_b200 import drive, precond as PC, pseudo as P, system as S
    from salmon_b200.rt import GpuSystem
    tabs = P.prepare(P.from_npz(os.path.join(ROOT, "tests", "golden", "si_rps_ky.npz"), lloc=2))
    ncell = (3, 3, 3)
    big, kS, vpsl, _ = S.si_pp_system(tabs, ncell=ncell, grid=(48, 48, 48), nkgrid=(2, 2, 1), NB=432, Nocc=432,
                                      with_orbitals=False)
    kU, ms = S.folded_kpoints(kS, ncell, big.aL)
    cell, _, vpsl_c, zu0 = S.si_pp_system(tabs, grid=(16, 16, 16), NB=20, Nocc=16, kpoints=kU)
    out = {"workload": "Si216 48^3, 4 k x 432 bands, physical Si pseudopotential (KY), PZ LDA; ground state "
                       "unfolded from the Si8 SCF at the 108 folded k-points; then "
                       f"{nsteps} complex(4) steps of dt = 0.08 under an Acos2 pulse (1.55 eV, 1e12 W/cm^2, 20 fs), "
                       "self-consistent Vloc every step"}
    t0 = time.perf_counter()
    with GpuSystem(cell, "c128") as g:
        g.gs_set_state(zu0)
        g.set_cg_preconditioner("tpa")
        esp, hist = drive.gs_scf(g, cell, kU, vpsl_c, nscf=nscf, ncg=4, threshold=1e-8)
        zgs = g.gs_get_state()
    out["ground_state"] = {"scf_iterations": len(hist), "ddns_last": hist[-1][0], "max_esp_var": hist[-1][1],
                           "seconds": time.perf_counter() - t0,
                           "gap_ha": float(np.sort(esp, axis=1)[:, 16].min() - np.sort(esp, axis=1)[:, 15].max())}
    zs_t = S.unfold_to_supercell(torch.from_numpy(np.ascontiguousarray(zgs[:, :16])).cuda(), ncell, ms,
                                 kS.shape[1], (16, 16, 16))
    zs = zs_t.cpu().numpy()
    del zs_t
    # the unfolded states are the supercell's to the grid error of the k+A treatment
    # (tests/test_unfold.py); a few supercell ground-state iterations in the
    # unfolded state's own potential remove it
    t0 = time.perf_counter()
    with GpuSystem(big, "c128") as g:
        g.set_vpsl(vpsl)
        g.set_vloc(vpsl)
        g.update_projector(kS)
        g.gs_set_state(zs)
        g.gs_to_rt()
        g.update_vloc()
        g.set_cg_preconditioner("tpa")
        res0 = None
        for it in range(npolish):
            _, ncg_it, res = PC.gs_iteration(g, 4)
            res0 = res if res0 is None else res0
        zs = g.gs_get_state()
    out["supercell_polish"] = {"iterations": npolish, "max_residual_first": res0, "max_residual_last": res,
                               "seconds": time.perf_counter() - t0}
    eion = P.ewald_energy(big.Rion, big.extra["zps"], big.aL, (big.NLx, big.NLy, big.NLz))
    dt = 0.08
    Ac = drive.init_Ac(nsteps + 1, dt, "Acos2", epdir=(0.0, 0.0, 1.0), rlaser_int_wcm2=1e12,
                       omega=1.55 / 27.211386245988, pulse_tw=20.0 * 41.341373335)
    runs = {}
    for prec, n in (("c64", nsteps), ("c128", check_steps)):
        with GpuSystem(big, "c128") as g:
            g.set_state(zs)
            if prec == "c64":
                g.set_precision("c64")
            g.update_projector(kS)
            g.synchronize()
            t1 = time.perf_counter()
            javt, energies = drive.rt_propagate(g, big, kS, vpsl, Ac, dt, n, energy_every=max(1, n // 10),
                                                scf=True, eion=eion)
            g.synchronize()
            sec = time.perf_counter() - t1
        runs[prec] = (javt, energies, sec, n)
    del zs
    j64, e64, s64, n64 = runs["c128"]
    j32, e32, s32, n32 = runs["c64"]
    norb = big.nk_local * big.NBoccmax
    out["c64"] = {"steps": n32, "seconds": s32, "ms_per_step_wall": 1e3 * s32 / n32,
                  "orbital_updates_per_s_wall": norb * n32 / s32,
                  "energy_change_ha": float(e32[max(e32)] - e32[0]), "max_abs_j": float(np.abs(j32).max())}
    out["c128"] = {"steps": n64, "seconds": s64, "ms_per_step_wall": 1e3 * s64 / n64}
    out["j_rel_err"] = drive.j_error(j64, j32[:n64 + 1])  # over the complex(8) run's steps
    out["energy_change_abs_diff_ha"] = float(max(abs((e32[t] - e32[0]) - (e64[t] - e64[0])) for t in e64 if t in e32))
    return out


def si8_bench(nsteps=50):
    """The Si8 RT shape of the plain FP64 run (16^3 grid, 4x4x4 k, 16 bands, 1024
    orbitals; synthetic Gaussian projectors and V_loc): Taylor-step time of the
    shared-memory resident form (the whole step in one kernel) against the four
    stencil passes, in both orbital precisions."""
    import torch
    from salmon_b200 import system as S
    from salmon_b200.rt import GpuSystem
    sysm, kAc, vloc, zu = S.si_supercell_system((1, 1, 1), (16, 16, 16), (4, 4, 4), 16, A=(1e-2, 0.0, 0.0))
    norb = sysm.nk_local * sysm.NBoccmax
    out = {"workload": "Si8 16^3, 64 k x 16 bands (1024 orbitals), synthetic Gaussian projectors / V_loc"}
    for prec in ("c64", "c128"):
        r = {}
        for name, tk in (("passes", 1), ("resident", 2)):
            with GpuSystem(sysm, prec) as g:
                g.set_state(zu)
                g.set_vloc(vloc)
                g.update_projector(kAc)
                g.set_param("taylor_kernel", tk)
                st = torch.cuda.ExternalStream(g.stream)
                for _ in range(5):
                    g.hamiltonian(DT)
                g.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(st)
                for _ in range(nsteps):
                    g.hamiltonian(DT)
                e1.record(st)
                e1.synchronize()
                ms = e0.elapsed_time(e1) / nsteps
                r[name] = {"ms_per_step": ms, "orbital_updates_per_s": norb / (ms * 1e-3)}
        r["resident_speedup"] = r["passes"]["ms_per_step"] / r["resident"]["ms_per_step"]
        out[prec] = r
    return out


def bench_config(args, sysm, norb, world):
    """The `config` of both arms' JSON lines (the same workload description)."""
    return {"workload": f"hpsi/Taylor microbench {args.grid}^3, {sysm.NK} k x {sysm.NBoccmax} bands per GPU",
            "grid": args.grid, "nk": sysm.NK, "nb": sysm.NBoccmax, "norb_per_gpu": norb,
            "l2": "inputs larger than L2 at every pass (no flush)", "parallelism": f"k-blocks x{world}"}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    sysm, kAc, vloc, zu = make_workload(args, 0, world)
    from oracle import oracle as O
    if not O.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref (SALMON AVX stencil build) missing"}))
        return 0
    secs = max(2.0, args.cpu_seconds / max(1, args.steps))
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(sysm, kAc, vloc, zu, 0.5)
    for _ in range(args.steps):
        vals.append(cpu_baseline(sysm, kAc, vloc, zu, secs))
    v = statistics.median(x["value"] for x in vals)
    norb = sysm.nk_local * sysm.NBoccmax
    out = {"metric": METRIC, "value": v, "unit": "orbital-updates/s", "n_gpus": 0, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": 1000.0 * norb / v, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c128", "data": "synthetic",
           "config": bench_config(args, sysm, norb, world),
           "impl": "reference", "cpu_baseline": {k: vals[-1][k] for k in ("kind", "cores", "sample")} | {"value": v, "unit": "orbital-updates/s"},
           "e2e": {"value": v, "unit": "orbital-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from salmon_b200 import build
    build.build()
    from salmon_b200.rt import GpuSystem

    sysm, kAc, vloc, zu = make_workload(args, rank, world)
    norb = sysm.nk_local * sysm.NBoccmax
    if args.profile_current:  # the current path as the end-to-end leg runs it (sphere values current)
        with GpuSystem(sysm, "c64") as g:
            g.set_state(zu)
            g.set_vloc(vloc)
            g.update_projector(kAc)
            g.hamiltonian(DT)
            for _ in range(2):
                g.current_RT(kAc)
            g.synchronize()
        return
    NL = sysm.NL
    hbm_peak, peak_kind = measured_peaks()
    res = {}

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([x], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())
        return x

    clocks = None
    for prec in ((args.only,) if args.only else ("c128", "c64")):
        S_bytes = 16 if prec == "c128" else 8
        g = GpuSystem(sysm, prec)
        g.set_state(zu)
        g.set_vloc(vloc)
        g.update_projector(kAc)
        g.set_param("kb_kernel", args.kb_kernel)
        g.set_param("pass_fixed", args.pass_fixed)
        g.set_param("taylor_kernel", args.taylor_kernel)
        stream = torch.cuda.ExternalStream(g.stream)
        for _ in range(args.warmup):
            g.hamiltonian(DT)
        g.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        ctx = Clocks(local) if prec == "c64" else None
        if ctx:
            ctx.__enter__()
        g.set_param("launches", 0)
        e0.record(stream)
        for _ in range(args.steps):
            g.hamiltonian(DT)
        e1.record(stream)
        launches = g.get_param("launches")
        e1.synchronize()
        if ctx:
            ctx.__exit__(None, None, None)
            clocks = ctx.summary()
        barrier()
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1))
        r = {"ms_per_step": ms / args.steps, "value": norb * world * args.steps / (ms / 1000.0), "launches": launches}
        # dominant kernel: one H application of all orbitals (stencil + KB scatter), events on its stream
        t_pass = g.time_kernel("stencil_pass", reps=10)
        t_last = g.time_kernel("taylor_last", reps=5)
        t_uv = g.time_kernel("uvpsi", reps=10)
        t_kb = g.time_kernel("kb_field", reps=10)
        t_kbt = g.time_kernel("kb_term", reps=10)
        alg = 2.0 * S_bytes * NL * norb  # algorithmic bytes of one H application over all orbitals
        r.update(t_pass_ms=t_pass, t_last_ms=t_last, t_uvpsi_ms=t_uv, t_kb_ms=t_kb, t_kbterm_ms=t_kbt,
                 achieved_gbs=alg / (t_last * 1e-3) / 1e9, pass_gbs=alg / (t_pass * 1e-3) / 1e9,
                 step_gbs=10.0 * S_bytes * NL * norb / (r["ms_per_step"] * 1e-3) / 1e9)
        if args.no_e2e:
            res[prec] = r
            g.close()
            continue
        # end to end through the C ABI: k+A(t) and V_loc from host memory in, rho and J
        # out to host memory, every step.  One rank: the host-result calls (the
        # library stages through its own pinned buffers).  Several ranks: rho and J
        # into device buffers, all-reduced on the device over NCCL (comm_summation
        # of psi_rho.f90:88 and current.f90:286), then read back.
        from salmon_b200 import dist as D
        kA = np.ascontiguousarray(kAc)
        rho_d = torch.empty(NL, dtype=torch.float64, device="cuda")
        jav_d = torch.empty(3, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        e0.record(stream)
        for it in range(args.steps):
            kt = kA + np.array([0.0, 0.0, 1e-4 * it])[:, None]
            g.update_projector(kt)
            g.set_vloc(vloc)
            g.hamiltonian(DT, flag_current=True)  # the current's stencil sums with the step
            if world == 1:
                rho = g.psi_rho_RT()
                jav = g.current_RT(kt)
            else:
                g.psi_rho_dev(rho_d.data_ptr())
                g.current_dev(kt, jav_d.data_ptr())
                D.comm_summation_dev(g, rho_d)
                D.comm_summation_dev(g, jav_d)
                with torch.cuda.stream(stream):
                    rho = rho_d.cpu().numpy()
                    jav = jav_d.cpu().numpy()
        e1.record(stream)
        e1.synchronize()
        ms_e2e = max_over_ranks(e0.elapsed_time(e1))
        r["e2e"] = {"value": norb * world * args.steps / (ms_e2e / 1000.0), "unit": "orbital-updates/s",
                    "h2d_bytes_per_step": 2 * kA.nbytes + vloc.nbytes, "d2h_bytes_per_step": rho.nbytes + jav.nbytes}
        res[prec] = r
        g.close()
        del stream

    # the other workloads' legs: one GPU only (a multi-GPU run reports the k-sharded step)
    legs = rank == 0 and world == 1 and not (args.only or args.no_e2e)
    prec_check = precision_check() if legs and not args.no_precision else None
    batched = batched_bench(args.batched_steps) if legs and not args.no_batched else None
    large = large_bench() if legs and not args.no_large else None
    si8 = si8_bench() if legs and not args.no_si8 else None
    pc = precond_bench("Si8") if legs and not args.no_precond else None
    pc64 = precond_bench("Si64") if rank == 0 and args.precond else None
    c5 = config5_bench(args.config5, check_steps=args.config5_check or args.config5) \
        if (rank == 0 and args.config5) else None
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(sysm, kAc, vloc, zu, args.cpu_seconds)
        except Exception as exc:  # the CPU baseline is reported, never required
            cpu = {"unavailable": str(exc)}
    if rank == 0 and (args.only or args.no_e2e):
        print(json.dumps({p: {k: v for k, v in r.items() if k != "e2e"} for p, r in res.items()} |
                         ({"config5": c5} if c5 else {}) | ({"precond_si64": pc64} if pc64 else {})))
    elif rank == 0:
        h = res["c64"]
        tpo = NCU_TRAFFIC_BYTES_PER_ORBITAL.get(("taylor_stage", "c64", args.grid))
        traffic = tpo * norb if tpo else None
        out = {
            "metric": METRIC, "value": h["value"], "unit": "orbital-updates/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": h["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "c64 orbitals (FP32 stencil), FP64 reductions", "data": "synthetic",
            "config": bench_config(args, sysm, norb, world),
            "fp64_path": {"value": res["c128"]["value"], "ms_per_step": res["c128"]["ms_per_step"],
                          "e2e": res["c128"]["e2e"], "taylor_stage_ms": res["c128"]["t_last_ms"],
                          "taylor_stage_gbs": res["c128"]["achieved_gbs"]},
            "fp32_over_fp64": h["value"] / res["c128"]["value"],
            "kernels_ms": {p: {"stencil_pass (H only)": res[p]["t_pass_ms"], "taylor_stage": res[p]["t_last_ms"],
                               "kb_term (in the step)": res[p]["t_kbterm_ms"], "uvpsi alone": res[p]["t_uvpsi_ms"],
                               "kb_field alone": res[p]["t_kb_ms"]} for p in res},
            "step_gbs_algorithmic": {p: res[p]["step_gbs"] for p in res},
            "roofline": {"bound": "hbm", "achieved": h["achieved_gbs"], "peak": hbm_peak, "unit": "GB/s",
                         "frac": h["achieved_gbs"] / hbm_peak, "traffic": traffic,
                         "kernel": "k_hpsi_pass<float,2,2> (one Taylor stage psi + c H psi, all orbitals)",
                         "peak_kind": peak_kind},
            "cpu_baseline": cpu,
            "e2e": h["e2e"],
            "gpu_launches": h["launches"],
            "precision": prec_check,
            "batched": batched,
            "large": large,
            "si8_resident_vs_passes": si8,
            "precond": pc,
            "precond_si64": pc64,
            "config5": c5,
            "clocks": clocks,
        }
        print(json.dumps(out))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
