"""The launch-shape table: for each system shape, the launch choices the step
tuner (sgpu_autotune_step) measured fastest, persisted as JSON so that a run
reuses them instead of tuning again.

Key: "<NLx>x<NLy>x<NLz> norb=<orbitals> nsp=<sphere points> <precision> <device>".
Value: {"params": {taylor_kernel, pass_fixed, pass_tables, nslab, kb_kernel,
uvpsi_split}, "ms_per_step": t, "dt": dt}.  tile_table.json beside this module
holds the entries measured on B200 for the benchmarked shapes; a run may pass
its own path to record new shapes.  No reference counterpart; the nearest is
auto_blocking (modules/opt_variables.f90:340-353), which measures cache-blocking
sizes at start-up and keeps them for the run.
"""
from __future__ import annotations

import json
import os
import tempfile

DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tile_table.json")


def device_name() -> str:
    try:
        import torch
        return torch.cuda.get_device_name().replace(" ", "_") if torch.cuda.is_available() else "cpu"
    except Exception:  # the name only labels table entries
        return "unknown"


def key(sysm, precision: str, nsp: int | None = None) -> str:
    n = nsp if nsp is not None else sysm.extra.get("nsp", -1)
    return (f"{sysm.NLx}x{sysm.NLy}x{sysm.NLz} norb={sysm.nk_local * sysm.NBoccmax} nsp={n} {precision} "
            f"{device_name()}")


def load(path: str = DEFAULT_TABLE) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def save(table: dict, path: str = DEFAULT_TABLE) -> None:
    d = os.path.dirname(os.path.abspath(path))
    fd, tmp = tempfile.mkstemp(dir=d, suffix=".tmp")
    with os.fdopen(fd, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply(g, sysm, precision: str, path: str = DEFAULT_TABLE, tune_if_missing: bool = True, dt: float = 0.02,
          reps: int = 3, write: bool = True):
    """Sets the handle's launch choices from the table entry of this shape; if
    there is none and tune_if_missing, runs the step tuner, records its choice
    (write=True) and returns it.  Returns (entry, "table" | "tuned" | "none")."""
    table = load(path)
    k = key(sysm, precision, nsp=g.get_nsp())
    if k in table:
        for p, v in table[k]["params"].items():
            g.set_param(p, v)
        return table[k], "table"
    if not tune_if_missing:
        return None, "none"
    params, ms = g.autotune_step(dt=dt, reps=reps)
    entry = {"params": params, "ms_per_step": ms, "dt": dt}
    if write:
        table = load(path)
        table[k] = entry
        save(table, path)
    return entry, "tuned"
