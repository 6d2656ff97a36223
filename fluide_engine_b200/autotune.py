"""The autotuner's host side: runs the library's search (fe_scene_autotune) and keeps its choices across processes.

fe_scene_autotune times every launch choice of a scene's pressure solve (plain CG at 256 / 512 / 1024 threads per
persistent block; multigrid-preconditioned CG at two block shapes and two one-block level thresholds) on the scene's own substeps, applies the fastest and stores it in the library's
per-process table, from which scenes created later with the automatic solver choice start.  This module persists
that table as JSON, one file per GPU model, so a later process starts tuned: load() puts the file's entries back
into the library, tune() runs the search and saves.  The reference has no counterpart (its CUDA Jacobi solver
uses fixed 4x4x4 blocks, linear_system/cuda_jacobi_iteration_solver.cu:41-63).
"""
import ctypes
import json
import os

from . import _abi

FIELDS = ("multigrid", "cg_block_threads", "mg_block_level_cells", "cg_cluster", "pressure_extrapolation")
SOLVER_NAMES = {_abi.PIC: "PIC", _abi.FLIP: "FLIP", _abi.APIC: "APIC"}


def cache_path(device_name):
    """JSON file of the tuning table for one GPU model ($FE_TUNING_CACHE overrides the directory)."""
    base = os.environ.get("FE_TUNING_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "fluide_b200")
    safe = "".join(ch if ch.isalnum() else "_" for ch in device_name)
    return os.path.join(base, "tuning_%s.json" % safe)


def device_name(device=0):
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:
        return "device%d" % device


def key_of(n, solver):
    return "%dx%dx%d/%s" % (n[0], n[1], n[2], SOLVER_NAMES.get(solver, str(solver)))


def parse_key(key):
    dims, solver = key.split("/")
    n = tuple(int(x) for x in dims.split("x"))
    inv = {v: k for k, v in SOLVER_NAMES.items()}
    return n, inv[solver]


def to_dict(t):
    return {f: int(getattr(t, f)) for f in FIELDS}


def store(n, solver, tuning, device=0):
    """Puts one choice into the library's table (fe_tuning_store)."""
    t = _abi.Tuning(*[int(tuning[f]) for f in FIELDS])
    n3 = (ctypes.c_int32 * 3)(*n)
    _abi.check(_abi.lib().fe_tuning_store(int(device), n3, int(solver), ctypes.byref(t)))


def lookup(n, solver, device=0):
    """The library's stored choice for (grid, transfer) on `device`, or None."""
    t = _abi.Tuning()
    n3 = (ctypes.c_int32 * 3)(*n)
    st = _abi.lib().fe_tuning_lookup(int(device), n3, int(solver), ctypes.byref(t))
    return to_dict(t) if st == _abi.FE_OK else None


def read_file(path):
    try:
        with open(path) as f:
            data = json.load(f)
    except (OSError, ValueError):
        return {}
    out = {}
    for key, val in data.get("entries", {}).items():
        try:
            n, solver = parse_key(key)
            out[(n, solver)] = {f: int(val[f]) for f in FIELDS}
        except (KeyError, ValueError, TypeError):
            continue  # an entry of another format version is skipped, not fatal
    return out


def write_file(path, entries, device_name_):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    data = {"device": device_name_, "format": 1,
            "entries": {key_of(n, solver): t for (n, solver), t in sorted(entries.items())}}
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def load(device=0, path=None):
    """Puts the saved choices for this GPU model into the library; returns how many."""
    path = path or cache_path(device_name(device))
    entries = read_file(path)
    for (n, solver), t in entries.items():
        store(n, solver, t, device)
    return len(entries)


def tune(scene, dt, substeps=6, device=0, path=None, save=True, shape_only=False):
    """Runs the search on `scene` (its state is restored afterwards), applies and returns the fastest choice with
    its ms per substep; shape_only keeps the scene's solver family (plain or multigrid CG) and searches its launch
    shapes; with save, merges the choice into this GPU model's file."""
    best = _abi.Tuning()
    ms = ctypes.c_float()
    scope = _abi.TUNE_SHAPE if shape_only else _abi.TUNE_ALL
    _abi.check(_abi.lib().fe_scene_autotune(scene.handle, float(dt), int(substeps), scope, ctypes.byref(best),
                                            ctypes.byref(ms)))
    choice = to_dict(best)
    if save:
        name = device_name(device)
        path = path or cache_path(name)
        entries = read_file(path)
        entries[(tuple(scene.n), scene.solver)] = choice
        write_file(path, entries, name)
    return choice, float(ms.value)


FLAT_CANDIDATES = (0, 32 ** 3, 48 ** 3, 64 ** 3, -1)


def tune_batch(batch, dt, substeps=3, candidates=FLAT_CANDIDATES, timer=None, rounds=2):
    """Picks which of a batch's scenes run in the flat launches (Batch.set_flat: scenes up to max_cells cells run
    every pre- and post-solve pass as one launch for all of them; the rest on their own streams).

    Every candidate computes the same substeps, so the search times them on the batch's own live substeps: per
    candidate and round one untimed substep (the batch graph's capture, once the batch is old enough to be captured)
    and `substeps` timed ones; the rounds visit the candidates in alternating order and each candidate keeps its best
    round, so a slow moment of the device does not decide.  The scenes advance by rounds * len(candidates) *
    (substeps + 1) substeps.  Applies the fastest and returns (max_cells, {candidate: ms per substep}).  `timer`
    (seconds, monotonic) defaults to time.perf_counter; the batch's step() synchronises before returning, so the wall
    clock spans the device work.
    """
    import time

    clock = timer or time.perf_counter
    times = {}
    order = list(candidates)
    for r in range(max(1, rounds)):
        for c in (order if r % 2 == 0 else order[::-1]):
            batch.set_flat(c)
            batch.step(dt, 1, stats=False)
            t0 = clock()
            batch.step(dt, substeps, stats=False)
            ms = (clock() - t0) / max(substeps, 1) * 1e3
            times[c] = min(times.get(c, ms), ms)
    best = min(times, key=times.get)
    batch.set_flat(best)
    return best, times
