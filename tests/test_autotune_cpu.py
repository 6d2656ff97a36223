"""The autotuner's host side without a GPU: the library's per-process tuning table (fe_tuning_store / lookup are
host code) and the JSON file that carries it across processes."""
import json
import os

import pytest

from fluide_engine_b200 import _abi, autotune


def test_store_and_lookup_per_device_grid_and_transfer():
    t = dict(multigrid=1, cg_block_threads=512, mg_block_level_cells=2048, cg_cluster=2, pressure_extrapolation=0)
    autotune.store((96, 64, 48), _abi.APIC, t, device=3)
    assert autotune.lookup((96, 64, 48), _abi.APIC, device=3) == t
    assert autotune.lookup((96, 64, 48), _abi.FLIP, device=3) is None      # another transfer
    assert autotune.lookup((96, 64, 48), _abi.APIC, device=2) is None      # another device
    assert autotune.lookup((96, 64, 49), _abi.APIC, device=3) is None      # another grid
    t2 = dict(t, cg_block_threads=1024)
    autotune.store((96, 64, 48), _abi.APIC, t2, device=3)                 # replaced, not duplicated
    assert autotune.lookup((96, 64, 48), _abi.APIC, device=3) == t2


def test_file_round_trip_and_load(tmp_path):
    path = str(tmp_path / "sub" / "tuning_B200.json")
    entries = {((128, 128, 128), _abi.FLIP): dict(multigrid=0, cg_block_threads=1024,
                                                  mg_block_level_cells=4096, cg_cluster=1,
                                                  pressure_extrapolation=1),
               ((256, 256, 256), _abi.APIC): dict(multigrid=1, cg_block_threads=512,
                                                  mg_block_level_cells=2048, cg_cluster=1,
                                                  pressure_extrapolation=0)}
    autotune.write_file(path, entries, "NVIDIA B200")
    with open(path) as f:
        data = json.load(f)
    assert data["device"] == "NVIDIA B200" and "128x128x128/FLIP" in data["entries"]
    assert autotune.read_file(path) == entries
    assert autotune.load(device=5, path=path) == 2
    assert autotune.lookup((256, 256, 256), _abi.APIC, device=5) == entries[((256, 256, 256), _abi.APIC)]


def test_unreadable_or_foreign_files_are_ignored(tmp_path):
    assert autotune.read_file(str(tmp_path / "missing.json")) == {}
    bad = tmp_path / "bad.json"
    bad.write_text("{not json")
    assert autotune.read_file(str(bad)) == {}
    odd = tmp_path / "odd.json"
    odd.write_text(json.dumps({"entries": {"12x12/FLIP": {"multigrid": 0}, "8x8x8/XYZ": {}}}))
    assert autotune.read_file(str(odd)) == {}


def test_cache_path_names_the_gpu_model(monkeypatch, tmp_path):
    monkeypatch.setenv("FE_TUNING_CACHE", str(tmp_path))
    p = autotune.cache_path("NVIDIA B200")
    assert p == os.path.join(str(tmp_path), "tuning_NVIDIA_B200.json")


def test_store_rejects_null_arguments():
    L = _abi.lib()
    assert L.fe_tuning_store(0, None, 1, None) == _abi.FE_ERR_BAD_ARG
    with pytest.raises(Exception):
        autotune.store((8, 8), _abi.FLIP, {})


def test_tune_batch_picks_the_fastest_threshold_and_applies_it():
    from fluide_engine_b200 import autotune

    # a stand-in batch whose substeps take a per-threshold time on a fake clock
    cost = {0: 10.0, 4096: 9.0, 32768: 8.5, -1: 12.0}

    class FakeBatch:
        def __init__(self):
            self.flat = None
            self.calls = []
            self.now = 0.0

        def set_flat(self, c):
            self.flat = c
            self.calls.append(("flat", c))

        def step(self, dt, nsub, stats=True):
            self.calls.append(("step", nsub))
            self.now += cost[self.flat] * 1e-3 * nsub

    b = FakeBatch()
    best, times = autotune.tune_batch(b, 1.0 / 240.0, substeps=3, candidates=tuple(cost), timer=lambda: b.now,
                                      rounds=2)
    assert best == 32768 and b.flat == 32768
    for c, ms in cost.items():
        assert abs(times[c] - ms) < 1e-9
    # every candidate: one untimed substep (the graph's capture), then the timed ones; the second round visits the
    # candidates in reverse order
    assert b.calls[:3] == [("flat", 0), ("step", 1), ("step", 3)]
    flats = [c for k, c in b.calls if k == "flat"]
    assert flats == list(cost) + list(cost)[::-1] + [32768]
