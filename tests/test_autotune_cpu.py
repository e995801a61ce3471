"""The launch-shape cache of pf_kks_gpu.autotune on the CPU, with a stand-in
cell: a miss times the cell (kks_autotune) and stores the choice under the
(GPU, grid, precision[, batch]) key; a hit applies the stored shape without
timing; ``force`` re-times; an unwritable cache file still tunes the cell."""

import json

from pf_kks_gpu import autotune


class FakeCell:
    def __init__(self, nx, ny, precision="mixed", shape=None, ms=0.25):
        self.nx, self.ny, self.precision = nx, ny, precision
        self.shape = shape or {"pipeline": 1, "cols": 3, "field_blocks": 296}
        self.ms = ms
        self.timed = 0
        self.applied = []

    def autotune(self, attempts, batchable=False):
        self.timed += 1
        self.batchable = batchable
        return dict(self.shape), self.ms

    def set_launch_shape(self, pipeline, cols, field_blocks):
        self.applied.append((pipeline, cols, field_blocks))


def test_miss_then_hit(tmp_path, monkeypatch):
    path = tmp_path / "shapes.json"
    monkeypatch.setenv("KKS_AUTOTUNE_CACHE", str(path))
    monkeypatch.setattr(autotune, "device_name", lambda device=0: "B200")
    a = FakeCell(1420, 1420, shape={"pipeline": 1, "cols": 2, "field_blocks": 592})
    r = autotune.tune(a, attempts=5)
    assert r["source"] == "measured" and a.timed == 1 and a.applied == []
    table = json.loads(path.read_text())
    assert table["B200|1420x1420|mixed"]["shape"] == {"pipeline": 1, "cols": 2, "field_blocks": 592}
    b = FakeCell(1420, 1420)
    r = autotune.tune(b)
    assert r["source"] == "cache" and b.timed == 0 and b.applied == [(1, 2, 592)]
    c = FakeCell(1420, 1420, shape={"pipeline": 0, "cols": 3, "field_blocks": 148})
    assert autotune.tune(c, force=True)["source"] == "measured" and c.timed == 1
    assert json.loads(path.read_text())["B200|1420x1420|mixed"]["shape"]["pipeline"] == 0


def test_keys_separate_grids_precisions_and_batches(tmp_path, monkeypatch):
    monkeypatch.setenv("KKS_AUTOTUNE_CACHE", str(tmp_path / "shapes.json"))
    monkeypatch.setattr(autotune, "device_name", lambda device=0: "B200")
    for cell, batchable in ((FakeCell(256, 256), False), (FakeCell(256, 256, "fp64"), False),
                            (FakeCell(256, 256), True), (FakeCell(512, 256), False)):
        assert autotune.tune(cell, batchable=batchable)["source"] == "measured"
        assert cell.batchable is batchable
    keys = set(json.loads((tmp_path / "shapes.json").read_text()))
    assert keys == {"B200|256x256|mixed", "B200|256x256|fp64", "B200|256x256|mixed|batch", "B200|512x256|mixed"}


def test_unwritable_cache_still_tunes(tmp_path, monkeypatch):
    blocker = tmp_path / "file"
    blocker.write_text("not a directory")
    monkeypatch.setenv("KKS_AUTOTUNE_CACHE", str(blocker / "shapes.json"))
    cell = FakeCell(128, 128)
    r = autotune.tune(cell)
    assert r["source"] == "measured" and r["shape"] == cell.shape and cell.timed == 1


def test_no_cache(tmp_path, monkeypatch):
    path = tmp_path / "shapes.json"
    monkeypatch.setenv("KKS_AUTOTUNE_CACHE", str(path))
    cell = FakeCell(128, 128)
    autotune.tune(cell, cache=False)
    autotune.tune(cell, cache=False)
    assert cell.timed == 2 and not path.exists()
