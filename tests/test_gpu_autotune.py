"""The launch-shape autotuner: every shape it may pick gives bit-identical
results (the shape changes the schedule, never the answer), and the tuner
returns, caches and reloads the fastest shape per K bucket and density."""
import json

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda"


@pytest.fixture(scope="module")
def fk():
    import flashknn_exprepo_b200 as fk
    from flashknn_exprepo_b200.build import build
    build()
    return fk


@pytest.mark.parametrize("k", [8, 16, 32])
def test_every_shape_gives_identical_results(fk, k):
    from flashknn_exprepo_b200 import _lib, autotune
    from flashknn_exprepo_b200 import synthetic as S
    b = S.first_clouds(S.uneven_batch(), 3)
    xyz = torch.from_numpy(b.xyz).to(DEV)
    off = torch.from_numpy(b.offsets).to(DEV)
    base = fk.ops.knn_offsets(xyz, off, k, S.C4_VOXEL, 2)
    seen = 0
    for w in autotune.WARPS:
        for t in autotune.TILES[::2]:
            for share in autotune.LANE_SHARES:
                for depth in autotune.DEPTHS:
                    try:
                        got = fk.ops.knn_offsets(xyz, off, k, S.C4_VOXEL, 2,
                                                 config=_lib.FknnConfig(w, t, share, 0, depth))
                    except _lib.FknnError:
                        continue                  # shared memory beyond a CTA's
                    assert torch.equal(got[0], base[0]) and torch.equal(got[1], base[1])
                    seen += 1
    assert seen >= 40


def test_tune_caches_and_reloads(fk, tmp_path, monkeypatch):
    from flashknn_exprepo_b200 import autotune
    from flashknn_exprepo_b200 import synthetic as S
    path = tmp_path / "tune.json"
    monkeypatch.setenv("FKNN_TUNE_CACHE", str(path))
    autotune._cache.clear()
    xyz = torch.from_numpy(S.lidar()).to(DEV)
    off = torch.tensor([len(xyz)], device=DEV)
    cfg = autotune.tune_offsets(xyz, off, 16, S.C3_VOXEL, 2, reps=2)
    stored = json.loads(path.read_text())
    (entry,) = stored.values()
    assert tuple(entry["config"]) == cfg.as_tuple()
    assert entry["ms"] <= entry["default_ms"] * 1.0001 or entry["default_ms"] is None
    autotune._cache.clear()                        # reload from the file
    dens = autotune.density_bucket(xyz, off, S.C3_VOXEL, 2)
    assert autotune.lookup(xyz.device, 16, dens).as_tuple() == cfg.as_tuple()
    assert autotune.tune_offsets(xyz, off, 16, S.C3_VOXEL, 2).as_tuple() == cfg.as_tuple()
    i1, d1 = fk.ops.knn_offsets(xyz, off, 16, S.C3_VOXEL, 2, config=cfg)
    i0, d0 = fk.ops.knn_offsets(xyz, off, 16, S.C3_VOXEL, 2)
    assert torch.equal(i0, i1) and torch.equal(d0, d1)


def test_concurrent_threads_with_different_shapes(fk):
    """Host threads querying one device at once, each with its own launch
    shape (different shared-memory sizes), on the same stream: every result
    equals the single-threaded one (per-thread workspaces, a launch cache
    shared under a lock)."""
    import threading

    from flashknn_exprepo_b200 import _lib
    from flashknn_exprepo_b200 import synthetic as S
    b = S.first_clouds(S.uneven_batch(), 3)
    xyz = torch.from_numpy(b.xyz).to(DEV)
    off = torch.from_numpy(b.offsets).to(DEV)
    base = fk.ops.knn_offsets(xyz, off, 16, S.C4_VOXEL, 2)
    torch.cuda.synchronize()
    shapes = [(4, 448, 8, 0, 1), (8, 1024, 8, 0, 1), (2, 256, 4, 0, 2), (4, 640, 16, 0, 2)]
    errors = []

    def worker(shape):
        try:
            cfg = _lib.FknnConfig(*shape)
            for _ in range(6):
                i, d = fk.ops.knn_offsets(xyz, off, 16, S.C4_VOXEL, 2, config=cfg)
                torch.cuda.current_stream().synchronize()
                if not (torch.equal(i, base[0]) and torch.equal(d, base[1])):
                    errors.append(f"shape {shape}: result differs")
        except Exception as exc:  # reported below, on the main thread
            errors.append(f"shape {shape}: {exc}")

    threads = [threading.Thread(target=worker, args=(s,)) for s in shapes]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not any(t.is_alive() for t in threads)
    assert not errors, errors
