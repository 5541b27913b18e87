"""CPU: argument validation of the drop-in API, mirroring the reference's
own checks (FlashKNN/functions/FlashKnnWrapper.py:193-219)."""
import pytest

from flashknn_exprepo_b200.wrapper import FlashKNN
from flashknn_exprepo_b200 import synthetic as S


def test_mode_validation_mirrors_reference():
    chk = FlashKNN._check_modes
    chk("SM", "PS", "register", True, None)
    chk("GM", "SS", "register", True, None)
    with pytest.raises(ValueError):
        chk("SM", "PS", "global", True, None)
    with pytest.raises(ValueError):
        chk("SM", "PS", "register", True, 12)
    with pytest.raises(ValueError):
        chk("GM", "PS", "shared", True, None)
    with pytest.raises(ValueError):
        chk("SM", "SS", "register", True, 16)
    with pytest.raises(ValueError):
        chk("XX", "PS", "register", True, None)


def test_constructor_limits():
    with pytest.raises(ValueError):
        FlashKNN(num_nbr=65)
    with pytest.raises(ValueError):
        FlashKNN(num_nbr=8, num_down=9)
    f = FlashKNN(num_nbr=16, num_down=2, debug=True)
    assert f.time_list == []
    assert f.rng_grid([0, -1, 1], device="cpu")[0].tolist() == [0, 0, 0]
    assert f.rng_grid([0, -1, 1], device="cpu").shape == (27, 3)


def test_synthetic_generators_are_seeded():
    a = S.uniform_cube(2048, voxel=0.05)
    b = S.uniform_cube(2048, voxel=0.05)
    assert (a == b).all() and a.shape == (2048, 3)
    r = S.room(target=5000)
    assert r.shape == (5000, 3)
    counts, seed = S.draw_counts()
    assert len(counts) == 16 and abs(counts.sum() - 1.5e6) <= 0.03 * 1.5e6
    assert counts.min() >= 20000 and counts.max() <= 200000


def test_autotune_buckets_and_cache_file(tmp_path, monkeypatch):
    from flashknn_exprepo_b200 import autotune
    assert [autotune.k_bucket(k) for k in (1, 2, 3, 16, 17, 33, 64)] == [1, 2, 4, 16, 32, 64, 64]
    path = tmp_path / "cache.json"
    monkeypatch.setenv("FKNN_TUNE_CACHE", str(path))
    autotune._cache.clear()
    autotune._cache["GPU|k16|d3"] = {"config": [8, 512, 4, 0], "ms": 1.0, "default_ms": 1.2}
    autotune._save_file()
    autotune._cache.clear()
    assert autotune._load_file()["GPU|k16|d3"]["config"] == [8, 512, 4, 0]
    autotune._cache.clear()
