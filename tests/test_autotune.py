"""The autotuner's cache logic on the CPU (the timing itself needs a GPU): size classes, the
default shape when tuning is off, and cached winners read back as Solver keywords."""
import json

import cfd_optimisations_b200 as H
from cfd_optimisations_b200 import autotune as A


def test_size_classes():
    assert A.size_class(1) == 10 and A.size_class(1 << 30) == 24
    assert A.size_class(4_000_000) == 22 and A.size_class(25_600) == 15


def test_shapes_are_valid_solver_keywords():
    for c in A.SOLVER_SHAPES:
        assert set(c) == {"kernel", "tile", "tile2", "block"}
        assert c["kernel"] in (H.KERNEL_TILED, H.KERNEL_CELL)
        assert c["tile"] % 32 == 0 and c["tile2"] % 32 == 0 and c["tile"] <= 512 and c["tile2"] <= 512
        if c["kernel"] == H.KERNEL_CELL:
            assert c["tile"] == 0 and c["tile2"] == 0
    assert A.DEFAULT_SHAPE == dict(kernel=H.KERNEL_TILED, tile=0, tile2=0, block=0)


def test_untuned_and_cached_shapes(tmp_path, monkeypatch):
    cache = tmp_path / "autotune.json"
    monkeypatch.setenv("HCFD_AUTOTUNE_CACHE", str(cache))
    monkeypatch.setattr(A, "gpu_name", lambda: "B200")
    assert A.best_solver_shape(4_000_000, tune=False) == A.DEFAULT_SHAPE
    assert A.best_arena_tile(20_000, H.FP32, tune=False) == 128
    key = A._key("solver", 22, H.FP64, H.LIMITER_BJ)
    # an entry written before the split tilings were tuned (no tile2) counts as missing
    cache.write_text(json.dumps({key: {"best": {"kernel": 1, "tile": 128, "block": 128}}}))
    assert A.best_solver_shape(4_000_000, tune=False) == A.DEFAULT_SHAPE
    best = dict(kernel=H.KERNEL_TILED, tile=256, tile2=128, block=0, ms_per_step=0.5)
    cache.write_text(json.dumps({key: {"best": best}}))
    assert A.best_solver_shape(4_000_000, tune=False) == dict(kernel=H.KERNEL_TILED, tile=256, tile2=128, block=0)
    akey = A._key("arena", 14, H.FP32, H.LIMITER_BJ)
    cache.write_text(json.dumps({akey: {"best": {"tile": 64, "ms_per_step": 0.2}}}))
    assert A.best_arena_tile(16_000, H.FP32, tune=False) == 64
