"""Host logic of the batch autotuner (no GPU): signatures, the pick, the cache file."""
import json

import pytest

from fluid_b200 import autotune


class FakeProjector:
    def __init__(self, dims, precision="fp16"):
        self.dims = dims
        self.precision = precision


def test_signature_names_sizes_in_order_and_precision():
    ps = [FakeProjector((24, 30, 28)), FakeProjector((64, 48, 64))]
    assert autotune.signature(ps) == "fp16:24x30x28,64x48x64"
    assert autotune.signature(ps[::-1]) != autotune.signature(ps)


def test_pick_takes_the_fastest_and_rejects_all_failed():
    table = [dict(tuning={"a": 1}, sweeps=(1, 1), ms=3.0), dict(tuning={"a": 2}, sweeps=(1, 1), ms=2.0),
             dict(tuning={"a": 3}, sweeps=(2, 2), ms=2.0)]
    assert autotune.pick(table)["tuning"] == {"a": 2}
    with pytest.raises(RuntimeError):
        autotune.pick([dict(tuning={}, sweeps=(1, 1), ms=float("inf"))])


def test_cached_choice_is_returned_without_measuring(tmp_path):
    ps = [FakeProjector((16, 16, 16))]
    key = autotune.signature(ps)
    path = tmp_path / "tune.json"
    stored = {"tuning": {"fill_tiles": 148, "chunk_planes": 0, "box_shape": -1}, "sweeps": [1, 1], "ms": 1.5,
              "default_ms": 2.0, "table": []}
    path.write_text(json.dumps({key: stored}))
    autotune._cache.pop(key, None)

    def never():
        raise AssertionError("a cached batch must not be measured")

    res = autotune.autotune_batch(ps, [1 / 60], never, cache_path=str(path))
    assert res.tuning == stored["tuning"] and res.sweeps == (1, 1) and res.ms == 1.5
    autotune._cache.pop(key, None)


def test_tuning_defaults_and_rejected_fields():
    """The library's default layout, and tunings it refuses before touching a GPU."""
    import ctypes

    from fluid_b200 import _abi
    from fluid_b200.projector import batch_tuning
    assert batch_tuning().as_dict() == {"fill_tiles": 148, "chunk_planes": 0, "box_shape": -1, "parts": 1}
    L = _abi.load()
    out = ctypes.c_void_p()
    for bad in (dict(fill_tiles=0), dict(chunk_planes=-8), dict(chunk_planes=12), dict(chunk_planes=264), dict(box_shape=5),
                dict(parts=0), dict(parts=17)):
        t = batch_tuning(**bad)
        assert L.fluid_pp_batch_create_tuned(None, 0, ctypes.byref(t), ctypes.byref(out)) == _abi.INVALID_ARG, bad
    good = batch_tuning(parts=4)
    assert L.fluid_pp_batch_create_tuned(None, 0, ctypes.byref(good), ctypes.byref(out)) == _abi.INVALID_ARG
