"""Host logic of the render autotuner (svraster_b200/autotune.py) on the CPU: the compiled
launch configurations the library reports, the process-wide selection, and the tuner's
choice and JSON cache with the kernel timings replaced by a table (no GPU launch)."""
import json

import pytest

from svraster_b200 import autotune


@pytest.fixture
def restore_config():
    before = autotune.get_config()
    yield
    autotune.set_config(*before)


def test_compiled_configurations():
    cfg = autotune.configs()
    assert [r[0] for r in cfg["fwd"]] == list(range(len(cfg["fwd"]))) and len(cfg["fwd"]) == 6
    assert [r[0] for r in cfg["bwd"]] == list(range(len(cfg["bwd"]))) and len(cfg["bwd"]) == 6
    for rows in cfg.values():
        variants = [(impl, ring, ctas) for _, impl, ring, ctas in rows]
        assert len(set(variants)) == len(variants)             # distinct schedules
        assert all(impl in (0, 1, 2, 3) and 3 <= ring <= 4 and 2 <= ctas <= 5 for impl, ring, ctas in variants)
        assert variants[0][0] == 3                             # the default family


def test_set_and_get_config(restore_config):
    autotune.set_config(2, 4)
    assert autotune.get_config() == (2, 4)
    with pytest.raises(RuntimeError):
        autotune.set_config(6, 0)
    with pytest.raises(RuntimeError):
        autotune.set_config(0, -1)
    assert autotune.get_config() == (2, 4)                      # a rejected choice changes nothing


def test_tuner_picks_fastest_and_caches(tmp_path, monkeypatch, restore_config):
    fwd_ms = [2.5, 2.4, 2.9, 3.0, 2.45, 2.6]
    bwd_ms = [3.0, 3.3, 3.7, 3.9, 2.8, 3.4]
    seen = []

    def fake_time(fn, reps):
        f, b = autotune.get_config()
        kind = fn()
        seen.append((kind, f, b))
        return fwd_ms[f] if kind == "fwd" else bwd_ms[b]

    monkeypatch.setattr(autotune, "_time", fake_time)
    cache = tmp_path / "sub" / "tune.json"
    res = autotune.tune_render(lambda: "fwd", lambda: "bwd", key="gpu|w", cache=str(cache))
    assert res["fwd"] == 1 and res["bwd"] == 4
    assert autotune.get_config() == (1, 4)
    cfg = autotune.configs()
    assert res["fwd_config"] == {"impl": cfg["fwd"][1][1], "ring": cfg["fwd"][1][2], "ctas_per_sm": cfg["fwd"][1][3]}
    # the adjoint configurations are timed with the chosen forward one in force
    assert all(f == 1 for kind, f, _ in seen if kind == "bwd")
    stored = json.loads(cache.read_text())["gpu|w"]
    assert (stored["fwd"], stored["bwd"]) == (1, 4)
    # a second call with the same key reuses the stored choice without timing anything
    autotune.set_config(0, 0)
    seen.clear()
    res2 = autotune.tune_render(lambda: "fwd", lambda: "bwd", key="gpu|w", cache=str(cache))
    assert res2["cached"] and not seen and autotune.get_config() == (1, 4)
    # another key is timed and added beside the first
    res3 = autotune.tune_render(lambda: "fwd", lambda: "bwd", key="gpu|other", cache=str(cache))
    assert "cached" not in res3 and set(json.loads(cache.read_text())) == {"gpu|w", "gpu|other"}
