"""Autotuner: the CTA-size variants per length, the measured choice being
installed for later plans, and the JSON cache round trip."""
import json

import pytest

from openvsip_b200 import autotune


def test_variants_per_length():
    assert autotune.variants(64) == (256,)
    assert autotune.variants(256) == (128, 256)
    assert autotune.variants(4096) == (128, 256, 512)
    assert autotune.variants(8192) == (128, 256, 512)
    assert autotune.variants(16384) == (256, 512, -256)
    assert autotune.variants(32768) == (256, 512, -256)


@pytest.mark.gpu
def test_tune_installs_choice_and_cache_round_trip(tmp_path, monkeypatch):
    from openvsip_b200 import _lib
    lib = _lib.lib()
    monkeypatch.setenv("FCB200_TUNE_CACHE", str(tmp_path / "tuning.json"))
    res = autotune.tune_plans(lengths=(1024, 16384), kinds=("fastconv",), samples=1 << 22)
    for n in (1024, 16384):
        r = res[f"fastconv:{n}"]
        assert r["threads"] in autotune.variants(n)
        assert set(r["ms"]) == set(autotune.variants(n)) and all(v > 0 for v in r["ms"].values())
        assert lib.fcb_tune_get(n, autotune.KINDS["fastconv"]) == r["threads"]
    path = autotune.save(res)
    assert "fastconv:1024" in next(iter(json.load(open(path)).values()))
    # overwrite the installed choice, then restore it from the cache
    other = [t for t in autotune.variants(1024) if t != res["fastconv:1024"]["threads"]][0]
    _lib.check(lib.fcb_tune_set(1024, autotune.KINDS["fastconv"], other))
    assert lib.fcb_tune_get(1024, autotune.KINDS["fastconv"]) == other
    autotune.load(path)
    assert lib.fcb_tune_get(1024, autotune.KINDS["fastconv"]) == res["fastconv:1024"]["threads"]
    # leave the library defaults for the tests that follow
    for n, t in ((1024, 128), (16384, -256)):
        _lib.check(lib.fcb_tune_set(n, autotune.KINDS["fastconv"], t))
