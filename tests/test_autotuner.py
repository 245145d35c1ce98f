"""Host-side parts of the autotuner: the reference interface's benchmark case
and sanity check (GPUSimulators/Autotuner.py:226-287), the cache lookup, and
the agreement of the tuned tile indices with the library's kernel tables."""

import numpy as np

from finitevolumegpu_b200.Autotuner import Autotuner, size_class


def test_gen_test_data_is_the_cosine_bump():
    h, hu, hv, dx, dy, dt = Autotuner.gen_test_data(128, 96, 9.81)
    assert h.shape == hu.shape == hv.shape == (96, 128)
    assert h.dtype == np.float32 and hu.dtype == np.float32
    assert dx == 100.0 / 128 and dy == 100.0 / 96
    # depth 0.5 outside the bump, up to 0.6 at its centre; momentum 0 .. 0.1
    assert abs(float(h.min()) - 0.5) < 1e-6 and abs(float(h.max()) - 0.6) < 1e-3
    assert np.array_equal(hu, hv) and float(hu.min()) >= 0.0 and float(hu.max()) <= 0.1 + 1e-6
    assert np.allclose(h - 0.5, hu, atol=1e-6)
    assert abs(dt - 0.7 * min(dx, dy) / (0.1 * np.sqrt(2.0) + np.sqrt(9.81 * 0.6))) < 1e-12
    # the bump (radius width / 5 = 20) is centred: symmetric under both flips
    assert np.allclose(h, h[:, ::-1]) and np.allclose(h, h[::-1, :])


def test_sanity_check():
    a = np.array([0.4, 0.5, 0.6], dtype=np.float32)
    assert Autotuner.sanity_check(a, 0.3, 0.7)
    assert not Autotuner.sanity_check(a, 0.45, 0.7)
    assert not Autotuner.sanity_check(a, 0.3, 0.55)
    assert not Autotuner.sanity_check(np.array([0.4, np.nan], dtype=np.float32), 0.3, 0.7)


def test_size_classes():
    assert size_class(4096, 4096) == "4^12"
    assert size_class(256, 256) == "4^8"
    assert size_class(4096, 1024) == size_class(2048, 2048) == "4^11"


SCHEME_OF = {"KP07_DIMSPLIT": "KP07_dimsplit", "HLL2": "HLL2", "WAF": "WAF", "FORCE": "FORCE", "HLL": "HLL",
             "EE2D_KP07_DIMSPLIT": "EE2D_KP07_dimsplit", "LXF": "LxF", "KP07": "KP07"}


def _table_counts(name):
    """Entries per scheme of a tile table in fv_api.cu (kTable, kBatchTable)."""
    import collections
    import os
    import re

    from conftest import ROOT

    src = open(os.path.join(ROOT, "finitevolumegpu_b200", "csrc", "fv_api.cu")).read()
    body = re.search(r"const \w+ %s\[\] = \{(.*?)\n\};" % name, src, re.S).group(1)
    return collections.Counter(SCHEME_OF[m] for m in re.findall(r"\{FV_(\w+), \d+, \d+, \d+", body))


def test_tile_tables_match_the_library():
    """The tile-configuration counts the tuner sweeps and every cached choice
    exist in the library's kernel tables (an index past them fails at create)."""
    import json

    from finitevolumegpu_b200.Autotuner import BATCH_TILE_CONFIGS, DEFAULT_CACHE, TILE_CONFIGS

    stage, batch = _table_counts("kTable"), _table_counts("kBatchTable")
    assert dict(stage) == TILE_CONFIGS
    assert dict(batch) == BATCH_TILE_CONFIGS
    cache = json.load(open(DEFAULT_CACHE))
    for device, schemes in cache.items():
        for key, entry in schemes.items():
            if key.startswith("batch:"):
                assert 0 <= int(entry["tile"]) < BATCH_TILE_CONFIGS[key[6:]], (device, key)
            else:
                for cls, best in entry.items():
                    assert 0 <= int(best["tile"]) < TILE_CONFIGS[key], (device, key, cls)


def test_get_tile_falls_back(tmp_path):
    import json

    path = tmp_path / "cache.json"
    json.dump({"Dev": {"HLL": {"4^8": {"tile": 2}, "4^12": {"tile": 1}}, "batch:HLL": {"tile": 3}}}, open(path, "w"))
    t = Autotuner(cache_file=str(path))
    assert t.get_tile("HLL", 256, 256, "Dev") == 2
    assert t.get_tile("HLL", 4096, 4096, "Dev") == 1
    assert t.get_tile("HLL", 512, 512, "Dev") == 2      # 4^9: nearest tuned class is 4^8
    assert t.get_tile("HLL", 2048, 2048, "Dev") == 1    # 4^11: nearest tuned class is 4^12
    assert t.get_tile("WAF", 256, 256, "Dev") == -1     # scheme never tuned: library default
    assert t.get_tile("HLL", 256, 256, "Other") == -1   # device never tuned
    assert t.get_batch_tile("HLL", "Dev") == 3 and t.get_batch_tile("WAF", "Dev") == -1
