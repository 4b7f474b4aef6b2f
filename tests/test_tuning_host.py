"""The persisted autotuning table: round trip through its JSON file, and files
written for another device or library version are ignored (no GPU needed)."""
import json

from astro_transit_gpu_b200.tuning import TuningTable, key_str, table_path


def test_table_round_trip(tmp_path):
    path = table_path("NVIDIA B200", (10, 0), str(tmp_path))
    assert path.endswith("tuning-NVIDIA_B200-sm100.json")
    t = TuningTable(path, "NVIDIA B200", "lib 1").load()
    assert t.get(("fast", 13, 14, 15)) is None
    t.put(("fast", 13, 14, 15), {"tile_periods": 32, "search_ms": {"8": 2.0, "32": 1.5}})
    t.put(("parity", 12, 13, 12), {"tile_periods": 64})
    t.save()
    u = TuningTable(path, "NVIDIA B200", "lib 1").load()
    assert u.get(("fast", 13, 14, 15)) == {"tile_periods": 32, "search_ms": {"8": 2.0, "32": 1.5}}
    assert u.get(("parity", 12, 13, 12))["tile_periods"] == 64
    assert json.load(open(path))["entries"][key_str(("parity", 12, 13, 12))]["tile_periods"] == 64


def test_table_ignores_other_devices_versions_and_bad_files(tmp_path):
    path = str(tmp_path / "t.json")
    t = TuningTable(path, "NVIDIA B200", "lib 1")
    t.put(("fast", 1, 2, 3), {"tile_periods": 8})
    t.save()
    assert TuningTable(path, "NVIDIA B200", "lib 2").load().get(("fast", 1, 2, 3)) is None
    assert TuningTable(path, "Other GPU", "lib 1").load().get(("fast", 1, 2, 3)) is None
    with open(path, "w") as f:
        f.write("{not json")
    assert TuningTable(path, "NVIDIA B200", "lib 1").load().entries == {}
    assert TuningTable(str(tmp_path / "missing.json"), "x", "y").load().entries == {}


def test_tuned_config_fills_only_knobs_left_at_zero(tmp_path):
    """BLSEngine.tuned_config takes every knob the config leaves at 0 (tile
    size, fold threshold, CTA size) from the table entry of the batch's kind,
    and keeps the ones the caller set; no entry, no change."""
    from types import SimpleNamespace
    from astro_transit_gpu_b200.engine import BLSEngine, SearchConfig
    table = TuningTable(str(tmp_path / "t.json"), "NVIDIA B200", "lib 1")
    key = ("fast", 11, 14, 15)
    table.put(key, {"tile_periods": 32, "merge_run": 16, "cta_threads": 256, "best_ms": 1.0})
    fake = SimpleNamespace(tuning=table, tune_key=lambda batch, config: key)
    cfg = BLSEngine.tuned_config(fake, None, SearchConfig("fast", n_bins=200))
    assert (cfg.tile_periods, cfg.merge_run, cfg.cta_threads) == (32, 16, 256)
    cfg = BLSEngine.tuned_config(fake, None, SearchConfig("fast", tile_periods=8, cta_threads=512))
    assert (cfg.tile_periods, cfg.merge_run, cfg.cta_threads) == (8, 16, 512)
    # an entry from before the CTA-size knob existed leaves it at the default
    table.put(key, {"tile_periods": 16, "merge_run": 0})
    cfg = BLSEngine.tuned_config(fake, None, SearchConfig("fast"))
    assert (cfg.tile_periods, cfg.merge_run, cfg.cta_threads) == (16, 0, 0)
    fake.tune_key = lambda batch, config: ("parity", 1, 1, 1)
    assert BLSEngine.tuned_config(fake, None, SearchConfig("parity")) == SearchConfig("parity")


def test_autotune_searches_cta_then_tile_then_fold(tmp_path):
    """BLSEngine.autotune with a stand-in timer: it keeps the fastest CTA
    size, then the fastest tile at that size, then the fastest fold threshold
    at both, stores the result for the batch's kind and persists it."""
    from types import SimpleNamespace
    from astro_transit_gpu_b200.engine import BLSEngine, SearchConfig
    cost = {"cta": {512: 10.0, 256: 8.0}, "tile": {8: 3.0, 16: 1.0, 32: 2.0, 64: 2.5},
            "fold": {0: 0.5, -1: 0.9, 4: 0.2, 16: 0.7}}
    seen = []

    def timer(batch, cfg, repeats):
        seen.append((cfg.cta_threads, cfg.tile_periods, cfg.merge_run))
        return (cost["cta"][cfg.cta_threads] + cost["tile"].get(cfg.tile_periods, 0.0)
                + cost["fold"][cfg.merge_run])

    table = TuningTable(str(tmp_path / "t.json"), "NVIDIA B200", "lib 1")
    key = ("fast", 11, 14, 15)
    fake = SimpleNamespace(tuning=table, tune_key=lambda batch, config: key, _time_search=timer)
    best = BLSEngine.autotune(fake, None, SearchConfig("fast"))
    assert best == {"cta_threads": 256, "tile_periods": 16, "merge_run": 4}
    # the CTA sizes first (tile and fold at the config's), then tiles, then folds
    assert seen[:2] == [(512, 0, 0), (256, 0, 0)]
    assert seen[2:6] == [(256, tp, 0) for tp in (8, 16, 32, 64)]
    assert seen[6:] == [(256, 16, mr) for mr in (0, -1, 4, 16)]
    again = TuningTable(table.path, "NVIDIA B200", "lib 1").load().get(key)
    assert {k: again[k] for k in best} == best
