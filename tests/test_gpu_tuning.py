"""Autotuner on the GPU (b2f_autotune through the C ABI): the recorded
tuning is the fastest candidate that agrees with the default plan, a plan
built from the tuned configuration still matches the FP64 oracle, and a
snapshot saved on this device loads back with the device check."""
import pytest

import wgpufft_b200 as w
from tests.gpu_util import check_c2c

pytestmark = pytest.mark.gpu

K = w.FftTransformKind


@pytest.fixture(autouse=True)
def clean_snapshot():
    w.tuning_snapshot_clear()
    yield
    w.tuning_snapshot_clear()


@pytest.mark.parametrize("cfg", [
    w.FftConfig.new(1024).with_batch(512),
    w.FftConfig.new(4099).with_batch(8),
    w.FftConfig.new_nd([96, 40]).with_batch(3),
    w.FftConfig.new(4096).with_batch(16).with_precision(w.FftPrecision.F64),
])
def test_autotune_records_a_matching_fastest_candidate(cuda, cfg):
    rep = w.autotune(cfg, K.C2c, device=0, reps=5)
    assert rep["default_us"] > 0 and 0 < rep["best_us"] <= rep["default_us"]
    ok = [c for c in rep["candidates"] if c["ok"]]
    assert ok, rep
    assert all(c["us"] >= rep["best_us"] - 1e-3 for c in ok)
    best = rep["best"]
    tuned, found = w.tuned_config(cfg)
    assert found
    t = tuned.tuning()
    assert (t.lines_per_block, t.threads_per_block, int(t.twiddle_table), t.radix_order) == \
        (best["lines_per_block"], best["threads_per_block"], best["twiddle_table"],
         best["radix_order"])
    assert any(c["radix_order"] == 1 for c in rep["candidates"])
    check_c2c(tuned, seed=3)


def test_autotune_real_transform_and_device_checked_load(cuda, tmp_path):
    cfg = w.FftConfig.new_nd([256, 64])
    rep = w.autotune(cfg, K.R2c, device=0, reps=5)
    assert rep["key"].startswith("r2c/f32/forward/")
    snap = w.tuning_snapshot_json()
    assert snap["device"].startswith("NVIDIA") and len(snap["entries"]) == 1
    path = tmp_path / "snap.json"
    w.tuning_snapshot_save(str(path))
    w.tuning_snapshot_clear()
    w.tuning_snapshot_load(str(path), device=0)
    assert w.tuning_snapshot_json() == snap
    assert w.tuned_config(cfg, K.R2c)[1]
