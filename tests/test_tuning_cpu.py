"""Tuning snapshot on the host: record / apply / save / load round trips and
the load-time checks (the crate's pipeline-cache snapshot contract,
src/runtime/pipeline_cache.rs:14-99, 160-260: JSON, schema, version and
integrity errors; a rejected file leaves the snapshot unchanged).  No GPU:
nothing here creates a plan."""
import json

import pytest

import wgpufft_b200 as w

K = w.FftTransformKind


@pytest.fixture(autouse=True)
def clean_snapshot():
    w.tuning_snapshot_clear()
    yield
    w.tuning_snapshot_clear()


def _seed():
    a = w.FftConfig.new(1024).with_batch(512)
    b = w.FftConfig.new_nd([64, 48])
    w.tuning_snapshot_record(a, K.C2c, 4, 256, 1, 10.5, 12.25)
    w.tuning_snapshot_record(b, K.R2c, 2, 0, 0, 3.0, 3.5, radix_order=1)
    return a, b


def test_record_apply_and_canonical_json():
    a, b = _seed()
    snap = w.tuning_snapshot_json()
    assert snap["schema"] == "wgpufft_b200.tuning" and snap["version"] == 2
    keys = [e["key"] for e in snap["entries"]]
    assert keys == sorted(keys)
    assert "c2c/f32/forward/inverse/shape=1024/axes=0/batch=512" in keys
    assert "r2c/f32/forward/inverse/shape=64,48/axes=0,1/batch=1" in keys
    tuned, found = w.tuned_config(a)
    assert found
    assert (tuned.tuning().lines_per_block, tuned.tuning().threads_per_block) == (4, 256)
    tuned_b, found_b = w.tuned_config(b, K.R2c)
    assert found_b and tuned_b.tuning().twiddle_table is False
    assert tuned_b.tuning().radix_order == 1 and tuned.tuning().radix_order == 0
    # the key covers kind, shape, batch and precision
    assert not w.tuned_config(b, K.C2c)[1]
    assert not w.tuned_config(a.with_batch(511))[1]
    assert not w.tuned_config(a.with_precision(w.FftPrecision.F64))[1]


def test_save_load_round_trip(tmp_path):
    _seed()
    path = tmp_path / "snap.json"
    w.tuning_snapshot_save(str(path))
    before = w.tuning_snapshot_json()
    w.tuning_snapshot_clear()
    assert w.tuning_snapshot_json()["entries"] == []
    w.tuning_snapshot_load(str(path))
    assert w.tuning_snapshot_json() == before


def test_record_rejects_invalid_tuning():
    c = w.FftConfig.new(1024)
    with pytest.raises(w.FftError) as e:
        w.tuning_snapshot_record(c, K.C2c, 1, 100, 1)  # threads_per_block not a power of two
    assert e.value.kind == "InvalidTuning"
    with pytest.raises(w.FftError):
        w.tuning_snapshot_record(c, K.C2c, 1, 64, 2)
    with pytest.raises(w.FftError) as e:
        w.tuning_snapshot_record(c, K.C2c, 1, 64, 1, radix_order=2)
    assert e.value.kind == "InvalidTuning"


def _load_bad(tmp_path, text, kind):
    path = tmp_path / "bad.json"
    path.write_text(text)
    with pytest.raises(w.FftError) as e:
        w.tuning_snapshot_load(str(path))
    assert e.value.kind == kind, e.value


def test_load_rejections_keep_the_snapshot(tmp_path):
    _seed()
    path = tmp_path / "snap.json"
    w.tuning_snapshot_save(str(path))
    good = json.loads(path.read_text())
    before = w.tuning_snapshot_json()

    _load_bad(tmp_path, "{not json", "SnapshotJson")
    _load_bad(tmp_path, json.dumps({**good, "extra": 1}), "SnapshotJson")
    _load_bad(tmp_path, json.dumps({**good, "schema": "wgpu-fft.pipeline-cache"}),
              "SnapshotSchemaMismatch")
    _load_bad(tmp_path, json.dumps({**good, "version": 1}), "SnapshotVersionMismatch")
    # an edited value: the checksum no longer matches
    edited = json.loads(json.dumps(good))
    edited["entries"][0]["lines_per_block"] = 8
    _load_bad(tmp_path, json.dumps(edited), "SnapshotIntegrity")
    # an edited device: the checksum covers it too
    _load_bad(tmp_path, json.dumps({**good, "device": "NVIDIA B200 sm_100"}), "SnapshotIntegrity")
    # unordered (and duplicate) keys
    swapped = json.loads(json.dumps(good))
    swapped["entries"] = swapped["entries"][::-1]
    _load_bad(tmp_path, json.dumps(swapped), "SnapshotIntegrity")
    dup = json.loads(json.dumps(good))
    dup["entries"] = [dup["entries"][0], dup["entries"][0]]
    _load_bad(tmp_path, json.dumps(dup), "SnapshotIntegrity")
    # a key that does not re-derive from its fields
    noncanon = json.loads(json.dumps(good))
    noncanon["entries"][0]["key"] = noncanon["entries"][0]["key"].replace("shape=1024", "shape=01024")
    _load_bad(tmp_path, json.dumps(noncanon), "SnapshotIntegrity")
    # a tuning value its configuration rejects
    badval = json.loads(json.dumps(good))
    badval["entries"][0]["threads_per_block"] = 100
    _load_bad(tmp_path, json.dumps(badval), "SnapshotIntegrity")
    badro = json.loads(json.dumps(good))
    badro["entries"][0]["radix_order"] = 3
    _load_bad(tmp_path, json.dumps(badro), "SnapshotIntegrity")

    assert w.tuning_snapshot_json() == before
