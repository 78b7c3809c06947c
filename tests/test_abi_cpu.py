"""C ABI and host planner checks that need no GPU: the library loads, exports
every symbol the public header declares, validates configurations the way
the crate's FftConfig/FftTuning do, and plans the routes and stages the
transform path needs (plan-only mode builds no device state)."""
import ctypes
import os
import re

import pytest

import wgpufft_b200 as w
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "wgpufft_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(b2f_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = w.lib()
    syms = header_symbols()
    assert len(syms) >= 30
    for s in syms:
        assert hasattr(L, s), s
    assert L.b2f_version().startswith(b"wgpufft_b200")


def test_python_binding_declares_every_symbol_with_its_arity():
    # a symbol without argtypes would pass 64-bit pointers as C ints
    src = open(os.path.join(ROOT, "include", "wgpufft_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    L = w.lib()
    protos = re.findall(r"\b(b2f_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", src)
    assert len(protos) >= 30
    for name, params in protos:
        params = params.strip()
        arity = 0 if params in ("", "void") else params.count(",") + 1
        fn = getattr(L, name)
        assert fn.argtypes is not None, name
        assert len(fn.argtypes) == arity, name


def test_status_strings_name_reference_variants():
    L = w.lib()
    assert L.b2f_status_string(1) == b"ZeroLength"
    assert L.b2f_status_string(12) == b"BufferViewTooSmall"
    assert L.b2f_status_string(14) == b"GpuPlanResourceAllocationFailed"


def kind_of(cfg):
    with pytest.raises(w.FftError) as e:
        cfg.validate()
    return e.value.kind


def test_config_validation_mirrors_reference():
    # src/config.rs tests: rejects_zero_length, validates_nd_axes_and_batch,
    # rejects_total_complex_count_above_u32_index_space.
    assert kind_of(w.FftConfig.new(0)) == "ZeroLength"
    assert kind_of(w.FftConfig.new_nd([])) == "ZeroLength"
    assert kind_of(w.FftConfig.new(8).with_batch(0)) == "ZeroBatch"
    assert kind_of(w.FftConfig.new_nd([2, 3]).with_axes([])) == "EmptyAxes"
    assert kind_of(w.FftConfig.new_nd([2, 3]).with_axes([2])) == "InvalidAxis"
    assert kind_of(w.FftConfig.new_nd([2, 3]).with_axes([1, 1])) == "DuplicateAxis"
    assert kind_of(w.FftConfig.new(1 << 16).with_batch(1 << 16)) == "LengthTooLarge"
    w.FftConfig.new(17).validate()
    w.FftConfig.new_nd([8, 29, 34]).validate()
    assert kind_of(w.FftConfig.new_nd([1, 4])) == "UnsupportedLength"
    w.FftConfig.new(1).validate()


def test_required_buffer_size_and_scale():
    # src/config.rs computes_required_buffer_size / applies_normalization_by_direction.
    assert w.FftConfig.new(8).with_batch(1).required_buffer_size_bytes() == 64
    assert w.FftConfig.new_nd([2, 3]).with_batch(4).required_buffer_size_bytes() == 192
    assert (w.FftConfig.new_nd([2, 3]).with_batch(4).with_precision(w.FftPrecision.F64)
            .required_buffer_size_bytes() == 384)
    assert (w.FftConfig.new_nd([2, 3]).with_batch(4).with_precision(w.FftPrecision.Df64)
            .required_buffer_size_bytes() == 384)
    assert w.FftConfig.inverse(4).scale() == 0.25
    assert w.FftConfig.new(4).scale() == 1.0
    assert w.FftConfig.inverse_nd([2, 3]).scale() == pytest.approx(1.0 / 6.0)
    assert (w.FftConfig.new(4).with_normalization(w.Normalization.Forward).scale() == 0.25)
    assert (w.FftConfig.new(4).with_normalization(w.Normalization.Orthogonal).scale() == 0.5)
    # f32 scale is computed in f32 as the reference does
    s = w.FftConfig.inverse(3).scale()
    assert s == O.scale_f32(3, True, O.NORM_INVERSE)


def test_tuning_validation_mirrors_reference():
    # src/config.rs validates_scalar_tuning_controls / validates_forced_axis_tuning.
    T = w.FftTuning
    bad = [
        T().with_workgroup_size(0), T().with_workgroup_size(48),
        T().with_fused_workgroup_size(3), T().with_rader_max_prime(1),
        T().with_segmented_burst_depth(4), T().with_threads_per_block(1024),
    ]
    for t in bad:
        assert kind_of(w.FftConfig.new(16).with_tuning(t)) == "InvalidTuning"
    assert kind_of(w.FftConfig.new(17).with_tuning(
        T().with_force_rader_axes([0]).with_force_bluestein_axes([0]))) == "InvalidTuning"
    assert kind_of(w.FftConfig.new(16).with_tuning(T().with_force_rader_axes([0]))) == "InvalidTuning"
    assert kind_of(w.FftConfig.new(16).with_tuning(T().with_force_rader_axes([1]))) == "InvalidTuning"
    assert kind_of(w.FftConfig.new_nd([17, 4]).with_axes([1]).with_tuning(
        T().with_force_rader_axes([0]))) == "InvalidTuning"
    assert kind_of(w.FftConfig.new(17).with_tuning(
        T().with_swap_to_2_stage_4_step(8).with_swap_to_3_stage_4_step(4))) == "InvalidTuning"
    w.FftConfig.new(17).with_tuning(T().with_force_rader_axes([0])).validate()
    w.FftConfig.new(17).with_tuning(T().with_force_bluestein_axes([0])).validate()


def plan_only(cfg, kind=w.FftTransformKind.C2c):
    return w.FftPlan.plan_only(cfg, kind)


def test_axis_kinds_and_routes():
    # src/runtime/axis_policy.rs classifies_smooth_prime_and_composite_lengths,
    # resolves_axis_kinds_for_shape_in_axis_order, config_tuning_changes_...
    for n, kind in [(8, "mixed"), (21, "mixed"), (17, "rader"), (29, "rader"),
                    (34, "bluestein"), (4099, "rader"), (8209, "bluestein")]:
        p = plan_only(w.FftConfig.new(n))
        assert p.axis_kinds() == [kind], n
    p = plan_only(w.FftConfig.new_nd([8, 29, 34]))
    assert p.axis_kinds() == ["mixed", "rader", "bluestein"]
    assert p.route() == "axis-sequence"
    p = plan_only(w.FftConfig.new_nd([8, 29, 34]).with_axes([2, 0]))
    assert p.axis_kinds() == ["bluestein", "mixed"]
    p = plan_only(w.FftConfig.new(17).with_tuning(w.FftTuning().with_rader_max_prime(13)))
    assert p.axis_kinds() == ["bluestein"]
    p = plan_only(w.FftConfig.new_nd([17, 8]).with_tuning(
        w.FftTuning().with_force_bluestein_axes([0])))
    assert p.axis_kinds() == ["bluestein", "mixed"]
    p = plan_only(w.FftConfig.new(8209).with_tuning(w.FftTuning().with_force_rader_axes([0])))
    assert p.axis_kinds() == ["rader"]
    assert plan_only(w.FftConfig.new(1024).with_batch(512)).route() == "mixed-radix"
    assert plan_only(w.FftConfig.new(1009)).route() == "rader"
    assert plan_only(w.FftConfig.new(34)).route() == "bluestein"
    assert plan_only(w.FftConfig.new(1)).route() == "direct-dft"


def test_factors_match_reference_factorisation():
    for n in [1024, 15015, 4096, 360, 2 ** 20]:
        assert plan_only(w.FftConfig.new(n)).factors() == O.factor_supported_length(n)


def test_single_pass_and_four_step_stages():
    d = plan_only(w.FftConfig.new(1024).with_batch(512)).diagnostics()
    assert [s["label"] for s in d["stages"]] == ["fused-pow2-workgroup-stage"]
    assert d["stages"][0]["radices"] == [16, 16, 4]
    d = plan_only(w.FftConfig.new(1 << 20).with_batch(2)).diagnostics()
    assert [s["label"] for s in d["stages"]] == ["smooth-axis-phase1-fused-pow2-stage",
                                                "smooth-axis-phase2-fused-pow2-stage"]
    p = plan_only(w.FftConfig.new(1 << 20).with_batch(2))
    assert p.workspace_size_bytes() == (1 << 21) * 8
    d = plan_only(w.FftConfig.new(1009)).diagnostics()
    assert d["stages"][0]["label"] == "rader-fused-workgroup-stage"
    assert d["stages"][0]["convolution_length"] == 1008
    d = plan_only(w.FftConfig.new(4099)).diagnostics()
    # p - 1 = 2*3*683 is not smooth: Bluestein over a 7-smooth length >= 2p-1
    assert d["stages"][0]["label"] == "bluestein-fused-workgroup-stage"
    m = d["stages"][0]["convolution_length"]
    assert 2 * 4099 - 1 <= m <= 9 * 4099 // 4
    # chosen by estimated cost among the 7-smooth lengths that fit one CTA:
    # 9216 = 2^10 * 3^2 (radix 16, 16, 4, 9) over 8232 = 2^3 * 3 * 7^3
    assert m == 9216 and sorted(d["stages"][0]["radices"]) == [4, 9, 16, 16]


def test_real_plans():
    p = plan_only(w.FftConfig.new_nd([256, 256, 256]), w.FftTransformKind.R2c)
    assert p.required_input_buffer_size_bytes() == 256 ** 3 * 4
    assert p.required_output_buffer_size_bytes() == 129 * 256 * 256 * 8
    assert p.packed_shape() == [129, 256, 256]
    assert not p.supports_in_place()
    with pytest.raises(w.FftError) as e:
        plan_only(w.FftConfig.new(8), w.FftTransformKind.C2r)
    assert e.value.kind == "InvalidRealTransformDirection"
    with pytest.raises(w.FftError) as e:
        plan_only(w.FftConfig.new_nd([4, 4]).with_axes([1]), w.FftTransformKind.R2c)
    assert e.value.kind == "UnsupportedRealAxes"
    with pytest.raises(w.FftError) as e:
        plan_only(w.FftConfig.new(8).with_precision(w.FftPrecision.Df64), w.FftTransformKind.R2c)
    assert e.value.kind == "PrecisionUnsupported"


def test_execute_on_plan_only_plan_fails_loudly():
    p = plan_only(w.FftConfig.new(16))
    with pytest.raises(w.FftError) as e:
        p.execute_checked((0x1000, 128), (0x2000, 128))
    assert e.value.kind == "DeviceError"


def test_tensor_core_knob_routes_and_validates():
    tc = w.FftTuning().with_tensor_cores(True)
    d = plan_only(w.FftConfig.new(64).with_batch(1000).with_tuning(tc)).diagnostics()
    assert [s["kind"] for s in d["stages"]] == ["tensor-core-dft"]
    # only length-64 f32 lines of axis 0 take the tensor-core layer
    for cfg in (w.FftConfig.new(128).with_tuning(tc),
                w.FftConfig.new(64).with_precision(w.FftPrecision.F64).with_tuning(tc),
                w.FftConfig.new_nd([32, 64]).with_tuning(tc)):
        assert all(s["kind"] != "tensor-core-dft" for s in plan_only(cfg).diagnostics()["stages"])
    with pytest.raises(w.FftError) as e:
        w.FftConfig.new(64).with_tuning(w.FftTuning().with_tensor_cores(2)).validate()
    assert e.value.kind == "InvalidTuning"


def test_batch_argument_checks_before_any_device_call():
    # b2f_batch_new validates lines on the host (the reference's checked
    # execution reports the same variants: src/error.rs)
    cases = [
        (([], []), {}, "InvalidArgument"),
        (([16, 0], [0, 16]), {}, "ZeroLength"),
        (([16, 16], [0, 8]), {}, "InvalidArgument"),          # overlapping lines
        (([1 << 33], [0]), {}, "LengthTooLarge"),
        (([16], [(1 << 64) - 8]), {}, "InvalidArgument"),     # beyond the address range
        (([16], [0]), {"direction": 2}, "InvalidArgument"),
        (([16], [0]), {"normalization": 7}, "InvalidArgument"),
    ]
    for (lengths, offsets), kw, kind in cases:
        with pytest.raises(w.FftError) as e:
            w.FftBatch(lengths, offsets, **kw)
        assert e.value.kind == kind, (lengths, offsets, kw, e.value)


def test_layout_status_strings():
    # src/error.rs:65-77
    L = w.lib()
    assert [L.b2f_status_string(c) for c in (22, 23, 24, 25)] == [
        b"BufferLayoutZeroStride", b"BufferLayoutBatchStrideTooSmall",
        b"BufferLayoutOutOfBounds", b"BufferLayoutTooLarge"]


def test_small_volume_eligibility():
    # src/runtime/small_volume.rs:223-272: f32, rank >= 2, every axis, at most
    # 4096 points, smooth axes, no forced axes, fuse_small_volumes on
    def labels(cfg):
        return [s["label"] for s in plan_only(cfg).diagnostics()["stages"]]
    for shape in ([8, 8, 8], [64, 64], [16, 16, 16], [3, 5, 7], [2, 2048]):
        assert labels(w.FftConfig.new_nd(shape).with_batch(3)) == ["small-volume-stage"], shape
    assert "small-volume-stage" not in labels(w.FftConfig.new_nd([64, 128]))       # 8192 points
    assert "small-volume-stage" not in labels(w.FftConfig.new_nd([8, 29, 4]))       # prime axis
    assert "small-volume-stage" not in labels(w.FftConfig.new(4096))               # rank 1
    assert "small-volume-stage" not in labels(w.FftConfig.new_nd([8, 8]).with_axes([1]))
    assert "small-volume-stage" not in labels(
        w.FftConfig.new_nd([8, 8]).with_precision(w.FftPrecision.F64))
    assert "small-volume-stage" not in labels(
        w.FftConfig.new_nd([8, 8]).with_tuning(w.FftTuning().with_fuse_small_volumes(False)))
