"""GPU parity of the complex transforms, through the C ABI, against the FP64
oracle: every codelet radix, mixed lengths, Rader primes, Bluestein lengths,
long axes (four-step), N-D shapes and axis subsets, all normalisations,
forward and inverse, f32 / f64 / df64, in place and out of place, and the
recorder.  Case lists follow the reference's tests/gpu_c2c.rs, gpu_f64.rs,
gpu_df64.rs, gpu_accuracy.rs and gpu_long_axes.rs."""
import numpy as np
import pytest

import wgpufft_b200 as w
from oracle import oracle as O
from tests.gpu_util import TOL, check_c2c, from_device, oracle_c2c, run_c2c, signal, to_device

pytestmark = pytest.mark.gpu

F32, F64, DF64 = w.FftPrecision.F32, w.FftPrecision.F64, w.FftPrecision.Df64
INV = w.FftDirection.Inverse


@pytest.mark.parametrize("n", list(range(2, 22)) + [32, 49, 64, 100, 121, 128, 169, 243, 256,
                                                     360, 512, 1000, 1024, 2048, 3003, 4096,
                                                     8192])
def test_f32_mixed_radix_lengths(cuda, n):
    check_c2c(w.FftConfig.new(n).with_batch(3))
    check_c2c(w.FftConfig.new(n).with_batch(2).with_direction(INV), seed=1)


@pytest.mark.parametrize("p", [17, 29, 31, 127, 1009, 2003, 4099, 6121, 8209])
def test_f32_prime_lengths(cuda, p):
    check_c2c(w.FftConfig.new(p).with_batch(2), seed=p)
    check_c2c(w.FftConfig.new(p).with_direction(INV), seed=p + 1)


@pytest.mark.parametrize("n", [34, 46, 58, 3256, 10001, 20000])
def test_f32_bluestein_lengths(cuda, n):
    check_c2c(w.FftConfig.new(n).with_batch(2), seed=n)
    check_c2c(w.FftConfig.new(n).with_direction(INV), seed=n + 1)


@pytest.mark.parametrize("n,prec,tuning", [
    (40961, F32, w.FftTuning().with_force_rader_axes([0])),        # 2^13 * 5 + 1, forced
    (7681, F64, None),                                             # too long for one CTA in f64
    (7681, DF64, None),
    (65537, F64, w.FftTuning().with_rader_max_prime(1 << 20)),     # 2^16 + 1
])
def test_multipass_rader(cuda, n, prec, tuning):
    # primes whose line does not fit one CTA and whose p - 1 is smooth: the
    # gather, FFT_{p-1}, spectrum product, FFT_{p-1}, scatter passes
    cfg = w.FftConfig.new(n).with_batch(2).with_precision(prec)
    if tuning is not None:
        cfg = cfg.with_tuning(tuning)
    check_c2c(cfg, seed=n)
    check_c2c(cfg.with_direction(INV).with_normalization(w.Normalization.Orthogonal), seed=n + 1)
    labels = [st["label"] for st in w.FftPlan.c2c(cfg).diagnostics()["stages"]]
    assert labels[0] == "rader-gather-stage" and labels[-1] == "rader-scatter-stage", labels


@pytest.mark.parametrize("n", [622423, 1268090])
def test_f32_long_bluestein_lines(cuda, n):
    # one line whose Bluestein convolution spans many CTAs (prime; 2*5*173*733):
    # the chirp and spectrum passes spread one line over the whole grid
    check_c2c(w.FftConfig.new(n), seed=n)
    check_c2c(w.FftConfig.new(n).with_batch(2).with_direction(INV), seed=n + 1)


@pytest.mark.parametrize("n", [15015, 16384, 65536, 1 << 20])
def test_f32_long_axes(cuda, n):
    check_c2c(w.FftConfig.new(n).with_batch(2), seed=3)
    check_c2c(w.FftConfig.new(n).with_direction(INV), seed=4)


@pytest.mark.parametrize("shape,axes", [([8, 29, 34], None), ([8, 29, 34], [2, 0]),
                                        ([64, 32], None), ([32, 64], [1]), ([12, 25, 2], None),
                                        ([5, 7, 9], [1, 2]), ([256, 16384], [1]),
                                        ([3, 8192], [1]), ([129, 256, 4], None)])
def test_f32_nd_and_axis_subsets(cuda, shape, axes):
    cfg = w.FftConfig.new_nd(shape).with_batch(2)
    if axes is not None:
        cfg = cfg.with_axes(axes)
    check_c2c(cfg, seed=5)
    check_c2c(cfg.with_direction(INV), seed=6)


@pytest.mark.parametrize("norm", list(w.Normalization))
def test_normalisations(cuda, norm):
    for d in (w.FftDirection.Forward, INV):
        check_c2c(w.FftConfig.new_nd([16, 12]).with_normalization(norm).with_direction(d), seed=2)


def test_length_one(cuda):
    check_c2c(w.FftConfig.new(1))
    check_c2c(w.FftConfig.new(1).with_direction(INV))


def test_known_length_four(cuda):
    # src/math/mod.rs:575-612
    import torch
    x = np.array([1, 2, 3, 4], dtype=np.complex64)
    t = torch.from_numpy(x.view(np.float32)).cuda()
    out = torch.empty_like(t)
    w.FftPlan.c2c(w.FftConfig.new(4).with_normalization(w.Normalization.NONE)).execute_checked(t, out)
    got = from_device(out, F32)
    assert np.max(np.abs(got - np.array([10, -2 + 2j, -2, -2 - 2j]))) < 1e-6


@pytest.mark.parametrize("prec", [F64, DF64])
@pytest.mark.parametrize("n", [2, 3, 5, 7, 11, 13, 16, 17, 100, 1000, 1009, 3000, 3256, 4096,
                               2999, 65536])
def test_extended_precision_lengths(cuda, prec, n):
    check_c2c(w.FftConfig.new(n).with_batch(2).with_precision(prec), seed=11)
    check_c2c(w.FftConfig.new(n).with_direction(INV).with_precision(prec), seed=12)


@pytest.mark.parametrize("prec", [F64, DF64])
def test_extended_precision_nd(cuda, prec):
    check_c2c(w.FftConfig.new_nd([12, 25, 2]).with_precision(prec), seed=13)
    check_c2c(w.FftConfig.new_nd([8, 29, 34]).with_precision(prec).with_direction(INV), seed=14)


@pytest.mark.parametrize("prec", [F64, DF64])
def test_extended_precision_2_20_batch_16(cuda, prec):
    # the precision configuration: 1D N = 2^20, batch 16
    check_c2c(w.FftConfig.new(1 << 20).with_batch(16).with_precision(prec), seed=8)


@pytest.mark.parametrize("shape,prec", [([1024], F32), ([8, 29, 34], F32), ([15015], F32),
                                        ([1 << 20], F32), ([4099], F32), ([1000], F64),
                                        ([4096], DF64)])
def test_in_place_equals_out_of_place(cuda, shape, prec):
    cfg = w.FftConfig.new_nd(shape).with_batch(2).with_precision(prec)
    x = signal(cfg.total_complex_len(), 21)
    a, _, _ = run_c2c(cfg, x, in_place=False)
    b, _, _ = run_c2c(cfg, x, in_place=True)
    assert O.rel_l2(b, a) <= (1e-6 if prec == F32 else 1e-13)


def test_recorder_equals_separate_executions(cuda):
    import torch
    cfgs = [w.FftConfig.new(1024).with_batch(8), w.FftConfig.new_nd([64, 64]),
            w.FftConfig.new(1009).with_batch(3)]
    plans = [w.FftPlan.c2c(c) for c in cfgs]
    ins, outs_sep, outs_rec = [], [], []
    for i, c in enumerate(cfgs):
        t, _ = to_device(signal(c.total_complex_len(), 30 + i), F32)
        ins.append(t)
        outs_sep.append(torch.empty_like(t))
        outs_rec.append(torch.empty_like(t))
    for p, a, b in zip(plans, ins, outs_sep):
        p.execute_checked(a, b)
    torch.cuda.synchronize()
    rec = w.FftRecorder()
    for p, a, b in zip(plans, ins, outs_rec):
        p.record(rec, a, b)
    rec.submit()
    rec.submit()
    torch.cuda.synchronize()
    for a, b in zip(outs_sep, outs_rec):
        assert torch.equal(a, b)


def test_buffer_too_small_is_reported(cuda):
    import torch
    plan = w.FftPlan.c2c(w.FftConfig.new(1024).with_batch(4))
    small = torch.empty(1024 * 2, dtype=torch.float32, device="cuda")
    big = torch.empty(1024 * 8, dtype=torch.float32, device="cuda")
    with pytest.raises(w.FftError) as e:
        plan.execute_checked(small, big)
    assert e.value.kind == "BufferViewTooSmall"
    with pytest.raises(w.FftError) as e:
        plan.execute_in_place(small)
    assert e.value.kind == "BufferViewTooSmall"


def test_forced_routes_agree(cuda):
    # forced Rader / Bluestein on the same prime give the same transform
    x = signal(2 * 127, 40)
    cfg = w.FftConfig.new(127).with_batch(2)
    a, exact, _ = run_c2c(cfg, x)
    b, _, p = run_c2c(cfg.with_tuning(w.FftTuning().with_force_bluestein_axes([0])), x)
    assert p.axis_kinds() == ["bluestein"]
    ref = O.c2c_nd_f64(exact, [127], batch=2)
    assert O.rel_l2(a, ref) < 2e-6 and O.rel_l2(b, ref) < 2e-6


@pytest.mark.parametrize("n", [360, 1000, 2048, 3003, 15015, 1009, 4099])
@pytest.mark.parametrize("prec", [F32, F64])
def test_reversed_radix_order(cuda, n, prec):
    # tuning radix_order = 1 runs every stage schedule of the shared-memory
    # engine in reverse (small odd radices first; power-of-two lines leave
    # the register kernel): same transform within the tolerance
    t = w.FftTuning().with_radix_order(1)
    check_c2c(w.FftConfig.new(n).with_batch(3).with_precision(prec).with_tuning(t), seed=n)
    check_c2c(w.FftConfig.new(n).with_direction(INV).with_precision(prec).with_tuning(t),
              seed=n + 1)


@pytest.mark.parametrize("shape,batch", [([2048, 4096], 1), ([64, 256, 128], 2), ([1 << 16], 3),
                                         ([100, 200], 2), ([256, 256, 256], 1)])
def test_tma_column_tiles_equal_plain_loads(cuda, shape, batch):
    # column passes of <= 256 points staged by TMA in a persistent grid agree
    # with the plain-load passes (the fixed-length register kernels, whose
    # arithmetic is compiled separately) and with the oracle
    import torch
    cfg = w.FftConfig.new_nd(shape).with_batch(batch)
    x = signal(cfg.total_complex_len(), 11)
    got, exact, plan = run_c2c(cfg.with_tuning(w.FftTuning().with_tma_tiles(True)), x)
    stages = plan.diagnostics()["stages"]
    if shape != [100, 200]:
        assert any(s.get("tma_tiles") for s in stages), stages
    off, _, plan_off = run_c2c(cfg.with_tuning(w.FftTuning().with_tma_tiles(False)), x)
    assert not any(s.get("tma_tiles") for s in plan_off.diagnostics()["stages"])
    assert O.rel_l2(got, off) <= 1e-6
    ref = oracle_c2c(cfg, exact)
    assert O.rel_l2(got, ref) <= 2e-6 and O.rel_l2(off, ref) <= 2e-6
    plan.device_status()


def test_computed_twiddles_match_table(cuda):
    x = signal(4 * 4096, 41)
    cfg = w.FftConfig.new(4096).with_batch(4)
    a, exact, _ = run_c2c(cfg, x)
    b, _, _ = run_c2c(cfg.with_tuning(w.FftTuning().with_twiddle_table(False)), x)
    ref = O.c2c_nd_f64(exact, [4096], batch=4)
    assert O.rel_l2(a, ref) < 2e-6 and O.rel_l2(b, ref) < 2e-6


def test_one_multipass_plan_on_two_streams(cuda):
    # a two-pass (four-step) plan shares its workspace between executions:
    # executions issued on two streams at once must be ordered by the plan
    import torch
    n, batch = 1 << 20, 4
    cfg = w.FftConfig.new(n).with_batch(batch)
    plan = w.FftPlan.c2c(cfg)
    assert plan.workspace_size_bytes() > 0
    xs = [signal(n * batch, 50 + i) for i in range(2)]
    devs = [to_device(x, F32) for x in xs]
    outs = [torch.empty_like(d) for d, _ in devs]
    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    torch.cuda.synchronize()
    for _ in range(3):
        for (d, _), o, s in zip(devs, outs, streams):
            plan.execute_checked(d, o, stream=s)
    torch.cuda.synchronize()
    for (_, exact), o in zip(devs, outs):
        ref = O.c2c_nd_f64(exact, [n], batch=batch)
        assert O.rel_l2(from_device(o, F32), ref) <= 2e-6


def test_df64_canary_exact_words(cuda):
    # src/df64_canary.rs: every error-free-transform word of the df64 route
    # on the device equals the host's IEEE single-precision evaluation
    rep = w.validate_df64_invariants()
    assert rep["cases"] == 4 and rep["exact_words"] == 88


@pytest.mark.parametrize("shape,batch", [([8, 8, 8], 1), ([16, 16, 16], 2), ([64, 64], 3),
                                         ([12, 25, 2], 2), ([3, 5, 7], 5), ([2, 2048], 1),
                                         ([13, 11, 9], 4)])
def test_small_volume_route(cuda, shape, batch):
    # src/runtime/small_volume.rs: every axis of a <= 4096-point f32 volume
    # in one kernel; same results as the oracle, forward and inverse, every
    # normalisation, in place
    cfg = w.FftConfig.new_nd(shape).with_batch(batch)
    labels = [s["label"] for s in w.FftPlan.c2c(cfg).diagnostics()["stages"]]
    if np.prod(shape) <= 4096 and min(shape) > 1:
        assert labels == ["small-volume-stage"], labels
    check_c2c(cfg, seed=60)
    check_c2c(cfg.with_direction(INV), seed=61)
    for norm in w.Normalization:
        check_c2c(cfg.with_normalization(norm).with_direction(INV), seed=62)
    check_c2c(cfg, seed=63, in_place=True)


def test_small_volume_knob_off_uses_axis_passes(cuda):
    cfg = w.FftConfig.new_nd([16, 16]).with_tuning(w.FftTuning().with_fuse_small_volumes(False))
    labels = [s["label"] for s in w.FftPlan.c2c(cfg).diagnostics()["stages"]]
    assert "small-volume-stage" not in labels and len(labels) == 2
    check_c2c(cfg, seed=64)
