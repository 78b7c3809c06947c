"""GPU tests of the serving loop (b2f_server_*): every request's result is
the same served in a mix (coalesced with other requests of its
configuration, overlapped with other groups) as run alone through its own
plan, within the f32 / f64 / df64 tolerances; admission refuses a request
larger than the budget."""
import numpy as np
import pytest

import wgpufft_b200 as w
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = {w.FftPrecision.F32: 2e-6, w.FftPrecision.F64: 1e-14, w.FftPrecision.Df64: 1e-13}


def host_arrays(cfg, kind, rng):
    import torch
    n = cfg.total_complex_len()
    prec = cfg.precision()
    packed = int(np.prod([cfg.shape()[0] // 2 + 1] + cfg.shape()[1:])) * cfg.batch()
    if kind == w.FftTransformKind.R2c:
        dt = np.float32 if prec == w.FftPrecision.F32 else np.float64
        x = rng.uniform(-1, 1, n).astype(dt)
        out_words = packed * 2
    elif kind == w.FftTransformKind.C2r:
        dt = np.float32 if prec == w.FftPrecision.F32 else np.float64
        r = rng.uniform(-1, 1, n)
        z = O.r2c_packed_f64(r, cfg.shape(), batch=cfg.batch())
        x = z.astype(np.complex64 if dt == np.float32 else np.complex128).view(dt)
        out_words = n
    else:
        z = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        if prec == w.FftPrecision.F32:
            x, dt = z.astype(np.complex64).view(np.float32), np.float32
        elif prec == w.FftPrecision.F64:
            x, dt = z.view(np.float64), np.float64
        else:
            x, dt = O.df64_split(z), np.float32
        out_words = x.size
    hin = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
    hout = torch.zeros(out_words, dtype=hin.dtype).pin_memory()
    return hin, hout


def alone(cfg, kind, hin):
    import torch
    plan = {0: w.FftPlan.c2c, 1: w.FftPlan.r2c, 2: w.FftPlan.c2r}[int(kind)](cfg)
    din = hin.cuda()
    n_out = plan.required_output_buffer_size_bytes() // hin.element_size()
    dout = torch.empty(n_out, dtype=hin.dtype, device="cuda")
    plan.execute_checked(din, dout)
    torch.cuda.synchronize()
    return dout.cpu().numpy()


def as_complex(a, prec):
    if prec == w.FftPrecision.Df64:
        return O.df64_join(a)
    if a.dtype == np.float32:
        return a.view(np.complex64).astype(np.complex128) if a.size % 2 == 0 else a.astype(np.complex128)
    return a.view(np.complex128) if a.size % 2 == 0 else a.astype(np.complex128)


def test_served_mix_equals_alone(cuda):
    rng = np.random.default_rng(1)
    F32, F64, DF = w.FftPrecision.F32, w.FftPrecision.F64, w.FftPrecision.Df64
    C2C, R2C, C2R = w.FftTransformKind.C2c, w.FftTransformKind.R2c, w.FftTransformKind.C2r
    kinds = [
        (w.FftConfig.new(1024).with_batch(3), C2C),
        (w.FftConfig.new(1024).with_batch(3), C2C),
        (w.FftConfig.new(1024).with_batch(5), C2C),
        (w.FftConfig.inverse(4099).with_batch(2), C2C),
        (w.FftConfig.new_nd([64, 128]).with_batch(2), C2C),
        (w.FftConfig.new_nd([64, 64, 64]), R2C),
        (w.FftConfig.inverse_nd([64, 64, 64]), C2R),
        (w.FftConfig.new(1 << 16).with_batch(2).with_precision(F64), C2C),
        (w.FftConfig.new(3000).with_batch(4).with_precision(DF), C2C),
        (w.FftConfig.new(1009).with_batch(7), C2C),
        (w.FftConfig.new(1009).with_batch(7), C2C),
    ]
    srv = w.FftServer(streams=3)
    reqs = []
    for cfg, kind in kinds * 3:
        hin, hout = host_arrays(cfg, kind, rng)
        rid = srv.submit(cfg, kind, hin, hout)
        reqs.append((cfg, kind, hin, hout, rid))
    for cfg, kind, hin, hout, rid in reqs:
        srv.wait(rid, 60.0)
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    for cfg, kind, hin, hout, rid in reqs:
        ref = alone(cfg, kind, hin)
        got = hout.numpy()
        prec = cfg.precision()
        err = O.rel_l2(as_complex(got, prec), as_complex(ref, prec))
        assert err <= TOL[prec], (cfg.shape(), kind, err)
    srv.close()


def test_served_results_match_oracle(cuda):
    rng = np.random.default_rng(2)
    srv = w.FftServer(streams=2)
    cfg = w.FftConfig.new(2048).with_batch(4)
    # a burst: the inputs are ready first, then eight identical requests
    # are queued while dispatch is held and released together
    ins, outs = zip(*[host_arrays(cfg, w.FftTransformKind.C2c, rng) for _ in range(8)])
    srv.hold()
    ids = [srv.submit(cfg, w.FftTransformKind.C2c, hin, hout) for hin, hout in zip(ins, outs)]
    srv.hold(False)
    srv.drain(60.0)
    for i, hin, hout in zip(ids, ins, outs):
        srv.wait(i, 10.0)
        x = hin.numpy().view(np.complex64).astype(np.complex128)
        ref = O.c2c_nd_f64(x, [2048], batch=4)
        assert O.rel_l2(hout.numpy().view(np.complex64), ref) < 2e-6
    assert srv.stats()["coalesced_requests"] > 0
    srv.close()


def test_admission_refuses_oversized_request(cuda):
    import torch
    srv = w.FftServer(hbm_budget_bytes=1 << 20)
    big = w.FftConfig.new(1 << 17)  # 1 MB in + 1 MB out > the 1 MB budget
    hin2 = torch.zeros(2 << 17, dtype=torch.float32).pin_memory()
    hout2 = torch.zeros(2 << 17, dtype=torch.float32).pin_memory()
    rid = srv.submit(big, w.FftTransformKind.C2c, hin2, hout2)
    with pytest.raises(w.FftError) as e:
        srv.wait(rid, 30.0)
    assert e.value.kind == "GpuPlanResourceAllocationFailed"
    srv.close()


def _line_requests(rng, lengths, batches, inverse=False):
    cfgs, ins, outs = [], [], []
    for n, b in zip(lengths, batches):
        cfg = w.FftConfig.new(int(n)).with_batch(int(b))
        if inverse:
            cfg = cfg.with_direction(w.FftDirection.Inverse)
        hin, hout = host_arrays(cfg, w.FftTransformKind.C2c, rng)
        cfgs.append(cfg)
        ins.append(hin)
        outs.append(hout)
    return cfgs, ins, outs


def test_lines_of_different_lengths_share_one_launch(cuda):
    # 1D complex f32 requests of any length are coalesced into one batched
    # launch of the mixed-length line kernels: short lines on the CTA queue,
    # Rader and Bluestein lengths, long smooth and long Bluestein lines; each
    # result matches the FP64 oracle and the same request served alone
    rng = np.random.default_rng(7)
    lengths = [16, 100, 127, 1009, 1024, 3003, 4099, 20000, 65536, 60013, 17, 243]
    batches = [5, 3, 2, 4, 8, 2, 1, 1, 1, 1, 64, 7]
    cfgs, ins, outs = _line_requests(rng, lengths, batches)
    srv = w.FftServer(streams=2)
    srv.hold()
    ids = [srv.submit(c, w.FftTransformKind.C2c, i, o) for c, i, o in zip(cfgs, ins, outs)]
    srv.hold(False)
    srv.drain(120.0)
    st = srv.stats()
    for i in ids:
        srv.wait(i, 10.0)
    assert st["line_groups"] >= 1 and st["coalesced_requests"] > 0, st
    assert st["groups"] < len(ids), st
    for cfg, hin, hout in zip(cfgs, ins, outs):
        n = cfg.shape()[0]
        x = hin.numpy().view(np.complex64).astype(np.complex128)
        ref = O.c2c_nd_f64(x, [n], batch=cfg.batch())
        got = hout.numpy().view(np.complex64).astype(np.complex128)
        assert O.rel_l2(got, ref) <= 2e-6, n
    srv.close()
    # alone: each request through a fresh server of its own
    for cfg, hin, hout in zip(cfgs, ins, outs):
        solo = w.FftServer(streams=1)
        _, out2 = host_arrays(cfg, w.FftTransformKind.C2c, rng)
        solo.wait(solo.submit(cfg, w.FftTransformKind.C2c, hin, out2), 60.0)
        a = hout.numpy().view(np.complex64).astype(np.complex128)
        b = out2.numpy().view(np.complex64).astype(np.complex128)
        assert O.rel_l2(a, b) <= 2e-6
        solo.close()


def test_device_buffer_requests(cuda):
    import torch
    rng = np.random.default_rng(8)
    srv = w.FftServer(streams=3)
    items = [(w.FftConfig.new(4096).with_batch(3), w.FftTransformKind.C2c),
             (w.FftConfig.new(777).with_batch(2), w.FftTransformKind.C2c),
             (w.FftConfig.inverse(30011), w.FftTransformKind.C2c),
             (w.FftConfig.new_nd([64, 48]).with_batch(2), w.FftTransformKind.C2c),
             (w.FftConfig.new_nd([32, 32, 32]), w.FftTransformKind.R2c),
             (w.FftConfig.new(1000).with_precision(w.FftPrecision.F64), w.FftTransformKind.C2c)]
    reqs = []
    srv.hold()
    for cfg, kind in items * 2:
        hin, hout = host_arrays(cfg, kind, rng)
        din, dout = hin.cuda(), torch.zeros_like(hout).cuda()
        reqs.append((cfg, kind, hin, din, dout, srv.submit_device(cfg, kind, din, dout)))
    srv.hold(False)
    for cfg, kind, hin, din, dout, rid in reqs:
        srv.wait(rid, 60.0)
        ref = alone(cfg, kind, hin)
        prec = cfg.precision()
        got = dout.cpu().numpy()
        assert O.rel_l2(as_complex(got, prec), as_complex(ref, prec)) <= TOL[prec], cfg.shape()
    st = srv.stats()
    assert st["failed"] == 0 and st["line_groups"] >= 1, st
    srv.close()


def test_plan_buckets_bound_the_resident_plans(cuda):
    # one configuration at batches 1..12: the executions run on plans of
    # power-of-two batches, so at most four plans (1, 2, 4, 8) become resident
    rng = np.random.default_rng(9)
    srv = w.FftServer(streams=1, coalesce=False)
    for b in range(1, 13):
        cfg = w.FftConfig.new_nd([32, 24]).with_batch(b)
        hin, hout = host_arrays(cfg, w.FftTransformKind.C2c, rng)
        srv.wait(srv.submit(cfg, w.FftTransformKind.C2c, hin, hout), 30.0)
        x = hin.numpy().view(np.complex64).astype(np.complex128)
        ref = O.c2c_nd_f64(x, [32, 24], batch=b)
        assert O.rel_l2(hout.numpy().view(np.complex64), ref) <= 2e-6
    assert srv.stats()["resident_plans"] <= 4
    srv.close()


def test_hold_releases_one_group_per_key(cuda):
    # requests queued while dispatch is held form one group per key when
    # released: three 1D f32 lengths (one line launch), two identical 2D
    # requests (one plan execution) and one f64 request
    rng = np.random.default_rng(10)
    C2C = w.FftTransformKind.C2c
    items = [w.FftConfig.new(1000).with_batch(2), w.FftConfig.new(4099),
             w.FftConfig.new(20000), w.FftConfig.new_nd([32, 48]).with_batch(3),
             w.FftConfig.new_nd([32, 48]).with_batch(3),
             w.FftConfig.new(512).with_precision(w.FftPrecision.F64)]
    srv = w.FftServer(streams=2)
    srv.hold()
    reqs = []
    for cfg in items:
        hin, hout = host_arrays(cfg, C2C, rng)
        reqs.append((cfg, hin, hout, srv.submit(cfg, C2C, hin, hout)))
    assert srv.stats()["completed"] == 0
    srv.hold(False)
    srv.drain(60.0)
    st = srv.stats()
    assert st["groups"] == 3 and st["line_groups"] == 1 and st["coalesced_requests"] == 5, st
    for cfg, hin, hout, rid in reqs:
        srv.wait(rid, 10.0)
        prec = cfg.precision()
        ref = alone(cfg, C2C, hin)
        assert O.rel_l2(as_complex(hout.numpy(), prec), as_complex(ref, prec)) <= TOL[prec]
    srv.close()
