"""GPU parity at the benchmark configurations' full sizes, through the C ABI,
against the FP64 oracle (oracle/fft_oracle.c, the restatement of the
reference's src/math/mod.rs:214-405) on the values the device saw.

  - 1D C2C f32 N = 1024, batch 512, uniform[-1, 1) inputs (seed 1);
  - 2D C2C f32 4096x2048 row-major (shape [2048, 4096]) and its transpose
    [4096, 2048], forward then inverse, both in place, N(0, 1) (seed 2);
  - 3D R2C then C2R f32 on 256^3 uniform[-1, 1) reals (seed 3);
  - awkward single-length batches at ~256 MiB (127, 1009, 4099, 15015,
    2^20 x 32), sampled lines, and 2^26 (the four-step route) in full;
  - the precision configuration: 1D 2^24 and 2D 8192^2 in f32 on N(0, 1)
    (seed 6) and on high-dynamic-range inputs (|z| log-uniform in
    [1e-6, 1e6], uniform phase, seed 7); native f64 and df64 at 2^24.

Bounds: relative L2 <= 2e-6 (f32), 1e-14 (f64), 1e-13 (df64); the
reference's long-axis tests (tests/gpu_long_axes.rs) use the same oracle
contract.  These cases take tens of seconds of FP64 host work each.
"""
import numpy as np
import pytest

import wgpufft_b200 as w
from oracle import oracle as O
from tests.gpu_util import TOL, from_device, to_device
from wgpufft_b200 import workloads as W

pytestmark = pytest.mark.gpu

F32, F64, DF64 = w.FftPrecision.F32, w.FftPrecision.F64, w.FftPrecision.Df64
INV = w.FftDirection.Inverse


def _normal(n, seed):
    return W.normal_complex(n, seed).astype(np.complex128)


def _forward_vs_oracle(cfg, x, tol=None):
    import torch
    prec = cfg.precision()
    dev, exact = to_device(x, prec)
    out = torch.empty_like(dev)
    plan = w.FftPlan.c2c(cfg)
    plan.execute_checked(dev, out)
    got = from_device(out, prec)
    del dev, out
    torch.cuda.empty_cache()
    ref = O.c2c_nd_f64(exact, cfg.shape(), axes=cfg.axes(), batch=cfg.batch(),
                       inverse=cfg.direction() == INV, normalization=int(cfg.normalization()))
    err = O.rel_l2(got, ref)
    lim = TOL[prec] if tol is None else tol
    assert err <= lim, (f"{cfg.shape()} batch={cfg.batch()} {prec.name}: rel_l2 {err:.3e} > "
                        f"{lim:.1e}, stages {[s['label'] for s in plan.diagnostics()['stages']]}")
    return err


def test_config1_1024_batch_512(cuda):
    x = W.uniform_complex(1024 * 512, 1).astype(np.complex128)
    _forward_vs_oracle(w.FftConfig.new(1024).with_batch(512), x)


@pytest.mark.parametrize("shape", [[2048, 4096], [4096, 2048]])
def test_config2_2d_forward_then_inverse_in_place(cuda, shape):
    import torch
    n = shape[0] * shape[1]
    x = _normal(n, 2)
    dev, exact = to_device(x, F32)
    fwd = w.FftPlan.c2c(w.FftConfig.new_nd(shape))
    inv = w.FftPlan.c2c(w.FftConfig.new_nd(shape).with_direction(INV))
    fwd.execute_in_place(dev)
    spec = from_device(dev, F32)
    ref = O.c2c_nd_f64(exact, shape)
    assert O.rel_l2(spec, ref) <= 2e-6
    inv.execute_in_place(dev)
    back = from_device(dev, F32)
    ref_back = O.c2c_nd_f64(spec, shape, inverse=True)
    assert O.rel_l2(back, ref_back) <= 2e-6
    assert O.rel_l2(back, exact) <= 4e-6
    del dev
    torch.cuda.empty_cache()


def test_config2_3d_256_r2c_then_c2r(cuda):
    import torch
    shape = [256, 256, 256]
    x = np.random.default_rng(3).uniform(-1, 1, 256 ** 3).astype(np.float32)
    dx = torch.from_numpy(x).cuda()
    spec = torch.empty(129 * 256 * 256 * 2, dtype=torch.float32, device="cuda")
    back = torch.empty_like(dx)
    w.FftPlan.r2c(w.FftConfig.new_nd(shape)).execute_checked(dx, spec)
    torch.cuda.synchronize()
    got_spec = spec.cpu().numpy().view(np.complex64).astype(np.complex128)
    ref_spec = O.r2c_packed_f64(x.astype(np.float64), shape)
    assert O.rel_l2(got_spec, ref_spec) <= 2e-6
    w.FftPlan.c2r(w.FftConfig.inverse_nd(shape)).execute_checked(spec, back)
    torch.cuda.synchronize()
    got = back.cpu().numpy().astype(np.float64)
    ref = O.c2r_from_packed_f64(got_spec, shape)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 2e-6
    assert np.linalg.norm(got - x) / np.linalg.norm(x) <= 4e-6


@pytest.mark.parametrize("n,batch", [(127, 264208), (1009, 33255), (4099, 8186), (15015, 2234),
                                     (1 << 20, 32)])
def test_config3_single_length_batches_sampled_lines(cuda, n, batch):
    import torch
    x = W.normal_complex(n * batch, 4)
    dx = torch.from_numpy(x.view(np.float32)).cuda()
    out = torch.empty_like(dx)
    w.FftPlan.c2c(w.FftConfig.new(n).with_batch(batch)).execute_checked(dx, out)
    torch.cuda.synchronize()
    y = out.cpu().numpy().view(np.complex64)
    rng = np.random.default_rng(n)
    lines = sorted({0, batch - 1, *rng.choice(batch, min(batch, 24), replace=False).tolist()})
    for line in lines:
        seg = slice(line * n, (line + 1) * n)
        ref = O.fft_f64(x[seg].astype(np.complex128))
        err = O.rel_l2(y[seg].astype(np.complex128), ref)
        assert err <= 2e-6, f"N={n} line {line}: rel_l2 {err:.3e}"


def test_config3_2pow26_four_step(cuda):
    n = 1 << 26
    _forward_vs_oracle(w.FftConfig.new(n), _normal(n, 4))


@pytest.mark.parametrize("inputs", ["normal", "hdr"])
def test_config4_1d_2pow24_f32(cuda, inputs):
    n = 1 << 24
    x = _normal(n, 6) if inputs == "normal" else W.hdr_complex(n, 7)
    _forward_vs_oracle(w.FftConfig.new(n), x)


def test_config4_1d_2pow24_f32_inverse(cuda):
    n = 1 << 24
    _forward_vs_oracle(w.FftConfig.new(n).with_direction(INV), _normal(n, 16))


@pytest.mark.parametrize("inputs", ["normal", "hdr"])
def test_config4_2d_8192_squared_f32(cuda, inputs):
    n = 8192 * 8192
    x = _normal(n, 6) if inputs == "normal" else W.hdr_complex(n, 7)
    _forward_vs_oracle(w.FftConfig.new_nd([8192, 8192]), x)


@pytest.mark.parametrize("prec", [F64, DF64])
def test_config4_1d_2pow24_extended_precision(cuda, prec):
    n = 1 << 24
    _forward_vs_oracle(w.FftConfig.new(n).with_precision(prec), _normal(n, 8))
