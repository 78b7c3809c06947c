"""GPU parity of the real transforms (R2C into the packed [N0/2+1, ...]
spectrum, C2R back), through the C ABI, against the FP64 oracle's
restatement of the reference's packed helpers (src/math/mod.rs:81-153)."""
import numpy as np
import pytest

import wgpufft_b200 as w
from oracle import oracle as O

pytestmark = pytest.mark.gpu

F32, F64 = w.FftPrecision.F32, w.FftPrecision.F64


def real_to_device(x, prec):
    import torch
    dt = np.float32 if prec == F32 else np.float64
    h = np.ascontiguousarray(x.astype(dt))
    return torch.from_numpy(h).cuda(), h.astype(np.float64)


def complex_to_device(z, prec):
    import torch
    if prec == F32:
        h = np.ascontiguousarray(z.astype(np.complex64))
        return torch.from_numpy(h.view(np.float32)).cuda(), h.astype(np.complex128)
    h = np.ascontiguousarray(z.astype(np.complex128))
    return torch.from_numpy(h.view(np.float64)).cuda(), h


def read_complex(t, prec):
    import torch
    torch.cuda.synchronize()
    h = t.cpu().numpy()
    return (h.view(np.complex64) if prec == F32 else h.view(np.complex128)).astype(np.complex128)


def run_r2c(shape, batch, prec, x, norm=w.Normalization.Inverse):
    import torch
    cfg = w.FftConfig.new_nd(shape).with_batch(batch).with_precision(prec).with_normalization(norm)
    plan = w.FftPlan.r2c(cfg)
    dev, exact = real_to_device(x, prec)
    nout = plan.required_output_buffer_size_bytes() // (4 if prec == F32 else 8)
    out = torch.empty(nout, dtype=dev.dtype, device="cuda")
    plan.execute_checked(dev, out)
    return read_complex(out, prec), exact, plan


def run_c2r(shape, batch, prec, z, norm=w.Normalization.Inverse):
    import torch
    cfg = (w.FftConfig.inverse_nd(shape).with_batch(batch).with_precision(prec)
           .with_normalization(norm))
    plan = w.FftPlan.c2r(cfg)
    dev, exact = complex_to_device(z, prec)
    nout = plan.required_output_buffer_size_bytes() // (4 if prec == F32 else 8)
    out = torch.empty(nout, dtype=dev.dtype, device="cuda")
    plan.execute_checked(dev, out)
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64), exact, plan


TOL = {F32: 2e-6, F64: 1e-14}

SHAPES = [[4], [5], [16], [17 * 2], [30], [1024], [1025], [6, 5], [64, 32, 16], [3, 2],
          [4096, 3], [9, 8, 7], [2048, 4], [47487], [2011186]]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("prec", [F32, F64])
def test_r2c_matches_oracle(cuda, shape, prec):
    batch = 2
    n = int(np.prod(shape)) * batch
    x = np.random.default_rng(len(shape) * 7 + n).uniform(-1, 1, n)
    got, exact, plan = run_r2c(shape, batch, prec, x)
    ref = O.r2c_packed_f64(exact, shape, batch=batch)
    assert O.rel_l2(got, ref) <= TOL[prec], plan.diagnostics()["stages"]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("prec", [F32, F64])
def test_c2r_matches_oracle(cuda, shape, prec):
    batch = 2
    n = int(np.prod(shape)) * batch
    x = np.random.default_rng(n + 3).uniform(-1, 1, n)
    packed = O.r2c_packed_f64(x, shape, batch=batch)
    # perturb the self-conjugate bins' imaginary parts: the C2R must ignore them
    got, exact, plan = run_c2r(shape, batch, prec, packed)
    ref = O.c2r_from_packed_f64(exact, shape, batch=batch)
    den = np.linalg.norm(ref)
    assert np.linalg.norm(got - ref) / den <= TOL[prec], plan.diagnostics()["stages"]


def test_known_packed_r2c(cuda):
    # src/math/mod.rs computes_known_r2c_packed_even_length
    got, _, _ = run_r2c([4], 1, F32, np.array([1.0, 2.0, 3.0, 4.0]), norm=w.Normalization.NONE)
    assert np.max(np.abs(got - np.array([10, -2 + 2j, -2]))) < 1e-6


def test_c2r_ignores_dc_and_nyquist_imaginary_parts(cuda):
    # src/cpu.rs:476-481: imaginary parts of the DC and Nyquist bins are ignored
    z = np.array([10 + 5j, -2 + 2j, -2 - 3j])
    got, _, _ = run_c2r([4], 1, F32, z, norm=w.Normalization.NONE)
    ref = O.c2r_from_packed_f64(np.array([10, -2 + 2j, -2]), [4], normalization=O.NORM_NONE)
    assert np.max(np.abs(got - ref)) < 1e-5


def test_3d_256_cube_round_trip_and_sampled_bins(cuda):
    # the 3D R2C -> C2R configuration: real 256^3, packed [129, 256, 256]
    import torch
    shape = [256, 256, 256]
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, 256 ** 3).astype(np.float32)
    fwd = w.FftPlan.r2c(w.FftConfig.new_nd(shape))
    inv = w.FftPlan.c2r(w.FftConfig.inverse_nd(shape))
    dx = torch.from_numpy(x).cuda()
    spec = torch.empty(129 * 256 * 256 * 2, dtype=torch.float32, device="cuda")
    back = torch.empty_like(dx)
    fwd.execute_checked(dx, spec)
    inv.execute_checked(spec, back)
    torch.cuda.synchronize()
    b = back.cpu().numpy()
    assert np.linalg.norm(b - x) / np.linalg.norm(x) < 2e-6
    # sampled bins against a direct FP64 evaluation
    s = spec.cpu().numpy().view(np.complex64).reshape(256, 256, 129)
    xr = x.astype(np.float64).reshape(256, 256, 256)
    X = np.fft.rfftn(xr, axes=(0, 1, 2))  # numpy axes (z, y, x): x fastest
    assert np.linalg.norm(s - X) / np.linalg.norm(X) < 2e-6
