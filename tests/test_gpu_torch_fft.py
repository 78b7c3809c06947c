"""The torch.fft-shaped front end (wgpufft_b200/torch_fft.py): dims, n / s
padding and truncation, norm, complex and real transforms, f32 and f64, on
CUDA tensors through the C ABI, against the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu

NORMS = {None: O.NORM_INVERSE, "backward": O.NORM_INVERSE, "forward": O.NORM_FORWARD,
         "ortho": O.NORM_ORTHO}


def _cplx(shape, dtype, seed):
    import torch
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    return torch.from_numpy(x.astype(dtype)).cuda(), x.astype(dtype).astype(np.complex128)


def _oracle_c2c(x, dims, inverse, norm):
    """numpy-ordered array x, torch dims -> the unnormalised oracle over the
    crate axes, scaled the way torch.fft scales (by the transformed
    dimensions only)."""
    k = x.ndim
    shape = list(x.shape)[::-1]
    axes = sorted(k - 1 - (d % k) for d in dims)
    y = O.c2c_nd_f64(x.reshape(-1), shape, axes=axes, inverse=inverse,
                     normalization=O.NORM_NONE).reshape(x.shape)
    n = int(np.prod([x.shape[d % k] for d in dims]))
    mode = norm or "backward"
    if mode == "ortho":
        return y / np.sqrt(n)
    return y / n if (mode == "backward") == inverse else y


@pytest.mark.parametrize("shape,dims,norm", [((3, 1000), [-1], None), ((48, 64), [-2, -1], "ortho"),
                                             ((16, 8, 4), [0], "forward"), ((5, 7, 9), None, None),
                                             ((4, 2048), [-1], "backward")])
@pytest.mark.parametrize("dtype", [np.complex64, np.complex128])
def test_complex_transforms(cuda, shape, dims, norm, dtype):
    from wgpufft_b200 import torch_fft as F
    x, exact = _cplx(shape, dtype, 1)
    tol = 2e-6 if dtype == np.complex64 else 1e-13
    d = list(range(len(shape))) if dims is None else dims
    got = F.fftn(x, dim=dims, norm=norm).cpu().numpy().astype(np.complex128)
    assert O.rel_l2(got, _oracle_c2c(exact, d, False, norm)) <= tol
    back = F.ifftn(F.fftn(x, dim=dims, norm=norm), dim=dims, norm=norm).cpu().numpy()
    assert O.rel_l2(back.astype(np.complex128), exact) <= 2 * tol


def test_fft_n_pads_and_truncates(cuda):
    import torch

    from wgpufft_b200 import torch_fft as F
    x, exact = _cplx((2, 100), np.complex64, 2)
    for n in (128, 60):
        got = F.fft(x, n=n).cpu().numpy().astype(np.complex128)
        ref_in = np.zeros((2, n), dtype=np.complex128)
        m = min(n, 100)
        ref_in[:, :m] = exact[:, :m]
        assert O.rel_l2(got, _oracle_c2c(ref_in, [-1], False, None)) <= 2e-6
    y = F.fft2(x.reshape(20, 10), s=(16, 12))
    assert tuple(y.shape) == (16, 12) and y.dtype == torch.complex64


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_real_transforms(cuda, dtype):
    import torch

    from wgpufft_b200 import torch_fft as F
    rng = np.random.default_rng(3)
    tol = 2e-6 if dtype == np.float32 else 1e-13
    # last dim, batched
    r = rng.uniform(-1, 1, (5, 30)).astype(dtype)
    X = F.rfft(torch.from_numpy(r).cuda())
    assert tuple(X.shape) == (5, 16)
    ref = O.r2c_packed_f64(r.astype(np.float64).reshape(-1), [30], batch=5)
    assert O.rel_l2(X.cpu().numpy().astype(np.complex128).reshape(-1), ref) <= tol
    back = F.irfft(X, n=30).cpu().numpy()
    assert np.linalg.norm(back - r) / np.linalg.norm(r) <= 2 * tol
    # every dim
    r3 = rng.uniform(-1, 1, (8, 6, 10)).astype(dtype)
    X3 = F.rfftn(torch.from_numpy(r3).cuda())
    ref3 = O.r2c_packed_f64(r3.astype(np.float64).reshape(-1), [10, 6, 8])
    assert O.rel_l2(X3.cpu().numpy().astype(np.complex128).reshape(-1), ref3) <= tol
    back3 = F.irfftn(X3, s=(8, 6, 10)).cpu().numpy()
    assert np.linalg.norm(back3 - r3) / np.linalg.norm(r3) <= 2 * tol
    # a leading dim (moved to the end and back)
    rl = rng.uniform(-1, 1, (30, 5)).astype(dtype)
    XL = F.rfft(torch.from_numpy(rl).cuda(), dim=0)
    assert tuple(XL.shape) == (16, 5)
    refl = O.r2c_packed_f64(np.ascontiguousarray(rl.T).astype(np.float64).reshape(-1), [30], batch=5)
    got_l = np.ascontiguousarray(XL.cpu().numpy().T).astype(np.complex128).reshape(-1)
    assert O.rel_l2(got_l, refl) <= tol
