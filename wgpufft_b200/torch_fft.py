"""A torch.fft-shaped front end over the C ABI: fft, ifft, fft2, ifft2,
fftn, ifftn, rfft, irfft, rfft2, irfft2, rfftn, irfftn on CUDA tensors,
with torch.fft's arguments (n / s, dim, norm) and dtypes (complex64 and
complex128 in, float32 and float64 for the real transforms).  Every call
runs a cached FftPlan of this library on the tensor's device and the
current stream; nothing falls back to another FFT implementation.

Layout mapping: a contiguous tensor of shape (d0, ..., d_{k-1}) (last
dimension fastest) is the crate's shape [d_{k-1}, ..., d0] (axis 0
fastest, README.md:111-128), so torch dimension `dim` is crate axis
k-1-dim.  Complex transforms run over any subset of dimensions directly;
real transforms halve the last transformed dimension (torch's convention),
so their dimensions are moved to the end first when they are not already
the trailing ones.
"""
from __future__ import annotations

from typing import Dict, Optional, Sequence, Tuple

import wgpufft_b200 as w

_NORM = {None: w.Normalization.Inverse, "backward": w.Normalization.Inverse,
         "forward": w.Normalization.Forward, "ortho": w.Normalization.Orthogonal}
_PLANS: Dict[tuple, w.FftPlan] = {}


def _plan(kind, shape, axes, batch, inverse, norm, prec, device):
    key = (int(kind), tuple(shape), tuple(axes), batch, inverse, int(norm), int(prec), device)
    p = _PLANS.get(key)
    if p is None:
        cfg = (w.FftConfig.new_nd(list(shape)).with_axes(list(axes)).with_batch(batch)
               .with_direction(w.FftDirection.Inverse if inverse else w.FftDirection.Forward)
               .with_normalization(norm).with_precision(prec))
        p = {0: w.FftPlan.c2c, 1: w.FftPlan.r2c, 2: w.FftPlan.c2r}[int(kind)](cfg, device=device)
        _PLANS[key] = p
    return p


def _dims(x, dim, s):
    if dim is None:
        dim = list(range(x.dim())) if s is None else list(range(x.dim() - len(s), x.dim()))
    elif isinstance(dim, int):
        dim = [dim]
    return [d % x.dim() for d in dim]


def _resize(x, dims, sizes):
    """Zero-pads or truncates x along dims to sizes (torch.fft's n / s)."""
    import torch
    for d, n in zip(dims, sizes):
        if n is None or n == x.shape[d]:
            continue
        if n < x.shape[d]:
            x = x.narrow(d, 0, n)
        else:
            pad = list(x.shape)
            pad[d] = n - x.shape[d]
            x = torch.cat([x, torch.zeros(pad, dtype=x.dtype, device=x.device)], dim=d)
    return x


def _c2c(x, s, dim, norm, inverse):
    import torch
    if not x.is_cuda:
        raise w.FftError("InvalidArgument", 15, "wgpufft_b200.torch_fft needs CUDA tensors")
    if not x.is_complex():
        x = x.to(torch.complex128 if x.dtype == torch.float64 else torch.complex64)
    dims = _dims(x, dim, s)
    if s is not None:
        x = _resize(x, dims, s)
    x = x.contiguous()
    prec = w.FftPrecision.F64 if x.dtype == torch.complex128 else w.FftPrecision.F32
    k = x.dim()
    out = torch.empty_like(x)
    if sorted(dims) == list(range(k - len(dims), k)):
        # trailing dimensions: the crate's shape is theirs (reversed), the
        # leading dimensions its batch, and its normalisation (1 / the
        # product of the shape) is torch's
        t = len(dims)
        shape = list(x.shape[k - t:])[::-1]
        batch = 1
        for d in x.shape[:k - t]:
            batch *= int(d)
        plan = _plan(w.FftTransformKind.C2c, shape, list(range(t)), batch, inverse, _NORM[norm],
                     prec, x.device.index)
        plan.execute_checked(torch.view_as_real(x), torch.view_as_real(out))
        return out
    # other subsets: the crate scales by its whole shape, torch by the
    # transformed dimensions only, so the plan runs unnormalised and the
    # scale is applied here
    shape = list(x.shape)[::-1]
    axes = sorted(k - 1 - d for d in dims)
    plan = _plan(w.FftTransformKind.C2c, shape, axes, 1, inverse, w.Normalization.NONE, prec,
                 x.device.index)
    plan.execute_checked(torch.view_as_real(x), torch.view_as_real(out))
    n = 1
    for d in dims:
        n *= int(x.shape[d])
    mode = norm or "backward"
    if mode == "ortho":
        out *= 1.0 / n ** 0.5
    elif (mode == "backward") == inverse:
        out *= 1.0 / n
    return out


def fft(x, n: Optional[int] = None, dim: int = -1, norm: Optional[str] = None):
    return _c2c(x, None if n is None else [n], [dim], norm, False)


def ifft(x, n: Optional[int] = None, dim: int = -1, norm: Optional[str] = None):
    return _c2c(x, None if n is None else [n], [dim], norm, True)


def fft2(x, s=None, dim: Tuple[int, int] = (-2, -1), norm: Optional[str] = None):
    return _c2c(x, s, list(dim), norm, False)


def ifft2(x, s=None, dim: Tuple[int, int] = (-2, -1), norm: Optional[str] = None):
    return _c2c(x, s, list(dim), norm, True)


def fftn(x, s=None, dim=None, norm: Optional[str] = None):
    return _c2c(x, s, dim, norm, False)


def ifftn(x, s=None, dim=None, norm: Optional[str] = None):
    return _c2c(x, s, dim, norm, True)


def _trailing(x, dims):
    """x with `dims` moved to the end (in order) and the permutation back."""
    k = x.dim()
    rest = [d for d in range(k) if d not in dims]
    order = rest + list(dims)
    if order == list(range(k)):
        return x, None
    back = [0] * k
    for i, d in enumerate(order):
        back[d] = i
    return x.permute(order), back


def rfftn(x, s=None, dim=None, norm: Optional[str] = None):
    import torch
    if not x.is_cuda:
        raise w.FftError("InvalidArgument", 15, "wgpufft_b200.torch_fft needs CUDA tensors")
    if x.is_complex():
        raise w.FftError("InvalidArgument", 15, "rfft takes a real tensor")
    dims = _dims(x, dim, s)
    if s is not None:
        x = _resize(x, dims, s)
    x, back = _trailing(x, dims)
    x = x.contiguous()
    t = len(dims)
    shape = list(x.shape[x.dim() - t:])[::-1]
    batch = 1
    for d in x.shape[:x.dim() - t]:
        batch *= int(d)
    prec = w.FftPrecision.F64 if x.dtype == torch.float64 else w.FftPrecision.F32
    plan = _plan(w.FftTransformKind.R2c, shape, list(range(t)), batch, False, _NORM[norm], prec,
                 x.device.index)
    oshape = list(x.shape)
    oshape[-1] = oshape[-1] // 2 + 1
    ctype = torch.complex128 if prec == w.FftPrecision.F64 else torch.complex64
    out = torch.empty(oshape, dtype=ctype, device=x.device)
    plan.execute_checked(x, torch.view_as_real(out))
    return out.permute(back) if back is not None else out


def irfftn(x, s=None, dim=None, norm: Optional[str] = None):
    import torch
    if not x.is_cuda:
        raise w.FftError("InvalidArgument", 15, "wgpufft_b200.torch_fft needs CUDA tensors")
    if not x.is_complex():
        x = x.to(torch.complex128 if x.dtype == torch.float64 else torch.complex64)
    dims = _dims(x, dim, s)
    t = len(dims)
    # output sizes: s, or the inputs' with the last one 2 * (m - 1)
    sizes = list(s) if s is not None else [x.shape[d] for d in dims[:-1]] + [2 * (x.shape[dims[-1]] - 1)]
    x = _resize(x, dims[:-1], sizes[:-1])
    x = _resize(x, [dims[-1]], [sizes[-1] // 2 + 1])
    x, back = _trailing(x, dims)
    x = x.contiguous()
    shape = sizes[::-1]
    batch = 1
    for d in x.shape[:x.dim() - t]:
        batch *= int(d)
    prec = w.FftPrecision.F64 if x.dtype == torch.complex128 else w.FftPrecision.F32
    plan = _plan(w.FftTransformKind.C2r, shape, list(range(t)), batch, True, _NORM[norm], prec,
                 x.device.index)
    oshape = list(x.shape[:x.dim() - t]) + sizes
    rtype = torch.float64 if prec == w.FftPrecision.F64 else torch.float32
    out = torch.empty(oshape, dtype=rtype, device=x.device)
    plan.execute_checked(torch.view_as_real(x), out)
    return out.permute(back) if back is not None else out


def rfft(x, n: Optional[int] = None, dim: int = -1, norm: Optional[str] = None):
    return rfftn(x, None if n is None else [n], [dim], norm)


def irfft(x, n: Optional[int] = None, dim: int = -1, norm: Optional[str] = None):
    return irfftn(x, None if n is None else [n], [dim], norm)


def rfft2(x, s=None, dim: Tuple[int, int] = (-2, -1), norm: Optional[str] = None):
    return rfftn(x, s, list(dim), norm)


def irfft2(x, s=None, dim: Tuple[int, int] = (-2, -1), norm: Optional[str] = None):
    return irfftn(x, s, list(dim), norm)


def clear_plan_cache() -> None:
    _PLANS.clear()
