"""Helpers for the GPU parity tests: move seeded inputs to the device in each
storage precision, run a plan through the C ABI, read results back, and
compare with the FP64 oracle on the values the device actually saw."""
import numpy as np

import wgpufft_b200 as w
from oracle import oracle as O

# Tolerances (relative L2 against the FP64 oracle).
TOL = {w.FftPrecision.F32: 2e-6, w.FftPrecision.F64: 1e-14, w.FftPrecision.Df64: 1e-13}


def signal(n, seed=None):
    """The reference tests' deterministic signal (tests/gpu_c2c.rs:391-402)
    or, with a seed, iid N(0,1) real and imaginary parts."""
    if seed is None:
        x = np.arange(n, dtype=np.float64)
        return (np.sin(0.37 * x) * 0.75 + np.cos(0.11 * x) * 0.25) + 1j * (
            np.cos(0.23 * x) * 0.5 - np.sin(0.19 * x) * 0.35)
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def to_device(x, prec):
    """complex128 values -> (torch CUDA tensor in storage layout, the exact
    complex128 values stored)."""
    import torch
    if prec == w.FftPrecision.F32:
        h = np.ascontiguousarray(x.astype(np.complex64))
        return torch.from_numpy(h.view(np.float32)).cuda(), h.astype(np.complex128)
    if prec == w.FftPrecision.F64:
        h = np.ascontiguousarray(x.astype(np.complex128))
        return torch.from_numpy(h.view(np.float64)).cuda(), h
    words = O.df64_split(x)
    return torch.from_numpy(words).cuda(), O.df64_join(words)


def from_device(t, prec):
    import torch
    torch.cuda.synchronize()
    h = t.cpu().numpy()
    if prec == w.FftPrecision.F32:
        return h.view(np.complex64).astype(np.complex128)
    if prec == w.FftPrecision.F64:
        return h.view(np.complex128).copy()
    return O.df64_join(h)


def run_c2c(cfg, x, in_place=False):
    prec = cfg.precision()
    dev, exact = to_device(x, prec)
    plan = w.FftPlan.c2c(cfg)
    if in_place:
        plan.execute_in_place(dev)
        out = dev
    else:
        import torch
        out = torch.empty_like(dev)
        plan.execute_checked(dev, out)
    return from_device(out, prec), exact, plan


def oracle_c2c(cfg, exact):
    return O.c2c_nd_f64(exact, cfg.shape(), axes=cfg.axes(), batch=cfg.batch(),
                        inverse=cfg.direction() == w.FftDirection.Inverse,
                        normalization=int(cfg.normalization()))


def check_c2c(cfg, seed=None, in_place=False, tol=None):
    n = cfg.total_complex_len()
    x = signal(n, seed)
    got, exact, plan = run_c2c(cfg, x, in_place)
    ref = oracle_c2c(cfg, exact)
    err = O.rel_l2(got, ref)
    lim = TOL[cfg.precision()] if tol is None else tol
    assert err <= lim, f"{cfg.shape()} axes={cfg.axes()} batch={cfg.batch()} " \
                       f"{cfg.direction().name} {cfg.precision().name}: rel_l2 {err:.3e} > {lim:.1e} " \
                       f"route={plan.route()} stages={[s['label'] for s in plan.diagnostics()['stages']]}"
    return err
