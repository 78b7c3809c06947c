"""The allocation-free entry point b2f_c2c_1d_f32_noalloc.

It exists for callers that cannot allocate device memory (a graph capture
that forbids allocation, a plug-in given a fixed memory budget, a real-time
path that must not touch the allocator); its multi-pass scratch is a static
device array inside the library instead of a plan workspace.  This test
calls it through the C ABI and checks two calls in a row against the
regular plan path (FftPlan::c2c + execute_checked) on the same input, at the
f32 tolerance of the other GPU tests.  The file name sorts last so that a
run stopping at the first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import wgpufft_b200 as w
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL = 2e-6  # relative L2, the f32 bound of the other parity tests


def _entry():
    L = w.lib()
    fn = L.b2f_c2c_1d_f32_noalloc
    fn.restype = ctypes.c_int32
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p,
                   ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int32,
                   ctypes.c_int32]
    return fn


@pytest.mark.parametrize("n,batch,direction", [(65536, 4, 0), (1 << 20, 2, 1), (15015, 3, 0)])
def test_noalloc_matches_plan_path_twice(cuda, n, batch, direction):
    import torch
    fn = _entry()
    rng = np.random.default_rng(n + batch)
    x = (rng.standard_normal(n * batch) + 1j * rng.standard_normal(n * batch)).astype(np.complex64)
    dx = torch.from_numpy(x.view(np.float32)).cuda()
    ref = torch.empty_like(dx)
    cfg = w.FftConfig.new(n).with_batch(batch).with_direction(w.FftDirection(direction))
    w.FftPlan.c2c(cfg).execute_checked(dx, ref)
    torch.cuda.synchronize()
    expect = ref.cpu().numpy().view(np.complex64)
    oracle = O.c2c_nd_f64(x.astype(np.complex128), [n], batch=batch, inverse=direction == 1)
    stream = torch.cuda.current_stream().cuda_stream
    nbytes = dx.numel() * 4
    for call in range(2):
        out = torch.full_like(dx, float("nan"))
        st = fn(stream, dx.data_ptr(), nbytes, out.data_ptr(), nbytes, n, batch, direction,
                int(w.Normalization.Inverse))
        assert st == 0, w.lib().b2f_status_string(st)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex64)
        err = O.rel_l2(got, expect)
        assert err <= TOL, f"call {call}: rel_l2 {err:.3e} against the plan path"
        err = O.rel_l2(got, oracle)
        assert err <= TOL, f"call {call}: rel_l2 {err:.3e} against the FP64 oracle"


def test_noalloc_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    fn = _entry()
    n, batch = 1 << 20, 8  # 64 MiB of workspace, above the 32 MiB static scratch
    t = torch.empty(2, dtype=torch.float32, device="cuda")
    st = fn(0, t.data_ptr(), n * batch * 8, t.data_ptr(), n * batch * 8, n, batch, 0, 2)
    assert w.lib().b2f_status_string(st) == b"WorkspaceTooSmall"
