"""The slab-decomposed single transform (wgpufft_b200/sharded.py): a 2D or
3D complex transform split over ranks by its slowest axis, with one
all-to-all between the local transforms.  On CPU (no GPU): world size 2 with
gloo, the local transforms injected (numpy), checked against a whole-array
FFT — this pins the decomposition, the exchange and the output layout.  On
the GPU: the same object with its FftPlans through the C ABI against the
FP64 oracle (world size 1: the exchange is a local copy)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _numpy_local(which, x, sh):
    import torch
    cdt = np.complex64 if x.dtype == torch.float32 else np.complex128
    a = x.numpy().view(cdt)
    shape = sh.shape
    if which == 0:
        arr = a.reshape([sh.slab] + shape[:-1][::-1])
        y = np.fft.fftn(arr, axes=tuple(range(1, arr.ndim))) if not sh.inverse else \
            np.fft.ifftn(arr, axes=tuple(range(1, arr.ndim))) * np.prod(shape[:-1])
    else:
        arr = a.reshape([shape[-1]] + shape[1:-1][::-1] + [sh.chunk])
        y = np.fft.fft(arr, axis=0) if not sh.inverse else np.fft.ifft(arr, axis=0) * shape[-1]
    return torch.from_numpy(np.ascontiguousarray(y.astype(cdt)).view(x.numpy().dtype).reshape(-1))


def _worker(rank, world, port, q, shape, inverse):
    os.environ.update({"WORLD_SIZE": str(world), "RANK": str(rank), "MASTER_ADDR": "127.0.0.1",
                       "MASTER_PORT": str(port)})
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    from wgpufft_b200.sharded import ShardedFft
    dist.init_process_group("gloo", timeout=timedelta(seconds=60))
    rng = np.random.default_rng(0)
    n = int(np.prod(shape))
    X = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    X = X.reshape(shape[::-1])
    sh = ShardedFft(shape, inverse=inverse, local_fft=_numpy_local)
    slab = np.ascontiguousarray(X[rank * sh.slab:(rank + 1) * sh.slab])
    out = sh.forward(torch.from_numpy(slab.view(np.float32).reshape(-1)))
    q.put((rank, out.numpy().view(np.complex64).reshape(sh.output_layout()[0]), sh.output_layout()[1]))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("shape,inverse", [([8, 12], False), ([6, 4, 10], False), ([16, 8], True)])
def test_two_rank_slab_transform_equals_whole_array(shape, inverse):
    from wgpufft_b200.sharded import assemble_output
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    world = 2
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, shape, inverse))
             for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=120) for _ in procs), key=lambda t: t[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, _, rng_ in res:
        c0 = shape[0] // world
        assert rng_ == (rank * c0, (rank + 1) * c0)
    full = assemble_output([r[1] for r in res], shape)
    rng = np.random.default_rng(0)
    n = int(np.prod(shape))
    X = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    X = X.reshape(shape[::-1]).astype(np.complex128)
    ref = np.fft.ifftn(X) if inverse else np.fft.fftn(X)
    assert np.linalg.norm(full - ref) / np.linalg.norm(ref) < 1e-5


def test_rejects_indivisible_shapes():
    from wgpufft_b200.sharded import ShardedFft
    with pytest.raises(ValueError):
        ShardedFft([8], local_fft=_numpy_local)


@pytest.mark.gpu
@pytest.mark.parametrize("shape,inverse", [([256, 128], False), ([64, 32, 16], True),
                                           ([8192, 64], False)])
def test_gpu_single_rank_matches_oracle(cuda, shape, inverse):
    import torch

    from oracle import oracle as O
    from wgpufft_b200.sharded import ShardedFft
    rng = np.random.default_rng(3)
    n = int(np.prod(shape))
    x = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    sh = ShardedFft(shape, inverse=inverse)
    out = sh.forward(torch.from_numpy(x.view(np.float32)).cuda())
    torch.cuda.synchronize()
    got = out.cpu().numpy().view(np.complex64).astype(np.complex128)
    ref = O.c2c_nd_f64(x.astype(np.complex128), shape, inverse=inverse)
    # one rank: the output layout is the natural one
    assert O.rel_l2(got, ref) <= 2e-6
