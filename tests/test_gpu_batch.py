"""GPU parity of the batched mixed-length launch (b2f_batch_*), through the
C ABI, against the FP64 oracle line by line."""
import numpy as np
import pytest

import wgpufft_b200 as w
from oracle import oracle as O
from wgpufft_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run_batch(lengths, inverse=False, norm=w.Normalization.Inverse, in_place=False, seed=1,
              clusters=False):
    import torch
    lengths = np.asarray(lengths, dtype=np.int64)
    off = W.packed_offsets(lengths)
    total = int(lengths.sum())
    x = W.normal_complex(total, seed)
    b = w.FftBatch(lengths, off, w.FftDirection.Inverse if inverse else w.FftDirection.Forward, norm,
                   clusters=clusters)
    dx = torch.from_numpy(x.view(np.float32)).cuda()
    if in_place:
        b.execute(dx, dx)
        out = dx
    else:
        out = torch.empty_like(dx)
        b.execute(dx, out)
    torch.cuda.synchronize()
    y = out.cpu().numpy().view(np.complex64)
    return x, y, off, b


def check_lines(x, y, lengths, off, idx, inverse=False, norm=O.NORM_INVERSE, tol=2e-6):
    worst = 0.0
    for i in idx:
        n, o = int(lengths[i]), int(off[i])
        ref = O.c2c_nd_f64(x[o:o + n].astype(np.complex128), [n], inverse=inverse,
                           normalization=norm)
        err = O.rel_l2(y[o:o + n], ref)
        worst = max(worst, err)
        assert err <= tol, f"line {i} (N={n}): rel_l2 {err:.3e}"
    return worst


SMALL = [16, 17, 31, 32, 34, 97, 100, 127, 128, 243, 256, 360, 1000, 1009, 1024, 2003, 3003,
         4096, 4099, 5000, 6121, 8192, 10007, 13013, 15015, 16384, 20000, 30011, 32768, 40000,
         46349, 65536, 60013, 65521, 14641]


def test_batch_lengths_match_oracle(cuda):
    lengths = np.array(SMALL * 2)
    x, y, off, b = run_batch(lengths)
    k = b.diagnostics()["kind_lines"]
    assert k["two_pass"] > 0 and k["two_pass_bluestein"] > 0 and k["mixed"] > 0
    assert k["rader"] > 0 and k["bluestein"] > 0
    check_lines(x, y, lengths, off, range(len(lengths)))


def test_batch_cluster_route_matches_oracle(cuda):
    # the distributed-shared-memory route for long lines (8/16-CTA clusters)
    lengths = np.array(SMALL)
    x, y, off, b = run_batch(lengths, clusters=True, seed=9)
    assert b.diagnostics()["cluster_lines"] > 0
    check_lines(x, y, lengths, off, range(len(lengths)))
    x, y, off, b = run_batch(lengths, clusters=True, inverse=True, seed=10)
    check_lines(x, y, lengths, off, range(len(lengths)), inverse=True)


def test_batch_inverse_and_normalisations(cuda):
    lengths = np.array([64, 1009, 4099, 20000, 65536, 360])
    for norm in w.Normalization:
        x, y, off, _ = run_batch(lengths, inverse=True, norm=norm, seed=3)
        check_lines(x, y, lengths, off, range(len(lengths)), inverse=True, norm=int(norm))


def test_batch_in_place(cuda):
    lengths = np.array([1024, 4099, 65536, 17, 30011])
    x, y, off, _ = run_batch(lengths, in_place=True, seed=4)
    check_lines(x, y, lengths, off, range(len(lengths)))


def test_batch_mixed_workload_sampled_lines(cuda):
    # the 20,000-line mixed workload: sampled lines against the oracle,
    # every line through a forward + inverse round trip
    import torch
    lengths = W.mixed_lengths()
    x, y, off, _ = run_batch(lengths, seed=5)
    rng = np.random.default_rng(0)
    idx = rng.choice(len(lengths), 60, replace=False)
    idx = np.concatenate([idx, np.argsort(lengths)[-10:]])
    check_lines(x, y, lengths, off, idx)
    inv = w.FftBatch(lengths, off, w.FftDirection.Inverse)
    dy = torch.from_numpy(y.view(np.float32).copy()).cuda()
    back = torch.empty_like(dy)
    inv.execute(dy, back)
    torch.cuda.synchronize()
    z = back.cpu().numpy().view(np.complex64)
    assert O.rel_l2(z, x) < 4e-6


def test_batch_rejects_overlap_and_small_buffers(cuda):
    import torch
    with pytest.raises(w.FftError):
        w.FftBatch([16, 16], [0, 8])
    b = w.FftBatch([16, 32], [0, 16])
    t = torch.empty(2 * 40, dtype=torch.float32, device="cuda")
    with pytest.raises(w.FftError) as e:
        b.execute(t, t)
    assert e.value.kind == "BufferViewTooSmall"


def _host_run(b, x, in_place=False):
    import torch
    hin = torch.from_numpy(x.view(np.float32).copy()).pin_memory()
    hout = hin if in_place else torch.empty_like(hin).pin_memory()
    din = torch.empty(hin.numel(), dtype=torch.float32, device="cuda")
    dout = din if in_place else torch.empty_like(din)
    b.execute_host(hin, hout, din, dout)
    torch.cuda.synchronize()
    return hout.numpy().view(np.complex64).copy()


@pytest.mark.parametrize("lengths", [
    W.mixed_lengths(),                      # the 20,000-line workload: 8 chunks
    np.array(SMALL),                        # every route, chunks of a few lines
    np.array([4099, 65536, 17]),            # fewer lines than chunks
])
def test_batch_execute_host_matches_device_execute(cuda, lengths):
    # chunked copy-in / transform / copy-out: the same bits as the
    # device-resident execution, in place too
    x, y, off, b = run_batch(lengths, seed=11)
    # chunks of ~32 MiB, at most 32: 32 for the 1.27 GB workload, 1 for the others
    assert b.diagnostics()["host_chunks"] == (32 if len(lengths) == 20000 else 1)
    assert np.array_equal(_host_run(b, x), y)
    assert np.array_equal(_host_run(b, x, in_place=True), y)


def test_batch_execute_host_gaps_inverse_and_clusters(cuda):
    import torch
    lengths = np.array([1024, 30011, 4096, 65536, 100])
    off = np.array([5, 2000, 40000, 50000, 130000])  # unpacked, out of order lines
    off = off[[2, 0, 4, 1, 3]]
    lengths = lengths[[2, 0, 4, 1, 3]]
    total = int((off + lengths).max())
    x = W.normal_complex(total, 12)
    for clusters in (False, True):
        b = w.FftBatch(lengths, off, w.FftDirection.Inverse, clusters=clusters)
        y = _host_run(b, x)
        check_lines(x, y, lengths, off, range(len(lengths)), inverse=True)
    hb = torch.empty(8, dtype=torch.float32)
    db = torch.empty(8, dtype=torch.float32, device="cuda")
    with pytest.raises(w.FftError) as e:
        b.execute_host(hb, hb, db, db)
    assert e.value.kind == "BufferViewTooSmall"


@pytest.mark.parametrize("world", [2, 3, 8])
def test_partitioned_batches_equal_the_whole_batch(cuda, world):
    # the multi-GPU split (one contiguous run of lines per rank, each run its
    # own batch over its own buffers) gives every line the same bits as one
    # batch over all lines; the runs execute one after the other on this GPU
    import torch

    from wgpufft_b200.replicas import partition_lines
    lengths = W.mixed_lengths(count=3000, seed=12)
    x, y_all, off, _ = run_batch(lengths, seed=4)
    for a, b in partition_lines(lengths, world):
        if a == b:
            continue
        sub = lengths[a:b]
        lo, hi = int(off[a]), int(off[a] + sub.sum())
        part = w.FftBatch(sub, W.packed_offsets(sub))
        dx = torch.from_numpy(x[lo:hi].view(np.float32).copy()).cuda()
        out = torch.empty_like(dx)
        part.execute(dx, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy().view(np.complex64)
        assert np.array_equal(got.view(np.uint32), y_all[lo:hi].view(np.uint32)), (a, b)
