"""GPU parity of plan execution between strided and offset caller views
(b2f_plan_execute_logical_views; the crate's FftPlan::execute_logical_views,
src/plan.rs:580-806, src/runtime/logical_io.rs:5-200), through the C ABI:
each view is filled from / read back into a dense array on the host, the
dense transform is checked against the FP64 oracle, and the layout errors
mirror the crate's BufferLayout* variants."""
import numpy as np
import pytest

import wgpufft_b200 as w
from oracle import oracle as O

pytestmark = pytest.mark.gpu

L = w.FftLogicalLayout
F32, F64 = w.FftPrecision.F32, w.FftPrecision.F64


def _place(dense, per_batch, batch, layout, dtype, total_elems):
    """Writes dense [batch, per_batch] values into a padded buffer following
    `layout`; the other elements hold a marker value."""
    buf = np.full(total_elems, 7.25 + 3.5j if np.iscomplexobj(dense) else 7.25, dtype=dtype)
    bs = layout.batch_stride or (layout.element_stride * (per_batch - 1) + 1)
    for b in range(batch):
        idx = layout.element_offset + b * bs + np.arange(per_batch) * layout.element_stride
        buf[idx] = dense[b * per_batch:(b + 1) * per_batch]
    return buf


def _take(buf, per_batch, batch, layout):
    bs = layout.batch_stride or (layout.element_stride * (per_batch - 1) + 1)
    out = []
    for b in range(batch):
        idx = layout.element_offset + b * bs + np.arange(per_batch) * layout.element_stride
        out.append(buf[idx])
    return np.concatenate(out)


def _span(per_batch, batch, layout):
    bs = layout.batch_stride or (layout.element_stride * (per_batch - 1) + 1)
    return layout.element_offset + (batch - 1) * bs + layout.element_stride * (per_batch - 1) + 1


@pytest.mark.parametrize("shape,batch,lin,lout", [
    ([1024], 3, L(5, 1), L(0, 1)),                     # offset input
    ([1024], 3, L(0, 1), L(9, 1)),                     # offset output
    ([256], 4, L(3, 2), L(1, 3)),                      # strided both sides
    ([16, 12], 2, L(0, 1, 300), L(4, 2, 500)),         # batch strides
    ([15015], 1, L(1, 5), None),                       # four-step route, strided input
    ([1009], 2, None, L(0, 2, 2100)),                  # Rader route, strided output
])
def test_c2c_views_match_dense(cuda, shape, batch, lin, lout):
    import torch
    cfg = w.FftConfig.new_nd(shape).with_batch(batch)
    plan = w.FftPlan.c2c(cfg)
    n = int(np.prod(shape))
    rng = np.random.default_rng(n)
    x = (rng.standard_normal(n * batch) + 1j * rng.standard_normal(n * batch)).astype(np.complex64)
    lin_ = lin or L()
    lout_ = lout or L()
    ib = _place(x, n, batch, lin_, np.complex64, _span(n, batch, lin_) + 3)
    ob = np.full(_span(n, batch, lout_) + 5, 7.25 + 3.5j, dtype=np.complex64)
    di = torch.from_numpy(ib.view(np.float32).copy()).cuda()
    do = torch.from_numpy(ob.view(np.float32).copy()).cuda()
    plan.execute_logical_views(di, lin, do, lout)
    torch.cuda.synchronize()
    got_buf = do.cpu().numpy().view(np.complex64)
    got = _take(got_buf, n, batch, lout_)
    ref = O.c2c_nd_f64(x.astype(np.complex128), shape, batch=batch)
    assert O.rel_l2(got.astype(np.complex128), ref) <= 2e-6
    # elements outside the output view are untouched
    mask = np.ones(got_buf.size, dtype=bool)
    bs = lout_.batch_stride or (lout_.element_stride * (n - 1) + 1)
    for b in range(batch):
        mask[lout_.element_offset + b * bs + np.arange(n) * lout_.element_stride] = False
    assert np.all(got_buf[mask] == np.complex64(7.25 + 3.5j))
    # the input view is not modified
    assert np.array_equal(di.cpu().numpy().view(np.complex64), ib)


@pytest.mark.parametrize("prec", [F32, F64])
def test_real_views(cuda, prec):
    import torch
    shape, batch = [30, 4], 2
    n, npk = 120, 16 * 4
    rdt, cdt = (np.float32, np.complex64) if prec == F32 else (np.float64, np.complex128)
    rng = np.random.default_rng(3)
    x = rng.uniform(-1, 1, n * batch)
    r2c = w.FftPlan.r2c(w.FftConfig.new_nd(shape).with_batch(batch).with_precision(prec))
    c2r = w.FftPlan.c2r(w.FftConfig.inverse_nd(shape).with_batch(batch).with_precision(prec))
    lin, lspec, lback = L(2, 3), L(1, 2, 200), L(0, 2)
    ib = _place(x.astype(rdt), n, batch, lin, rdt, _span(n, batch, lin))
    sb = np.zeros(_span(npk, batch, lspec), dtype=cdt)
    bb = np.zeros(_span(n, batch, lback), dtype=rdt)
    di = torch.from_numpy(ib.copy()).cuda()
    ds = torch.from_numpy(sb.view(rdt).copy()).cuda()
    db = torch.from_numpy(bb.copy()).cuda()
    r2c.execute_logical_views(di, lin, ds, lspec)
    c2r.execute_logical_views(ds, lspec, db, lback)
    torch.cuda.synchronize()
    spec = _take(ds.cpu().numpy().view(cdt), npk, batch, lspec).astype(np.complex128)
    ref = O.r2c_packed_f64(x.astype(rdt).astype(np.float64), shape, batch=batch)
    tol = 2e-6 if prec == F32 else 1e-14
    assert O.rel_l2(spec, ref) <= tol
    back = _take(db.cpu().numpy(), n, batch, lback).astype(np.float64)
    xr = x.astype(rdt).astype(np.float64)
    assert np.linalg.norm(back - xr) / np.linalg.norm(xr) <= 2 * tol


def test_layout_errors(cuda):
    import torch
    plan = w.FftPlan.c2c(w.FftConfig.new(64).with_batch(2))
    buf = torch.zeros(2 * 64 * 8, dtype=torch.float32, device="cuda")
    with pytest.raises(w.FftError) as e:
        plan.execute_logical_views(buf, L(0, 0), buf, None)
    assert e.value.kind == "BufferLayoutZeroStride"
    with pytest.raises(w.FftError) as e:
        plan.execute_logical_views(buf, L(0, 1, 63), buf, None)
    assert e.value.kind == "BufferLayoutBatchStrideTooSmall"
    with pytest.raises(w.FftError) as e:
        plan.execute_logical_views(buf, L(0, 8), buf, None)  # 8 * 63 + 1 + 8*... > buffer
    assert e.value.kind == "BufferLayoutOutOfBounds"
