"""The tensor-core DFT layer (tuning tensor_cores = 1): length-64 f32 lines
on tcgen05 with split-TF32 operands, through the C ABI, against the FP64
oracle at the f32 tolerance (2e-6 relative L2), forward and inverse, every
normalisation, a ragged last tile, in place, and lines of an N-D shape."""
import pytest

import wgpufft_b200 as w
from tests.gpu_util import check_c2c

pytestmark = pytest.mark.gpu

TC = w.FftTuning().with_tensor_cores(True)


def _tc(cfg):
    return cfg.with_tuning(TC)


def test_route_is_the_tensor_core_stage(cuda):
    plan = w.FftPlan.c2c(_tc(w.FftConfig.new(64).with_batch(4096)))
    kinds = [s["kind"] for s in plan.diagnostics()["stages"]]
    assert kinds == ["tensor-core-dft"]


@pytest.mark.parametrize("batch", [1, 63, 64, 65, 1000, 4096, 100000])
def test_forward_matches_oracle(cuda, batch):
    err = check_c2c(_tc(w.FftConfig.new(64).with_batch(batch)), seed=batch)
    assert err < 2e-6


@pytest.mark.parametrize("norm", list(w.Normalization))
def test_inverse_and_normalisations(cuda, norm):
    cfg = _tc(w.FftConfig.new(64).with_batch(777).with_direction(w.FftDirection.Inverse)
              .with_normalization(norm))
    check_c2c(cfg, seed=int(norm) + 11)


def test_in_place_and_nd_lines(cuda):
    check_c2c(_tc(w.FftConfig.new(64).with_batch(3000)), seed=5, in_place=True)
    check_c2c(_tc(w.FftConfig.new_nd([64, 48]).with_axes([0]).with_batch(3)), seed=6)


def test_other_shapes_ignore_the_knob(cuda):
    plan = w.FftPlan.c2c(_tc(w.FftConfig.new(128).with_batch(8)))
    assert all(s["kind"] != "tensor-core-dft" for s in plan.diagnostics()["stages"])
    check_c2c(_tc(w.FftConfig.new(128).with_batch(8)), seed=7)


def test_no_bounded_wait_gave_up(cuda):
    # every wait of the layer for its matrix products completes: the plan's
    # device status (the kernel's error flag, read on the host) stays clear
    import torch
    plan = w.FftPlan.c2c(_tc(w.FftConfig.new(64).with_batch(50000)))
    a = torch.randn(64 * 50000 * 2, device="cuda")
    o = torch.empty_like(a)
    for _ in range(3):
        plan.execute_checked(a, o)
    plan.device_status()
