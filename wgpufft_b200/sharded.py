"""Single transforms larger than one GPU: a 2D or 3D complex transform
sharded over the ranks of a process group as slabs of its slowest axis,
with one all-to-all transposition between the local transforms (the slab
decomposition).  The reference crate has no multi-GPU code; this is the
"one exchange step" of a distributed FFT:

    global data  X[n_{r-1}] ... [n_1][n_0]   (axis 0 contiguous, the crate's
                                              layout, README.md:111-128)
    rank p holds the slab of the slowest axis n_{r-1} in
    [p * S / P, (p + 1) * S / P), S = shape[-1]  (contiguous block)
    1. transform the other axes locally (one FftPlan over the slab);
    2. all-to-all: rank p sends to rank q the part of its slab whose axis-0
       index lies in q's chunk of axis 0 (shape[0] / P values);
    3. transform the slowest axis locally, now complete on every rank.
The result is distributed by chunks of axis 0: rank q holds, for every
index of the other axes, the axis-0 outputs [q * shape[0] / P, ...) in the
layout [n_{r-1}] ... [n_1][k_0 local] (documented by `output_layout`).

The local transforms run through the C ABI (FftPlan); the exchange is a
torch.distributed all_to_all_single (NCCL over NVLink on GPUs, gloo on
CPU), into local buffers.  No kernel reads another GPU's memory.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np


class ShardedFft:
    """A forward or inverse C2C transform of `shape` (2 or 3 axes, all
    transformed, f32 or f64) sharded over `group` (default: the world).
    shape[-1] and shape[0] must be divisible by the world size."""

    def __init__(self, shape: Sequence[int], inverse: bool = False, precision: int = 0,
                 group=None, local_fft: Optional[Callable] = None, device: Optional[int] = None):
        import torch.distributed as dist
        self.shape = [int(s) for s in shape]
        if len(self.shape) not in (2, 3):
            raise ValueError("sharded transforms take 2 or 3 axes")
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        P = self.world
        if self.shape[-1] % P or self.shape[0] % P:
            raise ValueError("shape[-1] and shape[0] must be divisible by the world size")
        self.inverse = inverse
        self.precision = precision
        self.slab = self.shape[-1] // P      # slowest-axis rows per rank
        self.chunk = self.shape[0] // P      # axis-0 values per rank after the exchange
        self.inner = int(np.prod(self.shape[:-1]))          # points per slowest-axis row
        self.local_points = self.slab * self.inner
        # the local transforms: injected (tests on CPU) or FftPlans on `device`
        self._local_fft = local_fft
        if local_fft is None:
            import wgpufft_b200 as w
            d = w.FftDirection.Inverse if inverse else w.FftDirection.Forward
            prec = w.FftPrecision(precision)
            norm = w.Normalization.NONE  # the global scale is applied once, at the end
            first = (w.FftConfig.new_nd(self.shape[:-1]).with_batch(self.slab)
                     .with_direction(d).with_precision(prec).with_normalization(norm))
            # after the exchange: [S][rest of the inner axes, axis 0 chunked]
            rest = [self.chunk] + self.shape[1:-1]
            second = (w.FftConfig.new_nd(rest + [self.shape[-1]]).with_axes([len(rest)])
                      .with_direction(d).with_precision(prec).with_normalization(norm))
            self._plans = (w.FftPlan.c2c(first, device=device),
                           w.FftPlan.c2c(second, device=device))
        self.logical = int(np.prod(self.shape))

    def output_layout(self):
        """Shape (slowest first) of the local output and the axis-0 range it
        holds: [shape[-1], ..., shape[1], chunk], [rank * chunk, ...)."""
        return [self.shape[-1]] + self.shape[1:-1][::-1] + [self.chunk], \
            (self.rank * self.chunk, (self.rank + 1) * self.chunk)

    def _run_local(self, which: int, x):
        if self._local_fft is not None:
            return self._local_fft(which, x, self)
        import torch
        out = torch.empty_like(x)
        self._plans[which].execute_checked(x, out)
        return out

    def forward(self, local_slab):
        """local_slab: this rank's slab as a flat tensor of interleaved
        complex values (2 * local_points real words); returns the local
        output (layout: output_layout), scaled by the crate's default
        normalisation (1/N on inverse transforms)."""
        import torch
        import torch.distributed as dist
        P, S, R, C0 = self.world, self.slab, self.inner, self.chunk
        x = self._run_local(0, local_slab)
        # [S rows][R inner] with R = rest * shape[0]: split axis 0 into P chunks
        rest = R // self.shape[0]
        v = x.view(S, rest, P, C0, 2)
        send = v.permute(2, 0, 1, 3, 4).contiguous()  # [q][S][rest][C0]
        recv = torch.empty_like(send)
        if P > 1:
            dist.all_to_all_single(recv.view(-1), send.view(-1), group=self.group)
        else:
            recv.copy_(send)
        # recv[s] = rows of rank s: [s][S][rest][C0] -> global slowest index s*S + row
        y = recv.view(P * S, rest, C0, 2).contiguous()
        z = self._run_local(1, y.view(-1))
        if self.inverse:
            z = z * (1.0 / self.logical)
        return z


def assemble_output(parts, shape):
    """Test helper: the full [shape[-1]]...[shape[0]] array from every rank's
    local output (a list in rank order of complex arrays [S, ..., chunk])."""
    P = len(parts)
    C0 = shape[0] // P
    full = np.empty([shape[-1]] + list(shape[1:-1])[::-1] + [shape[0]], dtype=parts[0].dtype)
    for q, part in enumerate(parts):
        full[..., q * C0:(q + 1) * C0] = part
    return full
