"""Profiling utility (not collected by pytest): a batch of lines of one
length through the mixed-length batch kernels (FftBatch) on cuda:0, about
256 MB of input, timed with CUDA events over 10 executions after 3 warm-up
ones; prints ms per execute and algorithmic GB/s.  One command line serves
as a plain timing run and as the target of an ncu capture.

python tests/profile_batch.py [--clusters] 65536 [20011 ...]
  --clusters: long lines on the thread-block-cluster kernels (one HBM pass,
              distributed shared memory) instead of the long-line passes
"""
from __future__ import annotations

import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main() -> None:
    import torch

    import wgpufft_b200 as w
    clusters = "--clusters" in sys.argv[1:]
    for arg in [a for a in sys.argv[1:] if not a.startswith("--")]:
        n = int(arg)
        lines = max(1, (256 << 20) // (8 * n))
        b = w.FftBatch([n] * lines, [i * n for i in range(lines)], clusters=clusters)
        x = torch.randn(2 * n * lines, device="cuda")
        y = torch.empty_like(x)
        for _ in range(3):
            b.execute(x, y)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(10):
            b.execute(x, y)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / 10
        d = b.diagnostics()
        print(json.dumps({"length": n, "lines": lines, "clusters": clusters, "ms": round(ms, 4),
                          "alg_gbs": round(16 * n * lines / ms / 1e6, 1),
                          "long_tasks": d.get("long_tasks"),
                          "kind_lines": d.get("kind_lines")}), flush=True)


if __name__ == "__main__":
    main()
