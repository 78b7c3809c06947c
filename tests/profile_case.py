"""Profiling utility (not collected by pytest): runs one plan configuration a
few times on cuda:0 and prints its CUDA-event time per execution, so that
one command line serves both as a plain timing run and as the target of an
ncu capture of a single kernel.

python tests/profile_case.py --shape 1024 --batch 32768 [--iters 5]
       [--precision f32|f64|df64] [--inverse] [--kind c2c|r2c|c2r]
       [--tensor-cores] [--tma] [--in-place]
"""
from __future__ import annotations

import argparse
import json
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", type=int, nargs="+", required=True)
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--iters", type=int, default=5)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64", "df64"])
    ap.add_argument("--kind", default="c2c", choices=["c2c", "r2c", "c2r"])
    ap.add_argument("--inverse", action="store_true")
    ap.add_argument("--in-place", action="store_true")
    ap.add_argument("--tensor-cores", action="store_true",
                    help="tuning tensor_cores = 1 (length-64 f32 lines on the tcgen05 layer)")
    ap.add_argument("--tma", action="store_true",
                    help="tuning tma_tiles = 1 (column tiles staged by TMA)")
    args = ap.parse_args()
    import torch

    import wgpufft_b200 as w
    prec = {"f32": w.FftPrecision.F32, "f64": w.FftPrecision.F64, "df64": w.FftPrecision.Df64}
    cfg = (w.FftConfig.new_nd(args.shape).with_batch(args.batch)
           .with_precision(prec[args.precision]))
    if args.tensor_cores:
        cfg = cfg.with_tuning(w.FftTuning().with_tensor_cores(True))
    if args.tma:
        cfg = cfg.with_tuning(cfg.tuning().with_tma_tiles(True))
    if args.inverse or args.kind == "c2r":
        cfg = cfg.with_direction(w.FftDirection.Inverse)
    plan = getattr(w.FftPlan, args.kind)(cfg, device=0)
    ib, ob = plan.required_input_buffer_size_bytes(), plan.required_output_buffer_size_bytes()
    a = torch.randn(max(ib, ob) // 4 + 4, device="cuda")
    o = torch.empty(ob // 4 + 4, device="cuda")

    def run():
        if args.in_place:
            plan.execute_in_place(a)
        else:
            plan.execute_checked(a, o)
    run()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.iters):
        run()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.iters
    print(json.dumps({"ms": ms, "stages": [s["kind"] + ":" + s["label"]
                                           for s in plan.diagnostics()["stages"]]}))


if __name__ == "__main__":
    main()
