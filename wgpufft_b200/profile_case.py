"""Runs one plan configuration a few times on cuda:0: a fixed, small case to
profile a kernel in isolation (e.g. under ncu).

python -m wgpufft_b200.profile_case --shape 1024 --batch 32768 [--iters 5]
       [--precision f32|f64|df64] [--inverse] [--kind c2c|r2c|c2r] [--tensor-cores]
"""
from __future__ import annotations

import argparse


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--shape", type=int, nargs="+", required=True)
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--iters", type=int, default=5)
    ap.add_argument("--precision", default="f32", choices=["f32", "f64", "df64"])
    ap.add_argument("--kind", default="c2c", choices=["c2c", "r2c", "c2r"])
    ap.add_argument("--inverse", action="store_true")
    ap.add_argument("--tensor-cores", action="store_true",
                    help="tuning tensor_cores = 1 (length-64 f32 lines on the tcgen05 layer)")
    args = ap.parse_args()
    import torch

    import wgpufft_b200 as w
    prec = {"f32": w.FftPrecision.F32, "f64": w.FftPrecision.F64, "df64": w.FftPrecision.Df64}
    cfg = (w.FftConfig.new_nd(args.shape).with_batch(args.batch)
           .with_precision(prec[args.precision]))
    if args.tensor_cores:
        cfg = cfg.with_tuning(w.FftTuning().with_tensor_cores(True))
    if args.inverse or args.kind == "c2r":
        cfg = cfg.with_direction(w.FftDirection.Inverse)
    plan = getattr(w.FftPlan, args.kind)(cfg, device=0)
    ib, ob = plan.required_input_buffer_size_bytes(), plan.required_output_buffer_size_bytes()
    a = torch.randn(ib // 4 + 4, device="cuda")
    o = torch.empty(ob // 4 + 4, device="cuda")
    for _ in range(args.iters):
        plan.execute_checked(a, o)
    torch.cuda.synchronize()
    print("ok", [s["kind"] for s in plan.diagnostics()["stages"]])


if __name__ == "__main__":
    main()
