#!/usr/bin/env python
"""Run a few steps of one workload of the step through the C ABI, for
profiler captures (ncu) and quick timings of a single workload.

  python general-simulator_b200/gs_profile.py --workload martensite|precipitate|cufft|plain|batch
      [--n 256] [--steps 3] [--warmup 2] [--dtype f32|f64] [--graph] [--tune]
      [--shape NX,NY,NZ] [--noise AMP]

martensite: the 3D three-variant workload (noise 1e-3, sigma_zz 0.005);
precipitate: concentration + 4 variants, semi-implicit; cufft / plain: the
two comparator steps on the martensite workload; batch: the 64-simulation
ensemble (--shape keeps only its simulations of one grid shape, to time a
shape group alone).  --noise sets the martensite workloads' noise amplitude
(0: the same kernels with the noise term skipped).  --graph replays the
steps as captured graphs, --tune runs the autotuner first.  Prints the
device time per step (CUDA events on the stepping stream, after the warm-up
steps)."""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="martensite",
                    choices=["martensite", "precipitate", "cufft", "plain", "batch"])
    ap.add_argument("--n", type=int, default=256)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--dtype", default="f32", choices=["f32", "f64"])
    ap.add_argument("--graph", action="store_true")
    ap.add_argument("--tune", action="store_true")
    ap.add_argument("--shape", default="")
    ap.add_argument("--noise", type=float, default=1e-3)
    args = ap.parse_args()

    import torch

    import gs_b200 as gb

    dt = gb.GS_DTYPE_F64 if args.dtype == "f64" else gb.GS_DTYPE_F32
    stream = torch.cuda.Stream()
    sh = stream.cuda_stream
    if args.workload == "batch":
        ps = gb.ensemble_params(dt)
        if args.shape:
            want = tuple(int(v) for v in args.shape.split(","))
            ps = [p for p in ps if (p.nx, p.ny, p.nz) == want]
            if not ps:
                raise SystemExit(f"no simulation of shape {want} in the ensemble")
        obj = gb.Batch(ps)
        for i, p in enumerate(ps):
            obj.set_eta(i, gb.initial_eta(p, 200 + i))
        cells = sum(p.ncells for p in ps)
    elif args.workload == "precipitate":
        p = gb.precip3d_params(args.n, dtype=dt)
        obj = gb.Sim(p)
        obj.set_field("concentration", gb.initial_c(p, 2))
        obj.set_field("eta", gb.initial_eta(p, 3))
        cells = p.ncells
    else:
        p = gb.mart3d_params(args.n, dtype=dt, noise=args.noise)
        obj = gb.Sim(p, plain=args.workload == "plain", cufft=args.workload == "cufft")
        obj.set_field("eta", gb.initial_eta(p, 1))
        cells = p.ncells
    if args.tune:
        obj.autotune(3, sh)
    if args.graph:
        obj.use_graph(True)
    with torch.cuda.stream(stream):
        obj.step(args.warmup, sh)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        obj.step(args.steps, sh)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / max(args.steps, 1)
    obj.close()
    print(json.dumps({"workload": args.workload, "n": args.n, "dtype": args.dtype, "steps": args.steps,
                      "shape": args.shape, "sims": len(ps) if args.workload == "batch" else 1,
                      "graph": args.graph, "tuned": args.tune,
                      "ms_per_step": ms, "cell_updates_per_s": cells * 1e3 / ms}))


if __name__ == "__main__":
    main()
