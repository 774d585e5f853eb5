"""The reference's own GPU writegrid (oracle/_ref/writegrid, its sources
compiled for sm_100a) beside this library on the same B200 and case: the
config-1 cell (cubic 25.8 A, 424 atoms, CH4, cutoff 12.5 A) at 0.2 A
resolution (129^3 points, N = ceil(25.8 / 0.2)).

Writes the project tree the reference reads into --tree and prints a JSON
line with this library's grid time (CUDA events, er_grid into device memory)
and the exact in-cutoff pair count. The reference's kernel times come from
an ncu launch list of its writegrid run in that tree (one ComputeGridSheet
launch per x-sheet).

Usage (GPU): python tests/ref_gpu_case.py --tree /tmp/rt
"""
from __future__ import annotations

import argparse
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, HERE)

import emptyroom_b200 as er  # noqa: E402
from emptyroom_b200 import synth  # noqa: E402
from fixture_tree import write_tree  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--tree", required=True)
    ap.add_argument("--resolution", type=float, default=0.2)
    args = ap.parse_args()
    import torch
    f = synth.config1(0)
    name, ads = write_tree(args.tree, f, resolution=args.resolution)
    dims = synth.grid_dims_for(f.abc, args.resolution)
    ctx = er.Context(0)
    fw = ctx.upload(f.particles(), f.t_matrix, f.rep, f.rc2)
    out = torch.empty(dims, dtype=torch.float32, device="cuda")
    s = torch.cuda.ExternalStream(ctx.stream_ptr)
    ts = []
    for k in range(6):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ctx.grid_device(fw, dims, out.data_ptr())
        e1.record(s)
        e1.synchronize()
        if k >= 2:
            ts.append(e0.elapsed_time(e1) * 1e-3)
    ctx.count_pairs_device(fw, dims, out.data_ptr())
    ctx.synchronize()
    pairs = float(out.double().sum().item())
    t = min(ts)
    print(json.dumps({"framework": name, "adsorbate": ads, "dims": list(dims), "pairs": pairs,
                      "ours_s": t, "ours_pair_terms_per_s": pairs / t}))


if __name__ == "__main__":
    main()
