"""Autotuner of the batched form: measures, for batches of tiles of one size
class, how many lanes (concurrent CUDA streams) give the highest throughput,
and writes the table cle_vol_batch_plan reads when it is given lanes = 0
(csrc/batch_tuning.h; rebuild the library afterwards).

    python -m pyclesperanto_prototype_b200.autotune [--write] [--reps 5]

Each size class is a batch of synthetic blob tiles (the batched workload's
generator: isotropic Gaussian blobs, Poisson noise, per-tile seeds) of one
shape, about 200 M voxels in all (at most 256 tiles).  Every candidate lane
count runs the batch as one captured CUDA graph; the time is the median of
`reps` replays (CUDA events).  A class's entry applies to batches whose mean
tile voxel count is at least the geometric mean of its own and the previous
class's tile size.
"""
from __future__ import annotations

import argparse
import json
import math
import os

import numpy as np
import torch

from . import _build, synthetic
from .batch import VolBatch

CLASSES = [(64, 64), (256, 256), (32, 128, 128), (64, 256, 256), (96, 512, 512)]
LANES = [1, 2, 4, 8, 12, 16]
HEADER = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "batch_tuning.h")


def _time(batch: VolBatch, reps: int) -> float:
    batch.capture()
    stream = torch.cuda.current_stream()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        batch.run()
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1) / 1e3)
    batch.check()
    return float(np.median(ts))


def tune(reps: int = 5, spot: float = 3.5, outline: float = 1.0):
    rows = []
    for k, shape in enumerate(CLASSES):
        vox = int(np.prod(shape))
        n = max(4, min(256, int(200e6 // vox)))
        tiles = [synthetic.blob_tile(shape, 2e-3 if len(shape) == 2 else 3e-4, seed=9000 + 100 * k + i)
                 for i in range(n)]
        res = {}
        for lanes in LANES:
            if lanes > n:
                continue
            t = _time(VolBatch(tiles, spot, outline, lanes=lanes), reps)
            res[lanes] = n * vox / t / 1e6
        best = max(res, key=res.get)
        rows.append({"shape": shape, "tiles": n, "voxels": vox, "mvoxels_per_s": res, "best_lanes": best})
        print(json.dumps(rows[-1]), flush=True)
        del tiles
        torch.cuda.empty_cache()
    return rows


def write_header(rows, path=HEADER):
    entries = []
    prev = None
    for r in rows:
        lo = 0.0 if prev is None else math.sqrt(prev * r["voxels"])
        entries.append((lo, r["best_lanes"], r))
        prev = r["voxels"]
    lines = [
        "// batch_tuning.h -- lane counts of the batched form per batch size class,",
        "// written by pyclesperanto_prototype_b200/autotune.py from measurements",
        "// (cle_vol_batch_plan with lanes = 0 reads it).  A class applies to batches",
        "// whose mean tile voxel count is at least min_mean_voxels; the last class",
        "// that applies wins.",
        "#pragma once",
        "",
        "namespace cle {",
        "",
        "struct BatchTuning {",
        "    double min_mean_voxels;",
        "    int lanes;",
        "};",
        "",
        "static const BatchTuning kBatchTuning[] = {",
    ]
    for lo, lanes, r in entries:
        meas = ", ".join("%d: %.0f" % (k, v) for k, v in sorted(r["mvoxels_per_s"].items()))
        lines.append("    {%.1f, %d},   // %s x %d tiles; Mvoxels/s by lanes {%s}"
                     % (lo, lanes, "x".join(map(str, r["shape"])), r["tiles"], meas))
    lines += ["};", "", "}  // namespace cle", ""]
    with open(path, "w") as f:
        f.write("\n".join(lines))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--write", nargs="?", const=HEADER, default=None,
                    help="write the table (default path: csrc/batch_tuning.h)")
    args = ap.parse_args()
    _build.build()
    torch.cuda.set_device(0)
    rows = tune(args.reps)
    if args.write:
        write_header(rows, args.write)
        print("wrote", args.write)


if __name__ == "__main__":
    main()
