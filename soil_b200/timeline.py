"""Kernel timeline of a bench workload's steps, recorded through CUPTI
(torch.profiler): the device's busy time per step and the gaps between
consecutive kernels, which CUDA events around a phase cannot separate.

    python -m soil_b200.timeline c3 [steps]

Run from the repository root (it builds the workload with bench.py).  Prints
one JSON object: span and busy time per step in microseconds, the largest
gaps with the kernels on either side, and the per-kernel mean durations.
With programmatic dependent launch a kernel's recorded span includes the
time it waits for its predecessor, so busy time can exceed the span."""
import json
import sys
from collections import defaultdict

import torch
from torch.profiler import ProfilerActivity, profile


def main(argv):
    import bench
    from soil_b200 import system

    cfg = argv[1] if len(argv) > 1 else "c3"
    steps = int(argv[2]) if len(argv) > 2 else 10
    w, _ = bench.make_workload(cfg, "fp64", None)
    ctx = system.Context(0)
    s = system.from_workload(ctx, w)
    s.step(5)
    s.sync()
    with profile(activities=[ProfilerActivity.CUDA, ProfilerActivity.CPU]) as prof:
        s.step(steps)
        s.sync()
    ev = sorted((e.time_range.start, e.time_range.end, e.name) for e in prof.events()
                if e.device_type == torch.autograd.DeviceType.CUDA)
    out = {"workload": cfg, "steps": steps, "records": len(ev)}
    if ev:
        t0, t1 = ev[0][0], ev[-1][1]
        gaps = sorted(((ev[k][0] - ev[k - 1][1], ev[k - 1][2][:48], ev[k][2][:48])
                       for k in range(1, len(ev))), reverse=True)
        per = defaultdict(list)
        for a, b, n in ev:
            per[n.split("(")[0]].append(b - a)
        out.update({
            "span_us_per_step": (t1 - t0) / steps,
            "busy_us_per_step": sum(b - a for a, b, _ in ev) / steps,
            "largest_gaps_us": [(round(g, 1), p, n) for g, p, n in gaps[:12]],
            "mean_us": {k: round(sum(v) / len(v), 1) for k, v in per.items()},
        })
    s.close()
    ctx.close()
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main(sys.argv)
