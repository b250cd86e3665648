"""Per-size-class autotuner of the bin size.

The reference's bin grid uses cells of at least `bin_size` (its
`bin_min_size`) and never smaller than the largest cutoff radius
(crates/soil_core/src/neighbor.rs:311-495).  The cell size trades grid
work (cells to count, scan and sort per rebuild) against candidates per row;
which side wins depends on the system's size and density.  This tuner times
a few candidate sizes on sample systems of each size class (floor(log2 N)
atoms) and keeps the fastest per class in a JSON table.

The bin size is part of a system's configuration: it decides the cell of
every atom, hence the CSR order and the force summation order.  A tuned
table is therefore applied to a workload's configuration before the system
is created (Table.apply), and every run of that workload - alone, batched,
served or in the CPU oracle - uses the same value and gives the same bits.
Timing never changes a result: candidates differ only in speed.

    table = autotune.tune(ctx, {cls: [workload, ...]})
    table.save(path); table = autotune.Table.load(path)
    for w in workloads: table.apply(w)
"""
import json
import math
import os

from . import system

# bin_size values tried; the grid clamps each to the largest cutoff radius
CANDIDATES = (0.65, 0.8, 1.0, 1.3)
DEFAULT_PATH = os.path.join(os.path.expanduser("~"), ".cache", "soil_b200", "autotune.json")


def size_class(n):
    """floor(log2 n) for n >= 1."""
    return max(0, int(n).bit_length() - 1)


class Table:
    """Tuned bin size per size class ({"<class>": {"bin_size": b, "rate": ...}})."""

    def __init__(self, entries=None):
        self.entries = {str(k): dict(v) for k, v in (entries or {}).items()}

    def bin_size(self, n, default=None):
        e = self.entries.get(str(size_class(n)))
        return e["bin_size"] if e else default

    def apply(self, w):
        """Set the workload's bin size from its class (unchanged if untuned)."""
        b = self.bin_size(w.n)
        if b is not None:
            w.cfg.bin_size = b
        return w

    def save(self, path=DEFAULT_PATH):
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = path + ".tmp"
        with open(tmp, "w") as f:
            json.dump({"version": 1, "classes": self.entries}, f, indent=1, sort_keys=True)
        os.replace(tmp, path)

    @staticmethod
    def load(path=DEFAULT_PATH):
        with open(path) as f:
            d = json.load(f)
        if d.get("version") != 1:
            raise ValueError(f"{path}: unknown autotune table version")
        return Table(d["classes"])


def measure(ctx, w, steps=20, warmup=5):
    """Atom-steps/s of workload w stepped alone, timed with CUDA events on
    the system's stream after `warmup` untimed steps."""
    import torch
    s = system.from_workload(ctx, w)
    try:
        s.step(warmup)
        st = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", ctx.device))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.step(steps)
        e1.record(st)
        s.sync()
        return w.n * steps / (e0.elapsed_time(e1) * 1e-3)
    finally:
        s.close()


def tune(ctx, samples, candidates=CANDIDATES, steps=20, warmup=5):
    """samples: {size class: [workload, ...]}.  Every candidate bin size is
    timed on every sample of a class (a copy of its configuration); the
    class keeps the candidate with the largest summed atom-steps/s."""
    import copy
    entries = {}
    for cls, ws in samples.items():
        best = None
        for b in candidates:
            rate = 0.0
            for w in ws:
                wc = copy.copy(w)
                wc.cfg = copy.copy(w.cfg)
                wc.cfg.bin_size = b
                rate += measure(ctx, wc, steps, warmup)
            if best is None or rate > best[1]:
                best = (b, rate)
        entries[str(cls)] = {"bin_size": best[0], "rate": best[1] / max(len(ws), 1),
                             "samples": len(ws)}
    return Table(entries)
