"""Per-size-class autotuner of the bin size.

The reference's bin grid uses cells of at least `bin_size` (its
`bin_min_size`), raised at setup to the largest pair cutoff
2 * max(cutoff_radius) * skin_fraction (neighbor_setup,
crates/soil_core/src/neighbor.rs:604-665).  Larger cells mean fewer cells to
count, scan and sort per rebuild (and thinner ghost layers of cells), but
more candidates per row; which side wins depends on the system's size.  This
tuner times a few cell sizes, as factors of the largest pair cutoff, on
sample systems of each size class (floor(log2 N) atoms) and keeps the
fastest factor per class in a JSON table.

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

# bin sizes tried, as factors of the largest pair cutoff
CANDIDATES = (1.0, 1.25, 1.5, 2.0)
DEFAULT_PATH = os.path.join(os.path.expanduser("~"), ".cache", "soil_b200", "autotune.json")


def size_class(n):
    """floor(log2 n) for n >= 1."""
    return max(0, int(n).bit_length() - 1)


def max_pair_cutoff(w):
    """The largest pair cutoff of a workload, as neighbor_setup computes it."""
    return 2.0 * float(w.cutoff.max()) * w.cfg.skin_fraction


def bin_size_of(w, factor):
    return factor * max_pair_cutoff(w)


class Table:
    """Tuned bin-size factor per size class
    ({"<class>": {"bin_factor": f, "rate": ...}})."""

    def __init__(self, entries=None):
        self.entries = {str(k): dict(v) for k, v in (entries or {}).items()}

    def factor(self, n, default=None):
        e = self.entries.get(str(size_class(n)))
        return e["bin_factor"] if e else default

    def apply(self, w):
        """Set the workload's bin size from its class (unchanged if untuned)."""
        f = self.factor(w.n)
        if f is not None:
            w.cfg.bin_size = bin_size_of(w, f)
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
    """samples: {size class: [workload, ...]}.  Every candidate factor is
    timed on every sample of a class (a copy of its configuration); the
    class keeps the factor with the largest summed atom-steps/s."""
    import copy
    entries = {}
    for cls, ws in samples.items():
        best = None
        for f in candidates:
            rate = 0.0
            for w in ws:
                wc = copy.copy(w)
                wc.cfg = copy.copy(w.cfg)
                wc.cfg.bin_size = bin_size_of(w, f)
                rate += measure(ctx, wc, steps, warmup)
            if best is None or rate > best[1]:
                best = (f, rate)
        entries[str(cls)] = {"bin_factor": best[0], "rate": best[1] / max(len(ws), 1),
                             "samples": len(ws)}
    return Table(entries)
