#!/usr/bin/env python
"""bench.py — atom-steps/s of the SOIL substrate hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl soil|reference]
                    [--config c1|c2|c3] [--filter fp64|fp32]

One "step" is one velocity-Verlet timestep of the whole hot path (integrate,
rebuild check, ghost comm, spatial sort + neighbor build when due, the
repulsion consumer, reverse comm) over one periodic system.  The default
workload is the large single system: 4,194,304 polydisperse spheres
(r ~ U[0.4, 0.6], packing fraction 0.50), harmonic repulsion k = 1e3,
dt = 1e-4, seeded synthetic inputs.  State is FP64 throughout.

A single system does not shard on one rank (no spatial decomposition), so
with --gpus N every rank runs an independent replica; `value` is the
atom-steps of all ranks over the slowest rank's device time (weak scaling).

Printed JSON keys beyond the base contract:
  timed_steps            light and rebuild steps inside the timed region
  ms_per_light_step, ms_per_rebuild_step
                         measured past the timed region until >= 3 rebuilds
  ms_per_step_at_rebuild_rate, neighbor_builds_per_s
                         the two mixed at the rebuild rate seen there
  roofline               dominant kernel: algorithmic bytes / mean launch time
  cpu_baseline           the CPU oracle on a bounded sample of the same system
  e2e                    the same metric through the C ABI from pinned host
                         buffers (upload, setup, K steps, download of pos/vel)
  phases                 device ms per phase over the timed region
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from soil_b200 import abi, dist, workloads  # noqa: E402

# Algorithmic bytes per unit of each timed phase (FP64 SoA; one read or
# write of each value the phase must touch).  c: the system's counts, fw: f64
# width of the #[forward] columns.
#   integrate: final(t) fused with initial(t+1) + displacement check:
#              R x,v,F,inv_m (80) + R last-build pos (24) + W x,v (48) = 152 B/local;
#              with forward comm fused in (light steps): R fold_start (4) per
#              local, and per ghost R fold_list + chain (8), W pos,vel (48),
#              R+W forward columns (16 B per f64)
#   force:     the consumer with the reverse fold: R x,y,z,radius (32) and
#              W force (24) of every atom, R list/fold metadata (12 B per
#              local, 8 B per ghost), R 5 B per pair side (each pair is read
#              from its owner's row and its partner's transposed list), and
#              the fold R ghost F (24) + R origin (4) + RMW owner F (48) per
#              ghost
#   forward:   R root+chain (8) + R root pos,vel (48) + W pos,vel (48)
#              + forward columns (16 B per f64) per ghost
#   reverse:   R send index (4) + R ghost F (24) + RMW owner F (48) per ghost
#   final:     80 B/local
BYTES_PER_UNIT = {
    "integrate": lambda c, fw: 156 * c.nlocal + (56 + 16 * fw) * c.nghost,
    "final": lambda c, fw: 80 * c.nlocal,
    "force": lambda c, fw: (60 * (c.nlocal + c.nghost) + 12 * c.nlocal + 8 * c.nghost
                            + 10 * c.npairs + 76 * c.nghost),
    "forward": lambda c, fw: (104 + 16 * fw) * c.nghost,
    "reverse": lambda c, fw: 76 * c.nghost,
}
# The kernel each timed phase launches on a light step (ncu names); the force
# phase's kernel depends on SOIL_FORCE and is asked of the library.
PHASE_KERNEL = {"integrate": "k_initial", "final": "k_final",
                "forward": "k_forward", "reverse": "k_reverse_fold_roots"}


def phase_kernel(lib, phase):
    if phase == "force":
        return lib.soil_consumer_kernel().decode()
    return PHASE_KERNEL.get(phase, phase)


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(kernel, workload):
    """DRAM bytes per atom of `kernel` (its ncu name) from a committed ncu
    summary of that kernel on `workload`, if any."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        d = json.load(f)
    for e in d.values():
        if e.get("kernel") == kernel and e.get("workload") == workload:
            return e
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=2)
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def make_workload(name, filt, natoms=None):
    f = abi.SOIL_FILTER_FP32_RECHECK if filt == "fp32" else abi.SOIL_FILTER_FP64
    if natoms:  # reduced size of the same configuration (profiling runs)
        w = {"c1": workloads.config1, "c2": workloads.config2,
             "c3": workloads.config3}[name](n=natoms)
        w.cfg.filter = f
        return w, f"{name} reduced to {natoms} atoms"
    if name == "c1":
        w = workloads.config1()
        w.cfg.filter = f
        desc = "C1 plain: 32,768 monodisperse spheres d=1, phi 0.30, F=0, dt 1e-3"
    elif name == "c3":
        w = workloads.config3()
        w.cfg.filter = f
        desc = ("C3 Lees-Edwards shear: 1,048,576 monodisperse spheres d=1, phi 0.40, "
                "xy rate 0.1, harmonic k=1e3, dt 1e-4")
    else:
        w = workloads.config2(filt=f)
        desc = ("C2 large single system: 4,194,304 polydisperse spheres r~U[0.4,0.6], "
                "phi 0.50, harmonic k=1e3, dt 1e-4")
    return w, desc


def rebuild_probe(s, stream, min_rebuilds=3, chunk=25, max_steps=800):
    """Light and rebuild step costs of a system past the timed region.

    Steps it in calls of about `chunk` steps (lengths varied), each timed with
    CUDA events on the library's stream, until at least `min_rebuilds` steps
    rebuilt the lists and the chunks separate the costs; then fits
    chunk_ms = L * steps + X * rebuilds + C over the chunks (least squares):
    L is the light (communicate-only) step, L + X the rebuild step, C the
    per-call cost (each call ends with the final half-kick, as every
    soil_step call does)."""
    import torch
    rows = []
    steps = rebuilds = 0
    # chunks of varying length, so that (steps, rebuilds) of the chunks are
    # not all proportional and the two costs separate
    lengths = (chunk, chunk // 2 + 1, chunk + chunk // 3, chunk // 3 + 1)

    def rank():
        return np.linalg.matrix_rank(np.array([[n, r, 1.0] for n, r, _ in rows]))

    while steps < max_steps and (rebuilds < min_rebuilds or len(rows) < 4 or
                                 (0 < rebuilds < steps and rank() < 3)):
        n = lengths[len(rows) % len(lengths)]
        r0 = s.counts().rebuilds
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.step(n)
        e1.record(stream)
        s.sync()
        r = int(s.counts().rebuilds - r0)
        rows.append((n, r, e0.elapsed_time(e1)))
        steps += n
        rebuilds += r
    # chunk_ms = L * steps + X * rebuilds + C, C the per-call cost (the
    # call's closing half-kick and launch latency)
    A = np.array([[n, r, 1.0] for n, r, _ in rows], dtype=np.float64)
    t = np.array([ms for _, _, ms in rows])
    out = {"steps": steps, "rebuilds": rebuilds, "chunk_steps": list(lengths),
           "rebuild_rate": rebuilds / steps}
    if rebuilds and np.linalg.matrix_rank(A) == 3:
        (light, extra, _), *_ = np.linalg.lstsq(A, t, rcond=None)
        out.update(ms_per_light_step=float(light), ms_per_rebuild_step=float(light + extra))
    elif rebuilds == steps:  # every step rebuilds (shear)
        out.update(ms_per_light_step=None, ms_per_rebuild_step=float(t.sum() / steps))
    else:
        out.update(ms_per_light_step=float(t.sum() / steps), ms_per_rebuild_step=None)
    L, R = out["ms_per_light_step"], out["ms_per_rebuild_step"]
    rate = out["rebuild_rate"]
    if L is not None and R is not None:
        out["ms_per_step_at_rebuild_rate"] = (1 - rate) * L + rate * R
    else:
        out["ms_per_step_at_rebuild_rate"] = L if R is None else R
    out["neighbor_builds_per_s"] = rate / (out["ms_per_step_at_rebuild_rate"] * 1e-3)
    return out


def cpu_baseline(w, budget_s=20.0, max_steps=10000, warmup=0):
    """The CPU oracle (single thread, as the reference path) on a bounded
    sample of the same system: setup, `warmup` untimed steps, then timed steps
    until ~budget_s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    t0 = time.perf_counter()
    o = oracle.from_workload(w)
    if warmup:
        o.step(warmup)
    t_setup = time.perf_counter() - t0
    steps, t = 0, 0.0
    while t < budget_s and steps < max_steps:
        t1 = time.perf_counter()
        o.step(1)
        t += time.perf_counter() - t1
        steps += 1
    c = o.counts()
    return {"value": w.n * steps / t, "unit": "atom-steps/s", "cores": 1, "kind": "port",
            "sample": (f"{steps} timesteps of the full {w.n}-atom system after {warmup} untimed "
                       f"ones, {c.rebuilds} neighbor builds in all (setup and warm-up "
                       f"{t_setup:.1f}s excluded), C++ oracle -O3, one thread"),
            "steps": steps, "seconds": t, "rebuilds": int(c.rebuilds)}


def run_reference(args, world, rank):
    if rank != 0:
        return 0
    w, desc = make_workload(args.config, args.filter, args.natoms)
    cb = cpu_baseline(w, budget_s=120.0, max_steps=args.steps, warmup=args.warmup)
    line = {
        "impl": "reference", "metric": "atom-steps/s", "value": cb["value"],
        "unit": "atom-steps/s", "n_gpus": args.gpus, "steps": cb["steps"],
        "warmup": args.warmup, "ms_per_step": 1e3 * cb["seconds"] / cb["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded SplitMix64 positions/radii, Box-Muller velocities)",
        "config": {"workload": desc, "n_atoms": w.n, "filter": args.filter},
        "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": cb["value"], "unit": "atom-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_soil(args, world, rank, local):
    import torch
    from soil_b200 import system

    w, desc = make_workload(args.config, args.filter, args.natoms)
    fwd_width = 1  # the radius column
    lib = abi.load_library()
    ctx = system.Context(local)
    s = system.from_workload(ctx, w)
    stream = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", local))

    # warm-up: the first step builds the neighbor list; time every phase on
    # the remaining warm-up steps to find the dominant kernel
    s.step(1)
    s.set_timing((1 << abi.SOIL_NUM_TIMERS) - 1)
    r_warm = s.counts().rebuilds
    n_warm = max(args.warmup - 1, 2)
    s.step(n_warm)
    all_rebuilds = s.counts().rebuilds - r_warm == n_warm
    ms0, _, iv0 = s.get_timing()
    light = {abi.TIMER_NAMES[t]: ms0[t] / max(iv0[t], 1) for t in range(abi.SOIL_NUM_TIMERS)
             if abi.TIMER_NAMES[t] in BYTES_PER_UNIT}
    dominant = max(light, key=light.get)
    # Systems up to 2^20 atoms run their communicate-only steps resident
    # (k_steps, one launch for many steps) unless SOIL_RESIDENT_STEPS=0; phase
    # timers would force the launch-per-phase path, so they stay off there and
    # the roofline comes from the light-step time of the rebuild probe.
    # A workload that rebuilds on every step has no communicate-only stretch
    # to run resident, and keeps its phase timer.
    resident = (w.n <= 2 ** 20 and os.environ.get("SOIL_RESIDENT_STEPS", "2") != "0"
                and not all_rebuilds)
    s.set_timing(0 if resident else 1 << abi.TIMER_NAMES.index(dominant))

    c0 = s.counts()
    launches0 = lib.soil_kernel_launches()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    s.sync()
    dist.barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.step(args.steps)
    ev1.record(stream)
    s.sync()
    torch.cuda.synchronize()
    dist.barrier(world)
    ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    launches = lib.soil_kernel_launches() - launches0
    c1 = s.counts()
    ms_dom, launches_dom, iv_dom = s.get_timing()
    k = abi.TIMER_NAMES.index(dominant)
    ms_max = dist.max_over_ranks(ms, world)

    value = world * w.n * args.steps / (ms_max * 1e-3)
    rebuilds = int(c1.rebuilds - c0.rebuilds)
    peak, peak_kind = load_peaks()
    per_launch_ms = ms_dom[k] / max(launches_dom[k], 1)
    alg_bytes = BYTES_PER_UNIT[dominant](c1, fwd_width)
    achieved = alg_bytes / (per_launch_ms * 1e-3) / 1e9
    kname = phase_kernel(lib, dominant)
    tr = load_traffic(kname, args.config)
    traffic = None
    if tr:
        traffic = tr["dram_bytes_per_atom"] * (c1.nlocal if dominant in ("integrate", "final")
                                               else c1.nlocal + c1.nghost)
    roofline = {"bound": "hbm", "kernel": kname, "phase": dominant,
                "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "peak_source": peak_kind,
                "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                "mean_launch_ms": per_launch_ms, "launches": int(launches_dom[k])}

    # per-phase breakdown (warm-up steps) for the record
    phases = {abi.TIMER_NAMES[t]: round(ms0[t], 4) for t in range(abi.SOIL_NUM_TIMERS) if iv0[t]}
    # the rebuild half of the metric: light and rebuild steps past the timed
    # region, until at least three rebuilds
    s.set_timing(0)
    probe = rebuild_probe(s, stream)
    if resident and probe["ms_per_light_step"]:
        # one k_steps launch runs many light steps: algorithmic bytes of a
        # light step (integration pass + consumer) over the light-step time
        step_bytes = BYTES_PER_UNIT["integrate"](c1, fwd_width) + (
            BYTES_PER_UNIT["force"](c1, fwd_width) if w.harmonic_k else 0)
        ach = step_bytes / (probe["ms_per_light_step"] * 1e-3) / 1e9
        roofline = {"bound": "hbm", "kernel": "k_steps", "phase": "light step (resident)",
                    "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                    "peak_source": peak_kind, "traffic": None,
                    "algorithmic_bytes_per_step": step_bytes,
                    "ms_per_light_step": probe["ms_per_light_step"],
                    "what": "light-step time from the rebuild probe (chunks of resident steps)"}
    del s

    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(ctx, w, args.steps, world)
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(w)
        cb = {k2: cb[k2] for k2 in ("value", "unit", "cores", "kind", "sample")}

    if rank == 0:
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded SplitMix64 positions/radii, Box-Muller velocities)",
            "config": {"workload": desc, "n_atoms": w.n, "filter": args.filter,
                       "box_L": w.L, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (per-atom state ~%d MB)" %
                             (c1.nlocal * 200 // 2**20),
                       "ghosts": int(c1.nghost), "pairs": int(c1.npairs)},
            "timed_steps": {"light": args.steps - rebuilds, "rebuild": rebuilds},
            "neighbor_builds_per_s": world * probe["neighbor_builds_per_s"],
            "neighbor_builds_in_timed_region_per_s": world * rebuilds / (ms_max * 1e-3),
            "rebuilds": rebuilds,
            "ms_per_light_step": probe["ms_per_light_step"],
            "ms_per_rebuild_step": probe["ms_per_rebuild_step"],
            "ms_per_step_at_rebuild_rate": probe["ms_per_step_at_rebuild_rate"],
            "rebuild_probe": {k: probe[k] for k in ("steps", "rebuilds", "chunk_steps",
                                                    "rebuild_rate")},
            "roofline": roofline,
            "cpu_baseline": cb,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "phases_warmup_ms": phases,
        }
        print(json.dumps(line), flush=True)
    return 0


# ---- batched configuration ------------------------------------------------------
C4_DESC = ("C4 batched: 4,096 independent periodic boxes, N log-uniform [256, 65,536] "
           "(47.3M atoms), phi U[0.20,0.55], r~U[0.4,0.6], half sheared at rate U[0.01,0.2], "
           "harmonic k=1e3, dt 1e-4")


def batched_cpu_baseline(ws, budget_s=15.0):
    """The CPU oracle on a sample of the boxes: one thread, and one thread per
    host core each stepping its own box (ctypes releases the GIL)."""
    import concurrent.futures as cf
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = os.cpu_count() or 1

    def run(w, budget):
        o = oracle.from_workload(w)
        steps, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < budget:
            o.step(1)
            steps += 1
        return w.n * steps, time.perf_counter() - t0

    one = run(ws[0], budget_s)
    sample = ws[:cores]
    t0 = time.perf_counter()
    with cf.ThreadPoolExecutor(max_workers=cores) as ex:
        res = list(ex.map(lambda w: run(w, budget_s), sample))
    wall = time.perf_counter() - t0
    return {"value": sum(r[0] for r in res) / wall, "unit": "atom-steps/s", "cores": cores,
            "kind": "port", "one_core_value": one[0] / one[1],
            "sample": (f"{len(sample)} boxes ({sum(w.n for w in sample)} atoms), one per host "
                       f"thread, ~{budget_s:.0f}s each from their initial state; one-core figure "
                       f"from box 0 ({ws[0].n} atoms) alone; C++ oracle -O3")}


def run_batched(args, world, rank, local):
    import torch
    from soil_b200 import system

    nbox = args.boxes
    sizes = [workloads.config4_size(i) for i in range(nbox)]
    mine = dist.lpt_partition(sizes, world)[rank]
    t0 = time.perf_counter()
    ws = [workloads.config4_box(i, steps=args.steps) for i in mine]
    natoms = sum(w.n for w in ws)
    log(f"[c4] rank {rank}: {len(ws)} boxes, {natoms} atoms generated in "
        f"{time.perf_counter() - t0:.1f}s")
    lib = abi.load_library()
    ctx = system.Context(local)
    tuned = None
    if args.tune:
        # bin size per size class, timed on up to two boxes of each class; the
        # table then configures every box (plain and batched runs alike)
        from soil_b200 import autotune
        t0 = time.perf_counter()
        samples = {}
        for w in ws:
            lst = samples.setdefault(autotune.size_class(w.n), [])
            if len(lst) < 2:
                lst.append(w)
        table = autotune.tune(ctx, samples)
        ws = [table.apply(w) for w in ws]
        tuned = {"classes": table.entries, "seconds": time.perf_counter() - t0}
        log(f"[c4] tuned {len(table.entries)} size classes in {tuned['seconds']:.1f}s")
    t0 = time.perf_counter()
    boxes = [system.from_workload(ctx, w) for w in ws]
    log(f"[c4] systems set up in {time.perf_counter() - t0:.1f}s")

    # plain per-system path: every box stepped alone through soil_step, one
    # after the other (each box's first step, which builds its lists, untimed)
    plain_ms = 0.0
    for s in (boxes if args.plain_steps > 0 else []):
        s.step(1)
        st = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", local))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.step(args.plain_steps)
        e1.record(st)
        s.sync()
        plain_ms += e0.elapsed_time(e1)
    plain_ms = dist.max_over_ranks(plain_ms, world)
    plain_value = (dist.sum_over_ranks(natoms, world) * args.plain_steps / (plain_ms * 1e-3)
                   if args.plain_steps > 0 else None)

    batch = system.Batch(ctx)
    for s in boxes:
        batch.add(s)
    stream = torch.cuda.ExternalStream(batch.stream(), device=torch.device("cuda", local))
    batch.step(args.warmup)
    batch.set_timing(True)
    rb0 = sum(s.counts().rebuilds for s in boxes)
    st0 = batch.stats()
    al0 = ctx.alloc_count()
    load0 = os.getloadavg()
    launches0 = lib.soil_kernel_launches()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    batch.sync()
    torch.cuda.synchronize()
    dist.barrier(world)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    batch.step(args.steps)
    ev1.record(stream)
    batch.sync()
    torch.cuda.synchronize()
    dist.barrier(world)
    ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    launches = lib.soil_kernel_launches() - launches0
    tim = batch.get_timing()
    st1 = batch.stats()
    al1 = ctx.alloc_count()
    load1 = os.getloadavg()
    cs = [s.counts() for s in boxes]
    rebuilds = sum(c.rebuilds for c in cs) - rb0
    ms_max = dist.max_over_ranks(ms, world)
    total_atoms = dist.sum_over_ranks(natoms, world)
    value = total_atoms * args.steps / (ms_max * 1e-3)

    # roofline of the consumer kernel (one launch per step over every box):
    # R pos+radius of every atom, W force, R offsets, R each pair twice
    force_ms = tim["force"][0] / max(tim["force"][1], 1)
    force_bytes = sum(64 * (c.nlocal + c.nghost) + 8 * c.npairs for c in cs)
    peak, peak_kind = load_peaks()
    achieved = force_bytes / (force_ms * 1e-3) / 1e9
    tr = load_traffic("batched_force", "c4")
    roofline = {"bound": "hbm", "kernel": "kb_harmonic (all boxes, one launch)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind,
                "traffic": tr["dram_bytes_per_launch"] if tr else None,
                "algorithmic_bytes_per_launch": force_bytes, "mean_launch_ms": force_ms,
                "launches": tim["force"][1]}
    stages = {k: round(v[0] / max(v[1], 1), 4) for k, v in tim.items()}
    host = {k: round(v / args.steps, 4) for k, v in batch.get_host_timing().items()}
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = batched_cpu_baseline(ws)
    if rank == 0:
        line = {
            "metric": "atom-steps/s", "value": value, "unit": "atom-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded SplitMix64 per box, Box-Muller velocities)",
            "config": {"workload": C4_DESC, "boxes": nbox, "n_atoms": total_atoms,
                       "parallelism": "boxes LPT-partitioned over ranks" if world > 1 else "single",
                       "l2": "inputs larger than L2 (~%d GB of per-atom state)" %
                             (total_atoms * 250 // 2**30)},
            "plain_per_system": {"value": plain_value, "unit": "atom-steps/s",
                                 "steps_per_box": args.plain_steps,
                                 "what": "each box alone through soil_step, one after another"},
            "batched_over_plain": value / plain_value if plain_value else None,
            "neighbor_builds_per_s": rebuilds / (ms_max * 1e-3),
            "host_waits_per_step": (st1["host_waits"] - st0["host_waits"]) / args.steps,
            "stage_ms_per_step": stages,
            "host_ms_per_step": host,
            "host_threads": os.environ.get("SOIL_HOST_THREADS", "default"),
            "host_loadavg_1min": [round(load0[0], 2), round(load1[0], 2)],
            "device_allocs_in_timed_region": al1[0] - al0[0],
            "autotune": tuned,
            "roofline": roofline,
            "cpu_baseline": cb,
            "e2e": None,
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    batch.close()
    return 0


# ---- served configuration ---------------------------------------------------------
C5_DESC = ("C5 served: Poisson arrivals at 80% of the plain path's measured throughput; "
           "jobs N log-uniform [1,024, 262,144], phi U[0.20,0.55], r~U[0.4,0.6], shear rate "
           "U[0,0.2], steps U[500,5,000], FP32+FP64-recheck filter, harmonic k=1e3, dt 1e-4, "
           "150 GB HBM budget")


def run_served(args, world, rank, local):
    """C5: continuous batching through soil_server_* against the plain path
    (each job alone through soil_step, one at a time in arrival order)."""
    import threading

    import torch
    from soil_b200 import serve, system

    jobs = [workloads.config5_job(i) for i in range(args.jobs)]
    # partition jobs over ranks (independent units); each rank serves its own
    mine = dist.lpt_partition([w.n * w.steps for w in jobs], world)[rank]
    jobs = [jobs[i] for i in mine]
    work = np.array([w.n * w.steps for w in jobs], dtype=np.float64)

    # plain path: every job alone, `sample` steps after one untimed step; its
    # service time is setup + steps x the sampled per-step time
    ctx = system.Context(local)
    lib = abi.load_library()
    sample = max(args.plain_steps, 20)
    service = []
    for w in jobs:
        t0 = time.perf_counter()
        s = system.from_workload(ctx, w)
        s.step(1)
        s.sync()
        t_setup = time.perf_counter() - t0
        st = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", local))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.step(sample)
        e1.record(st)
        s.sync()
        per_step = e0.elapsed_time(e1) * 1e-3 / sample
        service.append(t_setup + per_step * (w.steps - 1) + per_step)
        s.close()
    service = np.array(service)
    plain_rate = work.sum() / service.sum()           # atom-steps/s of the plain path
    rate = args.load * plain_rate / work.mean()        # jobs/s
    arrivals = serve.poisson_arrivals(rate, len(jobs), seed=5 + rank)
    plain_lat = serve.fifo_latencies(arrivals, service)
    del ctx

    sctx = system.Context(local)
    sv = serve.Server(sctx, hbm_budget_bytes=int(args.budget_gb * 1e9), quantum_steps=args.quantum)
    ids = [None] * len(jobs)
    launches0 = lib.soil_kernel_launches()
    sampler = ClockSampler(local)
    sampler.start()
    dist.barrier(world)
    t_start = time.perf_counter()

    def submitter():
        for k, w in enumerate(jobs):
            d = arrivals[k] - (time.perf_counter() - t_start)
            if d > 0:
                time.sleep(d)
            ids[k] = sv.submit(w)

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    infos = [sv.wait(j) for j in ids]
    t_end = time.perf_counter()
    clocks = sampler.stop()
    launches = lib.soil_kernel_launches() - launches0
    st = sv.stats()
    sv.close()
    states = [i["state"] for i in infos]
    lat = np.array([i["t_done"] - i["t_submit"] for i in infos])
    makespan = dist.max_over_ranks(t_end - t_start, world)
    total_work = dist.sum_over_ranks(float(work.sum()), world)
    if rank == 0:
        line = {
            "metric": "atom-steps/s", "value": total_work / makespan, "unit": "atom-steps/s",
            "n_gpus": world, "steps": int(sum(w.steps for w in jobs)), "warmup": 0,
            "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded SplitMix64 per job, Box-Muller velocities, seeded "
                    "Poisson arrivals)",
            "config": {"workload": C5_DESC, "jobs": len(jobs), "load": args.load,
                       "arrival_rate_per_s": rate, "quantum_steps": args.quantum,
                       "budget_gb": args.budget_gb},
            "served": {"p50_latency_s": float(np.percentile(lat, 50)),
                       "p99_latency_s": float(np.percentile(lat, 99)),
                       "mean_latency_s": float(lat.mean()),
                       "capacity_atom_steps_per_s": st["atom_steps"] / max(st["busy_s"], 1e-9),
                       "makespan_s": makespan, "max_resident_jobs": st["max_active"],
                       "states": {x: states.count(x) for x in set(states)}},
            "plain_per_job": {"value": plain_rate, "unit": "atom-steps/s",
                              "p50_latency_s": float(np.percentile(plain_lat, 50)),
                              "p99_latency_s": float(np.percentile(plain_lat, 99)),
                              "what": ("each job alone through soil_step, one at a time in "
                                       "arrival order (FIFO); service = measured setup + steps x "
                                       f"per-step time sampled over {sample} steps")},
            "served_over_plain_capacity": st["atom_steps"] / max(st["busy_s"], 1e-9) / plain_rate,
            "roofline": None, "cpu_baseline": None, "e2e": None,
            "gpu_launches": int(launches), "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    return 0


def run_e2e(ctx, w, steps, world):
    """Same metric through the C ABI from pinned host buffers: upload the
    initial state, set up, run `steps`, read back positions and velocities."""
    import torch
    from soil_b200 import system

    def pinned(a):
        t = torch.empty(a.shape, dtype={np.float64: torch.float64, np.uint32: torch.int32}[
            a.dtype.type], pin_memory=True)
        v = t.numpy().view(a.dtype)
        v[...] = a
        return t, v

    keep = []
    host = {}
    for name in ("tag", "pos", "vel", "mass", "cutoff", "radius"):
        t, v = pinned(getattr(w, name))
        keep.append(t)
        host[name] = v
    out_pos = pinned(np.zeros((w.n, 3)))
    out_vel = pinned(np.zeros((w.n, 3)))
    h2d = sum(host[k].nbytes for k in host)
    dist.barrier(world)
    t0 = time.perf_counter()
    s = system.System(ctx, w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    s.add_atoms(host["tag"], host["pos"], host["vel"], host["mass"], host["cutoff"],
                columns=[host["radius"]])
    if w.harmonic_k:
        s.set_harmonic(w.harmonic_k, rc)
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    s.setup()
    s.sync()
    t_setup = time.perf_counter()
    s.step(steps)
    s.sync()
    t_steps = time.perf_counter()
    s.read_local_state(out_pos[1], out_vel[1])
    t1 = time.perf_counter()
    dist.barrier(world)
    dt = dist.max_over_ranks(t1 - t0, world)
    d2h = out_pos[1].nbytes + out_vel[1].nbytes
    s.close()
    return {"value": world * w.n * steps / dt, "unit": "atom-steps/s",
            "h2d_bytes_per_step": h2d / steps, "d2h_bytes_per_step": d2h / steps,
            "seconds": dt, "what": "host arrays -> soil_sys_add_atoms/setup -> soil_step(K) "
                                   "-> soil_sys_get_atoms(pos, vel)",
            "breakdown_s": {"create_upload_setup": t_setup - t0, "steps": t_steps - t_setup,
                            "readback": t1 - t_steps}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["soil", "reference"], default="soil")
    ap.add_argument("--config", choices=["c1", "c2", "c3", "c4", "c5"], default="c2")
    ap.add_argument("--jobs", type=int, default=48, help="c5: number of jobs")
    ap.add_argument("--load", type=float, default=0.8,
                    help="c5: arrival rate as a fraction of the plain path's throughput")
    ap.add_argument("--quantum", type=int, default=50, help="c5: steps between admissions")
    ap.add_argument("--budget-gb", type=float, default=150.0, help="c5: HBM budget")
    ap.add_argument("--boxes", type=int, default=workloads.C4_BOXES,
                    help="c4: number of boxes (4096 is the configuration)")
    ap.add_argument("--plain-steps", type=int, default=4,
                    help="c4/c5: timed steps of each box alone (plain path; 0 skips it in c4)")
    ap.add_argument("--filter", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--tune", action="store_true",
                    help="c4: bin size per size class from the autotuner before the run")
    ap.add_argument("--natoms", type=int, default=None,
                    help="reduced system size (profiling only; not a bench line)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    world, rank, local = dist.init()
    try:
        if args.impl == "reference":
            return run_reference(args, world, rank)
        if args.config == "c4":
            return run_batched(args, world, rank, local)
        if args.config == "c5":
            return run_served(args, world, rank, local)
        return run_soil(args, world, rank, local)
    finally:
        dist.finalize(world)


if __name__ == "__main__":
    sys.exit(main())
