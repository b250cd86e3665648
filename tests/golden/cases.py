"""Workloads of the committed golden states (tests/golden/states.json).

Each case is a small seeded system covering one mix of the path's features;
`state_digest` reduces a system (GPU or oracle: both expose counts(),
atoms(), neighbor(), swaps(), box()) to counters and SHA-256 digests of the
IEEE bytes, so a fixture of a few hundred bytes pins a whole trajectory."""
import hashlib

import numpy as np

from soil_b200 import abi, workloads as W

P, F, S = abi.SOIL_BOUNDARY_PERIODIC, abi.SOIL_BOUNDARY_FIXED, abi.SOIL_BOUNDARY_SHRINK


def _w(name):
    if name == "mono-free":  # C1-like: no consumer
        return W.mono(name, 101, 2000, 0.30, 1e-3, 60), {}
    if name == "poly-harmonic":  # C2-like
        return W.poly(name, 102, 2000, 0.50, 1e-4, 60, harmonic_k=1e3), {}
    if name == "mono-shear":  # C3-like
        return W.mono(name, 103, 1500, 0.40, 1e-3, 60, harmonic_k=1e3, shear_rate=0.5), {}
    if name == "poly-newton-off-fp32":
        w = W.poly(name, 104, 1500, 0.45, 1e-4, 60, harmonic_k=1e3)
        w.cfg.newton = 0
        w.cfg.filter = abi.SOIL_FILTER_FP32_RECHECK
        return w, {}
    if name == "deform-z-erate":
        w = W.poly(name, 105, 1500, 0.40, 1e-3, 60, harmonic_k=1e3)
        return w, {"deform": [(2, abi.SOIL_DEFORM_ERATE, -1.0, 0.0, 0)]}
    if name == "registry-columns":  # every AtomData flag class, widths 1-3
        w = W.poly(name, 107, 1500, 0.45, 1e-3, 60, harmonic_k=1e3)
        w.vel *= 3.0  # a rebuild (sort, borders) every few steps
        return w, {"columns": True}
    if name == "fixed-z-shrink-x":
        w = W.poly(name, 106, 1500, 0.40, 1e-3, 60, harmonic_k=1e3)
        w.vel *= 10.0
        return w, {"boundary": ([S, P, F], 0.0)}
    raise KeyError(name)


CASES = ["mono-free", "poly-harmonic", "mono-shear", "poly-newton-off-fp32", "deform-z-erate",
         "fixed-z-shrink-x", "registry-columns"]

# Columns of the registry case beyond the radius (column 0): name, width,
# flags.  A consumer (the oracle's column probe, or tests/hooks/registry_hook.cu
# on the GPU) writes orient (locals), torque and zacc (every atom) in the
# Force phase; label is never written, only permuted and copied to ghosts.
REGISTRY_COLUMNS = [("orient", 3, abi.SOIL_COL_FORWARD), ("torque", 2, abi.SOIL_COL_REVERSE),
                    ("zacc", 1, abi.SOIL_COL_ZERO), ("label", 2, 0)]
REGISTRY_PROBE = {"rev_col": 2, "zero_col": 3, "fwd_col": 1}


def build(make, name, attach=None):
    """make(box, cfg, dt) -> an empty GPU or oracle system; returns (system, steps).
    attach(system, probe) installs the column-writing consumer of cases that
    register columns (probe: REGISTRY_PROBE)."""
    w, extra = _w(name)
    s = make(w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    data = [w.radius]
    if extra.get("columns"):
        for k, (cname, width, flags) in enumerate(REGISTRY_COLUMNS):
            s.register_column(cname, width, flags)
            vals = np.stack([W.uniform(w.seed, 0, 40 + 4 * k + c, w.n) for c in range(width)],
                            axis=1)
            data.append(vals if width > 1 else vals[:, 0])
    s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=data)
    if w.harmonic_k:
        s.set_harmonic(w.harmonic_k, rc)
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    for dim, style, a, b, stage in extra.get("deform", []):
        s.set_deform(dim, style, a, b, stage)
    if "boundary" in extra:
        s.set_boundary(*extra["boundary"])
    s.setup()
    if extra.get("columns"):
        if attach is None:
            raise ValueError(f"case {name} needs a column consumer (attach)")
        attach(s, REGISTRY_PROBE)
    return s, w.steps


def _h(*arrays):
    m = hashlib.sha256()
    for a in arrays:
        m.update(np.ascontiguousarray(a).tobytes())
    return m.hexdigest()


def state_digest(s):
    c = s.counts()
    a = s.atoms()
    off, idx = s.neighbor()
    sw = s.swaps()
    lo, hi, tilt = s.box()
    return {
        "nlocal": int(c.nlocal), "nghost": int(c.nghost), "npairs": int(c.npairs),
        "rebuilds": int(c.rebuilds), "step": int(c.step),
        "atoms": _h(a["tag"], a["pos"], a["vel"], a["force"], a["image"], a["origin"]),
        "lists": _h(off.astype(np.uint32), idx.astype(np.uint32)),
        "swaps": _h(*[np.array([x["recv_start"], x["recv_count"]], np.uint64) for x in sw],
                    *[x["send"].astype(np.uint32) for x in sw],
                    *[x["offset"] for x in sw], *[x["vel_offset"] for x in sw]),
        "box": _h(lo, hi, tilt),
        "columns": _h(*[s.column(k) for k in range(len(s.columns))]),
    }
