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
    if name == "fixed-z-shrink-x":
        w = W.poly(name, 106, 1500, 0.40, 1e-3, 60, harmonic_k=1e3)
        w.vel *= 10.0
        return w, {"boundary": ([S, P, F], 0.0)}
    raise KeyError(name)


CASES = ["mono-free", "poly-harmonic", "mono-shear", "poly-newton-off-fp32", "deform-z-erate",
         "fixed-z-shrink-x"]


def build(make, name):
    """make(box, cfg, dt) -> an empty GPU or oracle system; returns (system, steps)."""
    w, extra = _w(name)
    s = make(w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    if w.harmonic_k:
        s.set_harmonic(w.harmonic_k, rc)
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    for dim, style, a, b, stage in extra.get("deform", []):
        s.set_deform(dim, style, a, b, stage)
    if "boundary" in extra:
        s.set_boundary(*extra["boundary"])
    s.setup()
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
    }
