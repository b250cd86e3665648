"""Seeded synthetic inputs for the five benchmark configurations.

No dataset is involved: every input is generated on the host from SplitMix64
streams keyed by (seed, box id, stream id, atom id), so the CUDA path and the
CPU oracle consume identical bytes.  Uniform doubles take the top 53 bits;
normal deviates use the Box–Muller transform (Box & Muller, 1958).

Configurations (sizes as stated for the reference comparison):
  C1  plain      32,768 mono d=1, phi 0.30, F = 0, dt 1e-3, 2,000 steps
  C2  large      4,194,304 poly r~U[0.4,0.6], phi 0.50, harmonic k=1e3, dt 1e-4
  C3  shear      1,048,576 mono d=1, phi 0.40, LE rate 0.1, k=1e3, dt 1e-4
  C4  batched    4,096 boxes, N log-U[256, 65536], phi U[0.2,0.55]
  C5  served     Poisson jobs, N log-U[1024, 262144], steps U[500, 5000]
Mass is 1 for every atom (not given for the reference configs).
"""
import math

import numpy as np

from . import abi

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def splitmix64(x):
    """SplitMix64 finaliser applied to a uint64 array (vectorised)."""
    with np.errstate(over="ignore"):
        z = x + GOLDEN
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _key(seed, box, stream):
    with np.errstate(over="ignore"):
        k = splitmix64(np.uint64(seed) * np.uint64(0x100000001B3) + np.uint64(box))
        k = splitmix64(k ^ (np.uint64(stream) * np.uint64(0xD1B54A32D192ED03)))
    return k


def uniform(seed, box, stream, n):
    """n uniform doubles in [0, 1) from stream (seed, box, stream)."""
    k = _key(seed, box, stream)
    with np.errstate(over="ignore"):
        idx = np.arange(n, dtype=np.uint64) * GOLDEN + k
    bits = splitmix64(idx) >> np.uint64(11)
    return bits.astype(np.float64) * (1.0 / 9007199254740992.0)


def normal(seed, box, stream, n):
    """n N(0,1) deviates by Box–Muller from two uniform streams."""
    u1 = 1.0 - uniform(seed, box, 2 * stream + 1000, n)  # (0, 1]
    u2 = uniform(seed, box, 2 * stream + 1001, n)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * math.pi * u2)


def default_cfg(**kw):
    cfg = abi.SoilNeighCfg()
    cfg.skin_fraction = 1.0
    cfg.bin_size = 1.0
    cfg.every = 0
    cfg.sort_every = 1000
    cfg.check = 1
    cfg.newton = 1
    cfg.additive_skin = 0.0
    cfg.filter = abi.SOIL_FILTER_FP64
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


def make_box(L, lo=0.0):
    b = abi.SoilBox()
    for d in range(3):
        b.lo[d] = lo
        b.hi[d] = lo + L
    return b


class Workload:
    """One periodic system: host arrays + box + neighbor config + run knobs."""

    def __init__(self, name, n, L, pos, vel, radius, cutoff, cfg, dt, steps,
                 harmonic_k=0.0, shear_rate=0.0, seed=0):
        self.name = name
        self.n = n
        self.L = L
        self.pos = np.ascontiguousarray(pos, dtype=np.float64)
        self.vel = np.ascontiguousarray(vel, dtype=np.float64)
        self.radius = np.ascontiguousarray(radius, dtype=np.float64)
        self.cutoff = np.ascontiguousarray(cutoff, dtype=np.float64)
        self.mass = np.ones(n, dtype=np.float64)
        self.tag = np.arange(n, dtype=np.uint32)
        self.cfg = cfg
        self.box = make_box(L)
        self.dt = dt
        self.steps = steps
        self.harmonic_k = harmonic_k
        self.shear_rate = shear_rate
        self.seed = seed

    def state_bytes(self):
        # pos, vel, mass, cutoff, radius, tag
        return self.n * (24 + 24 + 8 + 8 + 8 + 4)


def _velocities(seed, box, n):
    v = np.stack([normal(seed, box, s, n) for s in range(3)], axis=1)
    v -= v.mean(axis=0)
    return v


def _positions(seed, box, n, L):
    return np.stack([uniform(seed, box, 10 + s, n) * L for s in range(3)], axis=1)


def mono(name, seed, n, phi, dt, steps, harmonic_k=0.0, shear_rate=0.0, box=0,
         skin=0.1, **cfg_kw):
    """Monodisperse spheres of diameter 1: reference-native skin mapping
    cutoff_radius = 0.5, skin_fraction = 1 + skin (pair cutoff 1 + skin,
    displacement budget skin/2)."""
    L = (n * math.pi / 6.0 / phi) ** (1.0 / 3.0)
    pos = _positions(seed, box, n, L)
    vel = _velocities(seed, box, n)
    radius = np.full(n, 0.5)
    cutoff = np.full(n, 0.5)
    cfg = default_cfg(skin_fraction=1.0 + skin, **cfg_kw)
    return Workload(name, n, L, pos, vel, radius, cutoff, cfg, dt, steps,
                    harmonic_k=harmonic_k, shear_rate=shear_rate, seed=seed)


def poly(name, seed, n, phi, dt, steps, harmonic_k=0.0, shear_rate=0.0, box=0,
         skin=0.1, rmin=0.4, rmax=0.6, **cfg_kw):
    """Polydisperse spheres r ~ U[rmin, rmax]: additive skin mapping
    cutoff_radius = r + skin/2, skin_fraction = 1, additive_skin = skin."""
    radius = rmin + (rmax - rmin) * uniform(seed, box, 20, n)
    vol = float(np.sum(4.0 / 3.0 * math.pi * radius ** 3))
    L = (vol / phi) ** (1.0 / 3.0)
    pos = _positions(seed, box, n, L)
    vel = _velocities(seed, box, n)
    cutoff = radius + 0.5 * skin
    cfg = default_cfg(skin_fraction=1.0, additive_skin=skin, **cfg_kw)
    return Workload(name, n, L, pos, vel, radius, cutoff, cfg, dt, steps,
                    harmonic_k=harmonic_k, shear_rate=shear_rate, seed=seed)


def config1(n=32768, steps=2000):
    return mono("C1-plain-32768", 1, n, 0.30, 1e-3, steps)


def config2(n=4194304, steps=1000, filt=abi.SOIL_FILTER_FP64):
    return poly("C2-large-4194304", 2, n, 0.50, 1e-4, steps, harmonic_k=1e3, filter=filt)


def config3(n=1048576, steps=5000):
    return mono("C3-shear-1048576", 3, n, 0.40, 1e-4, steps, harmonic_k=1e3, shear_rate=0.1)


C4_BOXES = 4096


def config4_size(i, nmin=256, nmax=65536):
    """Atom count of box i of the batched configuration (log-uniform)."""
    u = uniform(4, i, 90, 1)
    return int(round(math.exp(math.log(nmin) + (math.log(nmax) - math.log(nmin)) * u[0])))


def config4_box(i, nmin=256, nmax=65536, steps=1000):
    """Box i of the batched configuration (seed 4 + box id)."""
    s = 4
    u = uniform(s, i, 90, 4)
    n = config4_size(i, nmin, nmax)
    phi = 0.20 + 0.35 * u[1]
    rate = 0.0 if i % 2 == 0 else 0.01 + 0.19 * u[2]
    return poly(f"C4-box{i}", s, n, phi, 1e-4, steps, harmonic_k=1e3, shear_rate=rate, box=i)


def config5_job(i, nmin=1024, nmax=262144, smin=500, smax=5000):
    """Job i of the served configuration (seed 5 + job id)."""
    s = 5
    u = uniform(s, i, 91, 5)
    n = int(round(math.exp(math.log(nmin) + (math.log(nmax) - math.log(nmin)) * u[0])))
    phi = 0.20 + 0.35 * u[1]
    rate = 0.2 * u[2]
    steps = int(smin + (smax - smin) * u[3])
    return poly(f"C5-job{i}", s, n, phi, 1e-4, steps, harmonic_k=1e3, shear_rate=rate, box=i,
                filter=abi.SOIL_FILTER_FP32_RECHECK)
