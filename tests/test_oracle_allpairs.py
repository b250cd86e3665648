"""Pins the oracle's neighbor list against an independent O(N^2) periodic
all-pairs search (after neighbor.rs:1433-1454, extended to periodic images
and to equality instead of containment).

Every CSR entry (i, j) is mapped to a physical pair (tag_i, tag_j, image
shift); the set must equal the brute-force set of atom pairs over all
images whose distance passes the reference's pair test
fma(dx,dx,fma(dy,dy,dz*dz)) < cut^2.
"""
import itertools
from fractions import Fraction

import numpy as np
import pytest

import oracle
from soil_b200 import workloads as W


def fma(a, b, c):
    """Correctly rounded a*b+c (exact rational arithmetic, one rounding)."""
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def brute_force(pos, cut, L, sf):
    n = len(pos)
    res = set()
    shifts = np.array(list(itertools.product((-1, 0, 1), repeat=3)), dtype=np.float64)
    for a in range(n):
        for si, s in enumerate(shifts):
            d = pos[a:] + s * L - pos[a]          # candidates b >= a
            r2 = d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2]
            c = (cut[a] + cut[a:]) * sf
            c2 = c * c
            near = np.abs(r2 - c2) <= 1e-9 * c2
            hit = r2 < c2
            for k in np.nonzero(near)[0]:      # decide ties with the exact test
                dx, dy, dz = d[k]
                hit[k] = fma(dx, dx, fma(dy, dy, dz * dz)) < c2[k]
            st = tuple(int(v) for v in s)
            for k in np.nonzero(hit)[0]:
                b = a + int(k)
                if a == b and st <= (0, 0, 0):
                    continue  # each self-image pair once, never the atom itself
                res.add((a, b, st))
    return res


def csr_pairs(o, L):
    a = o.atoms()
    off, idx = o.neighbor()
    n = o.counts().nlocal
    tag, pos = a["tag"], a["pos"]
    owner_pos = {}
    for i in range(n):
        owner_pos[int(tag[i])] = pos[i]
    res = []
    for i in range(n):
        for k in range(off[i], off[i + 1]):
            j = int(idx[k])
            ti, tj = int(tag[i]), int(tag[j])
            s = tuple(int(v) for v in np.round((pos[j] - owner_pos[tj]) / L))
            if (ti, s) > (tj, tuple(-v for v in s)) if ti == tj else ti > tj:
                ti, tj, s = tj, ti, tuple(-v for v in s)
            res.append((ti, tj, s))
    return res


@pytest.mark.parametrize("kind", ["mono", "poly", "small"])
def test_csr_equals_periodic_all_pairs(kind):
    if kind == "mono":
        w = W.mono("ap", 21, 500, 0.35, 1e-3, 0)
    elif kind == "poly":
        w = W.poly("ap", 22, 500, 0.45, 1e-3, 0)
    else:
        w = W.mono("ap", 23, 30, 0.3, 1e-3, 0)
    o = oracle.from_workload(w)
    o.step(7)  # let the atoms move, then force a full rebuild at these positions
    o.set_state(0)
    for ph in ("remove_ghosts", "zero_forces", "pbc", "sort", "borders", "neighbor"):
        o.phase(ph)
    a = o.atoms(local_only=True)
    order = np.argsort(a["tag"])
    pos = a["pos"][order]
    cut = w.cutoff
    got = csr_pairs(o, w.L)
    assert len(got) == len(set(got)), "a physical pair appears twice"
    want = brute_force(pos, cut, w.L, w.cfg.skin_fraction)
    assert set(got) == want
