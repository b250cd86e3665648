"""The oracle's spatial sort and neighbor-list row order against a second,
independent restatement written here in plain Python/numpy:

  sort_atoms_by_bin (crates/soil_core/src/neighbor.rs:834-997): the cell of
      every local (lamda coordinates when triclinic), a stable counting sort,
      perm[new] = old;
  bin_neighbor_list (neighbor.rs:1013-1319): every atom (locals and ghosts)
      binned by a stable counting sort, then row i = the own cell's atoms after
      i's slot (newton) or the whole own cell without i (newton off), then the
      stencil cells in stencil order, each in bin order; a candidate j is kept
      when r2 = fma(dx, dx, fma(dy, dy, dz*dz)) is below the uniform cut^2, or
      below (s_i + s_j)^2 * sf^2 for mixed cutoffs.

The bin grid (origin, bin size, counts, stencils) is taken from the oracle;
what is checked is the order the lists and the permutation come out in, bit
for bit, which no reference test pins.  r2 is evaluated with numpy (never
fused); the few candidates within 1e-9 relative of their threshold are
re-evaluated with an exactly rounded fma (rational arithmetic)."""
from fractions import Fraction

import numpy as np
import pytest

import oracle
from soil_b200 import abi, workloads as W


def x2lamda(pos, lo, size, tilt):
    """Domain::x2lamda, domain.rs:211-217 (IEEE double, no contraction)."""
    xy, xz, yz = tilt
    lz = (pos[:, 2] - lo[2]) / size[2]
    ly = (pos[:, 1] - lo[1] - yz * lz) / size[1]
    lx = (pos[:, 0] - lo[0] - xy * ly - xz * lz) / size[0]
    return np.stack([lx, ly, lz], axis=1)


def cells(pos, origin, bin_size, bin_count, triclinic, lo, size, tilt):
    p = x2lamda(pos, lo, size, tilt) if triclinic else pos
    inv = [1.0 / b for b in bin_size]
    c = []
    for d in range(3):
        f = np.floor((p[:, d] - origin[d]) * inv[d])
        f = np.clip(f, -2.0 ** 31, 2.0 ** 31 - 1).astype(np.int64)  # `as i32` saturates
        c.append(np.clip(f, 0, bin_count[d] - 1))
    ny, nz = bin_count[1], bin_count[2]
    return (c[0] * ny * nz + c[1] * nz + c[2]).astype(np.int64)


def stable_counting_sort(cell, ncells):
    """perm[slot] = i in ascending i within each cell; start[c] = first slot of c."""
    counts = np.bincount(cell, minlength=ncells)
    start = np.zeros(ncells + 1, np.int64)
    np.cumsum(counts, out=start[1:])
    return np.argsort(cell, kind="stable"), start


def fma(a, b, c):
    return float(Fraction(a) * Fraction(b) + Fraction(c))


def py_neighbor_rows(pos, cut, nlocal, cell, ncells, stencil, has_self, newton, uniform_sq,
                     sf_sq):
    sorted_atoms, start = stable_counting_sort(cell, ncells)
    slot = np.empty(len(cell), np.int64)
    slot[sorted_atoms] = np.arange(len(cell))
    offsets, indices = [0], []
    for i in range(nlocal):
        c = cell[i]
        ranges = []
        if has_self:
            if newton:
                ranges.append(np.arange(slot[i] + 1, start[c + 1]))
            else:
                m = np.arange(start[c], start[c + 1])
                ranges.append(m[sorted_atoms[m] != i])
        for off in stencil:
            if not newton and off == 0:
                continue
            cc = c + off
            ranges.append(np.arange(start[cc], start[cc + 1]))
        m = np.concatenate(ranges) if ranges else np.zeros(0, np.int64)
        j = sorted_atoms[m]
        d = pos[j] - pos[i]
        r2 = d[:, 0] * d[:, 0] + (d[:, 1] * d[:, 1] + d[:, 2] * d[:, 2])
        if uniform_sq is not None:
            lim = np.full(len(j), uniform_sq)
        else:
            s = cut[i] + cut[j]
            lim = s * s * sf_sq
        keep = r2 < lim
        close = np.abs(r2 - lim) <= 1e-9 * lim
        for k in np.nonzero(close)[0]:  # exactly rounded nested fma near the threshold
            dx, dy, dz = (float(v) for v in d[k])
            keep[k] = fma(dx, dx, fma(dy, dy, dz * dz)) < lim[k]
        indices.extend(j[keep].tolist())
        offsets.append(len(indices))
    return np.array(offsets, np.uint32), np.array(indices, np.uint32)


def _oracle(w, newton=True):
    w.cfg.newton = 1 if newton else 0
    o = oracle.OracleSystem(w.box, w.cfg, w.dt)
    rc = o.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    o.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    o.set_harmonic(w.harmonic_k or 1e3, rc)
    if w.shear_rate:
        o.set_shear(w.shear_rate)
    o.setup()
    return o


CASES = {
    "mono-uniform": lambda: W.mono("rows-mono", 61, 1500, 0.35, 1e-3, 0),
    "poly-mixed": lambda: W.poly("rows-poly", 62, 1500, 0.45, 1e-3, 0, harmonic_k=1e3),
    "poly-newton-off": lambda: W.poly("rows-nn", 63, 1200, 0.45, 1e-3, 0, harmonic_k=1e3),
    "mono-sheared": lambda: W.mono("rows-shear", 64, 1500, 0.40, 1e-3, 0, harmonic_k=1e3,
                                   shear_rate=2.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
@pytest.mark.parametrize("steps", [0, 7])
def test_sort_and_rows_match_a_python_restatement(name, steps):
    w = CASES[name]()
    w.vel *= 4.0  # atoms change cells between rebuilds
    newton = name != "poly-newton-off"
    o = _oracle(w, newton)
    o.step(steps)
    o.set_state(abi.SOIL_FULL_REBUILD)
    for ph in ("deform", "initial", "decide_rebuild", "remove_ghosts", "zero_forces", "pbc"):
        o.phase(ph)
    o.set_state(abi.SOIL_FULL_REBUILD)
    c = o.counts()
    nl = c.nlocal
    before = o.atoms(local_only=True)
    o.phase("sort")
    fwd, origin, bin_size = o.stencil()
    full, has_self = o.stencil_full()
    c = o.counts()
    bc = list(c.bin_count)
    ncells = bc[0] * bc[1] * bc[2]
    lo, hi, tilt = o.box()
    tri = bool(c.triclinic)
    assert tri == (name == "mono-sheared")

    # sort_atoms_by_bin
    cell_before = cells(before["pos"], origin, bin_size, bc, tri, lo, hi - lo, tilt)
    perm, _ = stable_counting_sort(cell_before, ncells)
    np.testing.assert_array_equal(o.sort_perm(), perm.astype(np.uint32))

    # bin_neighbor_list over the bordered atoms
    o.phase("borders")
    o.phase("forward_comm")
    a = o.atoms()
    o.phase("neighbor")
    cut_of_tag = w.cutoff
    cut = cut_of_tag[a["tag"]]
    uniform_sq = None
    if cut[:nl].max() == cut[:nl].min():
        r = 2.0 * cut[0] * w.cfg.skin_fraction
        uniform_sq = r * r
    cell_all = cells(a["pos"], origin, bin_size, bc, tri, lo, hi - lo, tilt)
    want_off, want_idx = py_neighbor_rows(
        a["pos"], cut, nl, cell_all, ncells, fwd if newton else full, has_self, newton,
        uniform_sq, w.cfg.skin_fraction * w.cfg.skin_fraction)
    got_off, got_idx = o.neighbor()
    assert len(want_idx) > nl  # a non-trivial list
    np.testing.assert_array_equal(got_off, want_off)
    np.testing.assert_array_equal(got_idx, want_idx)
