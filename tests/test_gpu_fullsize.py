"""The full C2 system (4,194,304 polydisperse atoms) on the GPU, checked through
properties that do not need the oracle to run at that size:

- the spatial sort's permutation is a bijection and the locals sit in the box;
- every ghost is its origin plus its swap's offset, bit for bit (the border
  images and their chains);
- every listed pair lies inside its cutoff, and around sampled atoms the
  lists hold exactly the minimum-image pairs inside the cutoff (by tag);
- sampled interior atoms carry exactly the force the reference's pair order
  gives, recomputed here in Python doubles, bit for bit;
- the local forces sum to zero up to rounding (Newton's third law through
  the reverse comm).
"""
import math

import numpy as np
import pytest

from soil_b200 import system, workloads as W

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2(ctx):
    w = W.config2()
    s = system.from_workload(ctx, w)
    s.step(1)  # the first step builds ghosts and lists after the sort
    state = dict(w=w, c=s.counts(), a=s.atoms(), rad=s.column(0)[:, 0], lists=s.neighbor(),
                 swaps=s.swaps(), perm=s.sort_perm(), box=s.box())
    s.close()
    return state


def test_sort_is_a_bijection_and_locals_are_in_the_box(c2):
    nl = c2["c"].nlocal
    assert np.array_equal(np.sort(c2["perm"]), np.arange(nl, dtype=np.uint32))
    lo, hi, _ = c2["box"]
    p = c2["a"]["pos"][:nl]
    assert np.all(p >= lo) and np.all(p < hi)


def test_ghosts_are_their_origin_plus_the_swap_offset(c2):
    a, nl = c2["a"], c2["c"].nlocal
    pos, origin, tag = a["pos"], a["origin"], a["tag"]
    assert c2["c"].nghost > 0
    for sw in c2["swaps"]:
        g = np.arange(sw["recv_start"], sw["recv_start"] + sw["recv_count"])
        o = origin[g]
        assert np.array_equal(o, sw["send"].astype(np.int64))
        np.testing.assert_array_equal((pos[o] + sw["offset"]).view(np.uint64), pos[g].view(np.uint64))
        assert np.array_equal(tag[g], tag[o])
    assert len(pos) == nl + c2["c"].nghost


def _pairs(c2):
    off, idx = c2["lists"]
    nl = c2["c"].nlocal
    i = np.repeat(np.arange(nl), np.diff(off.astype(np.int64)))
    return i, idx.astype(np.int64)


def test_listed_pairs_are_inside_the_cutoff(c2):
    pos = c2["a"]["pos"]
    i, j = _pairs(c2)
    w = c2["w"]
    sf = w.cfg.skin_fraction
    # cutoff radii: r + skin/2 per atom, carried to ghosts through the tag
    r_of_tag = w.cutoff
    ci, cj = r_of_tag[c2["a"]["tag"][i]], r_of_tag[c2["a"]["tag"][j]]
    d = pos[j] - pos[i]
    r2 = np.einsum("ij,ij->i", d, d)
    lim = (ci + cj) * sf
    assert np.all(r2 < lim * lim * (1 + 1e-12))


def test_lists_around_sampled_atoms_are_complete(c2):
    w, a, nl = c2["w"], c2["a"], c2["c"].nlocal
    tag, pos = a["tag"], a["pos"]
    L = w.L
    sf = w.cfg.skin_fraction
    i, j = _pairs(c2)
    ti, tj = tag[i], tag[j]
    ploc = pos[:nl]
    cloc = w.cutoff[tag[:nl]]
    rng = np.random.default_rng(7)
    for a_idx in rng.choice(nl, 48, replace=False):
        t = tag[a_idx]
        d = ploc - ploc[a_idx]
        d -= L * np.round(d / L)
        r2 = np.einsum("ij,ij->i", d, d)
        lim2 = ((cloc + cloc[a_idx]) * sf) ** 2
        near = (r2 < lim2) & (np.arange(nl) != a_idx)
        clear = np.abs(r2 - lim2) > 1e-9 * lim2  # leave rounding ties at the edge aside
        want = set(tag[:nl][near & clear].tolist())
        listed = set(tj[ti == t].tolist()) | set(ti[tj == t].tolist())
        edge = set(tag[:nl][~clear].tolist())
        assert want == (listed - edge), f"atom tag {t}"


def _harmonic_f(K, xi, xj, ri, rj):
    sum_r = ri + rj
    dx, dy, dz = xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]
    dist_sq = dx * dx + dy * dy + dz * dz
    if dist_sq >= sum_r * sum_r or dist_sq == 0.0:
        return None
    dist = math.sqrt(dist_sq)
    overlap = sum_r - dist
    inv = 1.0 / dist
    fmag = K * overlap
    return (-fmag * dx * inv, -fmag * dy * inv, -fmag * dz * inv)


def test_sampled_interior_forces_follow_the_reference_pair_order(c2):
    w, a, nl = c2["w"], c2["a"], c2["c"].nlocal
    tag, pos, force, rad = a["tag"], a["pos"], a["force"], c2["rad"]
    off, idx = c2["lists"]
    i, j = _pairs(c2)
    imaged_tags = set(tag[nl:].tolist())
    rng = np.random.default_rng(11)
    done = 0
    for a_idx in rng.choice(nl, 400, replace=False):
        if tag[a_idx] in imaged_tags:
            continue  # its force also gets folded ghost contributions
        rows = np.sort(i[j == a_idx])  # rows that list a (ascending)
        F = [0.0, 0.0, 0.0]

        def sub(f):
            if f is not None:
                F[0], F[1], F[2] = F[0] - f[0], F[1] - f[1], F[2] - f[2]

        for r in rows[rows < a_idx]:
            sub(_harmonic_f(w.harmonic_k, pos[r], pos[a_idx], rad[r], rad[a_idx]))
        for k in range(int(off[a_idx]), int(off[a_idx + 1])):
            o = int(idx[k])
            f = _harmonic_f(w.harmonic_k, pos[a_idx], pos[o], rad[a_idx], rad[o])
            if f is not None:
                F[0], F[1], F[2] = F[0] + f[0], F[1] + f[1], F[2] + f[2]
        for r in rows[rows > a_idx]:
            sub(_harmonic_f(w.harmonic_k, pos[r], pos[a_idx], rad[r], rad[a_idx]))
        np.testing.assert_array_equal(np.array(F).view(np.uint64), force[a_idx].view(np.uint64),
                                      err_msg=f"atom {a_idx}")
        done += 1
    assert done > 300


def test_local_forces_sum_to_zero(c2):
    nl = c2["c"].nlocal
    f = c2["a"]["force"][:nl]
    total = np.abs(f).sum()
    assert total > 0
    assert np.all(np.abs(f.sum(axis=0)) < 1e-10 * total)
