"""The oracle's borders (comm.rs:288-369, 682-860, single rank) against a
second, independent restatement written here in plain Python, for orthogonal
boxes with periodic, fixed and shrink-wrapped axes: every swap's send list,
recv range and offset, and every ghost's position, tag and origin.  The
oracle is stepped first (integration, pbc, sort), then its locals are bordered
again here from scratch."""
import numpy as np
import pytest

import oracle
from soil_b200 import abi, workloads as W

P, F, S = abi.SOIL_BOUNDARY_PERIODIC, abi.SOIL_BOUNDARY_FIXED, abi.SOIL_BOUNDARY_SHRINK


def py_borders(pos, lo, hi, gc, periodic):
    """pack_border_atoms' orthogonal face test over [0, dim_scan_end) for each
    swap (lo face, then hi face, dims x, y, z); a periodic axis appends the
    packed atoms shifted by +-L as ghosts, a neighborless one packs only."""
    pos = [tuple(p) for p in pos]
    origin = list(range(len(pos)))
    swaps = []
    scan_end = len(pos)
    for dim in range(3):
        dim_scan_end = scan_end
        size = hi[dim] - lo[dim]
        for swap in range(2):
            po = (1.0 if swap == 0 else -1.0) if periodic[dim] else 0.0
            shift = [0.0, 0.0, 0.0]
            shift[dim] = po * size
            if swap == 0:
                thresh = lo[dim] + gc
                packed = [i for i in range(dim_scan_end) if pos[i][dim] < thresh]
            else:
                thresh = hi[dim] - gc
                packed = [i for i in range(dim_scan_end) if pos[i][dim] >= thresh]
            recv_start = len(pos)
            if periodic[dim]:
                for i in packed:
                    pos.append((pos[i][0] + shift[0], pos[i][1] + shift[1], pos[i][2] + shift[2]))
                    origin.append(i)
            swaps.append(dict(send=packed, recv_start=recv_start,
                              recv_count=len(pos) - recv_start, offset=shift))
        scan_end = len(pos)
    return np.array(pos), np.array(origin), swaps


@pytest.mark.parametrize("types", [[P, P, P], [P, P, F], [F, F, F], [S, P, F], [P, S, S]])
def test_oracle_borders_match_a_python_restatement(types):
    w = W.poly("borders", 51, 1200, 0.4, 1e-3, 5, harmonic_k=1e3)
    w.vel *= 5.0
    o = oracle.OracleSystem(w.box, w.cfg, w.dt)
    rc = o.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    o.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    o.set_harmonic(w.harmonic_k, rc)
    o.set_boundary(types, 0.3)
    o.setup()
    o.step(5)  # every step here rebuilds or not; force one more full rebuild:
    o.set_state(abi.SOIL_FULL_REBUILD)
    for ph in ("remove_ghosts", "shrink_wrap", "pbc", "sort", "borders"):
        o.phase(ph)
    c = o.counts()
    a = o.atoms()
    nl = c.nlocal
    lo, hi, _ = o.box()
    pos, origin, swaps = py_borders(a["pos"][:nl], lo, hi, c.ghost_cutoff,
                                    [t == P for t in types])
    assert c.nghost == len(pos) - nl
    np.testing.assert_array_equal(a["pos"].view(np.uint64), pos.view(np.uint64))
    np.testing.assert_array_equal(a["origin"][nl:], origin[nl:])
    np.testing.assert_array_equal(a["tag"][nl:], a["tag"][origin[nl:]])
    got = o.swaps()
    assert len(got) == 6
    for k, (g, want) in enumerate(zip(got, swaps)):
        assert g["recv_start"] == want["recv_start"] and g["recv_count"] == want["recv_count"], k
        np.testing.assert_array_equal(g["send"], np.array(want["send"], np.uint32), err_msg=str(k))
        np.testing.assert_array_equal(g["offset"], np.array(want["offset"]), err_msg=str(k))
