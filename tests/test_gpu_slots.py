"""Persistent per-neighbor slots (soil_sys_enable_slots, include/soil_slots.cuh).

The reference prototype's own test (crates/soil_gpu/src/neighbor_slots.rs:
211-275) lets every atom add 1 to a slot keyed by itself for K steps and
checks the payload is K; here the same runs through spatial sorts, which move
the slots with their atoms.  The contact test keeps a 5-wide history per
contact (steps in contact, summed overlap, summed x_j - x_i) and compares it
bit for bit with the same history kept on the host from the oracle's
positions and lists, through rebuilds, sorts, shear and pairs changing rows.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import oracle
from helpers import assert_same_state
from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
NONE = 0xFFFFFFFF


@pytest.fixture(scope="module")
def slots_lib(tmp_path_factory):
    out = tmp_path_factory.mktemp("hook") / "libslots_hook.so"
    subprocess.check_call(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-O3", "-fmad=false", "-shared", "-Xcompiler", "-fPIC",
                           "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "hooks", "slots_hook.cu"), "-o", str(out)])
    return C.CDLL(str(out))


class HistoryUser(C.Structure):
    _fields_ = [("K", C.c_double), ("overflow", C.c_void_p)]


def _system(ctx, w, max_contacts, width, enable_before_setup):
    s = system.System(ctx, w.box, w.cfg, w.dt)
    assert s.register_column("radius", 1, abi.SOIL_COL_FORWARD) == 0
    s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    if enable_before_setup:
        s.enable_slots(max_contacts, width)
    s.setup()
    if not enable_before_setup:
        s.enable_slots(max_contacts, width)
    return s


@pytest.mark.parametrize("enable_before_setup", [True, False])
def test_self_slot_persists_through_sorts(ctx, slots_lib, enable_before_setup):
    w = W.poly("slots-self", 21, 3000, 0.5, 1e-3, 30, harmonic_k=1e3, shear_rate=1.0)
    w.cfg.sort_every = 3
    s = _system(ctx, w, 4, 2, enable_before_setup)
    k = C.c_double(w.harmonic_k)
    s.set_force_hook_ptr(C.cast(slots_lib.self_count_hook, C.c_void_p).value,
                         C.cast(C.pointer(k), C.c_void_p))
    s.step(17)
    s.step(13)
    c = s.counts()
    assert c.sorts > 5
    tags, vals = s.slots()
    own = s.atoms(local_only=True)["tag"]
    np.testing.assert_array_equal(tags[:, 0], own)
    assert np.all(tags[:, 1:] == NONE)
    assert np.all(vals[:, 0, 0] == 30.0)
    s.close()


def _oracle_contacts(o, prev, stats):
    """One step of the contact history on the host, from the oracle's state
    after that step (positions at force time, the step's lists)."""
    nl = o.counts().nlocal
    off, idx = o.neighbor()
    a = o.atoms()
    tag, pos = a["tag"], a["pos"]
    rad = o.column(0)[:, 0]
    rows = np.repeat(np.arange(nl), np.diff(off[:nl + 1]).astype(np.int64))
    i, j = rows, idx.astype(np.int64)
    dx = pos[j, 0] - pos[i, 0]
    dy = pos[j, 1] - pos[i, 1]
    dz = pos[j, 2] - pos[i, 2]
    dist_sq = dx * dx + dy * dy + dz * dz
    sum_r = rad[i] + rad[j]
    hit = ~((dist_sq >= sum_r * sum_r) | (dist_sq == 0.0))
    overlap = sum_r - np.sqrt(dist_sq)
    new = {}
    for e in np.nonzero(hit)[0]:
        ti, tj = int(tag[i[e]]), int(tag[j[e]])
        key = (min(ti, tj), max(ti, tj))
        assert key not in new, "one pair twice in one step"
        old = prev.get(key)
        if old is None:
            st = [0.0, 0.0, 0.0, 0.0, 0.0]
        elif old[0] == ti:
            st = list(old[1])
        else:  # the pair was in the partner's row: orientation reversed
            stats["flips"] += 1
            st = [old[1][0], old[1][1], -old[1][2], -old[1][3], -old[1][4]]
        st = [st[0] + 1.0, st[1] + float(overlap[e]), st[2] + float(dx[e]),
              st[3] + float(dy[e]), st[4] + float(dz[e])]
        new[key] = (ti, st)
    return new


def test_contact_history_matches_host_history(ctx, slots_lib):
    w = W.poly("slots-contacts", 23, 2500, 0.55, 2e-3, 80, harmonic_k=1e3, shear_rate=2.0)
    w.vel *= 3.0  # atoms cross cells, so pairs change rows
    w.cfg.sort_every = 7
    w.cfg.newton = 1
    s = _system(ctx, w, 32, 5, True)
    import torch
    ov = torch.zeros(1, dtype=torch.int32, device="cuda")
    user = HistoryUser(w.harmonic_k, ov.data_ptr())
    s.set_force_hook_ptr(C.cast(slots_lib.contact_history_hook, C.c_void_p).value,
                         C.cast(C.pointer(user), C.c_void_p))
    o = oracle.from_workload(w)
    hist, stats = {}, {"flips": 0}
    for _ in range(w.steps):
        s.step(1)
        o.step(1)
        hist = _oracle_contacts(o, hist, stats)
    torch.cuda.synchronize()
    assert int(ov.item()) == 0, "a row had more contacts than slots"
    assert_same_state(s, o, "slots consumer")  # the hook's forces are the reference's
    assert s.counts().rebuilds > 3 and s.counts().sorts > 3
    assert stats["flips"] > 0, "no pair changed rows: the test lost its point"
    tags, vals = s.slots()
    own = s.atoms(local_only=True)["tag"]
    got = {}
    for r, c in zip(*np.nonzero(tags != NONE)):
        got[(int(own[r]), int(tags[r, c]))] = vals[r, c]
    want = {(v[0], k[0] if v[0] == k[1] else k[1]): np.array(v[1]) for k, v in hist.items()}
    assert set(got) == set(want)
    for key, v in want.items():
        np.testing.assert_array_equal(got[key].view(np.uint64), v.view(np.uint64),
                                      err_msg=f"contact {key}")
    assert max(v[0] for v in want.values()) > 10  # histories that outlived rebuilds
    s.close()


def test_slot_api_errors(ctx):
    w = W.config4_box(1, nmin=256, nmax=600, steps=5)
    s = system.from_workload(ctx, w)
    with pytest.raises(abi.SoilError):
        s.slots()  # not enabled
    with pytest.raises(abi.SoilError):
        s.enable_slots(0, 3)
    with pytest.raises(abi.SoilError):
        s.enable_slots(8, 65)
    s.enable_slots(8, 3)
    with pytest.raises(abi.SoilError):
        s.enable_slots(8, 3)  # twice
    b = system.Batch(ctx)
    with pytest.raises(abi.SoilError):
        b.add(s)  # batched systems have no slots
    tags, vals = s.slots()  # no hook ran: still all empty
    assert np.all(tags == NONE) and np.all(vals == 0.0)
    b.close()
    s.close()
