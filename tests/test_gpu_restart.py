"""Restart checkpoints in the reference's wire format (soil_sys_save_restart /
soil_sys_load_restart): the bytes a GPU system writes equal the format
restated in soil_b200.restart applied to the oracle's state after the same
steps, and a run continued from a restart matches the oracle continued from
the same restart, bit for bit."""
import numpy as np
import pytest

import oracle
from helpers import assert_same_lists, assert_same_state
from soil_b200 import abi, restart, system, workloads as W

pytestmark = pytest.mark.gpu


def oracle_restart(o, w, cycle):
    """RestartData of an oracle system: its locals in current order."""
    a = o.atoms(local_only=True)
    by_tag = {int(t): k for k, t in enumerate(w.tag)}
    idx = np.array([by_tag[int(t)] for t in a["tag"]])
    n = len(idx)
    return restart.encode({
        "natoms": n, "total_cycle": cycle, "dt": w.dt, "tag": a["tag"],
        "atom_type": np.zeros(n, np.uint32), "pos": a["pos"], "vel": a["vel"],
        "force": a["force"], "mass": np.asarray(w.mass)[idx],
        "cutoff_radius": np.asarray(w.cutoff)[idx],
        "atom_data_buffers": [o.column(0)[:n].reshape(-1)]})


def gpu_from_restart(ctx, w, data):
    s = system.System(ctx, w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    cyc = s.load_restart(data)
    s.set_harmonic(w.harmonic_k, rc)
    s.setup()
    return s, cyc


def oracle_from_restart(w, data):
    d = restart.decode(data)
    o = oracle.OracleSystem(w.box, w.cfg, d["dt"])
    rc = o.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    o.add_atoms(d["tag"], d["pos"], d["vel"], d["mass"], d["cutoff_radius"],
                columns=[d["atom_data_buffers"][0]], atom_type=d["atom_type"])
    for i in range(len(d["tag"])):
        o.set_atom_state(i, force=d["force"][i])
    o.set_harmonic(w.harmonic_k, rc)
    o.setup()
    return o


@pytest.mark.parametrize("filt", [abi.SOIL_FILTER_FP64, abi.SOIL_FILTER_FP32_RECHECK])
def test_restart_bytes_and_continuation(ctx, filt):
    w = W.poly("restart", 21, 3000, 0.5, 1e-4, 60, harmonic_k=1e3, filter=filt)
    g = system.from_workload(ctx, w)
    o = oracle.from_workload(w)
    g.step(30)
    o.step(30)
    data = g.save_restart()
    assert data == oracle_restart(o, w, 30)
    d = restart.decode(data)
    assert d["total_cycle"] == 30 and d["natoms"] == 3000 and d["dt"] == w.dt

    g2, cyc = gpu_from_restart(ctx, w, data)
    assert cyc == 30 and g2.counts().step == 30
    o2 = oracle_from_restart(w, data)
    g2.step(30)
    o2.step(30)
    assert g2.counts().step == 60  # the oracle does not read the step count
    assert_same_state(g2, o2, "continued from restart", skip=("step",))
    assert_same_lists(g2, o2, "continued from restart")
    # a restart of the continued run round-trips through the format
    assert restart.encode(restart.decode(g2.save_restart())) == g2.save_restart()


def test_malformed_restart_is_refused(ctx):
    w = W.poly("restart-bad", 22, 500, 0.5, 1e-4, 5, harmonic_k=1e3)
    g = system.from_workload(ctx, w)
    g.step(2)
    data = g.save_restart()
    s = system.System(ctx, w.box, w.cfg, w.dt)
    s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    with pytest.raises(abi.SoilError):
        s.load_restart(data[:-50])  # truncated
    t = system.System(ctx, w.box, w.cfg, w.dt)  # no radius column registered
    with pytest.raises(abi.SoilError):
        t.load_restart(data)
