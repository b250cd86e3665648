"""The restart wire format (RestartData under bincode 1's default encoding,
soil_print/src/lib.rs:318-418, 1390-1445) restated in soil_b200.restart: the
byte layout of a hand-built two-atom state, round trips, and refusal of
malformed data."""
import struct

import numpy as np
import pytest

from soil_b200 import restart


def tiny():
    return {"natoms": 2, "total_cycle": 7, "dt": 1e-3,
            "tag": np.array([5, 9], np.uint32), "atom_type": np.array([0, 1], np.uint32),
            "pos": np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]]),
            "vel": np.array([[0.5, -0.5, 0.0], [0.0, 0.25, -1.0]]),
            "force": np.zeros((2, 3)), "mass": np.array([1.0, 2.0]),
            "cutoff_radius": np.array([0.55, 0.6]),
            "atom_data_buffers": [np.array([0.5, 0.55])]}


def test_byte_layout_of_a_two_atom_state():
    b = restart.encode(tiny())
    want = struct.pack("<QQd", 2, 7, 1e-3)
    want += struct.pack("<QII", 2, 5, 9) + struct.pack("<QII", 2, 0, 1)
    cols = [(1.0, 4.0), (2.0, 5.0), (3.0, 6.0), (0.5, 0.0), (-0.5, 0.25), (0.0, -1.0),
            (0.0, 0.0), (0.0, 0.0), (0.0, 0.0), (1.0, 2.0), (0.55, 0.6)]
    for c in cols:  # pos_x .. cutoff_radius: x/y/z split into separate vectors
        want += struct.pack("<Qdd", 2, *c)
    want += struct.pack("<Q", 1) + struct.pack("<Qdd", 2, 0.5, 0.55)  # atom_data_buffers
    want += struct.pack("<Q", 0) * 9 + struct.pack("<Q", 0)  # legacy vectors, quaternion
    assert b == want
    assert len(b) == 8 * 3 + 2 * (8 + 8) + 11 * (8 + 16) + 8 + (8 + 16) + 80


def test_round_trip():
    d = tiny()
    e = restart.decode(restart.encode(d))
    for k in ("natoms", "total_cycle", "dt"):
        assert e[k] == d[k]
    for k in ("tag", "atom_type", "pos", "vel", "force", "mass", "cutoff_radius"):
        np.testing.assert_array_equal(e[k], d[k])
    np.testing.assert_array_equal(e["atom_data_buffers"][0], d["atom_data_buffers"][0])
    assert e["quaternion"].shape == (0, 4)


@pytest.mark.parametrize("cut", [1, 20, 100])
def test_truncated_data_is_refused(cut):
    b = restart.encode(tiny())
    with pytest.raises(ValueError):
        restart.decode(b[:-cut])


def test_reference_file_names():
    assert restart.filename(1500) == "restart_1500_rank0.bin"
    assert restart.filename(3, rank=2, fmt="json") == "restart_3_rank2.json"
