"""The reference's restart wire format in Python (RestartData,
soil_print/src/lib.rs:318-418, serialised by write_restart with bincode 1,
soil_print/src/lib.rs:1390-1445).

bincode 1's default encoding: fields in declaration order, little endian,
fixed-width integers (usize as u64), a u64 length before every Vec, fixed
arrays without one.  ``encode``/``decode`` restate that layout for the
fields the substrate owns; the library's soil_sys_save_restart writes the
same bytes from device state.  ``filename`` gives write_restart's naming.
"""
import struct

import numpy as np

_VEC_F64 = ("pos_x", "pos_y", "pos_z", "vel_x", "vel_y", "vel_z", "force_x", "force_y",
            "force_z", "mass", "cutoff_radius")
_LEGACY = ("omega_x", "omega_y", "omega_z", "torque_x", "torque_y", "torque_z",
           "ang_mom_x", "ang_mom_y", "ang_mom_z")


def filename(step, rank=0, fmt="bin"):
    """restart_{step}_rank{rank}.{bin|json} (soil_print/src/lib.rs:1434-1440)."""
    return f"restart_{step}_rank{rank}.{'json' if fmt == 'json' else 'bin'}"


def encode(d):
    """Bytes of a RestartData given as a dict: natoms, total_cycle, dt, tag,
    atom_type, pos/vel/force as [n][3], mass, cutoff_radius and
    atom_data_buffers (list of flat f64 arrays); legacy fields empty."""
    n = len(d["tag"])
    out = [struct.pack("<QQd", d["natoms"], d["total_cycle"], d["dt"])]

    def vec(a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        out.append(struct.pack("<Q", a.size))
        out.append(a.astype(np.dtype(dtype).newbyteorder("<"), copy=False).tobytes())

    vec(d["tag"], np.uint32)
    vec(d.get("atom_type", np.zeros(n, np.uint32)), np.uint32)
    cols = {}
    for k, name in enumerate(("pos", "vel", "force")):
        a = np.asarray(d[name], dtype=np.float64).reshape(n, 3)
        for c in range(3):
            cols[f"{name}_{'xyz'[c]}"] = a[:, c]
    cols["mass"] = d["mass"]
    cols["cutoff_radius"] = d["cutoff_radius"]
    for name in _VEC_F64:
        vec(cols[name], np.float64)
    bufs = d.get("atom_data_buffers", [])
    out.append(struct.pack("<Q", len(bufs)))
    for b in bufs:
        vec(b, np.float64)
    for _ in _LEGACY:
        out.append(struct.pack("<Q", 0))
    out.append(struct.pack("<Q", 0))  # quaternion: Vec<[f64; 4]>
    return b"".join(out)


def decode(b):
    """Inverse of encode; raises ValueError on truncated or malformed data."""
    at = 0

    def take(n):
        nonlocal at
        if n < 0 or at + n > len(b):
            raise ValueError("restart data is truncated")
        v = b[at:at + n]
        at += n
        return v

    def u64():
        return struct.unpack("<Q", take(8))[0]

    def vec(dtype, width=1):
        n = u64()
        size = np.dtype(dtype).itemsize * width
        if n > (len(b) - at) // max(size, 1):
            raise ValueError("restart vector longer than the data")
        return np.frombuffer(take(n * size), dtype=np.dtype(dtype).newbyteorder("<")).astype(dtype)

    natoms, total_cycle = u64(), u64()
    dt = struct.unpack("<d", take(8))[0]
    d = {"natoms": natoms, "total_cycle": total_cycle, "dt": dt,
         "tag": vec(np.uint32), "atom_type": vec(np.uint32)}
    cols = {name: vec(np.float64) for name in _VEC_F64}
    for name in ("pos", "vel", "force"):
        d[name] = np.stack([cols[f"{name}_{c}"] for c in "xyz"], axis=1)
    d["mass"] = cols["mass"]
    d["cutoff_radius"] = cols["cutoff_radius"]
    d["atom_data_buffers"] = [vec(np.float64) for _ in range(u64())]
    for name in _LEGACY:
        d[name] = vec(np.float64)
    d["quaternion"] = vec(np.float64, 4).reshape(-1, 4)
    if at != len(b):
        raise ValueError("trailing bytes after RestartData")
    return d
