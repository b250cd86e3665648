"""Python binding of the soil_b200 C ABI (include/soil_cuda.h).

``Context`` owns a CUDA device handle and an optional HBM budget; ``System``
is one periodic simulation (the reference's Atom + Domain + Neighbor +
CommTopology resources) whose every phase runs in libsoil_cuda.so.  There is
no CPU path: a missing library or device raises.
"""
import ctypes as C

import numpy as np

from . import abi


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


class Context:
    def __init__(self, device=0, hbm_budget_bytes=0):
        self.lib = abi.load_library()
        self.device = device
        h = C.c_void_p()
        st = self.lib.soil_ctx_create(device, hbm_budget_bytes, C.byref(h))
        if st != abi.SOIL_OK:
            raise abi.SoilError(st, "soil_ctx_create", f"(device {device})")
        self.h = h

    def error(self):
        return self.lib.soil_last_error(self.h).decode(errors="replace")

    def check(self, st, where):
        if st != abi.SOIL_OK:
            raise abi.SoilError(st, where, self.error())

    def bytes_in_use(self):
        v = C.c_uint64()
        self.check(self.lib.soil_ctx_bytes_in_use(self.h, C.byref(v)), "bytes_in_use")
        return v.value

    def alloc_count(self):
        """(device allocations, frees) made through this context so far."""
        a, f = C.c_uint64(), C.c_uint64()
        self.check(self.lib.soil_ctx_alloc_count(self.h, C.byref(a), C.byref(f)), "alloc_count")
        return a.value, f.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.soil_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


class System:
    """One simulation on the GPU; mirrors oracle.OracleSystem method by method."""

    def __init__(self, ctx, box, cfg, dt):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        ctx.check(self.lib.soil_sys_create(ctx.h, C.byref(box), C.byref(cfg), dt, C.byref(h)),
                  "soil_sys_create")
        self.h = h
        self.columns = []
        self._hook = None

    def close(self):
        if getattr(self, "h", None):
            self.lib.soil_sys_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _c(self, st, where):
        self.ctx.check(st, where)

    def register_column(self, name, width, flags):
        c = C.c_int32()
        self._c(self.lib.soil_sys_register_column(self.h, name.encode(), width, flags, C.byref(c)),
                "register_column")
        self.columns.append((name, width, flags))
        return c.value

    def add_atoms(self, tag, pos, vel, mass, cutoff, columns=None, atom_type=None):
        n = len(tag)
        tag = np.ascontiguousarray(tag, dtype=np.uint32)
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(n, 3)
        vel = np.ascontiguousarray(vel, dtype=np.float64).reshape(n, 3)
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        cutoff = np.ascontiguousarray(cutoff, dtype=np.float64)
        ty = np.ascontiguousarray(atom_type, dtype=np.uint32) if atom_type is not None else None
        keep = []
        arr = None
        if self.columns:
            arr = (C.POINTER(C.c_double) * len(self.columns))()
            for c in range(len(self.columns)):
                if columns is not None and columns[c] is not None:
                    a = np.ascontiguousarray(columns[c], dtype=np.float64)
                    keep.append(a)
                    arr[c] = _p(a, C.c_double)
        self._c(self.lib.soil_sys_add_atoms(self.h, n, _p(tag, C.c_uint32), _p(ty, C.c_uint32),
                                            _p(pos, C.c_double), _p(vel, C.c_double),
                                            _p(mass, C.c_double), _p(cutoff, C.c_double), arr),
                "add_atoms")

    def setup(self):
        self._c(self.lib.soil_sys_setup(self.h), "setup")

    def set_shear(self, rate):
        self._c(self.lib.soil_sys_set_shear(self.h, rate), "set_shear")

    def set_harmonic(self, k, radius_col):
        self._c(self.lib.soil_sys_set_harmonic(self.h, k, radius_col), "set_harmonic")

    def set_deform(self, dim, style, a=0.0, b=0.0, stage_steps=0):
        """Orthogonal deform of axis `dim` (abi.SOIL_DEFORM_*), before setup."""
        self._c(self.lib.soil_sys_set_deform(self.h, dim, style, a, b, stage_steps), "set_deform")

    def set_boundary(self, types, shrink_padding=0.0):
        """Boundary type per axis (abi.SOIL_BOUNDARY_*), before setup."""
        t = (C.c_int32 * 3)(*types)
        self._c(self.lib.soil_sys_set_boundary(self.h, t, shrink_padding), "set_boundary")

    def set_deform_remap(self, remap):
        self._c(self.lib.soil_sys_set_deform_remap(self.h, 1 if remap else 0), "set_deform_remap")

    def box(self):
        """(lo[3], hi[3], tilt[3]) of the domain as it stands."""
        lo, hi, tilt = np.zeros(3), np.zeros(3), np.zeros(3)
        self._c(self.lib.soil_sys_get_box(self.h, _p(lo, C.c_double), _p(hi, C.c_double),
                                          _p(tilt, C.c_double)), "get_box")
        return lo, hi, tilt

    def set_force_hook(self, fn, user=None):
        """fn(view: SoilDevView, user) -> int, called once per step."""
        if fn is None:
            self._hook = None
            self._c(self.lib.soil_sys_set_force_hook(self.h, abi.SOIL_FORCE_FN(), None), "hook")
            return
        cb = abi.SOIL_FORCE_FN(lambda v, u: fn(v.contents, user))
        self._hook = cb
        self._c(self.lib.soil_sys_set_force_hook(self.h, cb, None), "hook")

    def set_force_hook_ptr(self, fn_addr, user_addr=None):
        """Install a native hook by address (a soil_force_fn exported by a
        shared library); user_addr is passed through to it."""
        cb = abi.SOIL_FORCE_FN(fn_addr)
        self._hook = cb
        self._c(self.lib.soil_sys_set_force_hook(self.h, cb, user_addr), "hook")

    def step(self, n=1):
        self._c(self.lib.soil_step(self.h, n), "soil_step")

    def sync(self):
        self._c(self.lib.soil_sys_sync(self.h), "sync")

    def stream(self):
        v = C.c_void_p()
        self._c(self.lib.soil_sys_stream(self.h, C.byref(v)), "stream")
        return v.value

    def phase(self, name):
        self._c(getattr(self.lib, "soil_phase_" + name)(self.h), "phase " + name)

    def counts(self):
        c = abi.SoilCounts()
        self._c(self.lib.soil_sys_counts(self.h, C.byref(c)), "counts")
        return c

    def atoms(self, first=0, n=None, local_only=False):
        c = self.counts()
        total = c.nlocal + (0 if local_only else c.nghost)
        if n is None:
            n = total - first
        tag = np.zeros(n, np.uint32)
        pos = np.zeros((n, 3))
        vel = np.zeros((n, 3))
        force = np.zeros((n, 3))
        image = np.zeros((n, 3), np.int32)
        origin = np.zeros(n, np.int32)
        self._c(self.lib.soil_sys_get_atoms(self.h, first, n, _p(tag, C.c_uint32),
                                            _p(pos, C.c_double), _p(vel, C.c_double),
                                            _p(force, C.c_double), _p(image, C.c_int32),
                                            _p(origin, C.c_int32)), "get_atoms")
        return dict(tag=tag, pos=pos, vel=vel, force=force, image=image, origin=origin)

    def column(self, col, first=0, n=None):
        c = self.counts()
        total = c.nlocal + c.nghost
        if n is None:
            n = total - first
        w = self.columns[col][1]
        out = np.zeros(n * w)
        self._c(self.lib.soil_sys_get_column(self.h, col, first, n, _p(out, C.c_double)), "column")
        return out.reshape(n, w)

    def neighbor(self):
        c = self.counts()
        off = np.zeros(c.nlocal + 1, np.uint32)
        idx = np.zeros(c.npairs, np.uint32)
        self._c(self.lib.soil_sys_get_neighbor(self.h, _p(off, C.c_uint32), _p(idx, C.c_uint32)),
                "neighbor")
        return off, idx

    def swaps(self):
        n = C.c_int32()
        self._c(self.lib.soil_sys_num_swaps(self.h, C.byref(n)), "num_swaps")
        out = []
        for s in range(n.value):
            rs, rc = C.c_uint64(), C.c_uint64()
            off = np.zeros(3)
            voff = np.zeros(3)
            self._c(self.lib.soil_sys_get_swap(self.h, s, C.byref(rs), C.byref(rc),
                                               _p(off, C.c_double), _p(voff, C.c_double), None),
                    "get_swap")
            ns = C.c_uint64()
            self._c(self.lib.soil_sys_get_swap_sends(self.h, s, C.byref(ns)), "get_swap_sends")
            send = np.zeros(ns.value, np.uint32)
            self._c(self.lib.soil_sys_get_swap(self.h, s, None, None, None, None,
                                               _p(send, C.c_uint32)), "get_swap")
            out.append(dict(recv_start=rs.value, recv_count=rc.value, offset=off,
                            vel_offset=voff, send=send))
        return out

    def sort_perm(self):
        n = self.counts().nlocal
        perm = np.zeros(n, np.uint32)
        self._c(self.lib.soil_sys_get_sort_perm(self.h, _p(perm, C.c_uint32)), "sort_perm")
        return perm

    def read_local_state(self, pos_out, vel_out):
        """Positions and velocities of the locals into caller arrays ([n][3] f64,
        pinned or pageable), without other copies."""
        n = self.counts().nlocal
        assert pos_out.shape == (n, 3) and vel_out.shape == (n, 3)
        self._c(self.lib.soil_sys_get_atoms(self.h, 0, n, None, _p(pos_out, C.c_double),
                                            _p(vel_out, C.c_double), None, None, None),
                "get_atoms")

    def set_timing(self, mask):
        self._c(self.lib.soil_sys_set_timing(self.h, mask), "set_timing")

    def get_timing(self):
        ms = np.zeros(abi.SOIL_NUM_TIMERS)
        la = np.zeros(abi.SOIL_NUM_TIMERS, np.uint64)
        iv = np.zeros(abi.SOIL_NUM_TIMERS, np.uint64)
        self._c(self.lib.soil_sys_get_timing(self.h, _p(ms, C.c_double), _p(la, C.c_uint64),
                                             _p(iv, C.c_uint64)), "get_timing")
        return ms, la, iv

    def save_restart(self, total_cycle=None):
        """The reference's restart bytes (soil_sys_save_restart); total_cycle
        defaults to the steps taken."""
        cyc = self.counts().step if total_cycle is None else total_cycle
        n = C.c_uint64()
        self._c(self.lib.soil_sys_save_restart(self.h, cyc, None, 0, C.byref(n)), "save_restart")
        buf = (C.c_uint8 * n.value)()
        self._c(self.lib.soil_sys_save_restart(self.h, cyc, buf, n.value, C.byref(n)), "save_restart")
        return bytes(buf)

    def load_restart(self, data):
        """Load restart bytes into this (empty, columns registered) system; returns
        the step count stored in them."""
        buf = (C.c_uint8 * len(data)).from_buffer_copy(data)
        cyc = C.c_uint64()
        self._c(self.lib.soil_sys_load_restart(self.h, buf, len(data), C.byref(cyc)), "load_restart")
        return cyc.value

    def view(self):
        v = abi.SoilDevView()
        self._c(self.lib.soil_sys_view(self.h, C.byref(v)), "view")
        return v

    def enable_slots(self, max_contacts, width):
        """Persistent per-neighbor slots for a force hook (soil_sys_enable_slots)."""
        self._c(self.lib.soil_sys_enable_slots(self.h, max_contacts, width), "enable_slots")
        self._slots = (max_contacts, width)

    def slots(self):
        """(partner tags [nlocal, max], payload [nlocal, max, width]) written by
        the last hook call, rows in the current local order; empty slots have
        tag 0xFFFFFFFF."""
        m, w = getattr(self, "_slots", (1, 1))
        n = self.counts().nlocal
        tags = np.empty((n, m), np.uint32)
        vals = np.empty((n, m, w))
        self._c(self.lib.soil_sys_get_slots(self.h, _p(tags, C.c_uint32), _p(vals, C.c_double)),
                "get_slots")
        return tags, vals


class Batch:
    """Many set-up systems stepped together (soil_batch_*): one launch per phase
    over every member, each member bit-identical to stepping it alone."""

    def __init__(self, ctx):
        self.ctx = ctx
        self.lib = ctx.lib
        h = C.c_void_p()
        ctx.check(self.lib.soil_batch_create(ctx.h, C.byref(h)), "soil_batch_create")
        self.h = h
        self.members = []

    def close(self):
        if getattr(self, "h", None):
            self.lib.soil_batch_destroy(self.h)
            self.h = None
            self.members = []

    def __del__(self):
        self.close()

    def add(self, system):
        self.ctx.check(self.lib.soil_batch_add(self.h, system.h), "soil_batch_add")
        self.members.append(system)

    def remove(self, system):
        self.ctx.check(self.lib.soil_batch_remove(self.h, system.h), "soil_batch_remove")
        self.members.remove(system)

    def __len__(self):
        n = C.c_uint32()
        self.ctx.check(self.lib.soil_batch_size(self.h, C.byref(n)), "soil_batch_size")
        return n.value

    def step(self, n=1):
        self.ctx.check(self.lib.soil_batch_step(self.h, n), "soil_batch_step")

    def sync(self):
        self.ctx.check(self.lib.soil_batch_sync(self.h), "soil_batch_sync")

    def stream(self):
        v = C.c_void_p()
        self.ctx.check(self.lib.soil_batch_stream(self.h, C.byref(v)), "soil_batch_stream")
        return v.value

    def set_timing(self, on=True):
        self.ctx.check(self.lib.soil_batch_set_timing(self.h, 1 if on else 0), "batch timing")

    def get_timing(self):
        """{stage: (ms, intervals)} summed since set_timing."""
        ms = np.zeros(abi.SOIL_BATCH_NUM_TIMERS)
        iv = np.zeros(abi.SOIL_BATCH_NUM_TIMERS, np.uint64)
        self.ctx.check(self.lib.soil_batch_get_timing(self.h, _p(ms, C.c_double),
                                                      _p(iv, C.c_uint64)), "batch timing")
        return {n: (float(ms[k]), int(iv[k])) for k, n in enumerate(abi.BATCH_TIMER_NAMES)}

    def get_host_timing(self):
        """{section: host ms} of step planning since set_timing."""
        ms = np.zeros(len(abi.BATCH_HOST_TIMER_NAMES))
        self.ctx.check(self.lib.soil_batch_get_host_timing(self.h, _p(ms, C.c_double)),
                       "batch host timing")
        return {n: float(ms[k]) for k, n in enumerate(abi.BATCH_HOST_TIMER_NAMES)}

    def stats(self):
        st, w, b, r = C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.ctx.check(self.lib.soil_batch_stats(self.h, C.byref(st), C.byref(w), C.byref(b),
                                                 C.byref(r)), "soil_batch_stats")
        return dict(steps=st.value, host_waits=w.value, device_bytes=b.value,
                    border_retries=r.value)


def from_workload(ctx, w):
    """GPU system for a workloads.Workload (radius registered as column 0)."""
    s = System(ctx, w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    if w.harmonic_k:
        s.set_harmonic(w.harmonic_k, rc)
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    s.setup()
    return s


def pairs(offsets, indices, nlocal):
    """Neighbor::pairs(nlocal) (neighbor.rs:224-242): every (i, j) of the CSR
    half list, rows ascending, CSR order inside a row."""
    for i in range(nlocal):
        for k in range(int(offsets[i]), int(offsets[i + 1])):
            yield i, int(indices[k])


def classify_boundary_atoms(offsets, indices, nlocal):
    """classify_boundary_atoms (neighbor.rs:1327-1336): True for a local atom
    with at least one ghost neighbour (index >= nlocal)."""
    out = np.zeros(nlocal, dtype=bool)
    for i in range(nlocal):
        row = indices[int(offsets[i]):int(offsets[i + 1])]
        out[i] = bool(np.any(row >= nlocal))
    return out
