"""ctypes wrapper of the CPU oracle (oracle/build/libsoil_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "build", "libsoil_oracle.so")

from soil_b200 import abi  # struct layouts of include/soil_cuda.h

_lib = None


def build(force=False):
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    if force or not os.path.exists(LIB) or \
            os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "soil_oracle.cpp")):
        subprocess.check_call(["make", "-s", "-C", HERE])
    return LIB


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(LIB)
        P = C.c_void_p
        pu32, pi32, pdbl, pu64 = (C.POINTER(C.c_uint32), C.POINTER(C.c_int32),
                                  C.POINTER(C.c_double), C.POINTER(C.c_uint64))
        sig = {
            "orc_create": (P, [C.POINTER(abi.SoilBox), C.POINTER(abi.SoilNeighCfg), C.c_double]),
            "orc_destroy": (None, [P]),
            "orc_register_column": (C.c_int, [P, C.c_int32, C.c_uint32]),
            "orc_add_atoms": (C.c_int, [P, C.c_uint64, pu32, pu32, pdbl, pdbl, pdbl, pdbl,
                                        C.POINTER(pdbl)]),
            "orc_setup": (C.c_int, [P]),
            "orc_set_shear": (C.c_int, [P, C.c_double]),
            "orc_set_deform": (C.c_int, [P, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                         C.c_uint64]),
            "orc_set_deform_remap": (C.c_int, [P, C.c_int32]),
            "orc_set_boundary": (C.c_int, [P, C.POINTER(C.c_int32), C.c_double]),
            "orc_get_swap_sends": (C.c_int, [P, C.c_int32, C.POINTER(C.c_uint64)]),
            "orc_get_box": (C.c_int, [P, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                      C.POINTER(C.c_double)]),
            "orc_set_harmonic": (C.c_int, [P, C.c_double, C.c_int32]),
            "orc_set_column_probe": (C.c_int, [P, C.c_int32, C.c_int32, C.c_int32]),
            "orc_step": (C.c_int, [P, C.c_uint64]),
            "orc_phase": (C.c_int, [P, C.c_int]),
            "orc_counts": (C.c_int, [P, C.POINTER(abi.SoilCounts)]),
            "orc_get_atoms": (C.c_int, [P, C.c_uint64, C.c_uint64, pu32, pdbl, pdbl, pdbl, pi32, pi32]),
            "orc_get_column": (C.c_int, [P, C.c_int32, C.c_uint64, C.c_uint64, pdbl]),
            "orc_get_neighbor": (C.c_int, [P, pu32, pu32]),
            "orc_num_offsets": (C.c_int, [P]),
            "orc_num_swaps": (C.c_int, [P]),
            "orc_get_swap": (C.c_int, [P, C.c_int32, pu64, pu64, pdbl, pdbl, pu32]),
            "orc_get_sort_perm": (C.c_int, [P, pu32]),
            "orc_get_stencil": (C.c_int, [P, pi32, pi32, pdbl, pdbl]),
            "orc_get_stencil_full": (C.c_int, [P, pi32, pi32, pi32]),
            "orc_set_state": (C.c_int, [P, C.c_int]),
            "orc_set_domain_tilt": (C.c_int, [P, C.c_double, C.c_double, C.c_int]),
            "orc_set_atom_state": (C.c_int, [P, C.c_uint64, pdbl, pdbl, pdbl]),
            "orc_x2lamda": (C.c_int, [P, pdbl, pdbl]),
            "orc_lamda2x": (C.c_int, [P, pdbl, pdbl]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


PHASE_INDEX = {
    "deform": 0, "initial": 1, "decide_rebuild": 2, "remove_ghosts": 3, "zero_forces": 4,
    "pbc": 5, "sort": 6, "borders": 7, "forward_comm": 8, "neighbor": 9, "force": 10,
    "reverse_comm": 11, "final": 12, "shrink_wrap": 13,
}


class OracleSystem:
    """Same surface as soil_b200.System, computed on the CPU."""

    def __init__(self, box, cfg, dt):
        self._L = lib()
        self.h = self._L.orc_create(C.byref(box), C.byref(cfg), dt)
        self.columns = []

    def __del__(self):
        if getattr(self, "h", None):
            self._L.orc_destroy(self.h)
            self.h = None

    def register_column(self, name, width, flags):
        c = self._L.orc_register_column(self.h, width, flags)
        assert c >= 0
        self.columns.append((name, width, flags))
        return c

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
                else:
                    arr[c] = None
        st = self._L.orc_add_atoms(self.h, n, _p(tag, C.c_uint32), _p(ty, C.c_uint32),
                                   _p(pos, C.c_double), _p(vel, C.c_double), _p(mass, C.c_double),
                                   _p(cutoff, C.c_double), arr)
        assert st == 0, st

    def setup(self):
        assert self._L.orc_setup(self.h) == 0

    def set_shear(self, rate):
        self._L.orc_set_shear(self.h, rate)

    def set_harmonic(self, k, radius_col):
        self._L.orc_set_harmonic(self.h, k, radius_col)

    def set_column_probe(self, rev_col=-1, zero_col=-1, fwd_col=-1):
        """Test consumer writing registered columns in the Force phase (the
        oracle's counterpart of tests/hooks/registry_hook.cu)."""
        assert self._L.orc_set_column_probe(self.h, rev_col, zero_col, fwd_col) == 0

    def set_deform(self, dim, style, a=0.0, b=0.0, stage_steps=0):
        assert self._L.orc_set_deform(self.h, dim, style, a, b, stage_steps) == 0

    def set_boundary(self, types, padding=0.0):
        t = (C.c_int32 * 3)(*types)
        assert self._L.orc_set_boundary(self.h, t, padding) == 0

    def set_deform_remap(self, remap):
        self._L.orc_set_deform_remap(self.h, 1 if remap else 0)

    def box(self):
        lo, hi, tilt = np.zeros(3), np.zeros(3), np.zeros(3)
        self._L.orc_get_box(self.h, _p(lo, C.c_double), _p(hi, C.c_double), _p(tilt, C.c_double))
        return lo, hi, tilt

    def try_step(self, n=1):
        """Status of n steps (SOIL_ERR_INVALID when a deforming axis collapses)."""
        return self._L.orc_step(self.h, n)

    def step(self, n=1):
        assert self._L.orc_step(self.h, n) == 0

    def phase(self, name):
        assert self._L.orc_phase(self.h, PHASE_INDEX[name]) == 0

    def counts(self):
        c = abi.SoilCounts()
        self._L.orc_counts(self.h, C.byref(c))
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
        st = self._L.orc_get_atoms(self.h, first, n, _p(tag, C.c_uint32), _p(pos, C.c_double),
                                   _p(vel, C.c_double), _p(force, C.c_double),
                                   _p(image, C.c_int32), _p(origin, C.c_int32))
        assert st == 0
        return dict(tag=tag, pos=pos, vel=vel, force=force, image=image, origin=origin)

    def column(self, col, first=0, n=None):
        c = self.counts()
        total = c.nlocal + c.nghost
        if n is None:
            n = total - first
        w = self.columns[col][1]
        out = np.zeros(n * w)
        assert self._L.orc_get_column(self.h, col, first, n, _p(out, C.c_double)) == 0
        return out.reshape(n, w)

    def neighbor(self):
        c = self.counts()
        noff = self._L.orc_num_offsets(self.h)
        off = np.zeros(noff, np.uint32)
        idx = np.zeros(c.npairs, np.uint32)
        self._L.orc_get_neighbor(self.h, _p(off, C.c_uint32), _p(idx, C.c_uint32))
        return off, idx

    def swaps(self):
        out = []
        for s in range(self._L.orc_num_swaps(self.h)):
            rs, rc = C.c_uint64(), C.c_uint64()
            off = np.zeros(3)
            voff = np.zeros(3)
            self._L.orc_get_swap(self.h, s, C.byref(rs), C.byref(rc), _p(off, C.c_double),
                                 _p(voff, C.c_double), None)
            ns = C.c_uint64()
            self._L.orc_get_swap_sends(self.h, s, C.byref(ns))
            send = np.zeros(ns.value, np.uint32)
            self._L.orc_get_swap(self.h, s, None, None, None, None, _p(send, C.c_uint32))
            out.append(dict(recv_start=rs.value, recv_count=rc.value, offset=off,
                            vel_offset=voff, send=send))
        return out

    def sort_perm(self):
        n = self.counts().nlocal
        perm = np.zeros(n, np.uint32)
        k = self._L.orc_get_sort_perm(self.h, _p(perm, C.c_uint32))
        return perm[:k]

    def stencil(self):
        n = C.c_int32()
        self._L.orc_get_stencil(self.h, None, C.byref(n), None, None)
        fwd = np.zeros(n.value, np.int32)
        origin = np.zeros(3)
        bs = np.zeros(3)
        self._L.orc_get_stencil(self.h, _p(fwd, C.c_int32), C.byref(n), _p(origin, C.c_double),
                                _p(bs, C.c_double))
        return fwd, origin, bs

    def stencil_full(self):
        """(full stencil offsets, bin_stencil_self)"""
        n, hs = C.c_int32(), C.c_int32()
        self._L.orc_get_stencil_full(self.h, None, C.byref(n), C.byref(hs))
        full = np.zeros(n.value, np.int32)
        self._L.orc_get_stencil_full(self.h, _p(full, C.c_int32), C.byref(n), C.byref(hs))
        return full, bool(hs.value)

    # single-function access for known-answer tests
    def set_state(self, state):
        self._L.orc_set_state(self.h, state)

    def set_domain_tilt(self, xy, bvel_x, triclinic=True):
        self._L.orc_set_domain_tilt(self.h, xy, bvel_x, 1 if triclinic else 0)

    def set_atom_state(self, i, pos=None, vel=None, force=None):
        a = [np.ascontiguousarray(v, dtype=np.float64) if v is not None else None
             for v in (pos, vel, force)]
        self._L.orc_set_atom_state(self.h, i, *[_p(v, C.c_double) for v in a])

    def x2lamda(self, r):
        r = np.ascontiguousarray(r, dtype=np.float64)
        lam = np.zeros(3)
        self._L.orc_x2lamda(self.h, _p(r, C.c_double), _p(lam, C.c_double))
        return lam

    def lamda2x(self, lam):
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        r = np.zeros(3)
        self._L.orc_lamda2x(self.h, _p(lam, C.c_double), _p(r, C.c_double))
        return r


def from_workload(w, steps_override=None):
    """Oracle system for a soil_b200.workloads.Workload (radius as column 0)."""
    s = OracleSystem(w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    if w.harmonic_k:
        s.set_harmonic(w.harmonic_k, rc)
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    s.setup()
    return s
