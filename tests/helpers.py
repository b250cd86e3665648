"""Shared helpers of the parity tests: build the same system on the GPU and
in the CPU oracle from one seeded workload, and compare every observable."""
import ctypes as C
import os
import subprocess

import numpy as np

import oracle
from soil_b200 import abi, system, workloads

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def build_hook(out_dir, name):
    """Compile tests/hooks/<name>.cu (a consumer built apart from the library,
    against include/ only) into out_dir and load it."""
    out = os.path.join(str(out_dir), f"lib{name}.so")
    subprocess.check_call(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-O3", "-fmad=false", "-shared", "-Xcompiler", "-fPIC",
                           "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "hooks", f"{name}.cu"), "-o", out])
    return C.CDLL(out)


class RegistryProbe(C.Structure):
    """User data of tests/hooks/registry_hook.cu."""
    _fields_ = [("K", C.c_double), ("rev", C.c_int32), ("zero", C.c_int32), ("fwd", C.c_int32)]


def attach_registry_hook(lib, K):
    """attach(system, probe) for tests/golden/cases.build on the GPU: installs
    registry_hook (harmonic forces in the reference order + column writes)."""
    def attach(s, probe):
        u = RegistryProbe(K, probe["rev_col"], probe["zero_col"], probe["fwd_col"])
        s._probe = u  # lives as long as the system
        s.set_force_hook_ptr(C.cast(lib.registry_hook, C.c_void_p).value,
                             C.cast(C.pointer(u), C.c_void_p))
    return attach


def attach_oracle_probe(s, probe):
    s.set_column_probe(**probe)


def pair(ctx, w):
    return system.from_workload(ctx, w), oracle.from_workload(w)


def assert_same_state(g, o, what="", skip=()):
    cg, co = g.counts(), o.counts()
    for k in ("nlocal", "nghost", "npairs", "step", "rebuilds", "comm_state", "triclinic",
              "steps_since_build"):
        if k in skip:
            continue
        assert getattr(cg, k) == getattr(co, k), f"{what} counts.{k}: {getattr(cg, k)} != {getattr(co, k)}"
    assert list(cg.bin_count) == list(co.bin_count), what
    assert cg.tilt_xy == co.tilt_xy, what
    ag, ao = g.atoms(), o.atoms()
    for k in ("tag", "image", "origin"):
        np.testing.assert_array_equal(ag[k], ao[k], err_msg=f"{what} {k}")
    for k in ("pos", "vel", "force"):
        # bit-exact: compare the IEEE bit patterns
        bg, bo = ag[k].view(np.uint64), ao[k].view(np.uint64)
        bad = np.nonzero(bg != bo)
        if len(bad[0]):
            i = bad[0][0]
            raise AssertionError(f"{what} {k} differs at {len(bad[0])} entries; first atom {i}: "
                                 f"gpu {ag[k][i]} oracle {ao[k][i]}")
    for c in range(len(g.columns)):
        np.testing.assert_array_equal(g.column(c).view(np.uint64), o.column(c).view(np.uint64),
                                      err_msg=f"{what} column {c}")


def assert_same_lists(g, o, what=""):
    og, ig = g.neighbor()
    oo, io = o.neighbor()
    np.testing.assert_array_equal(og, oo, err_msg=f"{what} neighbor_offsets")
    np.testing.assert_array_equal(ig, io, err_msg=f"{what} neighbor_indices")
    sg, so = g.swaps(), o.swaps()
    assert len(sg) == len(so)
    for k, (a, b) in enumerate(zip(sg, so)):
        assert a["recv_start"] == b["recv_start"] and a["recv_count"] == b["recv_count"], (what, k)
        np.testing.assert_array_equal(a["send"], b["send"], err_msg=f"{what} swap {k} send")
        np.testing.assert_array_equal(a["offset"].view(np.uint64), b["offset"].view(np.uint64))
        np.testing.assert_array_equal(a["vel_offset"].view(np.uint64), b["vel_offset"].view(np.uint64))
