"""The device force-hook ABI (soil_sys_set_force_hook, soil_dev_view): an
external consumer compiled apart from the library (tests/hooks) runs inside
soil_step on the view's device pointers; ghost forces it leaves are folded by
reverse comm, and the integration uses its forces.  Its atomic summation
order differs from the reference's, so forces are compared within 1e-12
relative to the built-in (bit-exact) consumer after one step."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from soil_b200 import abi, system, workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _build(tmp_path_factory, name):
    out = tmp_path_factory.mktemp("hook") / f"lib{name}.so"
    subprocess.check_call(["/usr/local/cuda/bin/nvcc", "-gencode", "arch=compute_100a,code=sm_100a",
                           "-O3", "-fmad=false", "-shared", "-Xcompiler", "-fPIC",
                           "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "hooks", f"{name}.cu"), "-o", str(out)])
    return C.CDLL(str(out))


@pytest.fixture(scope="module")
def hook_lib(tmp_path_factory):
    return _build(tmp_path_factory, "harmonic_hook")


@pytest.fixture(scope="module")
def gather_lib(tmp_path_factory):
    return _build(tmp_path_factory, "gather_hook")


def _with_hook(ctx, w, lib, name, k):
    s = system.System(ctx, w.box, w.cfg, w.dt)
    rc = s.register_column("radius", 1, abi.SOIL_COL_FORWARD)
    s.add_atoms(w.tag, w.pos, w.vel, w.mass, w.cutoff, columns=[w.radius])
    if w.shear_rate:
        s.set_shear(w.shear_rate)
    s.setup()
    kbox = C.c_double(k)
    s._kbox = kbox  # lives as long as the system
    s.set_force_hook_ptr(C.cast(getattr(lib, name), C.c_void_p).value,
                         C.cast(C.pointer(kbox), C.c_void_p))
    assert rc == 0
    return s


@pytest.mark.parametrize("shear", [0.0, 2.0])
def test_hook_forces_match_builtin(ctx, hook_lib, shear):
    w = W.poly("hook", 13, 5000, 0.5, 1e-4, 1, harmonic_k=1e3, shear_rate=shear)
    ref = system.from_workload(ctx, w)
    hk = _with_hook(ctx, w, hook_lib, "harmonic_hook", w.harmonic_k)
    ref.step(1)
    hk.step(1)
    a, b = ref.atoms(local_only=True), hk.atoms(local_only=True)
    np.testing.assert_array_equal(a["tag"], b["tag"])
    np.testing.assert_array_equal(a["pos"], b["pos"])  # first half-kick uses F = 0
    scale = np.abs(a["force"]).max()
    assert scale > 0
    np.testing.assert_allclose(b["force"], a["force"], rtol=0, atol=1e-12 * scale)
    np.testing.assert_allclose(b["vel"], a["vel"], rtol=1e-12, atol=1e-12)
    # the view the hook saw describes the same system
    v, c = hk.view(), hk.counts()
    assert (v.nlocal, v.nghost, v.npairs, v.ncolumns, v.newton) == \
        (c.nlocal, c.nghost, c.npairs, 1, 1)
    ref.close()
    hk.close()


def test_failing_hook_stops_the_step(ctx, hook_lib):
    w = W.poly("hookfail", 14, 2000, 0.5, 1e-4, 1, harmonic_k=1e3)
    s = _with_hook(ctx, w, hook_lib, "failing_hook", 1.0)
    with pytest.raises(abi.SoilError) as e:
        s.step(1)
    assert e.value.status == abi.SOIL_ERR_INVALID and "hook" in str(e.value)
    s.close()


@pytest.mark.parametrize("shear,newton", [(0.0, 1), (2.0, 1), (0.0, 0)])
def test_external_gather_consumer_is_bit_exact(ctx, gather_lib, shear, newton):
    """A consumer written against include/soil_consumer.cuh, outside the
    library, reproduces the built-in consumer's trajectory bit for bit."""
    from helpers import assert_same_lists, assert_same_state
    w = W.poly("gather", 15, 4000, 0.5, 1e-4, 40, harmonic_k=1e3, shear_rate=shear)
    w.cfg.newton = newton
    ref = system.from_workload(ctx, w)
    hk = _with_hook(ctx, w, gather_lib, "gather_harmonic_hook", w.harmonic_k)
    ref.step(20)
    hk.step(20)
    ref.step(20)
    hk.step(20)
    assert_same_state(hk, ref, "external gather consumer")
    assert_same_lists(hk, ref, "external gather consumer")
    assert np.any(hk.atoms()["force"] != 0.0)
    v = hk.view()
    assert v.in_start and v.in_list and v.origin and v.fold_start
    ref.close()
    hk.close()
