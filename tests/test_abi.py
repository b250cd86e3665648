"""The C ABI library loads without a GPU and matches include/soil_cuda.h.

No compute entry point is called here; only symbol presence, the version
query, struct layouts and the no-device error path are checked.
"""
import ctypes as C
import os
import re
import subprocess

import pytest

from soil_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "soil_cuda.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(soil_\w+)\s*\(", text, flags=re.M)
    return sorted(set(n for n in names if not n.startswith("soil_force_fn")))


def test_library_exports_every_declared_symbol():
    lib = abi.load_library()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_prototype_table_matches_header():
    assert sorted(abi.PROTOTYPES) == declared_functions()


def test_abi_version():
    assert abi.load_library().soil_abi_version() == 1


def test_no_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    h = C.c_void_p()
    st = abi.load_library().soil_ctx_create(0, 0, C.byref(h))
    assert st == abi.SOIL_ERR_NO_DEVICE and not h.value


def test_struct_layouts_match_header(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text(r'''
#include <stdio.h>
#include <stddef.h>
#include "soil_cuda.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(soil_box), sizeof(soil_neigh_cfg), sizeof(soil_counts),
         sizeof(soil_dev_view));
  printf("%zu %zu %zu\n", offsetof(soil_neigh_cfg, additive_skin), offsetof(soil_counts, comm_state),
         offsetof(soil_counts, tilt_xy));
  printf("%zu %zu\n", offsetof(soil_dev_view, columns), offsetof(soil_dev_view, stream));
  printf("%zu %zu\n", offsetof(soil_dev_view, in_start), offsetof(soil_dev_view, fold_list));
  printf("%zu %zu %zu\n", offsetof(soil_dev_view, ghost_root), offsetof(soil_dev_view, slot_width),
         offsetof(soil_dev_view, slot_new_val));
  printf("%zu %zu %zu %zu\n", sizeof(soil_server_cfg), sizeof(soil_job_spec), sizeof(soil_job_info),
         sizeof(soil_server_stats));
  printf("%zu %zu %zu %zu\n", offsetof(soil_job_spec, natoms), offsetof(soil_job_spec, steps),
         offsetof(soil_job_info, t_done), offsetof(soil_server_stats, max_active));
  return 0;
}
''')
    exe = tmp_path / "layout"
    subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)])
    out = subprocess.check_output([str(exe)]).decode().split()
    got = [int(x) for x in out]
    want = [C.sizeof(abi.SoilBox), C.sizeof(abi.SoilNeighCfg), C.sizeof(abi.SoilCounts),
            C.sizeof(abi.SoilDevView),
            abi.SoilNeighCfg.additive_skin.offset, abi.SoilCounts.comm_state.offset,
            abi.SoilCounts.tilt_xy.offset,
            abi.SoilDevView.columns.offset, abi.SoilDevView.stream.offset,
            abi.SoilDevView.in_start.offset, abi.SoilDevView.fold_list.offset,
            abi.SoilDevView.ghost_root.offset, abi.SoilDevView.slot_width.offset,
            abi.SoilDevView.slot_new_val.offset,
            C.sizeof(abi.SoilServerCfg), C.sizeof(abi.SoilJobSpec), C.sizeof(abi.SoilJobInfo),
            C.sizeof(abi.SoilServerStats),
            abi.SoilJobSpec.natoms.offset, abi.SoilJobSpec.steps.offset,
            abi.SoilJobInfo.t_done.offset, abi.SoilServerStats.max_active.offset]
    assert got == want


def test_missing_library_raises(tmp_path):
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        abi.load_library(str(tmp_path / "nope.so"))


def test_consumer_headers_compile_for_sm100a(tmp_path):
    """include/soil_consumer.cuh and include/soil_slots.cuh are what an external
    force hook includes: they compile on their own (and together) for sm_100a,
    and so do the example hooks under tests/hooks."""
    src = tmp_path / "hook.cu"
    src.write_text(r'''
#include "soil_consumer.cuh"
#include "soil_slots.cuh"
__global__ void k(soil_dev_view v) {
    const soil_harmonic_pair pair{v.x, v.y, v.z, v.columns[0], 1.0};
    double F[3], s[4];
    soil_gather_force(v, threadIdx.x, pair, F);
    if (v.slot_max) {
        const int side = soil_slot_find(v, 0, 1, s);
        s[0] = F[0] + side;
        soil_slot_put(v, 0, 0, v.tag[1], s);
        soil_slot_clear_from(v, 0, 1);
    }
}
''')
    nvcc = "/usr/local/cuda/bin/nvcc"
    base = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O2", "-fmad=false",
            "-I", os.path.join(ROOT, "include"), "-c"]
    subprocess.check_call(base + [str(src), "-o", str(tmp_path / "hook.o")])
    for name in ("harmonic_hook", "gather_hook", "slots_hook"):
        subprocess.check_call(base + [os.path.join(ROOT, "tests", "hooks", f"{name}.cu"),
                                      "-o", str(tmp_path / f"{name}.o")])


@pytest.mark.parametrize("counts", [
    (1 << 22, 1 << 21, 1 << 21),   # 64-bit product is exactly 2**64 (wraps to 0)
    (2147483647, 2147483647, 5),   # product far past 2**64
    (200, 200, 200),               # 8,000,000 cells, no wrap, still above the limit
])
def test_no_alloc_sort_refuses_large_or_wrapping_grids(counts):
    """Grid checks run before any device call, so they work without a GPU."""
    lib = abi.load_library()
    one = (C.c_double * 3)(1.0, 1.0, 1.0)
    zero = (C.c_double * 3)(0.0, 0.0, 0.0)
    bc = (C.c_int32 * 3)(*counts)
    st = lib.soil_bin_sort_noalloc(None, None, None, None, 0, zero, one, bc, zero, one, zero, 0,
                                   None, None, None)
    assert st == abi.SOIL_ERR_CAPACITY
