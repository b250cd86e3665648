"""ctypes mirror of include/soil_cuda.h (structs, constants, prototypes).

The CUDA library ``soil_b200/libsoil_cuda.so`` is built in-tree by
``soil_b200/build.py``.  Loading fails loudly when it is missing: there is no
CPU fallback for any entry point.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsoil_cuda.so")

SOIL_OK = 0
SOIL_ERR_INVALID = 1
SOIL_ERR_CUDA = 2
SOIL_ERR_CAPACITY = 3
SOIL_ERR_OOM = 4
SOIL_ERR_STATE = 5
SOIL_ERR_TIMEOUT = 6
SOIL_ERR_NOT_FOUND = 7
SOIL_ERR_NO_DEVICE = 8

STATUS_NAMES = {
    0: "SOIL_OK", 1: "SOIL_ERR_INVALID", 2: "SOIL_ERR_CUDA", 3: "SOIL_ERR_CAPACITY",
    4: "SOIL_ERR_OOM", 5: "SOIL_ERR_STATE", 6: "SOIL_ERR_TIMEOUT",
    7: "SOIL_ERR_NOT_FOUND", 8: "SOIL_ERR_NO_DEVICE",
}

SOIL_FULL_REBUILD = 0
SOIL_COMMUNICATE_ONLY = 1

SOIL_COL_FORWARD = 1
SOIL_COL_REVERSE = 2
SOIL_COL_ZERO = 4

SOIL_FILTER_FP64 = 0
SOIL_DEFORM_NONE, SOIL_DEFORM_ERATE, SOIL_DEFORM_VEL, SOIL_DEFORM_FINAL = range(4)
SOIL_BOUNDARY_PERIODIC, SOIL_BOUNDARY_FIXED, SOIL_BOUNDARY_SHRINK = range(3)
SOIL_FILTER_FP32_RECHECK = 1


class SoilBox(C.Structure):
    _fields_ = [("lo", C.c_double * 3), ("hi", C.c_double * 3)]


class SoilNeighCfg(C.Structure):
    _fields_ = [
        ("skin_fraction", C.c_double),
        ("bin_size", C.c_double),
        ("every", C.c_uint64),
        ("sort_every", C.c_uint64),
        ("check", C.c_int32),
        ("newton", C.c_int32),
        ("additive_skin", C.c_double),
        ("filter", C.c_int32),
        ("reserved", C.c_int32),
    ]


class SoilCounts(C.Structure):
    _fields_ = [
        ("nlocal", C.c_uint64),
        ("nghost", C.c_uint64),
        ("npairs", C.c_uint64),
        ("step", C.c_uint64),
        ("rebuilds", C.c_uint64),
        ("sorts", C.c_uint64),
        ("steps_since_build", C.c_uint64),
        ("filter_candidates", C.c_uint64),
        ("filter_rechecked", C.c_uint64),
        ("comm_state", C.c_int32),
        ("triclinic", C.c_int32),
        ("bin_count", C.c_int32 * 3),
        ("nstencil_forward", C.c_int32),
        ("ghost_cutoff", C.c_double),
        ("max_cutoff", C.c_double),
        ("tilt_xy", C.c_double),
    ]

    def as_dict(self):
        d = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            d[name] = list(v) if name == "bin_count" else v
        return d


class SoilDevView(C.Structure):
    _fields_ = [
        ("nlocal", C.c_uint64),
        ("nghost", C.c_uint64),
        ("npairs", C.c_uint64),
        ("stride", C.c_uint64),
        ("x", C.c_void_p), ("y", C.c_void_p), ("z", C.c_void_p),
        ("vx", C.c_void_p), ("vy", C.c_void_p), ("vz", C.c_void_p),
        ("fx", C.c_void_p), ("fy", C.c_void_p), ("fz", C.c_void_p),
        ("mass", C.c_void_p), ("inv_mass", C.c_void_p), ("cutoff_radius", C.c_void_p),
        ("tag", C.c_void_p),
        ("neighbor_offsets", C.c_void_p),
        ("neighbor_indices", C.c_void_p),
        ("ncolumns", C.c_int32),
        ("newton", C.c_int32),
        ("columns", C.c_void_p),
        ("stream", C.c_void_p),
        ("in_start", C.c_void_p),
        ("in_list", C.c_void_p),
        ("origin", C.c_void_p),
        ("fold_start", C.c_void_p),
        ("fold_list", C.c_void_p),
        ("ghost_root", C.c_void_p),
        ("slot_max", C.c_uint32),
        ("slot_width", C.c_uint32),
        ("slot_old_tag", C.c_void_p),
        ("slot_old_val", C.c_void_p),
        ("slot_new_tag", C.c_void_p),
        ("slot_new_val", C.c_void_p),
    ]


SOIL_FORCE_FN = C.CFUNCTYPE(C.c_int, C.POINTER(SoilDevView), C.c_void_p)

SOIL_JOB_QUEUED, SOIL_JOB_RUNNING, SOIL_JOB_DONE, SOIL_JOB_FAILED, SOIL_JOB_CANCELLED = range(5)
JOB_STATES = ["queued", "running", "done", "failed", "cancelled"]


class SoilServerCfg(C.Structure):
    _fields_ = [
        ("hbm_budget_bytes", C.c_uint64),
        ("max_active", C.c_uint32),
        ("quantum_steps", C.c_uint32),
        ("bytes_per_atom", C.c_uint32),
        ("bytes_per_job", C.c_uint32),
    ]


class SoilJobSpec(C.Structure):
    _fields_ = [
        ("box", SoilBox),
        ("cfg", SoilNeighCfg),
        ("dt", C.c_double),
        ("natoms", C.c_uint64),
        ("tag", C.POINTER(C.c_uint32)),
        ("pos3", C.POINTER(C.c_double)),
        ("vel3", C.POINTER(C.c_double)),
        ("mass", C.POINTER(C.c_double)),
        ("cutoff_radius", C.POINTER(C.c_double)),
        ("radius", C.POINTER(C.c_double)),
        ("harmonic_k", C.c_double),
        ("shear_rate", C.c_double),
        ("steps", C.c_uint64),
    ]


class SoilJobInfo(C.Structure):
    _fields_ = [
        ("state", C.c_int32),
        ("natoms", C.c_uint64),
        ("steps", C.c_uint64),
        ("steps_done", C.c_uint64),
        ("t_submit", C.c_double),
        ("t_admit", C.c_double),
        ("t_done", C.c_double),
    ]


class SoilServerStats(C.Structure):
    _fields_ = [
        ("queued", C.c_uint64),
        ("admitted", C.c_uint64),
        ("completed", C.c_uint64),
        ("failed", C.c_uint64),
        ("atom_steps", C.c_uint64),
        ("batch_steps", C.c_uint64),
        ("busy_s", C.c_double),
        ("elapsed_s", C.c_double),
        ("reserved_bytes", C.c_uint64),
        ("max_active", C.c_int32),
    ]

P = C.c_void_p
PP = C.POINTER(C.c_void_p)
u64 = C.c_uint64
i32 = C.c_int32
u32 = C.c_uint32
dbl = C.c_double
pu32 = C.POINTER(C.c_uint32)
pi32 = C.POINTER(C.c_int32)
pu64 = C.POINTER(C.c_uint64)
pdbl = C.POINTER(C.c_double)

# name -> (restype, argtypes); the exact set declared in include/soil_cuda.h
PROTOTYPES = {
    "soil_abi_version": (C.c_int, []),
    "soil_ctx_create": (C.c_int, [C.c_int, u64, PP]),
    "soil_ctx_destroy": (C.c_int, [P]),
    "soil_last_error": (C.c_char_p, [P]),
    "soil_ctx_bytes_in_use": (C.c_int, [P, pu64]),
    "soil_ctx_alloc_count": (C.c_int, [P, pu64, pu64]),
    "soil_sys_create": (C.c_int, [P, C.POINTER(SoilBox), C.POINTER(SoilNeighCfg), dbl, PP]),
    "soil_sys_destroy": (C.c_int, [P]),
    "soil_sys_register_column": (C.c_int, [P, C.c_char_p, i32, u32, pi32]),
    "soil_sys_add_atoms": (C.c_int, [P, u64, pu32, pu32, pdbl, pdbl, pdbl, pdbl, C.POINTER(pdbl)]),
    "soil_sys_setup": (C.c_int, [P]),
    "soil_sys_set_shear": (C.c_int, [P, dbl]),
    "soil_sys_set_harmonic": (C.c_int, [P, dbl, i32]),
    "soil_sys_set_force_hook": (C.c_int, [P, SOIL_FORCE_FN, P]),
    "soil_step": (C.c_int, [P, u64]),
    "soil_sys_sync": (C.c_int, [P]),
    "soil_sys_stream": (C.c_int, [P, PP]),
    "soil_phase_deform": (C.c_int, [P]),
    "soil_phase_initial": (C.c_int, [P]),
    "soil_phase_decide_rebuild": (C.c_int, [P]),
    "soil_phase_remove_ghosts": (C.c_int, [P]),
    "soil_phase_zero_forces": (C.c_int, [P]),
    "soil_phase_shrink_wrap": (C.c_int, [P]),
    "soil_phase_pbc": (C.c_int, [P]),
    "soil_phase_sort": (C.c_int, [P]),
    "soil_phase_borders": (C.c_int, [P]),
    "soil_phase_forward_comm": (C.c_int, [P]),
    "soil_phase_neighbor": (C.c_int, [P]),
    "soil_phase_force": (C.c_int, [P]),
    "soil_phase_reverse_comm": (C.c_int, [P]),
    "soil_phase_final": (C.c_int, [P]),
    "soil_sys_counts": (C.c_int, [P, C.POINTER(SoilCounts)]),
    "soil_sys_get_atoms": (C.c_int, [P, u64, u64, pu32, pdbl, pdbl, pdbl, pi32, pi32]),
    "soil_sys_get_column": (C.c_int, [P, i32, u64, u64, pdbl]),
    "soil_sys_get_neighbor": (C.c_int, [P, pu32, pu32]),
    "soil_sys_num_swaps": (C.c_int, [P, pi32]),
    "soil_sys_get_swap": (C.c_int, [P, i32, pu64, pu64, pdbl, pdbl, pu32]),
    "soil_sys_get_sort_perm": (C.c_int, [P, pu32]),
    "soil_sys_view": (C.c_int, [P, C.POINTER(SoilDevView)]),
    "soil_sys_enable_slots": (C.c_int, [P, C.c_uint32, C.c_uint32]),
    "soil_sys_set_deform": (C.c_int, [P, C.c_int32, C.c_int32, C.c_double, C.c_double,
                                      C.c_uint64]),
    "soil_sys_set_deform_remap": (C.c_int, [P, C.c_int32]),
    "soil_sys_get_box": (C.c_int, [P, pdbl, pdbl, pdbl]),
    "soil_sys_set_boundary": (C.c_int, [P, pi32, C.c_double]),
    "soil_sys_get_swap_sends": (C.c_int, [P, C.c_int32, pu64]),
    "soil_sys_get_slots": (C.c_int, [P, pu32, pdbl]),
    "soil_bin_sort_noalloc": (C.c_int, [P, P, P, P, u64, pdbl, pdbl, pi32, pdbl, pdbl, pdbl, i32,
                                        P, P, P]),
    "soil_batch_create": (C.c_int, [P, PP]),
    "soil_batch_destroy": (C.c_int, [P]),
    "soil_batch_add": (C.c_int, [P, P]),
    "soil_batch_remove": (C.c_int, [P, P]),
    "soil_batch_size": (C.c_int, [P, pu32]),
    "soil_batch_step": (C.c_int, [P, u64]),
    "soil_batch_sync": (C.c_int, [P]),
    "soil_batch_stream": (C.c_int, [P, PP]),
    "soil_batch_stats": (C.c_int, [P, pu64, pu64, pu64, pu64]),
    "soil_batch_set_timing": (C.c_int, [P, i32]),
    "soil_batch_get_timing": (C.c_int, [P, pdbl, pu64]),
    "soil_batch_get_host_timing": (C.c_int, [P, pdbl]),
    "soil_server_create": (C.c_int, [P, C.POINTER(SoilServerCfg), PP]),
    "soil_server_destroy": (C.c_int, [P]),
    "soil_server_submit": (C.c_int, [P, C.POINTER(SoilJobSpec), pu64]),
    "soil_server_poll": (C.c_int, [P, u64, C.POINTER(SoilJobInfo)]),
    "soil_server_wait": (C.c_int, [P, u64, dbl, C.POINTER(SoilJobInfo)]),
    "soil_server_cancel": (C.c_int, [P, u64]),
    "soil_server_result": (C.c_int, [P, u64, pu32, pdbl, pdbl, pi32]),
    "soil_server_release": (C.c_int, [P, u64]),
    "soil_server_job_error": (C.c_int, [P, u64, C.c_char_p, u64]),
    "soil_server_get_stats": (C.c_int, [P, C.POINTER(SoilServerStats)]),
    "soil_sys_save_restart": (C.c_int, [P, u64, P, u64, pu64]),
    "soil_sys_load_restart": (C.c_int, [P, P, u64, pu64]),
    "soil_kernel_launches": (C.c_uint64, []),
    "soil_consumer_kernel": (C.c_char_p, []),
    "soil_sys_set_timing": (C.c_int, [P, u32]),
    "soil_sys_get_timing": (C.c_int, [P, pdbl, pu64, pu64]),
    "soil_timer_name": (C.c_char_p, [i32]),
}

SOIL_NUM_TIMERS = 10
TIMER_NAMES = ["integrate", "zero", "pbc", "sort", "borders", "forward", "neighbor", "force",
               "reverse", "final"]

SOIL_BATCH_NUM_TIMERS = 8
BATCH_TIMER_NAMES = ["integrate", "sort", "borders", "neighbor", "lists", "force", "reverse",
                     "step"]

BATCH_HOST_TIMER_NAMES = ["integrate", "sort", "border_plan", "borders", "neighbor", "lists",
                          "wait"]

PHASES = [
    "deform", "initial", "decide_rebuild", "remove_ghosts", "zero_forces", "pbc",
    "sort", "borders", "forward_comm", "neighbor", "force", "reverse_comm", "final",
]

_lib = None


def load_library(path=None):
    """Load libsoil_cuda.so and attach prototypes; raises if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"soil_b200: CUDA library {p} is missing; build it with "
            "`python -m soil_b200.build` (there is no CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class SoilError(RuntimeError):
    def __init__(self, status, where, message=""):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)} {message}".strip())
