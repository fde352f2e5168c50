"""ctypes binding of libymflow.so (the C ABI in include/ymflow.h).

The library is built in-tree (latticeyangmills_b200/libymflow.so) by
``__graft_entry__.build()`` (or ``make -C latticeyangmills_b200/csrc``).  There is no CPU fallback: if the
library is missing, importing the binding raises.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libymflow.so"

# status codes (include/ymflow.h)
OK = 0
ERR_ARG = -1
ERR_CUDA = -2
ERR_OOM = -3
ERR_NONFINITE = -4
ERR_UNITARITY = -5
ERR_CAPACITY = -6
ERR_STATE = -7
ERR_NODEVICE = -8
NOALLOC_MAX_SITES = 8388608  # YMFLOW_NOALLOC_MAX_SITES

FP64, FP32_18, FP32_12 = 0, 1, 2
PRECISIONS = {"fp64": FP64, "fp32_18": FP32_18, "fp32_12": FP32_12}
FIELD_COLD, FIELD_EXPIAH, FIELD_HOT, FIELD_CURRENT = 0, 1, 2, 3
IO_BIG_ENDIAN = 1
NCCL_ID_BYTES = 128
OPT_BLOCK, OPT_GRAPH, OPT_OBS_BLOCK, OPT_STAGE_FORM, OPT_TILE, OPT_TIMED_REUNIT = 1, 2, 3, 4, 5, 6
STAGE_FUSED, STAGE_SPLIT, STAGE_TILE = 0, 1, 2
ENS_SPLIT_RUNS = 3  # ensembles: the two-kernel stage per run of equal extents

# every symbol include/ymflow.h declares
EXPORTS = (
    "ymflow_version", "ymflow_device_count", "ymflow_create", "ymflow_destroy", "ymflow_last_error",
    "ymflow_upload", "ymflow_download", "ymflow_upload_sites", "ymflow_download_sites", "ymflow_load_file",
    "ymflow_init_links",
    "ymflow_generate_metropolis", "ymflow_observables", "ymflow_flow", "ymflow_derivative", "ymflow_su3_exp",
    "ymflow_reset_time", "ymflow_set_time", "ymflow_time_steps", "ymflow_time_kernels", "ymflow_set_option", "ymflow_get_option",
    "ymflow_autotune",
    "ymflow_host_alloc", "ymflow_host_free", "ymflow_device_bytes", "ymflow_fma_peak",
    "ymflow_ensemble_create", "ymflow_ensemble_destroy", "ymflow_ensemble_last_error",
    "ymflow_ensemble_upload", "ymflow_ensemble_download", "ymflow_ensemble_init_links",
    "ymflow_ensemble_flow", "ymflow_ensemble_reset_time", "ymflow_ensemble_time_steps",
    "ymflow_ensemble_autotune", "ymflow_ensemble_tuning", "ymflow_ensemble_set_tuning", "ymflow_observables_noalloc",
    "ymflow_create_slab", "ymflow_nccl_unique_id", "ymflow_slab_connect", "ymflow_slab_group_flow",
    "ymflow_create_block", "ymflow_block_group_flow",
)
NON_INT = ("ymflow_version", "ymflow_create", "ymflow_create_slab", "ymflow_create_block", "ymflow_destroy",
           "ymflow_last_error",
           "ymflow_ensemble_create",
           "ymflow_ensemble_destroy", "ymflow_ensemble_last_error")


class Obs(ctypes.Structure):
    """ymflow_obs: one measurement row."""
    _fields_ = [
        ("step", ctypes.c_int32), ("pad", ctypes.c_int32), ("t", ctypes.c_double),
        ("plaq", ctypes.c_double), ("topc", ctypes.c_double), ("energy", ctypes.c_double),
        ("t2E", ctypes.c_double),
    ]

    def as_tuple(self):
        return (self.step, self.t, self.plaq, self.topc, self.energy, self.t2E)


class YmflowError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"ymflow status {status}: {message}")
        self.status = status


_lib = None
_D = ctypes.POINTER(ctypes.c_double)
_I4 = ctypes.c_int * 4


def load():
    """Load libymflow.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -c 'import "
                           "__graft_entry__ as g; g.build()'` from the repository root, or "
                           "`make -C latticeyangmills_b200/csrc` (nvcc, sm_100a)")
    l = ctypes.CDLL(str(LIB_PATH))
    vp = ctypes.c_void_p
    l.ymflow_version.restype = ctypes.c_char_p
    l.ymflow_device_count.argtypes = [ctypes.POINTER(ctypes.c_int)]
    l.ymflow_create.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    l.ymflow_create.restype = vp
    l.ymflow_destroy.argtypes = [vp]
    l.ymflow_destroy.restype = None
    l.ymflow_last_error.argtypes = [vp]
    l.ymflow_last_error.restype = ctypes.c_char_p
    l.ymflow_upload.argtypes = [vp, vp]
    l.ymflow_download.argtypes = [vp, vp]
    l.ymflow_init_links.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_uint64, ctypes.c_uint32,
                                    ctypes.c_double]
    l.ymflow_observables.argtypes = [vp, ctypes.POINTER(Obs)]
    l.ymflow_fma_peak.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    l.ymflow_load_file.argtypes = [vp, ctypes.c_char_p, ctypes.c_int, ctypes.c_int64]
    l.ymflow_upload_sites.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
    l.ymflow_download_sites.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int]
    l.ymflow_generate_metropolis.argtypes = [vp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                             ctypes.c_int, ctypes.c_uint64, ctypes.POINTER(ctypes.c_double)]
    l.ymflow_flow.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.POINTER(Obs), ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    l.ymflow_derivative.argtypes = [vp, ctypes.c_int, vp]
    l.ymflow_su3_exp.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_int]
    l.ymflow_reset_time.argtypes = [vp]
    l.ymflow_set_time.argtypes = [vp, ctypes.c_int64, ctypes.c_double]
    l.ymflow_time_steps.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                    ctypes.POINTER(ctypes.c_float)]
    l.ymflow_time_kernels.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_float),
                                      ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    l.ymflow_set_option.argtypes = [vp, ctypes.c_int, ctypes.c_int64]
    l.ymflow_get_option.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int64)]
    l.ymflow_autotune.argtypes = [vp, ctypes.c_double, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                  ctypes.POINTER(ctypes.c_int)]
    l.ymflow_host_alloc.argtypes = [ctypes.c_int64, ctypes.POINTER(vp)]
    l.ymflow_host_free.argtypes = [vp]
    l.ymflow_device_bytes.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
    IP = ctypes.POINTER(ctypes.c_int)
    l.ymflow_ensemble_create.argtypes = [ctypes.c_int, IP, ctypes.c_int, ctypes.c_int, IP]
    l.ymflow_ensemble_create.restype = vp
    l.ymflow_ensemble_destroy.argtypes = [vp]
    l.ymflow_ensemble_destroy.restype = None
    l.ymflow_ensemble_last_error.argtypes = [vp]
    l.ymflow_ensemble_last_error.restype = ctypes.c_char_p
    l.ymflow_ensemble_upload.argtypes = [vp, ctypes.c_int, vp]
    l.ymflow_ensemble_download.argtypes = [vp, ctypes.c_int, vp]
    l.ymflow_ensemble_init_links.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_uint64,
                                             ctypes.c_uint32, ctypes.c_double]
    l.ymflow_ensemble_flow.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(Obs), ctypes.c_int, IP]
    l.ymflow_ensemble_reset_time.argtypes = [vp]
    l.ymflow_ensemble_time_steps.argtypes = [vp, ctypes.c_double, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    l.ymflow_ensemble_autotune.argtypes = [vp, ctypes.c_double, IP, IP]
    l.ymflow_ensemble_tuning.argtypes = [vp, IP, IP, IP]
    l.ymflow_ensemble_set_tuning.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    l.ymflow_observables_noalloc.argtypes = [vp, ctypes.POINTER(ctypes.c_int), vp, vp]
    l.ymflow_create_slab.argtypes = [IP, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, IP]
    l.ymflow_create_slab.restype = vp
    l.ymflow_nccl_unique_id.argtypes = [vp]
    l.ymflow_slab_connect.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    l.ymflow_slab_group_flow.argtypes = [ctypes.POINTER(vp), ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.POINTER(Obs), ctypes.c_int, IP]
    l.ymflow_create_block.argtypes = [IP, IP, IP, ctypes.c_int, ctypes.c_int, IP]
    l.ymflow_create_block.restype = vp
    l.ymflow_block_group_flow.argtypes = [ctypes.POINTER(vp), ctypes.c_int, IP, ctypes.c_double, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.POINTER(Obs), ctypes.c_int, IP]
    for name in EXPORTS:
        if name not in NON_INT:
            getattr(l, name).restype = ctypes.c_int
    _lib = l
    return l


def check(status: int, ctx=None) -> None:
    if status != OK:
        msg = load().ymflow_last_error(ctx).decode(errors="replace")
        raise YmflowError(status, msg)
