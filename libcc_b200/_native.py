"""ctypes binding of ``libcc_b200/_lib/libcc_b200.so`` (C ABI of include/libcc_b200.h).

There is no CPU fallback: if the shared library is missing or cannot be loaded
every entry point raises ``NativeLibraryError``.
"""
from __future__ import annotations

import ctypes
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "_lib" / "libcc_b200.so"

CCT_OK = 0
STATUS_NAMES = {
    0: "CCT_OK", 1: "CCT_ERR_INVALID", 2: "CCT_ERR_CUDA", 3: "CCT_ERR_NOMEM", 4: "CCT_ERR_NONFINITE",
    5: "CCT_ERR_DENOMINATOR", 6: "CCT_ERR_STATE", 7: "CCT_ERR_TIMEOUT", 8: "CCT_ERR_UNSUPPORTED",
}
CCT_PREC_FP64, CCT_PREC_INT8_EMU = 0, 1
CCT_MEM_HOST, CCT_MEM_DEVICE = 0, 1
CCT_VVVO_AUTO, CCT_VVVO_EXPANDED, CCT_VVVO_PACKED = 0, 1, 2

# every symbol include/libcc_b200.h declares
EXPORTS = [
    "ccT_options_default", "ccT_plan_create", "ccT_set_inputs", "ccT_num_tuples", "ccT_forward",
    "ccT_set_stream", "ccT_time_wbuild", "ccT_set_profiling", "ccT_last_kernel_ms", "ccT_last_forward_ms", "ccT_last_forward_launches", "ccT_plan_destroy", "ccT_status_string",
    "ccT_last_error", "ccT_measure_fp64_peak", "ccT_measure_int8_peak", "ijk_gpu_init_", "ijk_gpu_driver_", "ijk_gpu_finalize_",
    "cc_triples_b200_", "ccT_reduce_w_noalloc", "ccT_backward", "ccT_last_backward_ms", "ccT_kept_tuples", "ccT_emu_slice_histogram",
    "ccT_batch_create", "ccT_batch_set_inputs", "ccT_batch_forward", "ccT_batch_v1", "ccT_batch_configure",
    "ccT_batch_tune", "ccT_batch_last_ms", "ccT_batch_work_items", "ccT_batch_destroy", "ccT_emu_digits",
    "ccT_tuple_w", "ccT_batch_debug_stall", "ccT_batch_emu_digits", "ccT_ccsd_terms_29_31", "ccT_ccsd_terms_32_35", "ccT_ccsd_release_workspace",
]


class NativeLibraryError(RuntimeError):
    pass


class CctError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        self.status = status
        super().__init__(f"{where}: {STATUS_NAMES.get(status, status)}: {detail}")


class Options(ctypes.Structure):
    _fields_ = [("precision", ctypes.c_int32), ("device", ctypes.c_int32), ("check_inputs", ctypes.c_int32),
                ("emu_slices", ctypes.c_int32), ("emu_tol", ctypes.c_double), ("emu_tol_rel", ctypes.c_double),
                ("vvvo_mode", ctypes.c_int32), ("keep_w", ctypes.c_int32)]


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise NativeLibraryError(f"{LIB_PATH} is missing: build it with `python -m libcc_b200.build`")
    try:
        lib = ctypes.CDLL(str(LIB_PATH))
    except OSError as e:
        raise NativeLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    vp, dp, i64, i32 = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double), ctypes.c_int64, ctypes.c_int32
    i64p = ctypes.POINTER(ctypes.c_int64)
    lib.ccT_options_default.argtypes = [ctypes.POINTER(Options)]
    lib.ccT_options_default.restype = None
    lib.ccT_plan_create.argtypes = [ctypes.POINTER(vp), i64, i64, ctypes.POINTER(Options)]
    lib.ccT_plan_create.restype = ctypes.c_int
    lib.ccT_set_inputs.argtypes = [vp] + [vp] * 7 + [i32]
    lib.ccT_set_inputs.restype = ctypes.c_int
    lib.ccT_num_tuples.argtypes = [i64]
    lib.ccT_num_tuples.restype = i64
    lib.ccT_forward.argtypes = [vp, i64, i64, dp, dp, vp]
    lib.ccT_forward.restype = ctypes.c_int
    lib.ccT_set_stream.argtypes = [vp, vp]
    lib.ccT_set_stream.restype = ctypes.c_int
    lib.ccT_time_wbuild.argtypes = [vp, i64, i32, dp]
    lib.ccT_time_wbuild.restype = ctypes.c_int
    lib.ccT_set_profiling.argtypes = [vp, i32]
    lib.ccT_set_profiling.restype = ctypes.c_int
    lib.ccT_last_kernel_ms.argtypes = [vp, i32, dp, i64p]
    lib.ccT_last_kernel_ms.restype = ctypes.c_int
    lib.ccT_last_forward_ms.argtypes = [vp]
    lib.ccT_last_forward_ms.restype = ctypes.c_double
    lib.ccT_last_forward_launches.argtypes = [vp]
    lib.ccT_last_forward_launches.restype = i64
    lib.ccT_plan_destroy.argtypes = [vp]
    lib.ccT_plan_destroy.restype = ctypes.c_int
    lib.ccT_status_string.argtypes = [ctypes.c_int]
    lib.ccT_status_string.restype = ctypes.c_char_p
    lib.ccT_last_error.argtypes = []
    lib.ccT_last_error.restype = ctypes.c_char_p
    lib.ccT_measure_fp64_peak.argtypes = [i32]
    lib.ccT_measure_fp64_peak.restype = ctypes.c_double
    lib.ccT_measure_int8_peak.argtypes = [i32]
    lib.ccT_measure_int8_peak.restype = ctypes.c_double
    lib.ijk_gpu_init_.argtypes = [i64p, i64p, dp, dp, dp, dp, dp, dp]
    lib.ijk_gpu_init_.restype = None
    lib.ijk_gpu_driver_.argtypes = [i64p] * 5 + [dp] * 7
    lib.ijk_gpu_driver_.restype = None
    lib.ijk_gpu_finalize_.argtypes = [i64p, i64p, dp]
    lib.ijk_gpu_finalize_.restype = None
    lib.cc_triples_b200_.argtypes = [i64p, i64p] + [dp] * 10
    lib.cc_triples_b200_.restype = None
    lib.ccT_reduce_w_noalloc.argtypes = [i64] * 5 + [vp] * 6 + [vp]
    lib.ccT_reduce_w_noalloc.restype = ctypes.c_int
    lib.ccT_backward.argtypes = [vp, i64, i64] + [vp] * 7 + [i32]
    lib.ccT_backward.restype = ctypes.c_int
    lib.ccT_last_backward_ms.argtypes = [vp]
    lib.ccT_last_backward_ms.restype = ctypes.c_double
    lib.ccT_kept_tuples.argtypes = [vp]
    lib.ccT_kept_tuples.restype = ctypes.c_int64
    lib.ccT_emu_slice_histogram.argtypes = [vp, i64p, i32]
    lib.ccT_emu_slice_histogram.restype = i32
    lib.ccT_batch_create.argtypes = [ctypes.POINTER(vp), i64, i64p, i64p, ctypes.POINTER(Options)]
    lib.ccT_batch_create.restype = ctypes.c_int
    lib.ccT_batch_set_inputs.argtypes = [vp, i64] + [vp] * 7 + [i32]
    lib.ccT_batch_set_inputs.restype = ctypes.c_int
    lib.ccT_batch_forward.argtypes = [vp, dp, dp]
    lib.ccT_batch_forward.restype = ctypes.c_int
    lib.ccT_batch_v1.argtypes = [vp, i64, dp]
    lib.ccT_batch_v1.restype = ctypes.c_int
    lib.ccT_batch_configure.argtypes = [vp, i32, i32, i32, i64]
    lib.ccT_batch_configure.restype = ctypes.c_int
    lib.ccT_batch_tune.argtypes = [vp, ctypes.POINTER(i32), ctypes.POINTER(i32), ctypes.POINTER(i32), dp]
    lib.ccT_batch_tune.restype = ctypes.c_int
    lib.ccT_batch_last_ms.argtypes = [vp]
    lib.ccT_batch_last_ms.restype = ctypes.c_double
    lib.ccT_batch_work_items.argtypes = [vp]
    lib.ccT_batch_work_items.restype = i64
    lib.ccT_batch_destroy.argtypes = [vp]
    lib.ccT_batch_destroy.restype = ctypes.c_int
    lib.ccT_emu_digits.argtypes = [vp, ctypes.POINTER(i32), dp, dp]
    lib.ccT_emu_digits.restype = ctypes.c_int
    lib.ccT_tuple_w.argtypes = [vp, i64, vp, i32]
    lib.ccT_tuple_w.restype = ctypes.c_int
    lib.ccT_batch_debug_stall.argtypes = [vp, i64, i64]
    lib.ccT_batch_debug_stall.restype = ctypes.c_int
    lib.ccT_batch_emu_digits.argtypes = [vp, i64, ctypes.POINTER(i32)]
    lib.ccT_batch_emu_digits.restype = ctypes.c_int
    lib.ccT_ccsd_terms_29_31.argtypes = [i64, i64] + [vp] * 5 + [i32]
    lib.ccT_ccsd_terms_29_31.restype = ctypes.c_int
    lib.ccT_ccsd_terms_32_35.argtypes = [i64, i64] + [vp] * 6 + [i32]
    lib.ccT_ccsd_terms_32_35.restype = ctypes.c_int
    lib.ccT_ccsd_release_workspace.argtypes = []
    lib.ccT_ccsd_release_workspace.restype = ctypes.c_int
    _lib = lib
    return lib


def check(status: int, where: str):
    if status != CCT_OK:
        lib = load()
        raise CctError(status, where, lib.ccT_last_error().decode(errors="replace"))
