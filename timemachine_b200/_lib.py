"""Loader and build recipe of the native library (libtmnb.so, C ABI in include/tmnb.h).

The library is built in-tree for sm_100a. There is no fallback: importing a
potential whose library is missing raises immediately.
"""

import ctypes
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB_PATH = os.path.join(HERE, "libtmnb.so")
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(REPO, "include")

NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-gencode",
    "arch=compute_100a,code=sm_100a",
    "-Xcompiler",
    "-fPIC",
]

# The pair-kernel variants are split over their own translation units
# (pair_*.cu) so that they compile in parallel.
SOURCES = [
    "nonbonded.cu",
    "md.cu",
    "bonded.cu",
    "batch.cu",
    "static_pairlist.cu",
    "pair_f32_r32.cu",
    "pair_f32_r32_interp.cu",
    "pair_f32_r16.cu",
    "pair_f32_r16_interp.cu",
    "pair_f32_r8.cu",
    "pair_f32_r8_interp.cu",
    "pair_f64_r16.cu",
    "pair_f64_r16_interp.cu",
]
BUILD_DIR = os.path.join(HERE, "_build")


def build(verbose: bool = False, jobs: int = 0) -> str:
    """Compile libtmnb.so for sm_100a (nvcc cross-compiles without a GPU).

    Each source compiles to its own object in parallel; an object is rebuilt
    when it is older than its source or than any header of csrc/ and include/.
    """
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(BUILD_DIR, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    newest_header = max(os.path.getmtime(h) for h in headers)
    objs, todo = [], []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD_DIR, src[:-3] + ".o")
        objs.append(obj)
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(path), newest_header):
            todo.append([nvcc, *NVCC_FLAGS, "-I" + INCLUDE, "-c", path, "-o", obj])
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 1))
    running = []
    failed = []
    while todo or running:
        while todo and len(running) < jobs:
            cmd = todo.pop(0)
            if verbose:
                print(" ".join(cmd), flush=True)
            running.append((cmd, subprocess.Popen(cmd)))
        cmd, proc = running.pop(0)
        if proc.wait() != 0:
            failed.append(cmd[-3])
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(failed))
    link = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB_PATH, *objs]
    if verbose:
        print(" ".join(link), flush=True)
    subprocess.run(link, check=True)
    return LIB_PATH


c_ull_p = ctypes.POINTER(ctypes.c_ulonglong)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int32)

_lib = None


class TmnbError(RuntimeError):
    """Error reported by the native library (subclass of RuntimeError, as the reference raises)."""

    def __init__(self, status, message):
        super().__init__(message)
        self.status = status


def _declare(lib):
    vp = ctypes.c_void_p
    i = ctypes.c_int
    d = ctypes.c_double
    lib.tmnb_last_error.restype = ctypes.c_char_p
    lib.tmnb_version.restype = ctypes.c_char_p
    lib.tmnb_all_pairs_create.argtypes = [i, vp, vp, d, d, vp, i, i, i, ctypes.POINTER(vp)]
    lib.tmnb_pair_list_create.argtypes = [i, vp, vp, i, vp, vp, d, d, i, i, i, ctypes.POINTER(vp)]
    lib.tmnb_interaction_group_create.argtypes = [i, vp, i, vp, vp, d, d, i, i, ctypes.POINTER(vp)]
    lib.tmnb_interaction_group_create.restype = ctypes.c_int
    lib.tmnb_nonbonded_create.argtypes = [i, vp, vp, i, vp, vp, d, d, i, i, ctypes.POINTER(vp)]
    lib.tmnb_potential_destroy.argtypes = [vp]
    lib.tmnb_potential_execute_device.argtypes = [vp, i, i, vp, vp, vp, d, vp, vp, vp, vp, vp]
    lib.tmnb_potential_execute_host.argtypes = [vp, i, i, vp, vp, vp, d, vp, vp, vp, vp]
    lib.tmnb_potential_execute_windows_device.argtypes = [vp, i, i, vp, vp, vp, i, vp, vp, vp, vp, vp, vp]
    lib.tmnb_potential_execute_windows_host.argtypes = [vp, i, i, vp, vp, vp, i, vp, vp, vp, vp, vp]
    lib.tmnb_potential_execute_batch_host.argtypes = [vp, i, i, i, i, i, vp, vp, vp, vp, vp, vp, vp, vp]
    lib.tmnb_potential_du_dp_fixed_to_float.argtypes = [vp, i, i, vp, vp]
    lib.tmnb_potential_set_nblist_padding.argtypes = [vp, d]
    lib.tmnb_potential_disable_hilbert_sort.argtypes = [vp]
    lib.tmnb_potential_check_device_error.argtypes = [vp, vp]
    lib.tmnb_potential_nblist_stats.argtypes = [vp, vp, c_int_p, c_int_p, c_int_p]
    lib.tmnb_potential_nblist_shape.argtypes = [vp, c_int_p, c_int_p, ctypes.POINTER(ctypes.c_longlong)]
    lib.tmnb_potential_copy_nblist.argtypes = [vp, vp, vp, vp, vp]
    lib.tmnb_potential_nblist_shape.restype = ctypes.c_int
    lib.tmnb_potential_copy_nblist.restype = ctypes.c_int
    lib.tmnb_potential_enable_timing.argtypes = [vp, i]
    lib.tmnb_potential_last_pair_kernel_ms.argtypes = [vp, ctypes.POINTER(ctypes.c_float)]
    lib.tmnb_potential_last_stage_ms.argtypes = [vp, i, ctypes.POINTER(ctypes.c_float)]
    lib.tmnb_potential_last_stage_ms.restype = ctypes.c_int
    lib.tmnb_probe_fp32_peak.argtypes = [ctypes.POINTER(ctypes.c_double)]
    ull = ctypes.c_ulonglong
    lib.tmnb_context_create.argtypes = [i, vp, vp, vp, d, d, vp, vp, ull, i, vp, vp, vp, ctypes.POINTER(vp)]
    lib.tmnb_context_set_barostat.argtypes = [vp, d, d, vp, i, ull]
    lib.tmnb_context_multiple_steps.argtypes = [vp, i, vp, i, vp, i, vp, vp, i]
    lib.tmnb_context_multiple_steps_U.argtypes = [vp, d, i, i, vp, i, i, vp, vp, vp, i]
    for nm in ["get_x", "get_v", "get_box", "set_x", "set_v", "set_box"]:
        getattr(lib, "tmnb_context_" + nm).argtypes = [vp, vp]
    lib.tmnb_context_barostat_stats.argtypes = [vp, c_int_p, c_int_p, c_double_p]
    lib.tmnb_context_barostat_set_pressure.argtypes = [vp, d]
    lib.tmnb_context_barostat_set_interval.argtypes = [vp, i]
    lib.tmnb_context_barostat_last_move.argtypes = [vp, vp, vp]
    lib.tmnb_context_destroy.argtypes = [vp]
    lib.tmnb_harmonic_bond_create.argtypes = [i, i, vp, vp, vp, ctypes.POINTER(vp)]
    lib.tmnb_harmonic_angle_create.argtypes = [i, i, vp, vp, vp, ctypes.POINTER(vp)]
    lib.tmnb_pair_list_execute_static.argtypes = [i, i, vp, vp, vp, vp, d, d, i, vp, vp, vp, d, vp, vp, vp, vp, vp]
    lib.tmnb_pair_list_execute_static.restype = ctypes.c_int
    cp = ctypes.c_char_p
    lib.tmnb_potential_set_lambda_transforms.argtypes = [vp, cp, cp, cp, cp]
    lib.tmnb_potential_set_lambda_transforms.restype = ctypes.c_int
    lib.tmnb_lambda_transform_eval.argtypes = [cp, d, c_double_p, c_double_p]
    lib.tmnb_lambda_transform_eval.restype = ctypes.c_int
    lib.tmnb_potential_set_tile_rows.argtypes = [vp, i]
    lib.tmnb_potential_set_tile_rows.restype = ctypes.c_int
    lib.tmnb_batch_set_tile_rows.argtypes = [vp, i]
    lib.tmnb_batch_set_tile_rows.restype = ctypes.c_int
    lib.tmnb_potential_nblist_rows.argtypes = [vp, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32)]
    lib.tmnb_potential_nblist_rows.restype = ctypes.c_int
    lib.tmnb_potential_adjoint_device.argtypes = [vp, i, i, vp, vp, vp, d, vp, d, vp, vp, vp]
    lib.tmnb_potential_adjoint_device.restype = ctypes.c_int
    lib.tmnb_batch_create.argtypes = [ctypes.POINTER(vp)]
    lib.tmnb_batch_destroy.argtypes = [vp]
    lib.tmnb_batch_add.argtypes = [vp, i, vp, vp, vp, vp, vp, vp, i, vp, vp, i, vp, vp, i, vp, vp, d, d, d, d, d, vp, vp,
                                   ull, c_int_p]
    lib.tmnb_batch_remove.argtypes = [vp, i]
    lib.tmnb_batch_footprint.argtypes = [vp, i, i, i, i, ctypes.POINTER(ull)]
    lib.tmnb_batch_bytes_in_use.argtypes = [vp, ctypes.POINTER(ull)]
    lib.tmnb_batch_set_tuning.argtypes = [vp, i, d, i, i]
    lib.tmnb_batch_evaluate.argtypes = [vp, i, i, i, i]
    lib.tmnb_batch_md.argtypes = [vp, i, i, i]
    lib.tmnb_batch_synchronize.argtypes = [vp]
    lib.tmnb_batch_get.argtypes = [vp, i, i, vp]
    lib.tmnb_batch_set.argtypes = [vp, i, i, vp]
    lib.tmnb_batch_error.argtypes = [vp, i, c_int_p]
    lib.tmnb_batch_stats.argtypes = [vp, i, c_int_p, c_int_p, c_int_p]
    lib.tmnb_batch_stream.argtypes = [vp, ctypes.POINTER(vp)]
    lib.tmnb_batch_set_priority.argtypes = [vp, i]
    lib.tmnb_batch_set_priority.restype = ctypes.c_int
    lib.tmnb_batch_size.argtypes = [vp]
    lib.tmnb_batch_size.restype = ctypes.c_int
    lib.tmnb_potential_num_params.argtypes = [vp]
    lib.tmnb_potential_num_atoms.argtypes = [vp]
    for name in [
        "tmnb_all_pairs_create",
        "tmnb_pair_list_create",
        "tmnb_nonbonded_create",
        "tmnb_potential_destroy",
        "tmnb_potential_execute_device",
        "tmnb_potential_execute_host",
        "tmnb_potential_execute_batch_host",
        "tmnb_potential_execute_windows_device",
        "tmnb_potential_execute_windows_host",
        "tmnb_potential_du_dp_fixed_to_float",
        "tmnb_potential_set_nblist_padding",
        "tmnb_potential_disable_hilbert_sort",
        "tmnb_potential_check_device_error",
        "tmnb_potential_nblist_stats",
        "tmnb_potential_enable_timing",
        "tmnb_potential_last_pair_kernel_ms",
        "tmnb_probe_fp32_peak",
        "tmnb_context_create",
        "tmnb_context_set_barostat",
        "tmnb_context_multiple_steps",
        "tmnb_context_multiple_steps_U",
        "tmnb_context_get_x",
        "tmnb_context_get_v",
        "tmnb_context_get_box",
        "tmnb_context_set_x",
        "tmnb_context_set_v",
        "tmnb_context_set_box",
        "tmnb_context_barostat_stats",
        "tmnb_context_destroy",
        "tmnb_harmonic_bond_create",
        "tmnb_harmonic_angle_create",
    ]:
        getattr(lib, name).restype = ctypes.c_int
    lib.tmnb_potential_num_params.restype = ctypes.c_int
    lib.tmnb_potential_num_atoms.restype = ctypes.c_int
    return lib


def lib():
    """The loaded native library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is missing: build it with timemachine_b200._lib.build() "
                "(there is no CPU fallback for the nonbonded potential)"
            )
        _lib = _declare(ctypes.CDLL(LIB_PATH))
    return _lib


def check(status):
    if status != 0:
        raise TmnbError(status, lib().tmnb_last_error().decode())
