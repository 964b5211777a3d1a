"""ctypes binding of ``libtg_b200.so`` (the C ABI of include/tractography_b200.h).

The library is built in-tree by ``__graft_entry__.build()`` (or ``make -C
tractography_b200/csrc``).  There is no CPU fallback: if the library is
missing, every GPU entry point raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libtg_b200.so"

TG_OK = 0
TG_ERR_INVALID_ARGUMENT = 1
TG_ERR_CUDA = 2
TG_ERR_OUT_OF_MEMORY = 3
TG_ERR_UNSUPPORTED = 4
TG_ERR_POOL_EXHAUSTED = 5

MODEL_SH = 0
MODEL_DTI = 1
ALGO_TRANSPORT = 0
ALGO_DIFFUSION = 1
RNG_MWC64X = 0
RNG_PHILOX = 1

# Every symbol the header declares; tests check the library exports them.
EXPORTS = (
    "tg_abi_version",
    "tg_status_string",
    "tg_last_error",
    "tg_field_create",
    "tg_field_destroy",
    "tg_domain_create",
    "tg_domain_destroy",
    "tg_domain_create_mesh",
    "tg_bvh_build_host",
    "tg_mesh_info",
    "tg_mesh_segment_hits",
    "tg_mesh_segments_blocked",
    "tg_tractogram",
    "tg_tractogram_host",
    "tg_tractogram_noalloc",
    "tg_tracker_create",
    "tg_tracker_destroy",
    "tg_tracker_run",
    "tg_tracker_run_jobs",
    "tg_tracker_stats",
    "tg_tracker_set_tuning",
    "tg_tracker_get_tuning",
    "tg_tracker_set_slicing",
    "tg_tracker_get_slicing",
    "tg_tracker_copy_points",
    "tg_server_create",
    "tg_server_destroy",
    "tg_server_submit",
    "tg_server_poll",
    "tg_server_result_size",
    "tg_server_take",
    "tg_server_stats",
    "tg_server_set_epoch_time",
    "tg_server_reserve",
    "tg_server_timing",
    "tg_seeds_from_fod",
    "tg_domain_contains",
    "tg_field_evaluate",
    "tg_boundary_seeds",
    "tg_tod",
    "tg_connectome",
    "tg_local_evaluate",
    "tg_update_orientation",
    "tg_rng_stream",
    "tg_step_bound",
)


class Algorithm(ctypes.Structure):
    """Mirror of ``tg_algorithm``."""

    _fields_ = [
        ("algorithm", ctypes.c_int32),
        ("step_size", ctypes.c_float),
        ("gamma", ctypes.c_float),
        ("noise_variance", ctypes.c_float),
        ("rng_mode", ctypes.c_int32),
        ("rng_seed", ctypes.c_uint32),
        ("philox_key", ctypes.c_uint64),
        ("seed_offset", ctypes.c_uint64),
    ]


class Job(ctypes.Structure):
    """Mirror of ``tg_job``."""

    _fields_ = [
        ("domain", ctypes.c_void_p),
        ("field", ctypes.c_void_p),
        ("algorithm", Algorithm),
        ("seeds", ctypes.c_void_p),
        ("n_seeds", ctypes.c_uint32),
        ("batch_size", ctypes.c_uint32),
        ("batch_rng_seeds", ctypes.c_void_p),
        ("save_at", ctypes.c_float),
        ("n_steps", ctypes.c_uint32),
    ]


class TgError(RuntimeError):
    """A failed library call; ``status`` holds the tg status code."""

    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


_lib = None


def load() -> ctypes.CDLL:
    """Load the library (once) and declare the signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"the CUDA library {LIB_PATH} is not built; run "
            "`python -c 'import __graft_entry__ as g; g.build()'` or "
            "`make -C tractography_b200/csrc`"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    P = ctypes.c_void_p
    U32, I32, U64, F = ctypes.c_uint32, ctypes.c_int32, ctypes.c_uint64, ctypes.c_float
    AP = ctypes.POINTER(Algorithm)
    sig = {
        "tg_abi_version": ([], ctypes.c_int),
        "tg_status_string": ([ctypes.c_int], ctypes.c_char_p),
        "tg_last_error": ([], ctypes.c_char_p),
        "tg_field_create": ([I32, P, U32, U32, U32, U32, P, P, ctypes.POINTER(P)], ctypes.c_int),
        "tg_field_destroy": ([P], ctypes.c_int),
        "tg_domain_create": ([P, U32, U32, U32, P, P, ctypes.POINTER(P)], ctypes.c_int),
        "tg_domain_destroy": ([P], ctypes.c_int),
        "tg_domain_create_mesh": ([P, U32, P, U32, P, ctypes.POINTER(P)], ctypes.c_int),
        "tg_bvh_build_host": ([P, U32, P, U32, ctypes.POINTER(U32), ctypes.POINTER(U32), P, P, P, P, P, P],
                              ctypes.c_int),
        "tg_mesh_info": ([P, ctypes.POINTER(U32), ctypes.POINTER(U32), P, ctypes.POINTER(U64)], ctypes.c_int),
        "tg_mesh_segment_hits": ([P, P, P, U32, P, P, P, P], ctypes.c_int),
        "tg_mesh_segments_blocked": ([P, P, P, U32, P, P], ctypes.c_int),
        "tg_tractogram": ([AP, P, P, P, U32, F, U32, P, P, P], ctypes.c_int),
        "tg_tractogram_host": ([AP, P, P, P, U32, F, U32, P, P, P], ctypes.c_int),
        "tg_tractogram_noalloc": ([AP, P, P, P, U32, U32, P, F, U32, P, P, P], ctypes.c_int),
        "tg_tracker_create": ([U64, ctypes.POINTER(P)], ctypes.c_int),
        "tg_tracker_destroy": ([P], ctypes.c_int),
        "tg_tracker_run": ([P, AP, P, P, P, ctypes.c_int, U32, U32, P, F, U32, P, P,
                            ctypes.POINTER(U64), ctypes.POINTER(U64), P], ctypes.c_int),
        "tg_tracker_run_jobs": ([P, ctypes.POINTER(Job), U32, ctypes.c_int, P, P, ctypes.POINTER(U64),
                                 ctypes.POINTER(U64), P], ctypes.c_int),
        "tg_tracker_stats": ([P, ctypes.POINTER(F), ctypes.POINTER(U32), ctypes.POINTER(U32)], ctypes.c_int),
        "tg_tracker_set_tuning": ([P, U32, U32, U32], ctypes.c_int),
        "tg_tracker_get_tuning": ([P, ctypes.POINTER(U32), ctypes.POINTER(U32), ctypes.POINTER(U32)], ctypes.c_int),
        "tg_tracker_set_slicing": ([P, U32], ctypes.c_int),
        "tg_tracker_get_slicing": ([P, ctypes.POINTER(U32)], ctypes.c_int),
        "tg_tracker_copy_points": ([P, P, U64, U64, ctypes.c_int, P], ctypes.c_int),
        "tg_server_create": ([U64, U64, U32, U32, ctypes.POINTER(P)], ctypes.c_int),
        "tg_server_destroy": ([P], ctypes.c_int),
        "tg_server_submit": ([P, ctypes.POINTER(Job), ctypes.POINTER(U64)], ctypes.c_int),
        "tg_server_poll": ([P, P, U32, ctypes.POINTER(U32), ctypes.POINTER(U32), ctypes.POINTER(U32)], ctypes.c_int),
        "tg_server_result_size": ([P, U64, ctypes.POINTER(U32), ctypes.POINTER(U64), ctypes.POINTER(ctypes.c_double)],
                                  ctypes.c_int),
        "tg_server_take": ([P, U64, P, P, P], ctypes.c_int),
        "tg_server_set_epoch_time": ([P, ctypes.c_double], ctypes.c_int),
        "tg_server_reserve": ([P, U64], ctypes.c_int),
        "tg_server_timing": ([P, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                              ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
        "tg_server_stats": ([P, ctypes.POINTER(U64), ctypes.POINTER(U64), ctypes.POINTER(ctypes.c_double),
                             ctypes.POINTER(U64)], ctypes.c_int),
        "tg_seeds_from_fod": ([I32, U32, P, P, U32, P, P, U32, P, P], ctypes.c_int),
        "tg_domain_contains": ([P, P, U32, P, P], ctypes.c_int),
        "tg_field_evaluate": ([P, P, U32, P, P], ctypes.c_int),
        "tg_boundary_seeds": ([P, U32, P, P, U32, U32, U32, P, P], ctypes.c_int),
        "tg_tod": ([AP, P, P, P, U32, P, P, U32, U32, U32, P, P, P, P, P], ctypes.c_int),
        "tg_connectome": ([AP, P, P, P, P, U32, P, P, U32, U32, U32, F, P, P, P, P, P], ctypes.c_int),
        "tg_local_evaluate": ([I32, U32, P, P, U32, P, P], ctypes.c_int),
        "tg_update_orientation": ([I32, U32, AP, P, P, U32, P, P], ctypes.c_int),
        "tg_rng_stream": ([I32, U32, U32, U32, U32, P, P], ctypes.c_int),
        "tg_step_bound": ([F, F, U32, ctypes.POINTER(U64)], ctypes.c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(status: int) -> None:
    """Raise the matching Python exception for a non-zero status."""
    if status == TG_OK:
        return
    message = load().tg_last_error().decode(errors="replace")
    if status == TG_ERR_INVALID_ARGUMENT:
        raise ValueError(message)
    if status == TG_ERR_UNSUPPORTED:
        raise NotImplementedError(message)
    if status == TG_ERR_OUT_OF_MEMORY:
        raise MemoryError(message)
    raise TgError(status, message)
