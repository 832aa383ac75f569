"""ctypes binding of ``libzvfv_b200.so`` (declarations in ``include/zvfv_b200.h``).

The conventions follow the reference's AmgX binding (``zvcfd/fv/linear.py:681-955``):
arrays are raw device pointers, every call returns an int status (0 = success), and a
failure raises ``RuntimeError(f"... failed (code {rc})")`` with the library's last error
text. There is no fallback: without the built library, importing this module raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libzvfv_b200.so"

P = ctypes.c_void_p
I32 = ctypes.c_int
I64 = ctypes.c_int64
F64 = ctypes.c_double

# name: (argtypes, restype); restype None means int status
_SIGNATURES = {
    "zvfv_version": ([], I32),
    "zvfv_launch_count": ([], I64),
    "zvfv_last_error": ([], ctypes.c_char_p),
    "zvfv_record_doubles": ([I32], I32),
    "zvfv_pattern_create": ([P, I64, I32, P, P, P, P, P], None),
    "zvfv_pattern_fill": ([P, P, P, P], None),
    "zvfv_pattern_destroy": ([P], None),
    "zvfv_colour": ([P, I32, I64, I64, I32, P, P, I64, P], None),
    "zvfv_slot_order": ([P, I64, I32, P, P, P], None),
    "zvfv_permute_rows": ([P, P, I64, I64, P, I32, P], None),
    "zvfv_geobuild": ([I32, P, I64, P, P, P], None),
    "zvfv_blockpos": ([I32, P, I64, P, P, P, P], None),
    "zvfv_statics": ([I32, I32, P, I32, P, P, P, P, F64, I32, P, P, P, P], None),
    "zvfv_diagonal": ([I32, I32, P, I32, P, P, P, P, P, I32, F64, F64, F64, F64, F64, I32, I32,
                       I32, P, P, P], None),
    "zvfv_assemble": ([I32, I32, P, I32, P, P, P, P, P, P, P, P, P, P, I32, F64, P, P, F64, P, P,
                       F64, I32, F64, F64, F64, F64, F64, I32, I32, I32, P, P, P, P, P, P], None),
    "zvfv_massflow": ([I32, I32, P, I32, P, P, P, P, P, P, P, P, I32, F64, P, P, F64, P, P, F64,
                       P, P, P, P], None),
    "zvfv_massflow_diag": ([I32, I32, P, I32, P, P, P, P, P, P, P, P, I32, F64, P, P, F64, P, P,
                            F64, I32, F64, F64, F64, F64, F64, I32, I32, P, P, P, P, P, P], None),
    "zvfv_limiter": ([I32, I32, P, I32, P, P, P, P, P, P, P, P, P], None),
    "zvfv_gradient": ([I64, I32, I32, P, P, P, P, P, P, P], None),
    "zvfv_minmax": ([I64, P, P, P, P, P, P], None),
    "zvfv_finalise_partials": ([I64], I64),
    "zvfv_finalise": ([I64, P, P, P, P, P, I32, P, P, P, P, P, P, P, P, P, I32, P, P, P, P, P,
                       I32, P, P, P, P, P, P, F64, P, P, P, P, P], None),
    "zvfv_update_partials": ([I64], I64),
    "zvfv_update": ([I64, P, P, P, P, P], None),
    "zvfv_fold": ([I64, I32, P, P, P, P], None),
    "zvfv_update_noalloc": ([I64, P, P, P, P, P], None),
    "zvfv_wall_shear": ([I64, P, P, P, P, P, P, I32, F64, F64, F64, F64, F64, P, P], None),
    "zvfv_bsr_spmv": ([I64, P, P, P, P, P, I32, P], None),
    "zvfv_bsr_residual": ([I64, P, P, P, P, P, P, I32, P], None),
    "zvfv_bsr_spmv_f32": ([I64, P, P, P, P, P, I32, P], None),
    "zvfv_bsr_transpose": ([I64, I64, P, P, P, P, P, P], None),
    "zvfv_bsr_spmv_t": ([I64, P, P, P, P, P, P, I32, P], None),
    "zvfv_solver_create": ([P, I32, I32, I32, I32, I32, I32, F64, I32, I32, I32, I32], None),
    "zvfv_solver_smooth": ([P, I32, I32, P], None),
    "zvfv_solver_vcycle_t": ([P, P, P, P], None),
    "zvfv_solver_setup": ([P, I64, I64, P, P, P, P], None),
    "zvfv_solver_solve": ([P, P, P, F64, I32, I32, P, P, P, P, P, P, P, P, P, P], None),
    "zvfv_solver_solve_t": ([P, P, P, F64, I32, I32, P, P, P, P, P, P, P, P, P, P], None),
    "zvfv_solver_solve_segmented": ([P, I32, P, P, P, P, F64, I32, I32, P, P, P, P, P, P, P, P,
                                     P, P], None),
    "zvfv_solver_vcycle": ([P, P, P, P], None),
    "zvfv_solver_set_option": ([P, ctypes.c_char_p, F64], None),
    "zvfv_solver_get_option": ([P, ctypes.c_char_p, P], None),
    "zvfv_solver_stats": ([P, I32, P, P, P], None),
    "zvfv_solver_level": ([P, I32, P, P, P, P, P], None),
    "zvfv_solver_destroy": ([P], None),
}


def _load():
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH.name} is not built: run `python -m zvcfd_b200.build` "
                           "(there is no CPU fallback)")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (args, res) in _SIGNATURES.items():
        f = getattr(lib, name)
        f.argtypes = args
        f.restype = I32 if res is None else res
    return lib


lib = _load()


def declared() -> list[str]:
    return list(_SIGNATURES)


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib.zvfv_last_error().decode(errors="replace")
        raise RuntimeError(f"{what} failed (code {rc}): {msg}")


def call(name: str, *args) -> None:
    """Call a status-returning entry point and raise on failure."""
    check(getattr(lib, name)(*args), name)


def ptr(t) -> int | None:
    """Device pointer of a torch tensor (None for None)."""
    return None if t is None else t.data_ptr()


def stream_ptr():
    import torch

    return torch.cuda.current_stream().cuda_stream
