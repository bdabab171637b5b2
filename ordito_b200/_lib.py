"""ctypes binding of ``include/ordito_b200.h`` (``libordito_b200.so``, built in-tree).

The product path has no CPU fallback: importing a function of this module on a machine without
the built library raises ``ImportError``, and a CUDA error in any call raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
from ctypes import POINTER, c_char_p, c_double, c_float, c_int, c_size_t, c_uint64, c_void_p
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "libordito_b200.so"

OB_OK = 0
OB_ERR_INVALID = 1
OB_ERR_CUDA = 2
OB_ERR_NOMEM = 3
OB_ERR_INDEX = 4
OB_ERR_NOT_CONVERGED = 5
OB_ERR_NONFINITE = 6
OB_ERR_INDEFINITE = 7
OB_ERR_TIMEOUT = 8
OB_ERR_BUDGET = 9

STATUS_CONVERGED = 0
STATUS_CAPPED = 1
STATUS_NONFINITE = 2
STATUS_SETTLED = 3
STATUS_SETTLE_BOUND = 4

P = c_void_p
I = c_int
D = c_double

# name -> argument types (every function returns int status unless listed in _RESTYPES).
SIGNATURES: dict[str, list] = {
    "ob_last_error": [],
    "ob_version": [],
    "ob_device_count": [POINTER(c_int)],
    "ob_set_device": [I],
    "ob_get_device": [POINTER(c_int)],
    "ob_malloc": [c_size_t, POINTER(c_void_p), P],
    "ob_free": [P, P],
    "ob_host_alloc": [c_size_t, POINTER(c_void_p)],
    "ob_host_free": [P],
    "ob_memcpy": [P, P, c_size_t, I, P, I],
    "ob_memset": [P, I, c_size_t, P],
    "ob_stream_create": [POINTER(c_void_p)],
    "ob_stream_destroy": [P],
    "ob_stream_synchronize": [P],
    "ob_device_synchronize": [],
    "ob_event_create": [POINTER(c_void_p)],
    "ob_event_destroy": [P],
    "ob_event_record": [P, P],
    "ob_event_elapsed_ms": [P, P, POINTER(c_float)],
    "ob_event_query": [P, POINTER(c_int)],
    "ob_event_synchronize": [P],
    "ob_stream_wait_event": [P, P],
    "ob_mem_info": [POINTER(c_size_t), POINTER(c_size_t)],
    "ob_mem_trim": [c_size_t],
    "ob_capture_begin": [P],
    "ob_capture_end": [P, POINTER(c_void_p), POINTER(c_int)],
    "ob_graph_launch": [P, P],
    "ob_graph_destroy": [P],
    "ob_launch_count": [POINTER(c_uint64)],
    "ob_pattern_workspace": [I, I, POINTER(c_size_t)],
    "ob_pattern_build": [P, I, I, P, P, P, P, P, P, c_size_t, P],
    "ob_face_terms": [P, P, I, I, P, P, P, P, P],
    "ob_voronoi_area_sums": [P, P, I, I, P, P],
    "ob_rim_vertices": [P, P, P, P, I, I, P, P, P],
    "ob_pinned_rows": [P, P, P, P, I, P, P],
    "ob_off_rim": [P, P, I, P, P],
    "ob_add_to_diagonal": [P, P, P, I, D, P, P],
    "ob_mollified_cot": [P, P, I, D, P, P, POINTER(c_double), P],
    "ob_edge_sums": [P, P, P, P, I, I, P, I, P, P],
    "ob_heat_rows": [P, P, P, P, I, P, I, P, D, P, I, P, D, P, P, P, P, P],
    "ob_heat_rows_f64": [P, P, P, P, I, P, I, P, D, P, I, P, D, P, P, P, P, P],
    "ob_cover_build": [P, P, P, P, I, P, I, P, P, I, D, D, I, P, P, P, POINTER(c_int), P],
    "ob_cover_face_terms": [P, P, I, I, P, P, P, P, P, P],
    "ob_cover_divergence": [P, P, P, I, P, P, P, I, P, P],
    "ob_seed": [P, I, I, P, P, P],
    "ob_grad_div": [P, P, I, I, P, P, P, P, I, P, P],
    "ob_shift": [P, I, P, I, P, I, I, P],
    "ob_shift_noalloc": [P, I, P, I, P, I, I, P],
    "ob_pcg_create": [I, P, P, P, I, I, I, POINTER(c_void_p), P],
    "ob_pcg_destroy": [P],
    "ob_pcg_rebind": [P, P, P, P, ctypes.c_longlong, P],
    "ob_pcg_solve": [P, P, P, D, I, POINTER(c_int), POINTER(c_double), P],
    "ob_pcg_settle": [P, P, P, I, D, I, I, POINTER(c_int), POINTER(c_int), P],
    "ob_pcg_time_matvec": [P, I, POINTER(c_float), P],
    "ob_pcg_info": [P, POINTER(ctypes.c_longlong)],
    "ob_backward_error": [I, P, P, P, P, P, I, D, P, P],
    "ob_spmv": [I, P, P, P, P, P, I, P],
    "ob_cast_scale": [P, I, P, I, ctypes.c_longlong, D, P],
    "ob_bounds": [P, I, P, P],
    "ob_axpby": [ctypes.c_longlong, D, P, D, P, P, P],
    "ob_fp64_peak": [POINTER(c_float), P],
    "ob_transpose": [I, I, P, P, P],
    "ob_seed_columns": [P, P, I, I, P, P, P],
    "ob_chol_analyse": [I, P, P, P, I, POINTER(c_void_p), P],
    "ob_chol_analysis_info": [P, POINTER(ctypes.c_longlong)],
    "ob_chol_host_analyse": [I, P, P, P, I, POINTER(c_void_p)],
    "ob_chol_analysis_nodes": [P, P],
    "ob_chol_analysis_destroy": [P],
    "ob_chol_factor": [P, P, I, I, POINTER(c_void_p), P],
    "ob_chol_values": [P, P, ctypes.c_longlong, POINTER(ctypes.c_longlong), P],
    "ob_divergence_tiles": [P, P, I, P, P, P, P],
    "ob_grad_div_tiled": [P, P, P, P, P, P, P, I, I, P, I, P, P, I, P, P, P],
    "ob_extend_seed": [P, P, I, I, P, P, P, P],
    "ob_halfedge_twins": [P, P, P, P, I, P, P, I, I, P, P, P],
    "ob_vertex_one_rings": [P, P, P, I, P, P, P, P],
    "ob_halfedge_tangent_angles": [P, P, I, I, P, P, P, P, P, P, P],
    "ob_vertex_tangent_frames": [P, P, I, I, P, P, P, P, P, P, P, P],
    "ob_tangent_to_world": [P, P, P, I, P, P],
    "ob_halfedge_transport": [P, P, I, P, P, P],
    "ob_half_cot_f64": [P, P, I, P, P],
    "ob_polar_unit": [P, I, P, P],
    "ob_block_pattern": [P, P, I, P, P, P],
    "ob_vector_heat_rows": [P, P, P, P, I, P, I, P, P, P, P, D, P, I, P, P],
    "ob_transport_seed": [P, P, I, I, P, P, P, P],
    "ob_transport_tail": [P, P, I, D, P, P, P],
    "ob_vertex_unit_gradient": [P, P, I, I, P, P, P, P, P, P, P, P],
    "ob_log_map_angles": [P, P, P, P, P, I, P, P],
    "ob_log_map_outward_ball": [P, P, P, P, P, P, I, I, P, P],
    "ob_radial_divergence": [P, P, I, I, P, P, P, I, P, P, P, P, P, P],
    "ob_log_map_fields": [P, P, I, I, P, P],
    "ob_chol_analyse_blocked": [I, I, P, P, P, I, POINTER(c_void_p), P],
    "ob_extend_ratio": [P, I, P, P, P],
    "ob_chol_set_deterministic": [P, I, P],
    "ob_chol_tile_columns": [P, I, P],
    "ob_amg_build_mode": [I],
    "ob_floor_f32": [P, ctypes.c_longlong, c_float, P],
    "ob_chol_nbytes": [P, POINTER(c_size_t)],
    "ob_chol_host_solve": [I, P, P, P, P, I, I, P, P, POINTER(ctypes.c_longlong)],
    "ob_chol_destroy": [P],
    "ob_chol_solve": [P, P, P, I, I, P, P, P, P],
    "ob_chol_buffers": [P, I, POINTER(c_void_p), POINTER(c_void_p), P],
    "ob_chol_work": [P, I, POINTER(c_void_p), POINTER(c_void_p), POINTER(c_int), POINTER(c_void_p),
                     POINTER(c_void_p), P],
    "ob_chol_solve_in_place": [P, I, P],
    "ob_renumber": [P, ctypes.c_longlong, P, P, P],
    "ob_corner_index_workspace": [I, I, POINTER(c_size_t)],
    "ob_corner_index": [P, I, I, P, P, P, c_size_t, P],
    "ob_grad_div_gather": [P, P, P, P, P, P, P, I, I, P, I, P, P, I, P, P, P],
    "ob_face_gradient_terms": [P, P, I, P, P, P, P, P],
    "ob_grad_div_terms": [P, P, P, P, I, I, P, I, P, P, I, P, P, P],
    "ob_corner_records": [P, P, P, I, P, P, P],
    "ob_grad_div_records": [P, P, P, I, I, P, I, P, P, I, P, P, P],
    "ob_seed_permuted": [P, P, I, I, P, P, I, P, P],
    "ob_shift_permuted": [P, I, I, P, P, P, I, I, P, P],
    "ob_chol_time_solve": [P, I, I, POINTER(c_float), P],
    "ob_chol_tile": [P, I, I, P],
    "ob_chol_solve_in_place_sources": [P, I, I, P, P, P],
    "ob_chol_info": [P, POINTER(ctypes.c_longlong)],
    "ob_chol_work_generation": [P, POINTER(ctypes.c_longlong)],
    "ob_chol_work_set": [P, I, I, POINTER(c_void_p), POINTER(c_void_p), POINTER(c_int), POINTER(c_void_p),
                         POINTER(c_void_p), P],
    "ob_chol_solve_in_place_set": [P, I, I, P],
    "ob_chol_work_generation_set": [P, I, POINTER(ctypes.c_longlong)],
    "ob_march_solve": [I, P, P, P, P, P, POINTER(ctypes.c_longlong), P],
    "ob_edge_sums_segments": [P, P, P, P, I, P, I, P, I, P, P],
    "ob_heat_rows_packed": [P, P, P, P, I, P, I, P, P, P, D, P, P, P, P, P],
    "ob_shift_packed": [P, I, I, P, P, I, P, I, P, P, P],
    "ob_amg_setup": [I, P, P, P, ctypes.c_uint, POINTER(c_void_p), P],
    "ob_amg_destroy": [P],
    "ob_amg_info": [P, POINTER(ctypes.c_longlong)],
    "ob_amg_levels": [P, POINTER(ctypes.c_longlong), POINTER(ctypes.c_longlong), I],
    "ob_amg_time_kernels": [P, I, I, POINTER(ctypes.c_float), POINTER(ctypes.c_longlong), P],
    "ob_amg_apply": [P, P, P, I, I, P],
    "ob_amg_solve": [P, P, P, I, I, D, I, I, D, P, P, P, P],
    "ob_amg_host_setup": [I, P, P, P, ctypes.c_uint, POINTER(ctypes.c_longlong),
                          POINTER(ctypes.c_longlong), I, POINTER(c_int)],
}
_RESTYPES = {"ob_last_error": c_char_p}


class _Library:
    """The loaded library with typed functions; missing library -> ImportError on first use."""

    def __init__(self) -> None:
        self._lib: ctypes.CDLL | None = None

    def load(self) -> ctypes.CDLL:
        if self._lib is None:
            if not LIBRARY_PATH.exists():
                raise ImportError(
                    f"{LIBRARY_PATH.name} is not built: run `python -m ordito_b200.build` "
                    "(nvcc, sm_100a); ordito_b200 has no CPU fallback"
                )
            lib = ctypes.CDLL(str(LIBRARY_PATH))
            for name, argtypes in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.argtypes = argtypes
                fn.restype = _RESTYPES.get(name, c_int)
            self._lib = lib
        return self._lib

    def __getattr__(self, name: str):
        return getattr(self.load(), name)


lib = _Library()


class CudaError(RuntimeError):
    """A CUDA runtime failure inside the library."""


def check(status: int, what: str = "") -> None:
    """Raise the Python exception an ``OB_ERR_*`` status maps to."""
    if status == OB_OK:
        return
    message = (lib.ob_last_error() or b"").decode(errors="replace")
    text = f"{what}: {message}" if what else message
    if status == OB_ERR_INVALID or status == OB_ERR_INDEX:
        raise ValueError(text)
    if status == OB_ERR_NOMEM:
        raise MemoryError(text)
    raise CudaError(f"[status {status}] {text}")


def call(name: str, *args) -> None:
    """Call ``name`` and raise on a non-zero status."""
    check(getattr(lib, name)(*args), name)


def launch_count() -> int:
    """Kernel launches this library made so far in the process."""
    value = c_uint64(0)
    check(lib.ob_launch_count(ctypes.byref(value)))
    return int(value.value)


def device_count() -> int:
    value = c_int(0)
    check(lib.ob_device_count(ctypes.byref(value)))
    return int(value.value)
