"""ctypes binding of the C ABI declared in include/gat_b200.h.

The shared library is built in-tree by gat_b200/build.py. There is no fallback: if the library
is missing or fails to load, importing this module raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgat_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(f"{LIB_PATH} is missing: run `python -m gat_b200.build` (needs nvcc)")

lib = C.CDLL(LIB_PATH)

c_int, c_i64, c_u64, c_f, c_d, c_p = C.c_int, C.c_int64, C.c_uint64, C.c_float, C.c_double, C.c_void_p
P_i32 = C.POINTER(C.c_int32)
P_i64 = C.POINTER(C.c_int64)
P_f32 = C.POINTER(C.c_float)


class MBB(C.Structure):
    """gat_mbb, field order of the reference's MBB (MBB.h:5)."""

    _fields_ = [("xmin", c_f), ("ymin", c_f), ("xmax", c_f), ("ymax", c_f)]


GAT_OK, GAT_ERR_ARG, GAT_ERR_OOM, GAT_ERR_CUDA, GAT_ERR_TRUNCATED, GAT_ERR_TIMEOUT, GAT_ERR_STATE = range(7)
GAT_INDEX_GRID, GAT_INDEX_STIG, GAT_INDEX_FSG, GAT_INDEX_MORTON = 0, 1, 2, 3
GAT_RESULT_IDS, GAT_RESULT_POINTS = 0, 1
GAT_EXEC_PLAIN, GAT_EXEC_BATCHED = 0, 1
GAT_LEN_UNIFORM, GAT_LEN_LOGNORMAL, GAT_LEN_LOGUNIFORM = 0, 1, 2
GAT_SIDE_FIXED, GAT_SIDE_LOGUNIFORM = 0, 1
GAT_EDR_MAX_LEN = 16384
GAT_EDR_NOALLOC_MAX_LEN = 4096
GAT_KERNEL_EDR, GAT_KERNEL_BOUNDS, GAT_KERNEL_RANGE_SCAN, GAT_KERNEL_INDEX_BUILD = 0, 1, 2, 3
class ServerConfig(C.Structure):
    """gat_server_config."""

    _fields_ = [("lanes", c_int), ("budget_bytes", c_i64), ("max_range_batch", c_int), ("max_topk_batch", c_int)]


(GAT_TUNE_EDR_ROWS, GAT_TUNE_EDR_TUNED, GAT_TUNE_TOPK_CHUNK, GAT_TUNE_TOPK_GROWTH, GAT_TUNE_EDR_FORM,
 GAT_TUNE_INDEX_BUILD, GAT_TUNE_DEP_LAUNCH, GAT_TUNE_TEST_STALL_CARRY, GAT_TUNE_SERVE_RESERVE,
 GAT_TUNE_RANGE_SHAPE, GAT_TUNE_EDR_RESERVE) = 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11

# (name, restype, argtypes) for every symbol of include/gat_b200.h
SIGNATURES = [
    ("gat_ctx_create", c_int, [c_int, C.POINTER(c_p)]),
    ("gat_ctx_destroy", None, [c_p]),
    ("gat_last_error", C.c_char_p, [c_p]),
    ("gat_ctx_stream", c_p, [c_p]),
    ("gat_ctx_sync", c_int, [c_p]),
    ("gat_ctx_launches", c_i64, [c_p]),
    ("gat_ctx_scratch_bytes", c_i64, [c_p]),
    ("gat_ctx_set_timing", c_int, [c_p, c_int]),
    ("gat_ctx_kernel_stats", c_int, [c_p, c_int, C.POINTER(c_d), P_i64, C.POINTER(c_d)]),
    ("gat_ctx_create_worker", c_int, [c_p, C.POINTER(c_p)]),
    ("gat_ctx_trim", c_int, [c_p]),
    ("gat_ctx_set_tuning", c_int, [c_p, c_int, c_int]),
    ("gat_ctx_get_tuning", c_int, [c_p, c_int, P_i32]),
    ("gat_db_create", c_int, [c_p, c_int, P_i32, P_f32, P_f32, C.POINTER(c_p)]),
    ("gat_db_destroy", None, [c_p]),
    ("gat_db_info", c_int, [c_p, P_i64]),
    ("gat_grid_build", c_int, [c_p, c_p, MBB, c_f, c_int, c_int, C.POINTER(c_p)]),
    ("gat_stig_build", c_int, [c_p, c_p, c_int, C.POINTER(c_p)]),
    ("gat_fsg_build", c_int, [c_p, c_p, MBB, c_f, C.POINTER(c_p)]),
    ("gat_morton_grid_build", c_int, [c_p, c_p, C.POINTER(c_p)]),
    ("gat_morton_grid_leaves", c_int, [c_p, c_p, P_i32, P_i32, c_i64, P_i64]),
    ("gat_index_destroy", None, [c_p]),
    ("gat_index_info", c_int, [c_p, P_i64]),
    ("gat_index_points", c_int, [c_p, c_p, c_i64, P_f32, P_f32, P_i32, P_i32]),
    ("gat_index_save", c_int, [c_p, c_p, C.c_char_p]),
    ("gat_index_load", c_int, [c_p, c_p, C.c_char_p, C.POINTER(c_p)]),
    ("gat_range_query", c_int, [c_p, c_p, c_p, c_int, c_int, c_int, P_i64, P_i32, P_i32, c_i64, P_i64]),
    ("gat_range_query_dev", c_int, [c_p, c_p, c_p, c_int, c_int, c_int, c_p, c_p, c_p, c_i64, P_i64]),
    ("gat_edr_pairs", c_int, [c_p, c_int, P_i32, P_i64, P_f32, c_i64, P_i32, P_i64, P_f32, c_i64, c_d, P_i32]),
    ("gat_edr_pairs_dev", c_int, [c_p, c_int, c_p, c_p, c_p, c_p, c_p, c_p, c_d, c_p]),
    ("gat_edr_pairs_dev_noalloc", c_int, [c_p, c_int, c_int, c_p, c_p, c_p, c_p, c_p, c_p, c_d, c_p]),
    ("gat_fv_lower_bounds", c_int, [c_p, c_p, c_int, P_i32, P_f32, P_f32, P_i32]),
    ("gat_topk", c_int, [c_p, c_p, c_int, P_i32, P_f32, P_f32, c_int, c_d, c_int, P_i32, P_i32, P_i64]),
    ("gat_topk_dev", c_int, [c_p, c_p, c_int, c_p, c_p, c_p, c_int, c_int, c_d, c_int, c_p, c_p, P_i64]),
    ("gat_topk_merge", c_int, [c_int, c_int, c_int, P_i32, P_i32, P_i32, P_i32]),
    ("gat_topk_merge_dev", c_int, [c_p, c_int, c_int, c_int, c_p, c_p, c_p, c_p]),
    ("gat_server_create", c_int, [c_p, c_p, c_p, c_p, C.POINTER(ServerConfig), C.POINTER(c_p)]),
    ("gat_server_destroy", None, [c_p]),
    ("gat_server_submit_range", c_int, [c_p, c_int, MBB, c_int, P_i64]),
    ("gat_server_submit_topk", c_int, [c_p, c_int, P_f32, P_f32, c_int, c_d, P_i64]),
    ("gat_server_wait", c_int, [c_p, c_i64, c_int, P_i32]),
    ("gat_server_range_result", c_int, [c_p, c_i64, P_i32, P_i32, c_i64, P_i64]),
    ("gat_server_topk_result", c_int, [c_p, c_i64, P_i32, P_i32, c_int]),
    ("gat_server_request_times", c_int, [c_p, c_i64, P_i64]),
    ("gat_server_release", c_int, [c_p, c_i64]),
    ("gat_server_stats", c_int, [c_p, P_i64]),
    ("gat_traj_file_info", c_int, [C.c_char_p, P_i32, P_i64, P_f32]),
    ("gat_traj_file_read", c_int, [C.c_char_p, c_int, c_i64, P_i32, P_f32, P_f32, P_i32]),
    ("gat_traj_file_write", c_int, [C.c_char_p, c_int, P_i32, P_f32, P_f32, P_i32, P_f32]),
    ("gat_gen_lengths", c_int, [c_int, c_int, c_d, c_d, c_int, c_int, c_u64, P_i32]),
    ("gat_gen_walks", c_int, [c_int, P_i32, P_f32, c_d, c_u64, P_f32, P_f32]),
    ("gat_gen_boxes", c_int, [c_int, c_int, c_d, c_d, P_f32, c_u64, P_f32]),
    ("gat_gen_sample_ids", c_int, [c_int, c_int, c_u64, P_i32]),
    ("gat_gen_pairs", c_int, [c_int, P_i32, P_i32, P_f32, c_d, c_d, c_u64, P_f32, P_f32]),
]

for _name, _res, _args in SIGNATURES:
    _fn = getattr(lib, _name)  # raises AttributeError when the library lacks a declared symbol
    _fn.restype = _res
    _fn.argtypes = _args

EXPORTED = [s[0] for s in SIGNATURES]
