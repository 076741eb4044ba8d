"""ctypes mirror of the C ABI in include/merle_b200.h.

The structs below must stay byte-for-byte equal to the C declarations;
tests/test_abi.py checks their sizes against the library's own view.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

MB_MAXCOLS = 8
MB_MAXBINS = 64
MB_MAXPTRS = 128
MB_MAXNINSTR = 16
MB_NREGS = 4
MB_MAXSRC = 8
MB_MAXCLAUSE = 6
MB_MAXTERM = 16
MB_MAXKEY = 4

# mb_status
(MB_OK, MB_ERR_INVALID, MB_ERR_OOM, MB_ERR_CUDA, MB_ERR_TIMEOUT, MB_ERR_UNSUPPORTED, MB_ERR_IO, MB_ERR_REJECTED,
 MB_ERR_CANCELLED) = range(9)
STATUS_NAMES = ["MB_OK", "MB_ERR_INVALID", "MB_ERR_OOM", "MB_ERR_CUDA", "MB_ERR_TIMEOUT",
                "MB_ERR_UNSUPPORTED", "MB_ERR_IO", "MB_ERR_REJECTED", "MB_ERR_CANCELLED"]

# mb_opcode (the reference's enum ops, primitive.cuh:169-173)
END, AND, OR, NOT, ANDM, ORM = range(6)
# mb_xform
X_ID, X_DIV, X_YEAR = range(3)
# mb_vkind
V_ONE, V_COL, V_MUL, V_SUB = range(4)
# mb_grp_strategy
GRP_AUTO, GRP_SHARED, GRP_GLOBAL, GRP_HASH = range(4)


class mb_instr(C.Structure):
    _fields_ = [("opcode", C.c_uint8), ("dstreg", C.c_uint8), ("src1", C.c_uint8), ("src2", C.c_uint8)]


class mb_col(C.Structure):
    _fields_ = [("nmiddle", C.c_uint32), ("middle", C.POINTER(C.c_void_p)),
                ("leftmost", C.c_void_p), ("rightmost", C.c_void_p)]


class mb_vprg(C.Structure):
    _fields_ = [("factsz", C.c_uint64), ("ncols", C.c_uint32), ("cols", mb_col * MB_MAXCOLS),
                ("instrs", mb_instr * MB_MAXNINSTR)]


class mb_src(C.Structure):
    _fields_ = [("col", C.c_void_p), ("fk", C.c_void_p), ("dimsz", C.c_uint64),
                ("width", C.c_uint32), ("pad_", C.c_uint32)]


class mb_level(C.Structure):
    _fields_ = [("lo", C.POINTER(C.c_uint64)), ("hi", C.POINTER(C.c_uint64)), ("nbins", C.c_uint32),
                ("pad_", C.c_uint32), ("out", C.c_void_p), ("popcounts", C.c_void_p)]


class mb_term(C.Structure):
    _fields_ = [("src", C.c_uint32), ("pad_", C.c_uint32), ("lo", C.c_uint64), ("hi", C.c_uint64)]


class mb_key(C.Structure):
    _fields_ = [("src", C.c_uint32), ("xform", C.c_uint32), ("div", C.c_uint32),
                ("base", C.c_uint32), ("mul", C.c_uint32)]


class mb_op(C.Structure):
    _fields_ = [("nsrc", C.c_uint32), ("src", mb_src * MB_MAXSRC),
                ("nclause", C.c_uint32), ("clause_len", C.c_uint32 * MB_MAXCLAUSE),
                ("terms", mb_term * MB_MAXTERM),
                ("nkey", C.c_uint32), ("keys", mb_key * MB_MAXKEY),
                ("vkind", C.c_uint32), ("va", C.c_uint32), ("vb", C.c_uint32), ("pad_", C.c_uint32)]


class mb_launch(C.Structure):
    _fields_ = [("grp_strategy", C.c_uint32), ("warps_per_cta", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("words_per_lane", C.c_uint32), ("staging", C.c_uint32)]


class mb_star_cols(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("custkey", "partkey", "suppkey", "orderdate", "quantity",
                                          "discount", "extendedprice", "revenue", "supplycost", "suppcity")]


MB_RECIPE_COLS = 4
RECIPE_PERFECT, RECIPE_MANY_OR, RECIPE_CANDCHK = range(3)


class mb_recipe(C.Structure):
    _fields_ = [("factsz", C.c_uint64), ("nbit", C.c_uint32 * MB_RECIPE_COLS),
                ("min", C.c_uint32 * MB_RECIPE_COLS), ("max", C.c_uint32 * MB_RECIPE_COLS),
                ("dimsz", C.c_uint32 * MB_RECIPE_COLS), ("fk", C.c_void_p * MB_RECIPE_COLS),
                ("attr", C.c_void_p * MB_RECIPE_COLS)]


class mb_owned_vprg(C.Structure):
    _fields_ = [("prg", mb_vprg), ("mid", (C.c_void_p * MB_MAXBINS) * MB_MAXCOLS),
                ("owned", C.c_void_p * MB_MAXPTRS), ("nowned", C.c_uint32)]


class mb_star_host(C.Structure):
    _fields_ = [("nrows", C.c_uint64), ("ncust", C.c_uint64), ("nsupp", C.c_uint64), ("npart", C.c_uint64)] + \
        [(n, C.c_void_p) for n in ("custkey", "partkey", "orderdate", "extendedprice", "revenue", "supplycost",
                                   "quantity", "discount", "suppcity", "custcity", "partmfgr")]


class mb_engine_info(C.Structure):
    _fields_ = [("nrows", C.c_uint64), ("fact_bytes", C.c_uint64), ("dim_bytes", C.c_uint64),
                ("index_bytes", C.c_uint64), ("k", C.c_uint32), ("width4", C.c_uint32),
                ("nbitmaps", C.c_uint32), ("sms", C.c_uint32), ("index_build_ms", C.c_float),
                ("denorm", C.c_uint32), ("denorm_bytes", C.c_uint64)]


class mb_query(C.Structure):
    _fields_ = [("tmpl", C.c_uint32), ("p", C.c_uint32 * 8)]


PLAN_FUSED, PLAN_SCAN, PLAN_MATERIALISED, PLAN_HASH = range(4)
MB_INDEX_PROBE_DIMS = 1
MB_INDEX_LEVELS = 10
MB_LEVELS_ALL = 0x3FF
MB_BATCH_MAX = 128
PREFETCH_AUTO, PREFETCH_NONE, PREFETCH_ALL = range(3)


class mb_batch_opts(C.Structure):
    _fields_ = [("words_per_lane", C.c_uint32), ("warps", C.c_uint32), ("stages", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("prefetch", C.c_uint32), ("table_kb", C.c_uint32),
                ("pad_", C.c_uint32 * 2)]


class mb_batch_launch_info(C.Structure):
    _fields_ = [(n, C.c_uint32) for n in ("queries", "staged_rows", "copies", "words_per_lane", "warps",
                                          "table_slots", "stages", "chain_entries", "pad_")]


class mb_plan(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("order_mode", C.c_uint32), ("materialise", C.c_uint32),
                ("launch", mb_launch), ("cover", C.c_uint32)]


COVER_RULE, COVER_NOEDGE, COVER_NOCOMPL, COVER_FINE = range(4)


MB_PLAN_FEATURES = 32
MB_BATCH_FEATURES = 32
MB_BATCH_CANDIDATES = 18
MB_PLAN_CANDIDATES = 16


class mb_mlp_config(C.Structure):
    _fields_ = [("in_", C.c_uint32), ("hidden", C.c_uint32), ("out", C.c_uint32), ("seed", C.c_uint32)]


class mb_mlp_train_opts(C.Structure):
    _fields_ = [("epochs", C.c_uint32), ("batch", C.c_uint32), ("lr", C.c_float), ("beta1", C.c_float),
                ("beta2", C.c_float), ("seed", C.c_uint32)]


SERVE_BATCHED, SERVE_PLAIN = range(2)
FAULT_NONE, FAULT_ALLOC, FAULT_LAUNCH, FAULT_SLOW = range(4)


class mb_server_opts(C.Structure):
    _fields_ = [("mem_budget", C.c_uint64), ("mode", C.c_uint32), ("max_batch", C.c_uint32),
                ("max_inflight", C.c_uint32), ("use_planner", C.c_uint32), ("min_batch", C.c_uint32),
                ("pad_", C.c_uint32), ("batch", mb_batch_opts)]


class mb_request_info(C.Structure):
    _fields_ = [("status", C.c_int32), ("launch", C.c_uint32), ("batch_size", C.c_uint32), ("plan", C.c_uint32),
                ("nqual", C.c_uint64), ("t_submit_us", C.c_double), ("t_launch_us", C.c_double),
                ("t_done_us", C.c_double), ("gpu_ms", C.c_float), ("pad_", C.c_float)]


class mb_server_stats(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in ("submitted", "completed", "rejected", "cancelled", "failed", "launches",
                                          "launched_queries", "peak_reserved")] + [("gpu_ms", C.c_double),
                                                                                   ("scan_launches", C.c_uint64)]


class mb_query_stats(C.Structure):
    _fields_ = [("ms", C.c_float), ("nbitmaps", C.c_uint32), ("chk", C.c_uint32), ("algo_bytes", C.c_uint64)]


def query(tmpl: int, *p: int) -> mb_query:
    q = mb_query()
    q.tmpl = tmpl
    for i, v in enumerate(p):
        q.p[i] = v
    return q


VOIDP = C.c_void_p
U32 = C.c_uint32
U64 = C.c_uint64
I32 = C.c_int

# name -> (restype, argtypes) of every C ABI entry point (include/merle_b200.h)
SIGNATURES: dict[str, tuple] = {
    "mb_last_error": (C.c_char_p, []),
    "mb_version": (C.c_char_p, []),
    "mb_bitmap_words": (U64, [U64]),
    "mb_bitmap_stride": (U64, [U64]),
    "mb_vprg_is_nochk": (I32, [C.POINTER(mb_vprg)]),
    "mb_bitmap_create": (I32, [C.POINTER(mb_src), U64, C.POINTER(U64), C.POINTER(U64), U32, VOIDP, U64,
                               VOIDP, VOIDP]),
    "mb_bitmap_create_levels": (I32, [C.POINTER(mb_src), U64, C.POINTER(mb_level), U32, U64, VOIDP]),
    "mb_engine_test_stall": (I32, [VOIDP, U32, U32]),
    "mb_engine_enqueue_batch_plans": (I32, [VOIDP, VOIDP, VOIDP, U32, VOIDP, VOIDP, VOIDP]),
    "mb_engine_batch_features": (I32, [VOIDP, VOIDP, U32, VOIDP]),
    "mb_engine_batch_candidate": (I32, [U32, VOIDP, VOIDP]),
    "mb_engine_set_batch_planner": (I32, [VOIDP, VOIDP]),
    "mb_engine_plan_batch": (I32, [VOIDP, VOIDP, U32, VOIDP, VOIDP, VOIDP]),
    "mb_batch_graph_create_plans": (I32, [VOIDP, VOIDP, VOIDP, U32, VOIDP, VOIDP, VOIDP, VOIDP]),
    "mb_vprg_eval": (I32, [C.POINTER(mb_vprg), I32, VOIDP, VOIDP, VOIDP, VOIDP]),
    "mb_bitmap_to_rows": (I32, [VOIDP, VOIDP, U64, VOIDP, VOIDP, VOIDP]),
    "mb_bitmap_to_rows_noalloc": (I32, [VOIDP, VOIDP, U64, VOIDP, VOIDP, VOIDP]),
    "mb_rows_grpby": (I32, [VOIDP, VOIDP, U64, C.POINTER(mb_op), U32, VOIDP, VOIDP, VOIDP]),
    "mb_vprg_grpby": (I32, [C.POINTER(mb_vprg), C.POINTER(mb_op), U32, VOIDP, VOIDP,
                            C.POINTER(mb_launch), VOIDP]),
    "mb_join_grpby": (I32, [U64, C.POINTER(mb_op), U32, VOIDP, VOIDP, VOIDP]),
    "mb_hash_join_grpby": (I32, [U64, C.POINTER(mb_op), U32, VOIDP, VOIDP, VOIDP]),
    "mb_col_from_bin": (I32, [U32, C.POINTER(C.c_void_p), C.POINTER(U64), U64, U64, C.POINTER(mb_col),
                               C.POINTER(C.c_void_p)]),
    "mb_col_from_bin2": (I32, [U32, C.POINTER(C.c_void_p), C.POINTER(U64), U32, C.POINTER(C.c_void_p),
                                C.POINTER(U64), U64, U64, C.POINTER(mb_col), C.POINTER(C.c_void_p)]),
    "mb_recipe_build": (I32, [C.POINTER(mb_recipe), I32, C.POINTER(mb_instr), C.POINTER(mb_owned_vprg), VOIDP]),
    "mb_owned_vprg_release": (I32, [C.POINTER(mb_owned_vprg)]),
    "mb_engine_create": (I32, [I32, C.POINTER(VOIDP)]),
    "mb_engine_destroy": (I32, [VOIDP]),
    "mb_engine_gen_star": (I32, [VOIDP, U64, U32, U64, U64, I32]),
    "mb_engine_load_star": (I32, [VOIDP, C.POINTER(mb_star_host)]),
    "mb_engine_build_index": (I32, [VOIDP]),
    "mb_engine_build_index_ex": (I32, [VOIDP, U32]),
    "mb_engine_save_index": (I32, [VOIDP, C.c_char_p]),
    "mb_write_column": (I32, [C.c_char_p, VOIDP, U64, U32]),
    "mb_engine_save_ssb": (I32, [VOIDP, C.c_char_p]),
    "mb_engine_build_index_levels": (I32, [VOIDP, U32, U32]),
    "mb_engine_plan_index": (I32, [VOIDP, C.POINTER(mb_query), U32, U64, C.POINTER(U32), C.POINTER(U64),
                                   C.POINTER(U64)]),
    "mb_engine_load_index": (I32, [VOIDP, C.c_char_p, U32]),
    "mb_engine_get_info": (I32, [VOIDP, C.POINTER(mb_engine_info)]),
    "mb_query_ngroups": (U32, [C.POINTER(mb_query)]),
    "mb_engine_plan_rule": (I32, [VOIDP, C.POINTER(mb_query), C.POINTER(mb_plan)]),
    "mb_engine_query": (I32, [VOIDP, C.POINTER(mb_query), C.POINTER(mb_plan), VOIDP, VOIDP,
                              C.POINTER(mb_query_stats)]),
    "mb_queries_layout": (U64, [C.POINTER(mb_query), U32, C.POINTER(U64)]),
    "mb_engine_enqueue": (I32, [VOIDP, C.POINTER(mb_query), U32, C.POINTER(mb_plan), VOIDP, VOIDP, I32]),
    "mb_engine_sync": (I32, [VOIDP, C.POINTER(C.c_float), U32]),
    "mb_engine_mark": (I32, [VOIDP, U32]),
    "mb_engine_marks_ms": (I32, [VOIDP, U32, U32, C.POINTER(C.c_float)]),
    "mb_engine_stream": (VOIDP, [VOIDP]),
    "mb_engine_enqueue_batch": (I32, [VOIDP, C.POINTER(mb_query), U32, C.POINTER(mb_batch_opts), VOIDP, VOIDP]),
    "mb_engine_query_batch": (I32, [VOIDP, C.POINTER(mb_query), U32, C.POINTER(mb_batch_opts), VOIDP, VOIDP]),
    "mb_mlp_create": (I32, [I32, C.POINTER(mb_mlp_config), C.POINTER(VOIDP)]),
    "mb_mlp_destroy": (I32, [VOIDP]),
    "mb_mlp_nparams": (U32, [VOIDP]),
    "mb_mlp_get_params": (I32, [VOIDP, VOIDP]),
    "mb_mlp_set_params": (I32, [VOIDP, VOIDP]),
    "mb_mlp_forward": (I32, [VOIDP, VOIDP, U32, I32, VOIDP]),
    "mb_mlp_gradients": (I32, [VOIDP, VOIDP, VOIDP, VOIDP, U32, VOIDP, C.POINTER(C.c_float)]),
    "mb_mlp_train": (I32, [VOIDP, VOIDP, VOIDP, VOIDP, U32, C.POINTER(mb_mlp_train_opts), C.POINTER(C.c_float)]),
    "mb_engine_query_features": (I32, [VOIDP, C.POINTER(mb_query), VOIDP]),
    "mb_engine_plan_candidate": (I32, [VOIDP, C.POINTER(mb_query), U32, C.POINTER(mb_plan)]),
    "mb_engine_set_planner": (I32, [VOIDP, VOIDP]),
    "mb_engine_plan_learned": (I32, [VOIDP, C.POINTER(mb_query), U32, C.POINTER(mb_plan), VOIDP]),
    "mb_engine_batch_info": (I32, [VOIDP, C.POINTER(mb_query), U32, C.POINTER(mb_batch_opts),
                                   C.POINTER(mb_batch_launch_info), U32, C.POINTER(U32), C.POINTER(U32)]),
    "mb_batch_graph_create": (I32, [VOIDP, C.POINTER(mb_query), U32, C.POINTER(mb_batch_opts), VOIDP, VOIDP,
                                    C.POINTER(VOIDP)]),
    "mb_batch_graph_launch": (I32, [VOIDP]),
    "mb_batch_graph_destroy": (I32, [VOIDP]),
    "mb_engine_tune_batch": (I32, [VOIDP, C.POINTER(mb_query), U32, U32, C.POINTER(mb_batch_opts),
                                   C.POINTER(C.c_float), C.POINTER(U32)]),
    "mb_server_create": (I32, [VOIDP, C.POINTER(mb_server_opts), C.POINTER(VOIDP)]),
    "mb_server_destroy": (I32, [VOIDP]),
    "mb_server_submit": (I32, [VOIDP, C.POINTER(mb_query), VOIDP, C.POINTER(U64)]),
    "mb_server_cancel": (I32, [VOIDP, U64]),
    "mb_server_wait": (I32, [VOIDP, U64, C.c_int64, C.POINTER(mb_request_info)]),
    "mb_server_get_stats": (I32, [VOIDP, C.POINTER(mb_server_stats)]),
    "mb_server_run_load": (I32, [VOIDP, C.POINTER(mb_query), U32, C.c_double, U64, VOIDP,
                                 C.POINTER(mb_request_info)]),
    "mb_poisson_arrivals": (I32, [U64, C.c_double, U32, VOIDP]),
    "mb_server_inject": (I32, [VOIDP, U32, U32, U32]),
    "mb_gen_flat": (I32, [U64, U64, U64, VOIDP, VOIDP, VOIDP, VOIDP, VOIDP, VOIDP]),
    "mb_gen_star": (I32, [U64, U32, U64, U64, I32, C.POINTER(mb_star_cols), VOIDP]),
    "mb_gen_star_dims": (I32, [U64, U32, VOIDP, VOIDP, VOIDP, VOIDP]),
    "mb_wah_groups": (U64, [U64]),
    "mb_wah_encode": (I32, [VOIDP, U64, U32, VOIDP, U64, C.POINTER(U64), VOIDP]),
    "mb_wah_decode": (I32, [VOIDP, U64, U32, U64, VOIDP, VOIDP]),
    "mb_wah_ngroups": (I32, [VOIDP, U64, C.POINTER(U64), VOIDP]),
    "mb_wah_op": (I32, [U32, VOIDP, U64, VOIDP, U64, U64, VOIDP, U64, C.POINTER(U64), VOIDP]),
    "mb_wah_op_ex": (I32, [U32, VOIDP, U64, VOIDP, U64, U64, U32, VOIDP, U64, C.POINTER(U64), VOIDP]),
    "mb_wah_save": (I32, [C.c_char_p, VOIDP, U64, U64]),
    "mb_wah_load": (I32, [C.c_char_p, VOIDP, U64, C.POINTER(U64), C.POINTER(U64)]),
}

WAH_LSB, WAH_MSB = 0, 1
WAH_AND, WAH_OR, WAH_XOR = 0, 1, 2
WAH_AUTO, WAH_EXPLICIT, WAH_DIRECT = 0, 1, 2


def bind(lib: C.CDLL, sigs: dict[str, tuple]) -> None:
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


def header_symbols(header: Path) -> list[str]:
    """Names of the functions declared MB_API in a C ABI header."""
    import re
    text = header.read_text()
    return re.findall(r"^MB_API[^(]*?\b(\w+)\s*\(", text, flags=re.M)
