"""ctypes binding of libop2b200.so, the C-ABI library of the B200 backend.

The library is built in-tree by :mod:`pyop2_b200.csrc.build`.  There is no
fallback: if it cannot be loaded the backend raises on ``op2.init``.
"""

import ctypes as C
import os

from .exceptions import DeviceError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libop2b200.so")

u64, i64, i32, u32 = C.c_uint64, C.c_int64, C.c_int32, C.c_uint32
P = C.c_void_p
u64p, i64p, i32p = C.POINTER(u64), C.POINTER(i64), C.POINTER(i32)
charp = C.c_char_p

# name -> argument types (every function returns int status)
_SIGS = {
    "op2b_init": [C.c_int],
    "op2b_shutdown": [],
    "op2b_version": [],
    "op2b_last_error": [C.c_char_p, C.c_size_t],
    "op2b_device_info": [i32p, i32p, i32p, i32p, u64p, u64p],
    "op2b_set_l2_fetch_granularity": [i32],
    "op2b_malloc": [u64p, u64],
    "op2b_free": [u64],
    "op2b_host_alloc": [u64p, u64],
    "op2b_host_free": [u64],
    "op2b_memcpy_h2d": [u64, P, u64, u64],
    "op2b_memcpy_d2h": [P, u64, u64, u64],
    "op2b_memcpy_d2h_async": [P, u64, u64, u64],
    "op2b_memcpy_h2d_small": [u64, P, u64, u64],
    "op2b_memcpy_d2d": [u64, u64, u64, u64],
    "op2b_memset": [u64, C.c_int, u64, u64],
    "op2b_transpose": [u64, u64, i64, i32, i32, i32, u64],
    "op2b_map_validate": [u64, i64, i32, i64p, u64],
    "op2b_default_stream": [u64p],
    "op2b_stream_create": [u64p],
    "op2b_stream_destroy": [u64],
    "op2b_stream_sync": [u64],
    "op2b_device_sync": [],
    "op2b_event_create": [u64p],
    "op2b_event_destroy": [u64],
    "op2b_event_record": [u64, u64],
    "op2b_event_record_node": [u64, u64],
    "op2b_event_sync": [u64],
    "op2b_event_query": [u64, i32p],
    "op2b_event_elapsed_ms": [u64, u64, C.POINTER(C.c_float)],
    "op2b_stream_wait_event": [u64, u64],
    "op2b_graph_begin": [u64],
    "op2b_graph_end": [u64, u64p],
    "op2b_graph_launch": [u64, u64],
    "op2b_graph_destroy": [u64],
    "op2b_graph_capture_tail": [u64, u64p],
    "op2b_graph_end_capture": [u64, u64p],
    "op2b_graph_chain_positions": [u64, u64p, i32, i64p, i64p],
    "op2b_graph_relax": [u64, i64p, i64p, i32, i32p, i32p, u64p],
    "op2b_graph_free": [u64],
    "op2b_halo_pack": [u64, u64, u64, i64, i32, u64],
    "op2b_halo_unpack": [u64, u64, u64, i64, i32, u64],
    "op2b_nvrtc_compile": [charp, charp, C.POINTER(charp), i32, C.POINTER(P), u64p, charp, u64],
    "op2b_cubin_free": [P],
    "op2b_module_load": [P, u64p],
    "op2b_module_unload": [u64],
    "op2b_module_function": [u64, charp, u64p],
    "op2b_module_global": [u64, charp, u64p, u64p],
    "op2b_function_set_smem": [u64, i32],
    "op2b_function_occupancy": [u64, u32, u32, i32p],
    "op2b_launch": [u64, u32, u32, u32, u64, P, u64],
    "op2b_set_programmatic_launch": [i32],
    "op2b_launch_colored": [u64, i32, i32p, u32, u32, u64, P, u64, u64],
    "op2b_plan_build": [i32, i32, i32, u64p, i32p, i32p, i32p, i32p, i32p,
                        i32, i32p, i32p, u64p, i32p, i32p, i32, u64, u64p],
    "op2b_plan_info": [u64, i32p, i32p, i32p, i32p, i32p, i64p, i32p],
    "op2b_plan_array": [u64, i32, u64p, i64p],
    "op2b_plan_ncolblk_host": [u64, i32p, i32],
    "op2b_plan_free": [u64],
    "op2b_region_plan_build": [i32, i32, i32, u64, i32, i32, i32, u64p, i32p, i32p, u64, u64p],
    "op2b_region_plan_info": [u64, i32p, i32p, i32p, i32p, i64p, i32p],
    "op2b_region_plan_array": [u64, i32, u64p, i64p],
    "op2b_region_plan_free": [u64],
    "op2b_region_plan_bank_slots": [u64, u64],
    "op2b_sparsity_build": [i32, i32, i32, i32, i32, u64p, i32p, u64p, i32p, i32p, u64, u64p],
    "op2b_sparsity_info": [u64, i32p, i64p],
    "op2b_sparsity_arrays": [u64, u64p, u64p, u64p],
    "op2b_sparsity_free": [u64],
    "op2b_incidence_build": [u64, i32, i32, i32, u64, u64p],
    "op2b_incidence_arrays": [u64, u64p, u64p, i32p],
    "op2b_incidence_free": [u64],
    "op2b_first_use_order": [u64, i32, i64, u64, i32, u64, u64],
    "op2b_rows_gather": [u64, u64, u64, i64, i32, u64],
    "op2b_map_renumber": [u64, u64, i64, u64, i32, u64],
    "op2b_mat_incidence_build": [u64, u64, u64, u64, i32, i32, i32, i32, u64, u64p],
    "op2b_lma_reduce": [u64, i32, u64, u64, i32, u64, i64, i32, u64, i32, u64],
    "op2b_mat_zero_rows": [u64, u64, u64, i32, i32p, i32, C.c_double, i32, u64],
    "op2b_csr_spmv": [u64, u64, u64, i32, i64, u64, u64, C.c_double, C.c_double, i32, u64],
    "op2b_vec_binop": [u64, u64, u64, C.c_double, i64, i32, i32, u64],
    "op2b_vec_dot": [u64, u64, i64, C.POINTER(C.c_double), u64],
    "op2b_cg_solve": [u64, u64, u64, i32, i64, u64, u64, i32, C.c_double, C.c_double, C.c_double,
                      i32, i32p, i32p, C.POINTER(C.c_double), u64],
    "op2b_mat_slots_rel_build": [u64, u64, u64, u64, i64, i32, i32, u64, u64],
    "op2b_mat_slots_build": [u64, u64, u64, u64, i64, i32, i32, u64, u64],
    "op2b_mat_zero_rows_static": [u64, u64, u64, i32, i32p, i32, C.c_double, i32, u64],
}

EXPORTED = tuple(sorted(_SIGS))

_lib = None


def load(path=LIB_PATH):
    """Load the library (no device call) and declare every entry point."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise DeviceError("B200 backend library %s is missing; build it with "
                          "`python -m pyop2_b200.csrc.build`" % path)
    lib = C.CDLL(path)
    for name, argtypes in _SIGS.items():
        fn = getattr(lib, name)
        fn.argtypes = argtypes
        fn.restype = C.c_int
    _lib = lib
    return lib


def last_error():
    buf = C.create_string_buffer(4096)
    _lib.op2b_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc, what=""):
    if rc != 0:
        raise DeviceError("%s: %s" % (what, last_error()))


def call(name, *args):
    """Call entry point ``name`` and raise DeviceError on a non-zero status."""
    rc = getattr(_lib, name)(*args)
    if rc != 0:
        raise DeviceError("%s failed (status %d): %s" % (name, rc, last_error()))
    return rc


def lib():
    return load()
