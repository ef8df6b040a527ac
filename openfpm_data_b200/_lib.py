"""ctypes binding of libsgb200.so (the C ABI declared in include/sgb200.h).

The library is the product: there is no CPU or PyTorch fallback.  Importing
this module on a machine without the built library raises ImportError with
the command that builds it.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsgb200.so")

# status codes (sgb_status)
OK, EINVAL, ECUDA, ENOMEM, ERANGE, ESTATE, ETIMEOUT, ENOTSUP = range(8)
# property types (sgb_type)
F32, I32, F64, U8 = 0, 1, 2, 3
# flush operators (sgb_op)
OP_NONE, OP_RIGHT, OP_LEFT, OP_ADD, OP_MAX, OP_MIN, OP_OR = range(7)
# neighbourhoods (sgb_nn)
NN_STAR, NN_FULL = 0, 1
# stencils (sgb_stencil)
HEAT7, GS7, BOX27, BOX27_NS = 0, 1, 2, 3
LIN_SMB, LIN_ZMB = 0, 1

# every entry point of include/sgb200.h: name -> (restype, argtypes)
_vp, _i32, _i64 = C.c_void_p, C.c_int, C.c_int64
_pvp = C.POINTER(C.c_void_p)
SIGNATURES = {
    "sgb_status_string": (C.c_char_p, [_i32]),
    "sgb_last_error_string": (C.c_char_p, []),
    "sgb_version": (_i32, []),
    "sgb_create": (_i32, [_pvp, _i32, _i32, _vp, _i32, _vp, _i32]),
    "sgb_destroy": (_i32, [_vp]),
    "sgb_set_background": (_i32, [_vp, _i32, _vp]),
    "sgb_insert": (_i32, [_vp, _i64, _vp, _vp, _vp]),
    "sgb_insert_lin": (_i32, [_vp, _i64, _vp, _vp, _vp]),
    "sgb_insert_pools": (_i32, [_vp, _i64, _i64, _vp, _vp, _vp, _vp]),
    "sgb_insert_blocks": (_i32, [_vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp]),
    "sgb_get_view": (_i32, [_vp, _i32, _vp, _vp]),
    "sgb_remove_boxes": (_i32, [_vp, _i64, _vp, _vp]),
    "sgb_existing_points": (_i32, [_vp, _vp, _vp, _i64, _vp, _vp]),
    "sgb_calc_existing_points": (_i32, [_vp, _vp, _vp]),
    "sgb_existing_point_list": (_i32, [_vp, _vp, _vp, _vp]),
    "sgb_set_linearizer": (_i32, [_vp, _i32]),
    "sgb_release_scratch": (_i32, [_vp]),
    "sgb_existence_changed": (_i32, [_vp]),
    "sgb_probe_bounded_waits": (_i32, [_i64, _i32, _vp]),
    "sgb_construct_link_dw": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "sgb_construct_link_up": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "sgb_get_links": (_i32, [_vp, _i32, _vp]),
    "sgb_pack_request": (_i32, [_vp, _i64, _vp, _i32, _vp, _vp, _vp]),
    "sgb_pack": (_i32, [_vp, _i64, _vp, _i32, _vp, _vp, _i64, _vp, _vp]),
    "sgb_unpack": (_i32, [_vp, _vp, _i64, _i32, _vp, _vp, _vp, _vp]),
    "sgb_unpack_boxes": (_i32, [_vp, _vp, _i64, _i32, _vp, _i64, _vp, _vp, _vp]),
    "sgb_flush": (_i32, [_vp, _vp, _vp]),
    "sgb_find_neighbours": (_i32, [_vp, _i32, _vp]),
    "sgb_neighbour_table": (_i32, [_vp, _i32, _vp, _vp]),
    "sgb_tag_boundaries": (_i32, [_vp, _i32, _vp]),
    "sgb_apply_stencil": (_i32, [_vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp]),
    "sgb_run_steps": (_i32, [_vp, _i32, _vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp]),
    "sgb_nchunks": (_i32, [_vp, _vp]),
    "sgb_index_buffer": (_i32, [_vp, _vp]),
    "sgb_data_buffer": (_i32, [_vp, _i32, _vp]),
    "sgb_mask_buffer": (_i32, [_vp, _vp]),
    "sgb_load_map": (_i32, [_vp, _i64, _vp, _vp, _vp, _vp]),
    "sgb_load_map_dev": (_i32, [_vp, _i64, _vp, _vp, _vp, _vp]),
    "sgb_download_map": (_i32, [_vp, _vp, _vp, _vp, _vp]),
    "sgb_count_existing": (_i32, [_vp, _vp, _vp, _vp]),
    "sgb_existing_offsets": (_i32, [_vp, _vp, _vp]),
    "sgb_existing_offsets_noalloc": (_i32, [_vp, _vp, _vp]),
    "sgb_get": (_i32, [_vp, _i64, _vp, _i32, _vp, _vp]),
    "sgb_build_balls": (_i32, [_vp, _i32, _vp, _i32, C.c_uint64, _vp, _vp]),
    "sgb_check_device_errors": (_i32, [_vp, _vp]),
    "sgb_device_bytes": (_i32, [_vp, _vp]),
    "sgb_set_launch_config": (_i32, [_vp, _i32, _i32]),
    "sgb_batch_create": (_i32, [_pvp, _i32]),
    "sgb_batch_destroy": (_i32, [_vp]),
    "sgb_batch_add": (_i32, [_vp, _vp, _i32, _vp, _vp, _vp, _i32, _i64, _vp, _vp]),
    "sgb_batch_remove": (_i32, [_vp, _i32, _vp]),
    "sgb_batch_step": (_i32, [_vp, _i32, _i32, _vp]),
    "sgb_batch_slot_steps": (_i32, [_vp, _i32, _vp]),
    "sgb_batch_extract": (_i32, [_vp, _i32, _vp, _vp, _vp]),
    "sgb_batch_read": (_i32, [_vp, _i32, _vp, _vp, _vp, _vp, _vp]),
    "sgb_batch_read_async": (_i32, [_vp, _i32, _vp, _vp, _vp, _vp, _vp]),
    "sgb_batch_info": (_i32, [_vp, _vp, _vp, _vp]),
    "sgb_batch_set_launch_config": (_i32, [_vp, _i32, _i32]),
}
# entry points outside the drop-in surface (cross-checks, tuning)
EXTRA_SIGNATURES = {
    "sgb_apply_stencil_tiled": (_i32, [_vp, _i32, _vp, _vp, _vp, _i32, _vp, _vp]),
}

_lib = None


class SgbError(RuntimeError):
    def __init__(self, status: int, what: str, detail: str = ""):
        self.status = status
        msg = f"{what}: {status_string(status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


def load():
    """Load libsgb200.so once; raise ImportError when it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `python -m openfpm_data_b200.build` "
            "(nvcc, sm_100a).  There is no fallback implementation."
        )
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in {**SIGNATURES, **EXTRA_SIGNATURES}.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def status_string(status: int) -> str:
    return load().sgb_status_string(status).decode()


def check(status: int, what: str) -> None:
    if status != OK:
        detail = load().sgb_last_error_string().decode()
        raise SgbError(status, what, detail)
