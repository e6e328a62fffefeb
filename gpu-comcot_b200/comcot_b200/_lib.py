"""ctypes binding of libgcomcot.so (the C ABI in include/gcomcot.h).

The library is built in-tree (``make -C gpu-comcot_b200``).  There is no
fallback: if it is missing or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import pathlib

LIB_PATH = pathlib.Path(__file__).resolve().parent / "libgcomcot.so"

_lib = None

P_I = C.POINTER(C.c_int)
P_F = C.POINTER(C.c_float)
VP = C.c_void_p


class Fault(C.Structure):
    """gc_fault (include/gcomcot.h)"""
    _fields_ = [(n, C.c_double) for n in ("hh", "l", "w", "d", "th", "dl", "rd", "x0", "y0", "xo", "yo")] + [
        ("sw", C.c_int)]


def faults_array(faults):
    """list of dicts (keys of gc_fault; missing ones 0) -> ctypes array"""
    arr = (Fault * max(1, len(faults)))()
    for k, f in enumerate(faults):
        for key, v in f.items():
            setattr(arr[k], key, v)
    return arr


class ChildDesc(C.Structure):
    """gc_child_desc (include/gcomcot.h)"""
    _fields_ = ([("nx", C.c_int), ("ny", C.c_int), ("corners", C.c_int * 4), ("rel_size", C.c_int),
                 ("rel_time", C.c_int)]
                + [(n, C.c_int) for n in ("laycord", "laygov", "linchk", "modscm", "fric_switch")]
                + [(n, C.c_float) for n in ("dt", "rx", "ry", "grx", "gry", "fric_coef")]
                + [(n, P_F) for n in ("h", "hp", "hq", "rows", "rows2")]
                + [("sc_pos", P_I), ("sc_cxy", P_F), ("sc_fix_top", C.c_int), ("parent_modscm", C.c_int)])


# name -> (restype, argtypes)
SIGNATURES = {
    "gcomcot_init_gpu_": (None, []),
    "gcomcot_init_layer_": (None, [P_I, P_I, P_I, P_I, P_I, P_I, P_F, P_F, P_F, P_F, P_F, P_F, P_F,
                                   P_F, P_F, P_F, P_F, P_I, P_I]),
    "mass_launch_": (None, [P_F, P_F, P_F, P_I]),
    "momt_launch_": (None, [P_F, P_F, P_F, P_I]),
    "openbd_launch_": (None, [P_F]),
    "all_grid_launch_": (None, []),
    "maxamp_launch_": (None, [P_I]),
    "cuda_update_layer_": (None, [P_I]),
    "gcomcot_get_z_": (None, [P_I, P_F, P_F, P_F, P_F, P_I, P_I]),
    "cuda_getz_": (None, [P_F, P_I]),
    "cuda_setz_": (None, [P_F, P_I]),
    "cuda_getz1_": (None, [P_F, P_I]),
    "cuda_setz1_": (None, [P_F, P_I]),
    "cuda_getmn_": (None, [P_F, P_F, P_I]),
    "cuda_setmn_": (None, [P_F, P_F, P_I]),
    "cuda_getmn1_": (None, [P_F, P_F, P_I]),
    "cuda_setmn1_": (None, [P_F, P_F, P_I]),
    "cuda_getzmax_": (None, [P_F, P_I]),
    "gcomcot_show_grids_": (None, []),
    "cuda_shutdown_": (None, []),
    "edgeinterp_dbglaunch_": (None, [P_F, P_F, P_I, P_F, P_F, P_I, P_I, P_F, P_F]),
    "jnz_dbglaunch_": (None, [P_F, P_I, P_I]),
    "gcomcot_set_layer_params_": (None, [P_I, P_I, P_I, P_F, P_F, P_F, P_F, P_F, P_I, P_F, P_I, P_I,
                                         P_I, P_I, P_F, P_F]),
    "gcomcot_set_layer_coefs_": (None, [P_I, P_F, P_F, P_F, P_I, P_I]),
    "gcomcot_set_sponge_": (None, [P_I, P_F, P_F, P_F, P_I, P_I]),
    "sponge_launch_": (None, [P_I]),
    "gcomcot_set_sc_tables_": (None, [P_I, P_I, P_F, P_I, P_I, P_I, P_I]),
    "gcomcot_set_arrival_": (None, [P_I, P_F]),
    "gcomcot_get_arrival_": (None, [P_I, P_I]),
    "gcomcot_launch_count": (C.c_longlong, []),
    "gcomcot_set_fusion": (None, [C.c_int]),
    "gcomcot_sync": (C.c_int, []),
    "gcomcot_stream": (VP, []),
    "gcomcot_set_wait_limit": (None, [C.c_int]),
    "gcomcot_inject_stall": (None, []),
    "gcomcot_drive": (C.c_int, [C.c_int, C.c_int, C.c_int, P_I, P_I, P_I, P_F]),
    "gc_engine_create": (C.c_int, [C.c_longlong, C.POINTER(VP)]),
    "gc_engine_destroy": (C.c_int, [VP]),
    "gc_engine_add_class": (C.c_int, [VP, C.c_int, C.c_int, P_F, P_F]),
    "gc_engine_add_member": (C.c_int, [VP, C.c_int, P_F, C.c_int, C.c_int, P_I, P_F, C.c_float]),
    "gc_engine_step": (C.c_int, [VP, C.c_int]),
    "gc_engine_member_done": (C.c_int, [VP, C.c_int]),
    "gc_engine_member_steps": (C.c_int, [VP, C.c_int]),
    "gc_engine_sync": (C.c_int, [VP]),
    "gc_engine_query": (C.c_int, [VP]),
    "gc_engine_read": (C.c_int, [VP, C.c_int, P_F, P_F, P_F, P_F, P_I, P_F]),
    "gc_engine_release": (C.c_int, [VP, C.c_int]),
    "gc_engine_read_async": (C.c_int, [VP, C.c_int, P_F, P_F, P_F, P_F, P_I, P_F, C.POINTER(VP)]),
    "gc_event_query": (C.c_int, [VP]),
    "gc_event_wait": (C.c_int, [VP]),
    "gc_event_release": (C.c_int, [VP]),
    "gc_host_alloc": (VP, [C.c_longlong]),
    "gc_host_free": (C.c_int, [VP]),
    "gc_engine_bytes_in_use": (C.c_longlong, [VP]),
    "gc_engine_member_bytes": (C.c_longlong, [VP, C.c_int]),
    "gc_engine_config": (C.c_int, [VP, C.c_int, C.c_int, C.c_int]),
    "gc_engine_autotune": (C.c_int, [VP, C.c_int]),
    "gc_engine_variant": (C.c_int, [VP]),
    "gc_engine_num_variants": (C.c_int, []),
    "gc_engine_num_candidates": (C.c_int, []),
    "gc_engine_prepare": (C.c_int, [C.c_void_p]),
    "gc_engine_launches": (C.c_longlong, [VP]),
    "gc_engine_stream": (VP, [VP]),
    "gc_engine_add_nested_class": (C.c_int, [VP, C.c_int, C.POINTER(ChildDesc)]),
    "gc_engine_add_nested_member": (C.c_int, [VP, C.c_int, P_F, P_F, C.c_int, C.c_int, P_I, P_I, P_F,
                                              C.c_float]),
    "gc_engine_read_child": (C.c_int, [VP, C.c_int, P_F, P_F, P_F]),
    "gcomcot_fused_step_noalloc": (C.c_int, [C.c_int, VP, VP]),
    "gc_engine_member_health": (C.c_int, [VP, C.c_int, C.c_float]),
    "gc_okada_apply": (C.c_int, [VP, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, VP, VP, C.c_float, C.c_float, VP,
                                 VP, VP]),
    "gc_engine_set_class_axes": (C.c_int, [VP, C.c_int, P_F, P_F]),
    "gc_pair_layout_tile": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P_I]),
    "gc_engine_add_member_faults": (C.c_int, [VP, C.c_int, VP, C.c_int, C.c_int, C.c_int, P_I, P_F, C.c_float]),
}


def load():
    """Loads the library once; raises RuntimeError when it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is not built: run `make -C gpu-comcot_b200` "
                           "(or __graft_entry__.build())")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def fptr(a):
    return a.ctypes.data_as(P_F) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(P_I) if a is not None else None


def ref(v, ctype=C.c_int):
    return C.byref(ctype(v))
