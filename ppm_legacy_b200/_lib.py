"""ctypes binding of libppmg.so (the C-ABI declared in include/ppmg.h).

The library is built in-tree (``python -m ppm_legacy_b200.build``).  Loading
fails loudly when it is missing: there is no CPU fallback for the hot path.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libppmg.so")

_i = C.c_int
_i64 = C.c_int64
_pi = C.POINTER(C.c_int)
_pi64 = C.POINTER(C.c_int64)
_pd = C.c_void_p  # data pointers are passed as raw addresses (host or device)
_vp = C.c_void_p

# name -> argtypes (restype int for the few functions that return a value)
_P2M_V = [_pd, _i64, _i64, _pd, _i64, _i, _i, _i, _i, _pi, _pd, _i64, _pi64, _pi64, _pi]
_P2M_S = [_pd, _i64, _i64, _pd, _i, _i, _i, _pi, _pd, _pi64, _pi64, _pi]
_ADJ = [_pd, _i64, _i64, _pd, _i64, _i, _i, _i, _i, _pd, _i64, _pi64, _pi64, _pd, _i64, _pd,
        _i64, _pi]
_GHOST = [_pd, _i64, _i, _pi64, _pi64, _i, _i, _pi, _i, _pi]
_RANK = [_pd, _i64, _i64, _pd, _pd, _pi, _pi, _pd, _pd, _pi64, _pi]

SIGNATURES = {
    "ppmg_version": ([], _i),
    "ppmg_last_error": ([_pi, C.c_char_p, _i], _i),
    "ppmg_set_precision": ([_i, _pi], None),
    "ppmg_get_precision": ([], _i),
    "ppmg_launch_count": ([], _i64),
    "ppmg_mesh_register": ([_i, _i, _i, _pd, _pd, _pi, _pi, _i, _pd, _pd, _pi, _pi, _pi, _pi],
                           None),
    "ppmg_mesh_unregister": ([_i, _i, _pi], None),
    "ppmg_mesh_set_local_sub": ([_i, _i, _i, _pi], None),
    "ppmg_sync_status": ([_i, _i, _vp, _pi], None),
    "ppmg_halo_set_transport": ([_i, _i, _vp, _vp, _pi], None),
    "ppmg_halo_plan": ([_i, _pd, _pd, _i, _i, _i64, _pi64, _pi64, _pi, _i, _pi64, _pi, _pi, _pi64,
                        _pi, _pi, _pi64, _pi], None),
    "ppmg_halo_neighbours": ([_i, _pd, _pd, _pi, _i, _i, _vp, _pi, _pi], None),
    "ppmg_halo_plan_boxes": ([_i, _pd, _pd, _pi, _i, _pi, _i, _i, _vp, _pi, _vp, _pi, _pi],
                             None),
    "ppmg_interp_p2m_adjoint_dv_3d": (_ADJ, None),
    "ppmg_interp_p2m_adjoint_dv_3d_dev": (_ADJ + [_vp], None),
    "ppmg_map_field_ghost_d": (_GHOST, None),
    "ppmg_map_field_ghost_s": (_GHOST, None),
    "ppmg_map_field_ghost_d_dev": (_GHOST + [_vp], None),
    "ppmg_map_field_ghost_s_dev": (_GHOST + [_vp], None),
    "ppmg_rmsh_comp_weights_d": ([_pd, _i64, _i64, _i, _i, _i, _pd, _pd, _pd, _pi], None),
    "ppmg_rmsh_comp_weights_d_dev": ([_pd, _i64, _i64, _i, _i, _i, _pd, _pd, _pd, _pi, _vp],
                                     None),
    "ppmg_rmsh_comp_weights_s": ([_pd, _i64, _i64, _i, _i, _i, _pd, _pd, _pd, _pi], None),
    "ppmg_rmsh_comp_weights_s_dev": ([_pd, _i64, _i64, _i, _i, _i, _pd, _pd, _pd, _pi, _vp],
                                     None),
    "ppmg_rmsh_remesh_sv_3d": (_P2M_V, None),
    "ppmg_rmsh_remesh_sv_2d": (_P2M_V, None),
    "ppmg_rmsh_remesh_sv_3d_dev": (_P2M_V + [_vp], None),
    "ppmg_rmsh_remesh_sv_2d_dev": (_P2M_V + [_vp], None),
    "ppmg_rmsh_remesh_dv_3d": (_P2M_V, None),
    "ppmg_rmsh_remesh_dv_2d": (_P2M_V, None),
    "ppmg_rmsh_remesh_dv_3d_dev": (_P2M_V + [_vp], None),
    "ppmg_rmsh_remesh_dv_2d_dev": (_P2M_V + [_vp], None),
    "ppmg_rmsh_create_part_d": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pd, _pd, _i, _pd, _i64, _i,
                                 _pi64, _pd, _pd, _pd, _pi], None),
    "ppmg_rmsh_create_part_d_dev": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pd, _pd, _i, _pd, _i64,
                                     _i, _pi64, _pd, _pd, _pd, _pi, _vp], None),
    "ppmg_rmsh_create_part_s": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pd, _pd, _i, _pd, _i64, _i,
                                 _pi64, _pd, _pd, _pd, _pi], None),
    "ppmg_rmsh_create_part_s_dev": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pd, _pd, _i, _pd, _i64,
                                     _i, _pi64, _pd, _pd, _pd, _pi, _vp], None),
    "ppmg_util_rank3d_d": (_RANK, None),
    "ppmg_util_rank2d_d": (_RANK, None),
    "ppmg_util_rank3d_s": (_RANK, None),
    "ppmg_util_rank2d_s": (_RANK, None),
    "ppmg_util_rank3d_d_dev": (_RANK + [_vp], None),
    "ppmg_fdsolver_poisson_3d_d": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pi, _pi], None),
    "ppmg_fdsolver_poisson_3d_s": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pi, _pi], None),
    "ppmg_fdsolver_poisson_3d_d_dev": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pi, _pi, _vp], None),
    "ppmg_fdsolver_poisson_3d_s_dev": ([_pd, _i64, _i, _pi64, _pi64, _i, _i, _pi, _pi, _vp], None),
    "ppmg_map_part_route_d_dev": ([_pd, _i64, _i64, _i, _i, _pd, _pi64, _pi, _vp], None),
    "ppmg_map_part_route_s_dev": ([_pd, _i64, _i64, _i, _i, _pd, _pi64, _pi, _vp], None),
    "ppmg_map_part_global_route_d_dev": ([_pd, _i64, _i64, _i, _i, _pd, _pi64, _pi, _vp], None),
    "ppmg_map_part_global_route_s_dev": ([_pd, _i64, _i64, _i, _i, _pd, _pi64, _pi, _vp], None),
    "ppmg_map_part_partial_route_d_dev": ([_pd, _i64, _i64, _i, _i, _pd, _pi64, _pi, _vp], None),
    "ppmg_map_part_partial_route_s_dev": ([_pd, _i64, _i64, _i, _i, _pd, _pi64, _pi, _vp], None),
    "ppmg_map_part_gather_d_dev": ([_pd, _i64, _i, _pd, _i64, _pd, _i64, _pi, _vp], None),
    "ppmg_map_part_gather_s_dev": ([_pd, _i64, _i, _pd, _i64, _pd, _i64, _pi, _vp], None),
    "ppmg_util_rank2d_d_dev": (_RANK + [_vp], None),
    "ppmg_util_rank3d_s_dev": (_RANK + [_vp], None),
    "ppmg_util_rank2d_s_dev": (_RANK + [_vp], None),
    "ppmg_interp_p2m_dv_3d_noalloc": (_P2M_V + [_vp], None),
    "ppmg_kernel_timing": ([_i], None),
    "ppmg_kernel_timing_read": ([_i, C.POINTER(C.c_double), _pi64], _i),
}
for _k in ("ss", "sv", "ds", "dv"):
    for _d in ("2d", "3d"):
        SIGNATURES[f"ppmg_interp_p2m_{_k}_{_d}"] = (_P2M_V if _k[1] == "v" else _P2M_S, None)
        SIGNATURES[f"ppmg_interp_m2p_{_k}_{_d}"] = (_P2M_V if _k[1] == "v" else _P2M_S, None)
        if _k[1] == "v":
            SIGNATURES[f"ppmg_interp_p2m_{_k}_{_d}_dev"] = (_P2M_V + [_vp], None)
            SIGNATURES[f"ppmg_interp_m2p_{_k}_{_d}_dev"] = (_P2M_V + [_vp], None)

_lib = None


class LibraryMissing(RuntimeError):
    pass


def lib():
    """The loaded library (raises LibraryMissing when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                f"{LIB_PATH} is missing: build it with `python -m ppm_legacy_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (args, res) in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def last_error():
    """(info, errno, message) of the calling thread's last library call."""
    e = C.c_int(0)
    buf = C.create_string_buffer(512)
    info = lib().ppmg_last_error(C.byref(e), buf, 512)
    return info, e.value, buf.value.decode(errors="replace")


def int_array(vals, ct=C.c_int):
    vals = list(vals)
    return (ct * max(len(vals), 1))(*vals)
