"""Host mirror of the reference's interpolation / remeshing API.

Each function keeps the reference routine's name and argument list
(ppm/src/ppm_interp_p2m.f:127-163, ppm_interp_m2p.f:126-162,
ppm_rmsh_comp_weights.f:96-103, ppm_rmsh_remesh.f:90-124,
ppm_rmsh_create_part.f:90-171, ppm_map_field_ghost.f:61-89) and resolves the
specific variant the way the Fortran generic interface does: kind from the
array type (float64 'd' / float32 's'), scalar or vector from the rank of
``up`` (vector variants take ``lda``), 2D or 3D from the rank of ``field_up``.
Every call goes through libppmg.so; ``info`` is returned (0 on success, the
reference's severities otherwise; see ``last_error``).

Arrays use the Fortran layout: ``xp`` (ldxp, Np), ``up`` (lda, Np) or (Np,),
``field_up`` (lda, nx, ny[, nz], 1) (vector) or (nx, ny[, nz], 1) (scalar),
all column-major.  ``field_up``'s lower bounds default to 1-ghostsize as the
reference allocates them; pass ``field_lb`` for a different allocation.
numpy arrays run the synchronous host entry points; CUDA torch tensors run the
``_dev`` entry points on the current torch stream.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import halo
from . import params as P
from . import topo as _topo
from ._lib import int_array, last_error, lib  # noqa: F401

try:  # torch is optional: only the device-pointer path needs it
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_dev(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _colmajor(a) -> bool:
    if _is_dev(a) or (torch is not None and isinstance(a, torch.Tensor)):
        exp = 1
        for n, s in zip(a.shape, a.stride()):
            if n > 1 and s != exp:
                return False
            exp *= n
        return True
    return a.flags.f_contiguous


def _addr(a) -> int:
    if torch is not None and isinstance(a, torch.Tensor):
        return a.data_ptr()
    return a.ctypes.data


def _kind(a) -> str:
    dt = a.dtype
    if torch is not None and isinstance(a, torch.Tensor):
        if dt == torch.float64:
            return "d"
        if dt == torch.float32:
            return "s"
    else:
        if dt == np.float64:
            return "d"
        if dt == np.float32:
            return "s"
    raise TypeError(f"unsupported dtype {dt}")


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _bounds(field, dim, vector, ghostsize, field_lb):
    shape = tuple(field.shape)
    sp = shape[1:1 + dim] if vector else shape[:dim]
    lb = [1 - int(ghostsize[a]) for a in range(dim)] if field_lb is None else list(field_lb)
    ub = [lb[a] + int(sp[a]) - 1 for a in range(dim)]
    return int_array(lb, C.c_int64), int_array(ub, C.c_int64)


def _check(*arrays):
    for a in arrays:
        if a is not None and not _colmajor(a):
            raise ValueError("arrays must be column-major (Fortran order)")


def _split(up, args, name):
    if len(args) == 6:
        lda, topo_id, mesh_id, kernel, ghostsize, field_up = args
        return True, int(lda), topo_id, mesh_id, kernel, ghostsize, field_up
    if len(args) == 5:
        topo_id, mesh_id, kernel, ghostsize, field_up = args
        return False, 1, topo_id, mesh_id, kernel, ghostsize, field_up
    raise TypeError(f"{name}: wrong number of arguments")


def _slab_exchange(field_up, topo_id, mesh_id, ghostsize, lb, put):
    """The ghost exchange of a handle on one subdomain of several (every rank
    takes it, also after a local error, so that no neighbour waits for a
    message never sent)."""
    t, isub = _topo.local_sub(topo_id, mesh_id)
    fn = halo.put if put else halo.get
    fn({isub: field_up}, t, list(ghostsize), [int(v) for v in lb], halo.comm_for(topo_id, mesh_id))


def _python_exchange(topo_id, mesh_id):
    """A handle on one subdomain of several whose exchange runs in Python
    (ppm_legacy_b200.halo):
    one without a transport registered in the library (halo.CTransport),
    whose C calls then leave the exchange to their caller."""
    return _topo.is_slab(topo_id, mesh_id) and not halo.has_c_transport(topo_id, mesh_id)


def ppm_interp_p2m(xp, Np, up, *args, field_lb=None, exchange=True):
    """ppm_interp_p2m(xp, Np, up, [lda,] topo_id, mesh_id, kernel, ghostsize, field_up).

    On one subdomain of several the ghost put with the neighbours follows the
    local deposit (as the reference's P2M ends with ppm_map_field_ghost put);
    exchange=False leaves it to the caller (halo.put).
    """
    vector, lda, topo_id, mesh_id, kernel, ghostsize, field_up = _split(up, args, "ppm_interp_p2m")
    _check(xp, up, field_up)
    dim = field_up.ndim - (2 if vector else 1)
    k = _kind(xp)
    lb, ub = _bounds(field_up, dim, vector, ghostsize, field_lb)
    info = C.c_int(0)
    g = int_array(ghostsize)
    dev = _is_dev(xp)
    name = f"ppmg_interp_p2m_{k}{'v' if vector else 's'}_{dim}d"
    if vector:
        a = (_addr(xp), xp.shape[0], int(Np), _addr(up), up.shape[0], lda, topo_id, mesh_id,
             kernel, g, _addr(field_up), field_up.shape[0], lb, ub, C.byref(info))
        if dev:
            getattr(lib(), name + "_dev")(*a, _stream())
        else:
            getattr(lib(), name)(*a)
    else:
        if dev:
            raise TypeError("device (torch) arrays use the vector variant (pass lda)")
        getattr(lib(), name)(_addr(xp), xp.shape[0], int(Np), _addr(up), topo_id, mesh_id,
                             kernel, g, _addr(field_up), lb, ub, C.byref(info))
    if exchange and _python_exchange(topo_id, mesh_id):
        _slab_exchange(field_up, topo_id, mesh_id, ghostsize, lb, True)
    return info.value


def ppm_interp_m2p(xp, Np, up, *args, field_lb=None):
    """ppm_interp_m2p(xp, Np, up, [lda,] topo_id, mesh_id, kernel, ghostsize, field_up)."""
    vector, lda, topo_id, mesh_id, kernel, ghostsize, field_up = _split(up, args, "ppm_interp_m2p")
    _check(xp, up, field_up)
    dim = field_up.ndim - (2 if vector else 1)
    k = _kind(xp)
    lb, ub = _bounds(field_up, dim, vector, ghostsize, field_lb)
    info = C.c_int(0)
    g = int_array(ghostsize)
    dev = _is_dev(xp)
    name = f"ppmg_interp_m2p_{k}{'v' if vector else 's'}_{dim}d"
    if vector:
        a = (_addr(xp), xp.shape[0], int(Np), _addr(up), up.shape[0], lda, topo_id, mesh_id,
             kernel, g, _addr(field_up), field_up.shape[0], lb, ub, C.byref(info))
        if dev:
            getattr(lib(), name + "_dev")(*a, _stream())
        else:
            getattr(lib(), name)(*a)
    else:
        if dev:
            raise TypeError("device (torch) arrays use the vector variant (pass lda)")
        getattr(lib(), name)(_addr(xp), xp.shape[0], int(Np), _addr(up), topo_id, mesh_id,
                             kernel, g, _addr(field_up), lb, ub, C.byref(info))
    return info.value


def ppm_interp_p2m_adjoint(xp, Np, up, lda, topo_id, mesh_id, kernel, r_field, dw, dx,
                           ghostsize=(0, 0, 0), field_lb=None, exchange=True):
    """Adjoint of P2M (3D, FP64): dw = M2P(r), dx = sum_a up(a) grad_x W . r(a).

    On one subdomain of several the adjoint of P2M's ghost put is a ghost
    get: r's ghost layers along the cut axes are filled from the neighbours
    first (exchange=False: the caller's); r then needs those ghost layers
    (ghostsize / field_lb).
    """
    _check(xp, up, r_field, dw, dx)
    lb, ub = _bounds(r_field, 3, True, ghostsize, field_lb)
    if exchange and _topo.is_slab(topo_id, mesh_id):
        if halo.has_c_transport(topo_id, mesh_id):
            info = ppm_map_field_ghost(r_field, int(lda), topo_id, mesh_id, ghostsize,
                                       P.ppm_param_map_ghost_get, field_lb=field_lb)
            if info != 0:
                return info
        else:
            _slab_exchange(r_field, topo_id, mesh_id, ghostsize, lb, False)
    info = C.c_int(0)
    a = (_addr(xp), xp.shape[0], int(Np), _addr(up), up.shape[0], int(lda), topo_id, mesh_id,
         kernel, _addr(r_field), r_field.shape[0], lb, ub, _addr(dw), dw.shape[0], _addr(dx),
         dx.shape[0], C.byref(info))
    if _is_dev(xp):
        lib().ppmg_interp_p2m_adjoint_dv_3d_dev(*a, _stream())
    else:
        lib().ppmg_interp_p2m_adjoint_dv_3d(*a)
    return info.value


def ppm_map_field_ghost(field_up, *args, field_lb=None):
    """ppm_map_field_ghost(field_up, [lda,] topo_id, mesh_id, ghostsize, maptype).

    maptype ppm_param_map_ghost_get or ppm_param_map_ghost_put; the
    init/push/send/pop steps of the reference happen inside the call.  On a
    handle on one subdomain of several this is the exchange with the
    neighbours (ppm_legacy_b200.halo); uncut axes are periodic within it.
    """
    if len(args) == 5:
        lda, topo_id, mesh_id, ghostsize, maptype = args
        vector = True
    else:
        topo_id, mesh_id, ghostsize, maptype = args
        lda, vector = 1, False
    _check(field_up)
    dim = field_up.ndim - (2 if vector else 1)
    lb, ub = _bounds(field_up, dim, vector, ghostsize, field_lb)
    if _python_exchange(topo_id, mesh_id):
        if int(maptype) not in (P.ppm_param_map_ghost_get, P.ppm_param_map_ghost_put):
            return -2
        _slab_exchange(field_up, topo_id, mesh_id, ghostsize, lb,
                       int(maptype) == P.ppm_param_map_ghost_put)
        return 0
    info = C.c_int(0)
    ldf = field_up.shape[0] if vector else 1
    a = (_addr(field_up), ldf, int(lda), lb, ub, topo_id, mesh_id, int_array(ghostsize),
         int(maptype), C.byref(info))
    k = _kind(field_up)
    if _is_dev(field_up):
        getattr(lib(), f"ppmg_map_field_ghost_{k}_dev")(*a, _stream())
    else:
        getattr(lib(), f"ppmg_map_field_ghost_{k}")(*a)
    return info.value


def ppm_fdsolver_poisson(field_up, lda, topo_id, mesh_id, ghostsize, field_lb=None):
    """Solve lap(phi) = omega in place on the periodic 3D mesh
    (ppm_fdsolver_solve_3d with ppm_fdsolver_poisson_3d): field_up(lda, ...)
    holds omega at the unique nodes on entry and phi, with its periodic
    images in the ghost layers, on return.  float32 arrays: the single
    variant; torch CUDA arrays: the device twin."""
    _check(field_up)
    lb, ub = _bounds(field_up, 3, True, ghostsize, field_lb)
    k = _kind(field_up)
    info = C.c_int(0)
    a = (_addr(field_up), field_up.shape[0], int(lda), lb, ub, topo_id, mesh_id,
         int_array(ghostsize), C.byref(info))
    if _is_dev(field_up):
        getattr(lib(), f"ppmg_fdsolver_poisson_3d_{k}_dev")(*a, _stream())
    else:
        getattr(lib(), f"ppmg_fdsolver_poisson_3d_{k}")(*a)
    return info.value


def ppm_rmsh_comp_weights(xp, Np, topo_id, mesh_id, kernel, wx1_user=None, wx2_user=None,
                          wx3_user=None):
    """ppm_rmsh_comp_weights(xp, Np, topo_id, mesh_id, kernel[, wx1, wx2, wx3]).

    The weights stay in the library (like the reference's module state); user
    arrays, when given, have xp's dtype and shape (2ks, 1, Np+2ks), column-major.
    float32 positions select ppm_rmsh_comp_weights_s (FP32 weights).
    """
    _check(xp)
    k = _kind(xp)
    for u in (wx1_user, wx2_user, wx3_user):
        if u is not None and _kind(u) != k:
            raise TypeError("ppm_rmsh_comp_weights: wx arrays must have the dtype of xp")
    info = C.c_int(0)
    w = [None if u is None else _addr(u) for u in (wx1_user, wx2_user, wx3_user)]
    a = (_addr(xp), xp.shape[0], int(Np), topo_id, mesh_id, kernel, w[0], w[1], w[2],
         C.byref(info))
    if _is_dev(xp):
        getattr(lib(), f"ppmg_rmsh_comp_weights_{k}_dev")(*a, _stream())
    else:
        getattr(lib(), f"ppmg_rmsh_comp_weights_{k}")(*a)
    return info.value


def ppm_rmsh_remesh(xp, Np, up, *args, field_lb=None, exchange=True):
    """ppm_rmsh_remesh(xp, Np, up, [lda,] topo_id, mesh_id, kernel, ghostsize, field_up).

    The reference puts ``info`` before ``field_up``; here ``field_up`` must be
    preallocated by the caller (the reference's ppm_alloc grow step) and is
    overwritten entirely (zeroed, then the remeshed field).  float32 arrays
    select the single-precision variants (_ss/_sv), which need weights from
    a single-precision ppm_rmsh_comp_weights.  On one subdomain of several
    the ghost put with the neighbours follows (exchange=False: the caller's).
    """
    vector, lda, topo_id, mesh_id, kernel, ghostsize, field_up = _split(up, args, "ppm_rmsh_remesh")
    _check(xp, up, field_up)
    k = _kind(xp)
    if _kind(up) != k or _kind(field_up) != k:
        raise TypeError("ppm_rmsh_remesh: xp, up and field_up must share one dtype")
    dim = field_up.ndim - (2 if vector else 1)
    lb, ub = _bounds(field_up, dim, vector, ghostsize, field_lb)
    info = C.c_int(0)
    ldup = up.shape[0] if vector else 1
    ldf = field_up.shape[0] if vector else 1
    a = (_addr(xp), xp.shape[0], int(Np), _addr(up), ldup, lda, topo_id, mesh_id, kernel,
         int_array(ghostsize), _addr(field_up), ldf, lb, ub, C.byref(info))
    if _is_dev(xp):
        getattr(lib(), f"ppmg_rmsh_remesh_{k}v_{dim}d_dev")(*a, _stream())
    else:
        getattr(lib(), f"ppmg_rmsh_remesh_{k}v_{dim}d")(*a)
    if exchange and _python_exchange(topo_id, mesh_id):
        _slab_exchange(field_up, topo_id, mesh_id, ghostsize, lb, True)
    return info.value


def ppm_rmsh_create_part(field_up, topo_id, mesh_id, cutoff, lda=None, resetpos=False,
                         cutoff_weights=None, field_wp=None, ghostsize=(0, 0, 0),
                         field_lb=None):
    """ppm_rmsh_create_part: returns (info, np, up, xp, wp).

    The reference reallocates xp/up/wp in place (POINTER arguments); this
    mirror returns the new arrays: up (lda, np), xp (dim, np) when resetpos,
    wp (lda2, np) when field_wp is given.  A float32 field selects
    ppm_rmsh_create_part_s* (FP32 cutoffs and outputs).
    """
    vector = lda is not None
    lda = int(lda) if vector else 1
    _check(field_up)
    k = _kind(field_up)
    ft = np.float64 if k == "d" else np.float32
    dim = field_up.ndim - (2 if vector else 1)
    lb, ub = _bounds(field_up, dim, vector, ghostsize, field_lb)
    ldf = field_up.shape[0] if vector else 1
    cut = np.ascontiguousarray(cutoff, dtype=ft)
    cw = None if cutoff_weights is None else np.ascontiguousarray(cutoff_weights, dtype=ft)
    lda2 = 0
    ldfw = 0
    if field_wp is not None:
        _check(field_wp)
        if _kind(field_wp) != k:
            raise TypeError("ppm_rmsh_create_part: field_wp must have the dtype of field_up")
        lda2 = field_wp.shape[0] if field_wp.ndim == dim + 2 else 1
        ldfw = lda2
    n = C.c_int64(0)
    info = C.c_int(0)
    dev = _is_dev(field_up)
    if dev:
        fn = lambda *a: getattr(lib(), f"ppmg_rmsh_create_part_{k}_dev")(*a, _stream())  # noqa: E731
    else:
        fn = getattr(lib(), f"ppmg_rmsh_create_part_{k}")
    common = (_addr(field_up), ldf, lda, lb, ub, topo_id, mesh_id, cut.ctypes.data,
              None if cw is None else cw.ctypes.data, int(bool(resetpos)),
              None if field_wp is None else _addr(field_wp), ldfw, lda2)
    fn(*common, C.byref(n), None, None, None, C.byref(info))
    if info.value != 0:
        return info.value, 0, None, None, None
    npn = n.value
    if dev:
        # device outputs, column-major like the host arrays
        def cm(rows):
            return torch.empty((max(npn, 1), rows), dtype=field_up.dtype,
                               device=field_up.device).t()[:, :npn]
        up = cm(lda)
        xp = cm(dim) if resetpos else None
        wp = cm(max(lda2, 1)) if field_wp is not None else None
        fn(*common, C.byref(n), _addr(up) if npn else None,
           None if xp is None or not npn else _addr(xp),
           None if wp is None or not npn else _addr(wp), C.byref(info))
        if not vector:
            up = up.reshape(-1)
        return info.value, npn, up, xp, wp
    up = np.zeros((lda, npn), dtype=ft, order="F")
    xp = np.zeros((dim, npn), dtype=ft, order="F") if resetpos else None
    wp = np.zeros((max(lda2, 1), npn), dtype=ft, order="F") if field_wp is not None else None
    fn(*common, C.byref(n), up.ctypes.data, None if xp is None else xp.ctypes.data,
       None if wp is None else wp.ctypes.data, C.byref(info))
    if not vector:
        up = up.reshape(-1)
    return info.value, npn, up, xp, wp


def ppm_util_rank(xp, Np, xmin, xmax, Nm, Ngl):
    """ppm_util_rank{2,3}d: returns (info, lpdx, lhbx) with 1-based entries.
    float32 positions select ppm_util_rank{2,3}d_s (bounds and spacing in FP32);
    torch CUDA positions the device twins (lpdx, lhbx as device int32 tensors)."""
    _check(xp)
    k = _kind(xp)
    dim = len(Nm)
    nbox = 1
    for a in range(dim):
        nbox *= int(Nm[a]) + int(Ngl[a]) + int(Ngl[dim + a])
    dev = _is_dev(xp)
    if dev:
        lpdx = torch.zeros(max(int(Np), 1), dtype=torch.int32, device=xp.device)
        lhbx = torch.zeros(nbox + 1, dtype=torch.int32, device=xp.device)
    else:
        lpdx = np.zeros(max(int(Np), 1), dtype=np.int32)
        lhbx = np.zeros(nbox + 1, dtype=np.int32)
    ic = C.c_int64(0)
    info = C.c_int(0)
    ft = np.float64 if k == "d" else np.float32
    xmin = np.ascontiguousarray(xmin, dtype=ft)
    xmax = np.ascontiguousarray(xmax, dtype=ft)
    a = (_addr(xp), xp.shape[0], int(Np), xmin.ctypes.data, xmax.ctypes.data, int_array(Nm),
         int_array(Ngl), _addr(lpdx), _addr(lhbx), C.byref(ic), C.byref(info))
    if dev:
        getattr(lib(), f"ppmg_util_rank{dim}d_{k}_dev")(*a, _stream())
    else:
        getattr(lib(), f"ppmg_util_rank{dim}d_{k}")(*a)
    return info.value, lpdx[: ic.value], lhbx


def ppm_neighlist_clist(xp, Np, cutoff, lsymm, topo, isub=0):
    """ppm_neighlist_clist for one sub (ppm/src/ppm_neighlist_clist.f:300-440).

    Returns (info, lpdx, lhbx, Nm): cells of size >= cutoff over the sub,
    one ghost layer on every side (or only on the upper sides when lsymm).
    """
    dim = topo.dim
    xmin = topo.min_sub[isub, :dim]
    xmax = topo.max_sub[isub, :dim]
    cutoff = np.resize(np.asarray(cutoff, dtype=np.float64), dim)
    Nm = [max(int((xmax[a] - xmin[a]) / cutoff[a]), 1) for a in range(dim)]
    if lsymm:
        Ngl = [0] * dim + [1] * dim
    else:
        Ngl = [1] * (2 * dim)
    info, lpdx, lhbx = ppm_util_rank(xp, Np, xmin, xmax, Nm, Ngl)
    Nm_out = [Nm[a] + Ngl[a] + Ngl[dim + a] for a in range(dim)]
    return info, lpdx, lhbx, Nm_out


def set_precision(mode: int) -> int:
    """0 = FP64 (default), 1 = mixed (FP64 offsets, FP32 weights, compensated sums)."""
    info = C.c_int(0)
    lib().ppmg_set_precision(int(mode), C.byref(info))
    return info.value


def sync_status(topo_id, mesh_id, stream=None) -> int:
    """Waits for a handle's device-pointer calls and returns their data-dependent info."""
    info = C.c_int(0)
    if stream is None and torch is not None and torch.cuda.is_available():
        stream = _stream()
    lib().ppmg_sync_status(topo_id, mesh_id, stream, C.byref(info))
    return info.value


PPM = P  # the reference constants, e.g. PPM.ppm_param_rmsh_kernel_mp4
