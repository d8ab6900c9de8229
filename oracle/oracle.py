"""ctypes wrapper of the CPU restatement (libppm_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/ (as the checker) and by bench.py's
CPU-baseline leg.  Parity with the reference is unpinned against reference
outputs (none exist; the Fortran reference cannot be built here) and pinned by
exact-rational golden vectors plus analytic identities instead.

Arrays follow the Fortran layout: xp(ldxp, Np), up(lda, Np) and
field(lda, lb:ub per axis, nsubs) as F-ordered numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libppm_oracle.so")


def build(force: bool = False) -> str:
    if force or not os.path.exists(_SO):
        subprocess.run(["make", "-C", _HERE], check=True, capture_output=True)
    return _SO


class _Geom(C.Structure):
    _fields_ = [
        ("dim", C.c_int), ("nsubs", C.c_int),
        ("min_phys", C.c_double * 3), ("max_phys", C.c_double * 3),
        ("Nm", C.c_int * 3), ("bcdef", C.c_int * 6),
        ("min_sub", C.POINTER(C.c_double)), ("max_sub", C.POINTER(C.c_double)),
        ("subs_bc", C.POINTER(C.c_int)), ("istart", C.POINTER(C.c_int)),
        ("nnodes", C.POINTER(C.c_int)),
    ]


class _Field(C.Structure):
    _fields_ = [("lda", C.c_int), ("lb", C.c_int * 3), ("ub", C.c_int * 3)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
    return _lib


def _ptr(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Geom:
    """Holds the ctypes geometry struct and keeps its arrays alive."""

    def __init__(self, topo):
        self.topo = topo
        self._min_sub = np.ascontiguousarray(topo.min_sub, dtype=np.float64)
        self._max_sub = np.ascontiguousarray(topo.max_sub, dtype=np.float64)
        self._subs_bc = np.ascontiguousarray(topo.subs_bc, dtype=np.int32)
        self._istart = np.ascontiguousarray(topo.istart, dtype=np.int32)
        self._nnodes = np.ascontiguousarray(topo.nnodes, dtype=np.int32)
        g = _Geom()
        g.dim = topo.dim
        g.nsubs = topo.nsubs
        for a in range(3):
            g.min_phys[a] = float(topo.min_phys[a])
            g.max_phys[a] = float(topo.max_phys[a])
            g.Nm[a] = int(topo.Nm[a])
        for f in range(6):
            g.bcdef[f] = int(topo.bcdef[f])
        g.min_sub = _ptr(self._min_sub, C.c_double)
        g.max_sub = _ptr(self._max_sub, C.c_double)
        g.subs_bc = _ptr(self._subs_bc, C.c_int)
        g.istart = _ptr(self._istart, C.c_int)
        g.nnodes = _ptr(self._nnodes, C.c_int)
        self.g = g

    def ref(self):
        return C.byref(self.g)


def field_desc(lda, lb, ub):
    f = _Field()
    f.lda = lda
    for a in range(3):
        f.lb[a] = int(lb[a]) if a < len(lb) else 0
        f.ub[a] = int(ub[a]) if a < len(ub) else 0
    return f


def field_bounds(topo, ghost):
    nn = topo.nnodes.max(axis=0)
    lb = [1 - int(ghost[a]) for a in range(topo.dim)]
    ub = [int(nn[a]) + int(ghost[a]) for a in range(topo.dim)]
    return lb, ub


def new_field(topo, lda, ghost, dtype=np.float64):
    lb, ub = field_bounds(topo, ghost)
    shape = (lda,) + tuple(ub[a] - lb[a] + 1 for a in range(topo.dim)) + (topo.nsubs,)
    return np.zeros(shape, dtype=dtype, order="F"), lb, ub


def _f64(a):
    return np.asfortranarray(a, dtype=np.float64)


def _f32(a):
    return np.asfortranarray(a, dtype=np.float32)


def _ghost(ghost):
    g = np.zeros(3, dtype=np.int32)
    g[: len(ghost)] = ghost
    return g


class OracleError(RuntimeError):
    def __init__(self, info, errno):
        super().__init__(f"oracle info={info} errno={errno}")
        self.info, self.errno = info, errno


def p2m(topo, xp, up, kernel, ghost, dtype=np.float64, put=True, field_lb_ub=None):
    """Reference P2M: returns (field, lb, ub).  xp (ldxp, Np), up (lda, Np)."""
    G = Geom(topo)
    cast = _f64 if dtype == np.float64 else _f32
    xp = cast(xp)
    up = cast(up if up.ndim == 2 else up.reshape(1, -1))
    lda, np_ = up.shape
    if field_lb_ub is None:
        field, lb, ub = new_field(topo, lda, ghost, dtype)
    else:
        lb, ub = field_lb_ub
        shape = (lda,) + tuple(ub[a] - lb[a] + 1 for a in range(topo.dim)) + (topo.nsubs,)
        field = np.zeros(shape, dtype=dtype, order="F")
    fd = field_desc(lda, lb, ub)
    err = C.c_int(0)
    gh = _ghost(ghost)
    ct = C.c_double if dtype == np.float64 else C.c_float
    if dtype == np.float64:
        fn = lib().orc_p2m_d if put else lib().orc_p2m_noput_d
    else:
        fn = lib().orc_p2m_s
    info = fn(G.ref(), _ptr(xp, ct), xp.shape[0], np_, _ptr(up, ct), lda, kernel,
              _ptr(gh, C.c_int), _ptr(field, ct), C.byref(fd), C.byref(err))
    if info != 0:
        raise OracleError(info, err.value)
    return field, lb, ub


def m2p(topo, xp, field, lb, ub, lda, kernel, ghost, dtype=np.float64):
    """Reference M2P on the field as given (ghosts must already be filled)."""
    G = Geom(topo)
    cast = _f64 if dtype == np.float64 else _f32
    xp = cast(xp)
    field = cast(field)
    np_ = xp.shape[1]
    up = np.zeros((lda, np_), dtype=dtype, order="F")
    fd = field_desc(lda, lb, ub)
    err = C.c_int(0)
    gh = _ghost(ghost)
    ct = C.c_double if dtype == np.float64 else C.c_float
    fn = lib().orc_m2p_d if dtype == np.float64 else lib().orc_m2p_s
    info = fn(G.ref(), _ptr(xp, ct), xp.shape[0], np_, _ptr(up, ct), lda, kernel,
              _ptr(gh, C.c_int), _ptr(field, ct), C.byref(fd), C.byref(err))
    if info != 0:
        raise OracleError(info, err.value)
    return up


def _check_inplace(field):
    if not field.flags.f_contiguous:
        raise ValueError("field must be a Fortran-ordered (column-major) array")


def ghost_get(topo, field, lb, ub, ghost):
    _check_inplace(field)
    G = Geom(topo)
    fd = field_desc(field.shape[0], lb, ub)
    gh = _ghost(ghost)
    if field.dtype == np.float64:
        lib().orc_ghost_get_d(G.ref(), _ptr(field, C.c_double), C.byref(fd), _ptr(gh, C.c_int))
    else:
        lib().orc_ghost_get_s(G.ref(), _ptr(field, C.c_float), C.byref(fd), _ptr(gh, C.c_int))
    return field


def ghost_put(topo, field, lb, ub, ghost):
    _check_inplace(field)
    G = Geom(topo)
    fd = field_desc(field.shape[0], lb, ub)
    gh = _ghost(ghost)
    if field.dtype == np.float64:
        lib().orc_ghost_put_d(G.ref(), _ptr(field, C.c_double), C.byref(fd), _ptr(gh, C.c_int))
    else:
        lib().orc_ghost_put_s(G.ref(), _ptr(field, C.c_float), C.byref(fd), _ptr(gh, C.c_int))
    return field


def assign(topo, xp):
    """Particle -> sub lists; float32 positions use the single-precision tests."""
    G = Geom(topo)
    k = "s" if np.asarray(xp).dtype == np.float32 else "d"
    xp = np.asfortranarray(xp, dtype=np.float32 if k == "s" else np.float64)
    np_ = xp.shape[1]
    lst = np.zeros(max(np_, 1), dtype=np.int32)
    si = np.zeros(topo.nsubs, dtype=np.int32)
    err = C.c_int(0)
    info = getattr(lib(), f"orc_assign_{k}")(G.ref(), _ptr(xp, _ctk(k)), xp.shape[0], np_,
                                             _ptr(lst, C.c_int), _ptr(si, C.c_int),
                                             C.byref(err))
    if info != 0:
        raise OracleError(info, err.value)
    return lst[:np_], si


def _kind(*arrays):
    """'s' when the arrays are float32 (the reference's single variants), else 'd'."""
    return "s" if any(a is not None and np.asarray(a).dtype == np.float32 for a in arrays) else "d"


def _fk(a, k):
    return np.asfortranarray(a, dtype=np.float32 if k == "s" else np.float64)


def _ctk(k):
    return C.c_float if k == "s" else C.c_double


def comp_weights(topo, xp, kernel):
    """Returns (wx list per axis shaped (2ks, nsubs, maxp+2ks) F-order, list, store_info).
    float32 positions run the single-precision routine (ppm_rmsh_comp_weights_s)."""
    G = Geom(topo)
    k = _kind(xp)
    xp = _fk(xp, k)
    lst, si = assign(topo, xp)
    maxp = int(si.max()) if si.size else 0
    ks = 2 if kernel == 2 else 1
    shape = (2 * ks, topo.nsubs, maxp + 2 * ks)
    ct = _ctk(k)
    wx = [np.zeros(shape, order="F", dtype=xp.dtype) for _ in range(3)]
    info = getattr(lib(), f"orc_comp_weights_{k}")(
        G.ref(), _ptr(xp, ct), xp.shape[0], xp.shape[1], kernel, _ptr(lst, C.c_int),
        _ptr(si, C.c_int), maxp, _ptr(wx[0], ct), _ptr(wx[1], ct), _ptr(wx[2], ct))
    if info != 0:
        raise OracleError(info, 0)
    return wx, lst, si


def remesh(topo, xp, up, kernel, ghost, wx, lst, si):
    G = Geom(topo)
    k = _kind(xp)
    xp = _fk(xp, k)
    up = _fk(up if up.ndim == 2 else up.reshape(1, -1), k)
    lda = up.shape[0]
    field, lb, ub = new_field(topo, lda, ghost)
    field = _fk(field, k)
    fd = field_desc(lda, lb, ub)
    gh = _ghost(ghost)
    err = C.c_int(0)
    maxp = int(si.max()) if si.size else 0
    ct = _ctk(k)
    wx = [_fk(w, k) for w in wx]
    info = getattr(lib(), f"orc_remesh_{k}")(
        G.ref(), _ptr(xp, ct), xp.shape[0], xp.shape[1], _ptr(up, ct), lda, kernel,
        _ptr(gh, C.c_int), _ptr(lst, C.c_int), _ptr(si, C.c_int), maxp, _ptr(wx[0], ct),
        _ptr(wx[1], ct), _ptr(wx[2], ct), _ptr(field, ct), C.byref(fd), C.byref(err))
    if info != 0:
        raise OracleError(info, err.value)
    return field, lb, ub


def create_part(topo, field, lb, ub, cutoff, cutoff_weights=None, resetpos=True,
                field_wp=None):
    G = Geom(topo)
    k = _kind(field)
    ct = _ctk(k)
    dt = np.float32 if k == "s" else np.float64
    field = _fk(field, k)
    lda = field.shape[0]
    fd = field_desc(lda, lb, ub)
    cut = np.asarray(cutoff, dtype=dt)
    cw = None if cutoff_weights is None else np.ascontiguousarray(cutoff_weights, dtype=dt)
    fw = None if field_wp is None else _fk(field_wp, k)
    lda2 = 0 if fw is None else fw.shape[0]
    npo = C.c_int(0)
    cwp = _ptr(cw, ct) if cw is not None else None
    fwp = _ptr(fw, ct) if fw is not None else None
    fn = getattr(lib(), f"orc_create_part_{k}")
    fn(G.ref(), _ptr(field, ct), C.byref(fd), _ptr(cut, ct), cwp, int(resetpos), fwp, lda2,
       C.byref(npo), None, None, None)
    n = npo.value
    up = np.zeros((lda, n), order="F", dtype=dt)
    xp = np.zeros((topo.dim, n), order="F", dtype=dt)
    wp = np.zeros((max(lda2, 1), n), order="F", dtype=dt) if fw is not None else None
    fn(G.ref(), _ptr(field, ct), C.byref(fd), _ptr(cut, ct), cwp, int(resetpos), fwp, lda2,
       C.byref(npo), _ptr(up, ct), _ptr(xp, ct), _ptr(wp, ct) if wp is not None else None)
    return n, up, (xp if resetpos else None), wp


def rank(xp, xmin, xmax, Nm, Ngl):
    """ppm_util_rank{2,3}d: returns (lpdx 1-based, lhbx 1-based, icount).
    float32 positions run ppm_util_rank{2,3}d_s (bounds and spacing in FP32)."""
    k = _kind(xp)
    ct = _ctk(k)
    xp = _fk(xp, k)
    dim = len(Nm)
    Ngl = np.asarray(Ngl, dtype=np.int32)
    Nm = np.asarray(Nm, dtype=np.int32)
    nbox = int(np.prod([Nm[a] + Ngl[a] + Ngl[dim + a] for a in range(dim)]))
    lpdx = np.zeros(max(xp.shape[1], 1), dtype=np.int32)
    lhbx = np.zeros(nbox + 1, dtype=np.int32)
    ic = C.c_int(0)
    xmin = np.ascontiguousarray(xmin, dtype=xp.dtype)
    xmax = np.ascontiguousarray(xmax, dtype=xp.dtype)
    fn = getattr(lib(), f"orc_rank{dim}d_{k}")
    fn(_ptr(xp, ct), xp.shape[0], xp.shape[1], _ptr(xmin, ct),
       _ptr(xmax, ct), _ptr(Nm, C.c_int), _ptr(Ngl, C.c_int), _ptr(lpdx, C.c_int),
       _ptr(lhbx, C.c_int), C.byref(ic))
    return lpdx[: ic.value], lhbx, ic.value


def p2m_adjoint(topo, xp, up, r_field, lb, ub, kernel):
    G = Geom(topo)
    xp = _f64(xp)
    up = _f64(up if up.ndim == 2 else up.reshape(1, -1))
    lda, np_ = up.shape
    r = _f64(r_field)
    fd = field_desc(lda, lb, ub)
    dw = np.zeros((lda, np_), order="F")
    dx = np.zeros((topo.dim, np_), order="F")
    lib().orc_p2m_adjoint_d(G.ref(), _ptr(xp, C.c_double), xp.shape[0], np_, _ptr(up, C.c_double),
                            lda, kernel, _ptr(r, C.c_double), C.byref(fd), _ptr(dw, C.c_double),
                            _ptr(dx, C.c_double))
    return dw, dx


def roundtrip_owned(topo, xp, owner, up, kernel, ghost, nthreads=0):
    """CPU baseline: P2M + ghost put + ghost get + M2P, one thread per sub."""
    G = Geom(topo)
    xp = _f64(xp)
    up = _f64(up)
    lda, np_ = up.shape
    field, lb, ub = new_field(topo, lda, ghost)
    fd = field_desc(lda, lb, ub)
    gh = _ghost(ghost)
    owner = np.ascontiguousarray(owner, dtype=np.int32)
    out = np.zeros((lda, np_), order="F")
    info = lib().orc_roundtrip_owned_d(G.ref(), _ptr(xp, C.c_double), xp.shape[0], np_,
                                       _ptr(owner, C.c_int), _ptr(up, C.c_double), lda, kernel,
                                       _ptr(gh, C.c_int), _ptr(field, C.c_double), C.byref(fd),
                                       _ptr(out, C.c_double), int(nthreads))
    if info != 0:
        raise OracleError(info, 0)
    return field, lb, ub, out


def poisson(U, lengths):
    """lap(phi) = omega on a periodic mesh, restated from the spectral step of
    ppm_fdsolver_poisson_3d.f:60-82 (every mode times -1/|k|^2, k_a = 2 pi /
    L_a times the wave number folded to |.| <= N_a/2, zero mode 0) between a
    forward and a backward FFT normalised by 1/(Nx Ny Nz).  U(lda, Nx, Ny, Nz)
    holds omega at the unique nodes; returns phi there (numpy FFTs)."""
    U = np.asarray(U, dtype=np.float64)
    nx, ny, nz = U.shape[1:]
    k = [2.0 * np.pi / float(lengths[a]) *
         np.minimum(np.arange(n), n - np.arange(n)).astype(np.float64)
         for a, n in enumerate((nx, ny, nz))]
    kx = k[0][: nx // 2 + 1]  # the real-to-complex axis: 0 .. nx/2
    k2 = kx[:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2
    k2[0, 0, 0] = 1.0
    out = np.empty_like(U)
    for a in range(U.shape[0]):
        spec = np.fft.rfftn(U[a], axes=(2, 1, 0))
        spec = -spec / k2
        spec[0, 0, 0] = 0.0
        out[a] = np.fft.irfftn(spec, s=(nz, ny, nx), axes=(2, 1, 0))
    return out

