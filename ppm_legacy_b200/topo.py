"""Topology and mesh geometry: the part of PPM's module state the hot path reads.

The reference keeps this state in ``ppm_module_data`` / ``ppm_module_data_mesh``
and fills it in ``ppm_topo_mkfield`` (ppm/src/ppm_topo_mkfield.f:311-319) and
``ppm_mesh_on_subs`` (ppm/src/ppm_mesh_on_subs.f:182-291).  This module builds
the same numbers for a cartesian decomposition of a box: per sub its extent
(``min_sub``/``max_sub``), which of its faces lie on the physical boundary
(``subs_bc``) and its mesh block (``istart`` = global 1-based index of its first
node, ``nnodes`` = Nc_sub + 1).

Arrays are sub-major: ``min_sub[isub, axis]``, ``subs_bc[isub, face]`` with faces
ordered (xmin, xmax, ymin, ymax, zmin, zmax) as in the reference.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import params as P


@dataclass
class Topology:
    dim: int
    min_phys: np.ndarray
    max_phys: np.ndarray
    Nm: np.ndarray  # global mesh nodes per axis (Nc + 1)
    bcdef: np.ndarray  # 2*dim boundary condition codes
    min_sub: np.ndarray  # (nsubs, 3)
    max_sub: np.ndarray
    subs_bc: np.ndarray  # (nsubs, 6): 1 if face lies on the physical boundary
    istart: np.ndarray  # (nsubs, 3) 1-based global index of first node
    nnodes: np.ndarray  # (nsubs, 3)
    topo_id: int = 1
    mesh_id: int = 1
    decomp: tuple = field(default=(1, 1, 1))

    @property
    def nsubs(self) -> int:
        return int(self.min_sub.shape[0])

    @property
    def Nc(self) -> np.ndarray:
        return self.Nm[: self.dim] - 1

    @property
    def h(self) -> np.ndarray:
        return (self.max_phys[: self.dim] - self.min_phys[: self.dim]) / self.Nc

    def field_shape(self, lda: int, ghostsize) -> tuple:
        """Shape of field_up(lda, 1-g:maxnn+g, ..., nsubs) (vector variant)."""
        g = np.asarray(ghostsize, dtype=np.int64)
        nn = self.nnodes.max(axis=0)[: self.dim]
        return (lda,) + tuple(int(nn[a] + 2 * g[a]) for a in range(self.dim)) + (self.nsubs,)


def cartesian(dim: int, Nc, decomp=None, min_phys=None, max_phys=None, bcdef=None,
              topo_id: int = 1, mesh_id: int = 1) -> Topology:
    """Cartesian split of a box into decomp[0] x decomp[1] (x decomp[2]) subs.

    The split follows mesh planes, as the reference's cartesian decomposition does
    for a field topology; sub s has index s = ix + nx*(iy + ny*iz).
    """
    Nc = np.asarray(Nc, dtype=np.int64).reshape(-1)
    if Nc.size == 1:
        Nc = np.repeat(Nc, dim)
    decomp = tuple(decomp) if decomp is not None else (1,) * dim
    min_phys = np.zeros(3) if min_phys is None else np.asarray(min_phys, dtype=np.float64)
    max_phys = np.ones(3) if max_phys is None else np.asarray(max_phys, dtype=np.float64)
    min_phys = np.resize(min_phys, 3).astype(np.float64)
    max_phys = np.resize(max_phys, 3).astype(np.float64)
    if bcdef is None:
        bcdef = [P.ppm_param_bcdef_periodic] * (2 * dim)
    bcdef6 = np.zeros(6, dtype=np.int32)
    bcdef6[: 2 * dim] = bcdef
    Nm = np.ones(3, dtype=np.int64)
    Nm[:dim] = Nc[:dim] + 1
    h = np.ones(3)
    h[:dim] = (max_phys[:dim] - min_phys[:dim]) / Nc[:dim]
    cuts = []
    for a in range(dim):
        nd = decomp[a]
        c = [int(round(Nc[a] * q / nd)) for q in range(nd + 1)]
        cuts.append(c)
    subs = []
    for iz in range(decomp[2] if dim == 3 else 1):
        for iy in range(decomp[1]):
            for ix in range(decomp[0]):
                subs.append((ix, iy, iz))
    ns = len(subs)
    min_sub = np.zeros((ns, 3))
    max_sub = np.zeros((ns, 3))
    subs_bc = np.zeros((ns, 6), dtype=np.int32)
    istart = np.ones((ns, 3), dtype=np.int32)
    nnodes = np.ones((ns, 3), dtype=np.int32)
    for s, idx in enumerate(subs):
        for a in range(dim):
            i0, i1 = cuts[a][idx[a]], cuts[a][idx[a] + 1]
            min_sub[s, a] = min_phys[a] + i0 * h[a] if i0 > 0 else min_phys[a]
            max_sub[s, a] = min_phys[a] + i1 * h[a] if i1 < Nc[a] else max_phys[a]
            subs_bc[s, 2 * a] = 1 if i0 == 0 else 0
            subs_bc[s, 2 * a + 1] = 1 if i1 == Nc[a] else 0
            # ppm_mesh_on_subs.f:219-291: ndata = NINT(len_sub/dx) + 1,
            # istart = NINT((min_sub - min_phys)/dx) + 1
            istart[s, a] = int(np.rint((min_sub[s, a] - min_phys[a]) / h[a])) + 1
            nnodes[s, a] = int(np.rint((max_sub[s, a] - min_sub[s, a]) / h[a])) + 1
    return Topology(dim=dim, min_phys=min_phys, max_phys=max_phys, Nm=Nm, bcdef=bcdef6,
                    min_sub=min_sub, max_sub=max_sub, subs_bc=subs_bc, istart=istart,
                    nnodes=nnodes, topo_id=topo_id, mesh_id=mesh_id,
                    decomp=tuple(decomp) + (1,) * (3 - len(decomp)))


# (topo_id, mesh_id) -> (Topology, local sub) of every registered handle
_registered: dict = {}


def local_sub(topo_id: int, mesh_id: int):
    """(Topology, isub) registered under (topo_id, mesh_id), or None."""
    return _registered.get((int(topo_id), int(mesh_id)))


def is_slab(topo_id: int, mesh_id: int) -> bool:
    """Whether the handle computes on one subdomain of several (a z-slab or
    any other cartesian cut): its exchange with the neighbours is then the
    caller's, or the registered transport's."""
    r = local_sub(topo_id, mesh_id)
    return r is not None and r[0].nsubs > 1


def register(topo: Topology, isub=None) -> int:
    """Hand the geometry to libppmg (ppmg_mesh_register); returns info.

    isub: the subdomain this process's GPU computes on (needed when the
    topology has several subdomains: a cartesian decomposition).
    """
    import ctypes as C

    from ._lib import int_array, lib

    info = C.c_int(0)
    ms = np.ascontiguousarray(topo.min_sub, dtype=np.float64)
    Ms = np.ascontiguousarray(topo.max_sub, dtype=np.float64)
    mp = np.ascontiguousarray(topo.min_phys, dtype=np.float64)
    Mp = np.ascontiguousarray(topo.max_phys, dtype=np.float64)
    lib().ppmg_mesh_register(
        int(topo.topo_id), int(topo.mesh_id), int(topo.dim), mp.ctypes.data, Mp.ctypes.data,
        int_array(topo.Nm), int_array(topo.bcdef), int(topo.nsubs), ms.ctypes.data,
        Ms.ctypes.data, int_array(topo.subs_bc.reshape(-1)), int_array(topo.istart.reshape(-1)),
        int_array(topo.nnodes.reshape(-1)), C.byref(info))
    if info.value == 0 and isub is not None:
        lib().ppmg_mesh_set_local_sub(int(topo.topo_id), int(topo.mesh_id), int(isub),
                                      C.byref(info))
    if info.value == 0:
        _registered[(int(topo.topo_id), int(topo.mesh_id))] = (
            topo, 0 if isub is None else int(isub))
    return info.value


def unregister(topo: Topology) -> int:
    import ctypes as C

    from ._lib import lib

    info = C.c_int(0)
    lib().ppmg_mesh_unregister(int(topo.topo_id), int(topo.mesh_id), C.byref(info))
    _registered.pop((int(topo.topo_id), int(topo.mesh_id)), None)
    return info.value
