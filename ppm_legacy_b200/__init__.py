"""B200-native particle <-> mesh interpolation and remeshing for PPM.

The hot path (P2M, M2P, remeshing, periodic ghost get/put, cell ranking) runs
as hand-written sm_100a CUDA kernels in libppmg.so behind a C-ABI
(include/ppmg.h).  This package is the host-side mirror of the reference's
API for that path.
"""
from . import halo, mapping, params
from .interp import (ppm_fdsolver_poisson, ppm_interp_m2p, ppm_interp_p2m, ppm_interp_p2m_adjoint,
                     ppm_map_field_ghost, ppm_neighlist_clist, ppm_rmsh_comp_weights,
                     ppm_rmsh_create_part, ppm_rmsh_remesh, ppm_util_rank, set_precision,
                     sync_status)
from ._lib import last_error, lib
from .topo import Topology, cartesian, register, unregister

__all__ = [
    "halo", "mapping", "params", "ppm_interp_p2m", "ppm_interp_m2p", "ppm_interp_p2m_adjoint",
    "ppm_map_field_ghost", "ppm_rmsh_comp_weights", "ppm_rmsh_remesh", "ppm_rmsh_create_part",
    "ppm_util_rank", "ppm_neighlist_clist", "ppm_fdsolver_poisson", "set_precision", "sync_status", "last_error",
    "lib", "Topology", "cartesian", "register", "unregister",
]
