"""Particle redistribution between subdomains: the host mirror of
``ppm_map_part_partial`` (ppm/src/ppm_map_part_partial.f with the push /
send / pop of ppm_map_part_push.f, ppm_map_part_send.f, ppm_map_part_pop.f)
and ``ppm_map_part_global`` for the decompositions of ppm_legacy_b200.halo.

After particles moved (and the client imposed the periodic bounds, as in
PPM), every particle goes to the subdomain that contains it among its own
and the neighbours: on slabs along z the two z neighbours
(ppmg_map_part_route), on other cartesian cuts up to 26 neighbours
(ppmg_map_part_partial_route).  The routing and the packing run on the GPU
(one stable grouping of the particles by destination, then a gather per
array, ppmg_map_part_gather); the blocks travel with the transports of
ppm_legacy_b200.halo.  Sizes go first, then the particle blocks, in the same
operation order on every rank.

The new particle list is the kept particles in their order, then the
arrivals: on slabs those from the slab below, then those from the slab
above; on other cuts by ascending source subdomain.  (The reference orders
arrivals by its communication sequence; the set of particles is the same.)
"""
from __future__ import annotations

import ctypes as C

from . import halo
from . import topo as _topo
from ._lib import lib

TAG_SIZE, TAG_DATA = 40, 60


def _rows(a):
    """The C-ordered (n, ld) tensor behind a column-major (ld, n) array."""
    t = a.t()
    if not t.is_contiguous():
        raise ValueError("particle arrays must be column-major (Fortran order)")
    return t


def device_gather(src, perm, n):
    """Columns src[:, perm[:n]] as a new column-major array
    (ppmg_map_part_gather on the current stream)."""
    import torch
    ld = src.shape[0]
    out = torch.empty((max(n, 1), ld), dtype=src.dtype, device=src.device).t()[:, :n]
    if n == 0:
        return out
    if src.element_size() not in (4, 8):
        raise TypeError("particle arrays must have 4- or 8-byte elements")
    k = "d" if src.element_size() == 8 else "s"
    info = C.c_int(0)
    getattr(lib(), f"ppmg_map_part_gather_{k}_dev")(
        src.data_ptr(), src.stride(1), ld, perm.data_ptr(), n, out.data_ptr(), ld,
        C.byref(info), torch.cuda.current_stream().cuda_stream)
    if info.value:
        raise RuntimeError("ppmg_map_part_gather failed")
    return out


def device_route(topo_id, mesh_id, xp):
    """(info, perm, [kept, to below, to above, in none]) of the slab's
    particles (ppmg_map_part_route on the current stream)."""
    import torch
    n = int(xp.shape[1])
    perm = torch.empty(max(n, 1), dtype=torch.int32, device=xp.device)
    cnt = (C.c_int64 * 4)()
    info = C.c_int(0)
    k = "d" if xp.dtype == torch.float64 else "s"
    getattr(lib(), f"ppmg_map_part_route_{k}_dev")(
        xp.data_ptr(), xp.stride(1), n, int(topo_id), int(mesh_id), perm.data_ptr(), cnt,
        C.byref(info), torch.cuda.current_stream().cuda_stream)
    return info.value, perm, [int(c) for c in cnt]


def map_subs(parts: dict, topo, comm, route=None, gather=device_gather):
    """parts {isub: (topo_id, mesh_id, xp, [props])} of the subdomains this
    process holds; returns (info, {isub: (xp_new, [props_new])}).  route /
    gather: the device kernels (replaceable, for tests of the exchange on
    CPU; route takes (topo_id, mesh_id, xp) on slabs, (topo_id, mesh_id, xp,
    nsubs) on other cuts)."""
    if not halo.is_slab_topology(topo):
        return map_global(parts, topo, comm, route=route or device_route_partial, gather=gather,
                          peers=lambda s: halo.cart_neighbours(topo, s))
    route = route or device_route
    import torch
    info_all = 0
    packed, counts = {}, {}
    for s, (tid, mid, xp, props) in parts.items():
        n = int(xp.shape[1])
        info, perm, cnt = route(tid, mid, xp)
        if info and not info_all:
            info_all = info
        counts[s] = cnt
        packed[s] = [gather(a, perm, n) for a in [xp] + list(props)]
    # sizes: [to above, to below] sent, [from below, from above] received
    sends, recvs = [], []
    dev = next(iter(parts.values()))[2].device
    for s, c in counts.items():
        below, above = halo.neighbours(topo, s)
        sends.append((s, above, TAG_SIZE, torch.tensor([c[2]], dtype=torch.int64, device=dev)))
        sends.append((s, below, TAG_SIZE + 1, torch.tensor([c[1]], dtype=torch.int64,
                                                            device=dev)))
        recvs.append((s, below, TAG_SIZE, torch.zeros(1, dtype=torch.int64, device=dev)))
        recvs.append((s, above, TAG_SIZE + 1, torch.zeros(1, dtype=torch.int64, device=dev)))
    got = comm.exchange(sends, recvs)
    arrive = {}
    for (s, src, tag, _), g in zip(recvs, got):
        arrive.setdefault(s, {})[tag] = int(g.item())
    # particle blocks of every array (empty blocks are skipped on both sides)
    sends, recvs, want = [], [], []
    for s, c in counts.items():
        below, above = halo.neighbours(topo, s)
        nb, na = arrive[s][TAG_SIZE], arrive[s][TAG_SIZE + 1]
        for k, P in enumerate(packed[s]):
            rows = _rows(P)
            lo_up, lo_dn = c[0] + c[1], c[0]
            if c[2]:
                sends.append((s, above, TAG_DATA + 2 * k, rows[lo_up:lo_up + c[2]]))
            if c[1]:
                sends.append((s, below, TAG_DATA + 2 * k + 1, rows[lo_dn:lo_dn + c[1]]))
            if nb:
                recvs.append((s, below, TAG_DATA + 2 * k,
                              torch.empty((nb, rows.shape[1]), dtype=P.dtype, device=P.device)))
                want.append((s, k, 0))
            if na:
                recvs.append((s, above, TAG_DATA + 2 * k + 1,
                              torch.empty((na, rows.shape[1]), dtype=P.dtype, device=P.device)))
                want.append((s, k, 1))
    got = comm.exchange(sends, recvs)
    blocks = {}
    for (s, k, side), g in zip(want, got):
        blocks[(s, k, side)] = g
    out = {}
    for s, c in counts.items():
        nb, na = arrive[s][TAG_SIZE], arrive[s][TAG_SIZE + 1]
        n_new = c[0] + nb + na
        arrays = []
        for k, P in enumerate(packed[s]):
            rows = _rows(P)
            res = torch.empty((max(n_new, 1), rows.shape[1]), dtype=P.dtype, device=P.device)
            res[:c[0]].copy_(rows[:c[0]])
            if nb:
                res[c[0]:c[0] + nb].copy_(blocks[(s, k, 0)])
            if na:
                res[c[0] + nb:n_new].copy_(blocks[(s, k, 1)])
            arrays.append(res.t()[:, :n_new])
        out[s] = (arrays[0], arrays[1:])
    return info_all, out


def ppm_map_part_partial(xp, Np, topo_id, mesh_id, props=(), comm=None):
    """ppm_map_part_partial for the subdomain this process holds: returns
    (info, Np_new, xp_new, [props_new]).  xp and props are column-major
    device arrays (ld, Np); every rank of the decomposition calls it.  info
    is -2 (errno 405) when particles lie in no neighbouring subdomain (they
    are dropped); the exchange takes place all the same."""
    r = _topo.local_sub(topo_id, mesh_id)
    if r is None:
        raise ValueError("ppm_map_part_partial: unknown topo_id/mesh_id")
    t, isub = r
    n = int(Np)
    c = comm if comm is not None else halo.comm_for(topo_id, mesh_id)
    info, out = map_subs({isub: (topo_id, mesh_id, xp[:, :n], list(p[:, :n] for p in props))},
                         t, c)
    x2, p2 = out[isub]
    return info, int(x2.shape[1]), x2, p2


# ---- ppm_map_part_global: every particle to the subdomain that contains it ----

TAG_GSIZE, TAG_GDATA = 80, 100


def device_route_global(topo_id, mesh_id, xp, nsubs):
    """(info, perm, [count to subdomain 0 .. nsubs-1, count in none]) of the
    local subdomain's particles (ppmg_map_part_global_route on the current
    stream)."""
    import torch
    n = int(xp.shape[1])
    perm = torch.empty(max(n, 1), dtype=torch.int32, device=xp.device)
    cnt = (C.c_int64 * (int(nsubs) + 1))()
    info = C.c_int(0)
    k = "d" if xp.dtype == torch.float64 else "s"
    getattr(lib(), f"ppmg_map_part_global_route_{k}_dev")(
        xp.data_ptr(), xp.stride(1), n, int(topo_id), int(mesh_id), perm.data_ptr(), cnt,
        C.byref(info), torch.cuda.current_stream().cuda_stream)
    return info.value, perm, [int(c) for c in cnt]


def device_route_partial(topo_id, mesh_id, xp, nsubs):
    """As device_route_global, with only the local subdomain and its
    neighbours as destinations (ppmg_map_part_partial_route): particles
    beyond them land in the last group and give info -2, errno 405."""
    import torch
    n = int(xp.shape[1])
    perm = torch.empty(max(n, 1), dtype=torch.int32, device=xp.device)
    cnt = (C.c_int64 * (int(nsubs) + 1))()
    info = C.c_int(0)
    k = "d" if xp.dtype == torch.float64 else "s"
    getattr(lib(), f"ppmg_map_part_partial_route_{k}_dev")(
        xp.data_ptr(), xp.stride(1), n, int(topo_id), int(mesh_id), perm.data_ptr(), cnt,
        C.byref(info), torch.cuda.current_stream().cuda_stream)
    return info.value, perm, [int(c) for c in cnt]


def map_global(parts: dict, topo, comm, route=device_route_global, gather=device_gather,
               peers=None):
    """parts {isub: (topo_id, mesh_id, xp, [props])} of the subdomains this
    process holds; returns (info, {isub: (xp_new, [props_new])}).  Sizes go
    first (one to every peer), then the non-empty particle blocks, in the same
    operation order on every rank.  peers(s): the subdomains s exchanges with
    (every other one by default, the global mapping; the neighbours for the
    partial mapping)."""
    import torch
    ns = int(topo.nsubs)
    if peers is None:
        def peers(s):
            return [q for q in range(ns) if q != s]
    info_all = 0
    packed, counts = {}, {}
    for s, (tid, mid, xp, props) in parts.items():
        n = int(xp.shape[1])
        info, perm, cnt = route(tid, mid, xp, ns)
        if info and not info_all:
            info_all = info
        counts[s] = cnt
        packed[s] = [gather(a, perm, n) for a in [xp] + list(props)]
    dev = next(iter(parts.values()))[2].device
    sends, recvs = [], []
    for s, c in counts.items():
        for q in peers(s):
            sends.append((s, q, TAG_GSIZE, torch.tensor([c[q]], dtype=torch.int64, device=dev)))
            recvs.append((s, q, TAG_GSIZE, torch.zeros(1, dtype=torch.int64, device=dev)))
    got = comm.exchange(sends, recvs)
    arrive = {}
    for (s, src, _, _), g in zip(recvs, got):
        arrive.setdefault(s, {})[src] = int(g.item())
    sends, recvs, want = [], [], []
    for s, c in counts.items():
        start = [0]
        for v in c:
            start.append(start[-1] + v)
        for k, P in enumerate(packed[s]):
            rows = _rows(P)
            for q in peers(s):
                if c[q]:
                    sends.append((s, q, TAG_GDATA + k, rows[start[q]:start[q] + c[q]]))
                nq = arrive[s].get(q, 0)
                if nq:
                    recvs.append((s, q, TAG_GDATA + k, torch.empty((nq, rows.shape[1]),
                                                                  dtype=P.dtype,
                                                                  device=P.device)))
                    want.append((s, k, q))
    got = comm.exchange(sends, recvs)
    blocks = {key: g for key, g in zip(want, got)}
    out = {}
    for s, c in counts.items():
        start = sum(c[:s])
        n_new = c[s] + sum(arrive[s].get(q, 0) for q in peers(s))
        arrays = []
        for k, P in enumerate(packed[s]):
            rows = _rows(P)
            res = torch.empty((max(n_new, 1), rows.shape[1]), dtype=P.dtype, device=P.device)
            res[:c[s]].copy_(rows[start:start + c[s]])
            pos = c[s]
            for q in peers(s):
                nq = arrive[s].get(q, 0)
                if nq:
                    res[pos:pos + nq].copy_(blocks[(s, k, q)])
                    pos += nq
            arrays.append(res.t()[:, :n_new])
        out[s] = (arrays[0], arrays[1:])
    return info_all, out


def ppm_map_part_global(xp, Np, topo_id, mesh_id, props=(), comm=None):
    """ppm_map_part_global for the subdomain this process holds: returns
    (info, Np_new, xp_new, [props_new]).  Every particle goes to the
    subdomain that contains it, however far it moved; particles in none are
    left out, without an error (ppm_map_part_global.f:437-442).  The new list
    is the kept particles in their order, then the arrivals by ascending
    source subdomain (each in the source's order).  xp and props are
    column-major device arrays (ld, Np); every rank of the decomposition
    calls it."""
    r = _topo.local_sub(topo_id, mesh_id)
    if r is None:
        raise ValueError("ppm_map_part_global: unknown topo_id/mesh_id")
    t, isub = r
    n = int(Np)
    c = comm if comm is not None else halo.comm_for(topo_id, mesh_id)
    info, out = map_global({isub: (topo_id, mesh_id, xp[:, :n], list(p[:, :n] for p in props))},
                           t, c)
    x2, p2 = out[isub]
    return info, int(x2.shape[1]), x2, p2
