"""Ghost exchange between z-slab subdomains: the inter-subdomain part of
``ppm_map_field_ghost`` (ppm/src/ppm_map_field_ghost.f:392-670 with
ppm_map_field_send.f and the add / replace pops of ppm_map_field_pop_3d.f).

A domain cut into slabs along z puts one slab on each GPU (the subdomain
that ``topo.register(topo, isub)`` selected).  On a slab the library's 3D P2M
leaves in the z ghost planes the contributions owed to the neighbouring
slabs, and its M2P reads the z ghost planes; x and y stay periodic within the
slab.  The exchange moves contiguous blocks of node planes: field_up's z
axis is the slowest, so planes z0..z1 of a Fortran-ordered
``field_up(ldn, x, y, z, 1)`` are one contiguous run of memory.

With ``nz`` the slab's cells (its real nodes 1..nz+1, node nz+1 shared with
the slab above, whose node 1 it is) and ``g`` the z ghost width:

* put (after P2M): planes nz+1 .. nz+1+g go up and are added to the upper
  neighbour's planes 1 .. 1+g; planes 1-g .. 1 go down and are added to the
  lower neighbour's planes nz_below+1-g .. nz_below+1.  Both copies of a
  shared plane end with the full sum, as in the reference.
* get (before M2P): real planes nz+1-g .. nz go up into the upper
  neighbour's ghost planes 1-g .. 0; real planes 2 .. 1+g go down into the
  lower neighbour's ghost planes nz_below+2 .. nz_below+1+g.

Transports: :class:`DistComm` (torch.distributed point-to-point, NCCL for
device tensors, gloo for host tensors; subdomain s on rank s by default) and
:class:`LocalComm` (every slab in this process).  Every rank posts the same
operations in the same order, and all receives complete before any block is
added, so the blocks sent are the pre-exchange values.
"""
from __future__ import annotations

import numpy as np

TAG_UP, TAG_DOWN = 17, 18   # messages travelling to the slab above / below

_comms: dict = {}


def set_exchange(topo_id: int, mesh_id: int, comm) -> None:
    """Use `comm` for the slab exchanges of handle (topo_id, mesh_id)."""
    _comms[(int(topo_id), int(mesh_id))] = comm


def comm_for(topo_id: int, mesh_id: int):
    """The transport of a slab handle: the one set with :func:`set_exchange`,
    else torch.distributed's default group (subdomain s on rank s)."""
    c = _comms.get((int(topo_id), int(mesh_id)))
    if c is not None:
        return c
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return DistComm()
    raise RuntimeError("slab subdomain: no exchange configured (initialise torch.distributed "
                       "or call ppm_legacy_b200.halo.set_exchange)")


def neighbours(topo, isub: int):
    """(sub below, sub above) of slab isub, periodic in z."""
    z0 = topo.istart[:, 2]
    z1 = z0 + topo.nnodes[:, 2] - 1          # top node (global, 1-based)
    top = int(topo.Nm[2])
    lo, hi = int(z0[isub]), int(z1[isub])
    below = [s for s in range(topo.nsubs) if int(z1[s]) == (lo if lo > 1 else top)]
    above = [s for s in range(topo.nsubs) if int(z0[s]) == (hi if hi < top else 1)]
    if len(below) != 1 or len(above) != 1:
        raise ValueError("topology is not a decomposition into z-slabs")
    return below[0], above[0]


def _base(field):
    """The C-ordered contiguous tensor behind a Fortran-ordered field view:
    dimension 1 is z (1-based plane z at index z - lb_z)."""
    import torch
    if isinstance(field, np.ndarray):
        field = torch.from_numpy(field)
    b = field.permute(*reversed(range(field.dim())))
    if not b.is_contiguous():
        raise ValueError("field_up must be a Fortran-ordered (column-major) array")
    return b


def _planes(base, lbz: int, z0: int, z1: int):
    """Planes z0..z1 (1-based, inclusive) of the local subdomain."""
    return base[0, z0 - lbz:z1 - lbz + 1]


def _check(base, lbz, nz, g):
    nzf = base.shape[1]
    if lbz > 1 - g or lbz + nzf - 1 < nz + 1 + g:
        raise ValueError("field_up bounds do not cover the z ghost planes 1-g .. Nm+g")
    if nz < g:
        raise ValueError("z ghost width exceeds the slab's cell layers")


def _exchange(fields, topo, ghost, field_lb, comm, put: bool):
    g = int(ghost[2]) if len(ghost) > 2 else int(ghost[-1])
    sends, recvs = [], []
    for s, f in fields.items():
        base = _base(f)
        lbz = int(field_lb[s][2] if isinstance(field_lb, dict) else field_lb[2])
        nz = int(topo.nnodes[s, 2]) - 1
        _check(base, lbz, nz, g)
        below, above = neighbours(topo, s)
        if put:
            up = _planes(base, lbz, nz + 1, nz + 1 + g)
            down = _planes(base, lbz, 1 - g, 1)
            into_from_below = _planes(base, lbz, 1, 1 + g)
            into_from_above = _planes(base, lbz, nz + 1 - g, nz + 1)
        else:
            if g == 0:
                continue
            up = _planes(base, lbz, nz + 1 - g, nz)
            down = _planes(base, lbz, 2, 1 + g)
            into_from_below = _planes(base, lbz, 1 - g, 0)
            into_from_above = _planes(base, lbz, nz + 2, nz + 1 + g)
        sends.append((s, above, TAG_UP, up))
        sends.append((s, below, TAG_DOWN, down))
        recvs.append((s, below, TAG_UP, into_from_below))
        recvs.append((s, above, TAG_DOWN, into_from_above))
    got = comm.exchange(sends, [(d, src, tag, t) for d, src, tag, t in recvs])
    for (d, src, tag, target), blk in zip(recvs, got):
        if put:
            target.add_(blk)
        else:
            target.copy_(blk)


def put(fields: dict, topo, ghost, field_lb, comm) -> None:
    """Ghost put between slabs: fields {isub: field_up} held by this process,
    field_lb their lower bounds (one triple, or {isub: triple})."""
    _exchange(fields, topo, ghost, field_lb, comm, True)


def get(fields: dict, topo, ghost, field_lb, comm) -> None:
    """Ghost get between slabs (fills the z ghost planes)."""
    _exchange(fields, topo, ghost, field_lb, comm, False)


class LocalComm:
    """Every slab in this process: each receive takes the matching send."""

    def exchange(self, sends, recvs):
        table = {(src, dst, tag): t for src, dst, tag, t in sends}
        out = []
        for dst, src, tag, like in recvs:
            blk = table[(src, dst, tag)]
            if blk.shape != like.shape:
                raise ValueError("slab exchange: block shapes differ between neighbours")
            out.append(blk.clone())
        return out


class DistComm:
    """torch.distributed point-to-point (one batch of isend / irecv).

    sub_to_rank maps a subdomain to its rank (default: the identity).
    """

    def __init__(self, group=None, sub_to_rank=None):
        self.group = group
        self.sub_to_rank = sub_to_rank

    def _rank(self, s):
        return int(s if self.sub_to_rank is None else self.sub_to_rank[s])

    def exchange(self, sends, recvs):
        import torch
        import torch.distributed as dist
        me = dist.get_rank(self.group)
        # NCCL moves device memory only, gloo host memory only: blocks on the
        # other side travel through copies
        if dist.get_backend(self.group) == "nccl":
            dev = torch.device("cuda", torch.cuda.current_device())
        else:
            dev = torch.device("cpu")

        def wire(t):
            return t.to(dev) if t.device != dev else t.contiguous()

        ops, bufs, local = [], [], {}
        for src, dst, tag, t in sends:
            if self._rank(dst) == me:
                local[(src, dst, tag)] = t
            else:
                ops.append(dist.P2POp(dist.isend, wire(t), self._peer(dst), self.group, tag))
        for dst, src, tag, like in recvs:
            buf = torch.empty_like(like, memory_format=torch.contiguous_format, device=dev)
            bufs.append(buf)
            if self._rank(src) != me:
                ops.append(dist.P2POp(dist.irecv, buf, self._peer(src), self.group, tag))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        out = []
        for (dst, src, tag, like), buf in zip(recvs, bufs):
            if self._rank(src) == me:
                buf.copy_(local[(src, dst, tag)])
            out.append(buf.to(like.device) if buf.device != like.device else buf)
        return out

    def _peer(self, s):
        # global rank of the subdomain's owner (group ranks -> global ranks)
        import torch.distributed as dist
        r = self._rank(s)
        return r if self.group is None else dist.get_global_rank(self.group, r)
