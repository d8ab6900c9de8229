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


def is_slab_topology(topo) -> bool:
    """Whether every subdomain spans x and y (cuts along z only)."""
    return all(int(topo.nnodes[s, a]) == int(topo.Nm[a])
               for s in range(topo.nsubs) for a in range(2))


def _exchange_boxes(fields, topo, ghost, field_lb, comm, put: bool):
    """The exchange of a decomposition cut along x or y as well: the boxes of
    ppmg_halo_plan_boxes, every send packed before any receive is applied,
    receives applied in the plan's order (adds of the put in that order)."""
    sends, recvs = [], []
    for s, f in fields.items():
        base = _base(f)
        lbv = field_lb[s] if isinstance(field_lb, dict) else field_lb
        lb = [int(v) for v in lbv]
        ext = [base.shape[3], base.shape[2], base.shape[1]]  # x, y, z nodes

        def view(lo, hi, base=base, lb=lb, ext=ext):
            for a in range(3):
                if lo[a] < lb[a] or hi[a] > lb[a] + ext[a] - 1:
                    raise ValueError("field_up bounds do not cover the ghost layers")
            return base[0, lo[2] - lb[2]:hi[2] - lb[2] + 1, lo[1] - lb[1]:hi[1] - lb[1] + 1,
                        lo[0] - lb[0]:hi[0] - lb[0] + 1]
        p = plan_boxes(topo, s, [int(v) for v in ghost], put)
        for peer, tag, lo, hi in p["send"]:
            sends.append((s, peer, tag, view(lo, hi).clone()))
        for peer, tag, lo, hi in p["recv"]:
            recvs.append((s, peer, tag, view(lo, hi)))
    got = comm.exchange(sends, recvs)
    for (_, _, _, target), blk in zip(recvs, got):
        if put:
            target.add_(blk)
        else:
            target.copy_(blk)


def _exchange(fields, topo, ghost, field_lb, comm, put: bool):
    if not is_slab_topology(topo):
        return _exchange_boxes(fields, topo, ghost, field_lb, comm, put)
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
    """Ghost put between subdomains: fields {isub: field_up} held by this
    process, field_lb their lower bounds (one triple, or {isub: triple}).
    Slabs along z exchange whole planes; other cartesian cuts the boxes of
    plan_boxes."""
    _exchange(fields, topo, ghost, field_lb, comm, True)


def get(fields: dict, topo, ghost, field_lb, comm) -> None:
    """Ghost get between subdomains (fills the ghost layers of the cut axes)."""
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

    def posting_order(self, sends, recvs):
        """The order in which this rank posts its sends and receives.

        NCCL pairs the point-to-point messages between two ranks in the
        order they are posted and ignores tags (gloo matches tags).  Sends
        are posted sorted by (destination rank, source subdomain, destination
        subdomain, tag) and receives by (source rank, the same triple), so
        the k-th send from rank A to rank B meets the k-th receive at B from
        A whatever order the plans list them in.
        """
        so = sorted(range(len(sends)),
                    key=lambda i: (self._rank(sends[i][1]), sends[i][0], sends[i][1], sends[i][2]))
        ro = sorted(range(len(recvs)),
                    key=lambda i: (self._rank(recvs[i][1]), recvs[i][1], recvs[i][0], recvs[i][2]))
        return so, ro

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

        so, ro = self.posting_order(sends, recvs)
        ops, local = [], {}
        bufs = [torch.empty_like(like, memory_format=torch.contiguous_format, device=dev)
                for _, _, _, like in recvs]
        for i in so:
            src, dst, tag, t = sends[i]
            if self._rank(dst) == me:
                local[(src, dst, tag)] = t
            else:
                ops.append(dist.P2POp(dist.isend, wire(t), self._peer(dst), self.group, tag))
        for i in ro:
            dst, src, tag, like = recvs[i]
            if self._rank(src) != me:
                ops.append(dist.P2POp(dist.irecv, bufs[i], self._peer(src), self.group, tag))
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


# ---- the library's own exchange (ppmg_halo_plan, ppmg_halo_set_transport) ----
#
# With a transport registered on a slab handle, the C-ABI performs the
# exchange itself: ppmg_map_field_ghost_* on the slab does the put or get, and
# the 3D P2M and remesh end with the put.  The library decides which planes
# travel where (ppmg_halo_plan) and adds or copies what arrives; the transport
# only moves bytes.  CTransport registers a Python mover as that transport.

import ctypes as _C  # noqa: E402
import threading as _threading  # noqa: E402


class HaloBlock(_C.Structure):
    """ppmg_halo_block: one contiguous block to send or receive."""
    _fields_ = [("peer", _C.c_int), ("tag", _C.c_int), ("buf", _C.c_void_p),
                ("bytes", _C.c_int64)]


HALO_FN = _C.CFUNCTYPE(_C.c_int, _C.c_void_p, _C.c_int, _C.POINTER(HaloBlock), _C.c_int,
                       _C.POINTER(HaloBlock), _C.c_int, _C.c_void_p)

_c_transports: dict = {}


def plan(topo, isub, ldf, field_lb, field_ub, ghost, put):
    """The library's blocks of one exchange of slab isub (ppmg_halo_plan):
    {"count": elements per block, "send": [(peer, tag, offset)] * 2,
    "recv": [(peer, tag, offset)] * 2}, offsets in elements into field_up,
    index 0 towards / from the slab above, 1 the slab below.  Host logic
    only: needs no GPU."""
    from ._lib import int_array, last_error, lib
    ist = np.ascontiguousarray(topo.istart, dtype=np.int32)
    nn = np.ascontiguousarray(topo.nnodes, dtype=np.int32)
    cnt = _C.c_int64(0)
    sp, st, rp, rt = ((_C.c_int * 2)() for _ in range(4))
    so, ro = (_C.c_int64 * 2)(), (_C.c_int64 * 2)()
    info = _C.c_int(0)
    lib().ppmg_halo_plan(int(topo.nsubs), ist.ctypes.data, nn.ctypes.data, int(topo.Nm[2]),
                         int(isub), int(ldf), int_array(field_lb, _C.c_int64),
                         int_array(field_ub, _C.c_int64), int_array(ghost), 6 if put else 5,
                         _C.byref(cnt), sp, st, so, rp, rt, ro, _C.byref(info))
    if info.value != 0:
        raise ValueError(last_error()[2])
    return {"count": cnt.value, "send": [(sp[b], st[b], so[b]) for b in range(2)],
            "recv": [(rp[b], rt[b], ro[b]) for b in range(2)]}


class HaloBox(_C.Structure):
    """ppmg_halo_box: one box of local field nodes (1-based, inclusive)."""
    _fields_ = [("peer", _C.c_int), ("tag", _C.c_int), ("lo", _C.c_int64 * 3),
                ("hi", _C.c_int64 * 3)]


def plan_boxes(topo, isub, ghost, put):
    """The library's boxes of one exchange of subdomain isub of a cartesian
    decomposition (ppmg_halo_plan_boxes): {"send": [...], "recv": [...]},
    each entry (peer, tag, lo(3), hi(3)) in local 1-based node indices,
    receives in the order they are applied.  Host logic only."""
    from ._lib import int_array, last_error, lib
    ist = np.ascontiguousarray(topo.istart, dtype=np.int32)
    nn = np.ascontiguousarray(topo.nnodes, dtype=np.int32)
    ns, nr, info = _C.c_int(0), _C.c_int(0), _C.c_int(0)
    args = (int(topo.nsubs), ist.ctypes.data, nn.ctypes.data, int_array(topo.Nm), int(isub),
            int_array(ghost), 6 if put else 5)
    lib().ppmg_halo_plan_boxes(*args, 0, None, _C.byref(ns), None, _C.byref(nr),
                               _C.byref(info))
    if info.value != 0:
        raise ValueError(last_error()[2])
    sb, rb = (HaloBox * max(ns.value, 1))(), (HaloBox * max(nr.value, 1))()
    cap = max(ns.value, nr.value)
    lib().ppmg_halo_plan_boxes(*args, cap, _C.addressof(sb), _C.byref(ns), _C.addressof(rb),
                               _C.byref(nr), _C.byref(info))

    def rows(b, n):
        return [(b[i].peer, b[i].tag, tuple(b[i].lo), tuple(b[i].hi)) for i in range(n)]
    return {"send": rows(sb, ns.value), "recv": rows(rb, nr.value)}


def cart_neighbours(topo, isub):
    """The neighbours of subdomain isub of a cartesian cut (ppmg_halo_neighbours):
    ascending, isub excluded; the subdomains whose boxes share a face, an
    edge or a corner with isub's, across the periodic faces too."""
    from ._lib import int_array, last_error, lib
    ist = np.ascontiguousarray(topo.istart, dtype=np.int32)
    nn = np.ascontiguousarray(topo.nnodes, dtype=np.int32)
    out = (_C.c_int * max(int(topo.nsubs), 1))()
    cnt, info = _C.c_int(0), _C.c_int(0)
    lib().ppmg_halo_neighbours(int(topo.nsubs), ist.ctypes.data, nn.ctypes.data,
                               int_array(topo.Nm), int(isub), int(topo.nsubs),
                               _C.addressof(out), _C.byref(cnt), _C.byref(info))
    if info.value != 0:
        raise ValueError(last_error()[2])
    return [out[i] for i in range(cnt.value)]


def has_c_transport(topo_id, mesh_id) -> bool:
    return (int(topo_id), int(mesh_id)) in _c_transports


def c_transport(topo_id, mesh_id):
    """The CTransport registered on a handle, or None."""
    return _c_transports.get((int(topo_id), int(mesh_id)))


class CTransport:
    """A Python mover registered as the halo transport of slab handle
    (topo_id, mesh_id) whose local subdomain is isub.  mover.exchange(me,
    sends, recvs, on_device, stream) moves blocks given as (peer, tag,
    address, nbytes); an exception becomes a nonzero status (the C call then
    fails with errno 2)."""

    def __init__(self, topo_id, mesh_id, isub, mover):
        from ._lib import last_error, lib
        self.key = (int(topo_id), int(mesh_id))
        self.isub = int(isub)
        self.mover = mover
        self._fn = HALO_FN(self._call)  # kept alive as long as the registration
        info = _C.c_int(0)
        lib().ppmg_halo_set_transport(self.key[0], self.key[1], _C.cast(self._fn, _C.c_void_p),
                                      None, _C.byref(info))
        if info.value != 0:
            raise RuntimeError(last_error()[2])
        _c_transports[self.key] = self

    def _call(self, ctx, ns, sends, nr, recvs, on_device, stream):
        try:
            s = [(sends[i].peer, sends[i].tag, sends[i].buf, sends[i].bytes) for i in range(ns)]
            r = [(recvs[i].peer, recvs[i].tag, recvs[i].buf, recvs[i].bytes) for i in range(nr)]
            self.mover.exchange(self.isub, s, r, bool(on_device), stream)
            return 0
        except Exception:  # noqa: BLE001 -- reported through the library's info
            import traceback
            traceback.print_exc()
            return 1

    def close(self):
        from ._lib import lib
        info = _C.c_int(0)
        lib().ppmg_halo_set_transport(self.key[0], self.key[1], None, None, _C.byref(info))
        _c_transports.pop(self.key, None)


def _cudart():
    from cuda.bindings import runtime as rt
    return rt


def _read_block(addr, nbytes, on_device, stream):
    """The bytes of a block (device blocks after the work on `stream`)."""
    if not on_device:
        return _C.string_at(addr, nbytes)
    rt = _cudart()
    (err,) = rt.cudaStreamSynchronize(stream or 0)
    out = bytearray(nbytes)
    buf = (_C.c_char * nbytes).from_buffer(out)
    (err2,) = rt.cudaMemcpy(_C.addressof(buf), addr, nbytes, rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    if err != rt.cudaError_t.cudaSuccess or err2 != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"halo block read failed: {err} {err2}")
    return bytes(out)


def _write_block(addr, data, on_device):
    if not on_device:
        _C.memmove(addr, data, len(data))
        return
    rt = _cudart()
    src = (_C.c_char * len(data)).from_buffer_copy(data)
    (err,) = rt.cudaMemcpy(addr, _C.addressof(src), len(data),
                           rt.cudaMemcpyKind.cudaMemcpyHostToDevice)
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"halo block write failed: {err}")


class ThreadMover:
    """Slabs held by one process, each exchanging from a host thread of its
    own (their C calls run concurrently): a send is matched with the receive
    of the same (source, destination, tag), in the order they were posted
    (a thread may post its next exchange before a peer took the last one).
    Blocks travel through host memory.  A receive waits at most `timeout`
    seconds."""

    def __init__(self, timeout=60.0):
        import collections
        self.cv = _threading.Condition()
        self.box = collections.defaultdict(collections.deque)
        self.timeout = timeout

    def exchange(self, me, sends, recvs, on_device, stream):
        posted = [((me, peer, tag), _read_block(addr, n, on_device, stream))
                  for peer, tag, addr, n in sends]
        with self.cv:
            for k, data in posted:
                self.box[k].append(data)
            self.cv.notify_all()
        for peer, tag, addr, n in recvs:
            key = (peer, me, tag)
            with self.cv:
                if not self.cv.wait_for(lambda: len(self.box[key]) > 0, timeout=self.timeout):
                    raise TimeoutError(f"slab {me}: no block from {peer} (tag {tag})")
                data = self.box[key].popleft()
            if len(data) != n:
                raise ValueError("slab exchange: block sizes differ between neighbours")
            _write_block(addr, data, on_device)


class DistMover:
    """torch.distributed point-to-point (subdomain s on rank s, or
    sub_to_rank[s]): one batch of isend / irecv.  Blocks go through tensors
    on the process group's side (host memory for gloo, the current device for
    NCCL)."""

    def __init__(self, group=None, sub_to_rank=None):
        self.group = group
        self.sub_to_rank = sub_to_rank

    def _peer(self, s):
        import torch.distributed as dist
        r = int(s if self.sub_to_rank is None else self.sub_to_rank[s])
        return r if self.group is None else dist.get_global_rank(self.group, r)

    def _rank(self, s):
        return int(s if self.sub_to_rank is None else self.sub_to_rank[s])

    def exchange(self, me, sends, recvs, on_device, stream):
        import torch
        import torch.distributed as dist
        nccl = dist.get_backend(self.group) == "nccl"
        dev = torch.device("cuda", torch.cuda.current_device()) if nccl else torch.device("cpu")

        def tensor_of(data):
            return torch.frombuffer(bytearray(data), dtype=torch.uint8).to(dev)

        # posted in the order of DistComm.posting_order: NCCL pairs the
        # messages of two ranks in posting order, not by tag
        sends = sorted(sends, key=lambda m: (self._rank(m[0]), me, m[0], m[1]))
        recvs = sorted(recvs, key=lambda m: (self._rank(m[0]), m[0], me, m[1]))
        ops, bufs = [], []
        for peer, tag, addr, n in sends:
            t = tensor_of(_read_block(addr, n, on_device, stream))
            ops.append(dist.P2POp(dist.isend, t, self._peer(peer), self.group, tag))
        for peer, tag, addr, n in recvs:
            t = torch.empty(n, dtype=torch.uint8, device=dev)
            bufs.append((t, addr))
            ops.append(dist.P2POp(dist.irecv, t, self._peer(peer), self.group, tag))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for t, addr in bufs:
            _write_block(addr, t.cpu().numpy().tobytes(), on_device)
