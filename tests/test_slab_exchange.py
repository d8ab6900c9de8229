"""The ghost exchange between z-slab subdomains (ppm_legacy_b200.halo) on CPU:
in one process (LocalComm) and as world_size 2 and 3 `gloo` process groups
(DistComm, the transport the multi-GPU path runs over NCCL).

Each slab's field is built as the library's slab P2M leaves it: the
deposit of the slab's own particles (the oracle's periodic deposit of those
particles alone) read over the slab's z planes 1-g .. nz+1+g, ghost planes
included.  After the put every slab's real planes must hold the deposit of
all particles (the oracle over the whole domain); after the get its ghost
planes must hold its neighbours' real planes."""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, ROOT)
from _util import random_particles, topo_for, unique_view  # noqa: E402
import _util as U  # noqa: E402
from oracle import oracle as O  # noqa: E402
from ppm_legacy_b200 import halo  # noqa: E402


def slab_of(t, xp):
    """0-based slab of every particle (z inside [min_sub, max_sub))."""
    z = xp[2]
    own = np.full(z.shape, -1)
    for s in range(t.nsubs):
        own[(z >= t.min_sub[s, 2]) & (z < t.max_sub[s, 2])] = s
    assert (own >= 0).all()
    return own


def box(U, z0, nz, g):
    """Planes 1-g .. nz+1+g of a slab whose node 1 is global node z0 (0-based),
    x and y over 1-g .. Nc+1+g, from unique periodic values U(lda, Nc, Nc, Nc)."""
    nc = U.shape[1]
    xi = (np.arange(1 - g, nc + 2 + g) - 1) % nc
    zi = (z0 + np.arange(1 - g, nz + 2 + g) - 1) % nc
    return np.asfortranarray(U[np.ix_(range(U.shape[0]), xi, xi, zi)][..., None])


def case(nc, nslab, kernel, g, lda, seed):
    rng = np.random.default_rng(seed)
    t = topo_for(3, nc, decomp=(1, 1, nslab))
    t1 = topo_for(3, nc)
    n = 3 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    own = slab_of(t, xp)
    gg = [g, g, g]
    fa, lba, _ = O.p2m(t1, xp, up, kernel, gg)
    Ua = unique_view(fa, lba, [nc] * 3, 3)
    local, want = {}, {}
    for s in range(nslab):
        sel = own == s
        fs, lbs, _ = O.p2m(t1, np.asfortranarray(xp[:, sel]), np.asfortranarray(up[:, sel]),
                           kernel, gg)
        Us = unique_view(fs, lbs, [nc] * 3, 3)
        z0 = int(t.istart[s, 2]) - 1
        nz = int(t.nnodes[s, 2]) - 1
        local[s] = box(Us, z0, nz, g)
        want[s] = box(Ua, z0, nz, g)
    return t, local, want


def check_put(t, s, f, want, g):
    nz = int(t.nnodes[s, 2]) - 1
    real = (slice(None), slice(None), slice(None), slice(g, g + nz + 1), 0)
    got, ref = f[real], want[real]
    assert np.abs(got - ref).max() <= 1e-13 * max(np.abs(ref).max(), 1.0)


def check_get(t, s, f, want, g):
    err = np.abs(f - want).max()
    assert err <= 1e-13 * max(np.abs(want).max(), 1.0)


@pytest.mark.parametrize("nc,nslab,kernel,g,lda", [
    (12, 2, 2, 2, 3), (12, 3, 2, 2, 1), (10, 2, 1, 1, 2), (16, 4, 2, 3, 1)])
def test_put_then_get_in_one_process(nc, nslab, kernel, g, lda):
    t, local, want = case(nc, nslab, kernel, g, lda, seed=nc + nslab)
    fields = {s: torch.from_numpy(local[s]) for s in local}
    lb = [1 - g] * 3
    halo.put(fields, t, [g] * 3, lb, halo.LocalComm())
    for s in fields:
        check_put(t, s, fields[s].numpy(), want[s], g)
    halo.get(fields, t, [g] * 3, lb, halo.LocalComm())
    for s in fields:
        check_get(t, s, fields[s].numpy(), want[s], g)


@pytest.mark.parametrize("nc,nslab,g", [(12, 2, 2), (12, 3, 1), (16, 4, 3)])
def test_put_then_get_with_nccl_pairing(nc, nslab, g):
    # NCCL pairs the messages of two ranks in posting order, not by tag: with
    # two slabs both neighbours are the same rank, and the up and down blocks
    # must still meet their own receives
    t, local, want = case(nc, nslab, 2, g, 2, seed=nc + 7 * nslab)
    fields = {s: torch.from_numpy(local[s]) for s in local}
    lb = [1 - g] * 3
    halo.put(fields, t, [g] * 3, lb, U.PairOrderComm())
    for s in fields:
        check_put(t, s, fields[s].numpy(), want[s], g)
    halo.get(fields, t, [g] * 3, lb, U.PairOrderComm())
    for s in fields:
        check_get(t, s, fields[s].numpy(), want[s], g)


def test_neighbours_wrap_periodically():
    t = topo_for(3, 12, decomp=(1, 1, 3))
    assert [halo.neighbours(t, s) for s in range(3)] == [(2, 1), (0, 2), (1, 0)]
    with pytest.raises(ValueError):
        halo.neighbours(topo_for(3, 12, decomp=(2, 1, 1)), 0)


def test_thin_slab_and_short_field_are_refused():
    t, local, _ = case(12, 4, 2, 2, 1, seed=1)
    fields = {s: torch.from_numpy(local[s]) for s in local}
    with pytest.raises(ValueError):
        halo.put(fields, t, [4] * 3, [1 - 4] * 3, halo.LocalComm())


def _rank_main(rank, world, port, nc, g, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, local, want = case(nc, world, 2, g, 3, seed=99)
        f = {rank: torch.from_numpy(local[rank])}
        lb = [1 - g] * 3
        halo.put(f, t, [g] * 3, lb, halo.DistComm())
        check_put(t, rank, f[rank].numpy(), want[rank], g)
        halo.get(f, t, [g] * 3, lb, halo.DistComm())
        check_get(t, rank, f[rank].numpy(), want[rank], g)
        dist.barrier()
        out.put((rank, "ok"))
    except Exception as e:  # reported to the parent, which fails the test
        out.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_put_then_get_over_gloo(world):
    """One slab per rank; with two ranks both neighbours are the same rank."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, 12, 2, out))
             for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(v == "ok" for v in res.values()), res


# ---- particle redistribution between slabs (ppm_legacy_b200.mapping) --------

def route_rule(topo, s, x):
    """Class of every particle of slab s (0 kept, 1 below, 2 above, 3 none):
    closed-lower / open-upper boxes, the first match in that order."""
    below, above = halo.neighbours(topo, s)
    inxy = np.ones(x.shape[1], bool)
    for a in range(2):
        inxy &= (x[a] >= topo.min_phys[a]) & (x[a] < topo.max_phys[a])
    cls = np.full(x.shape[1], 3)
    for c, q in reversed(list(enumerate([s, below, above]))):
        cls[inxy & (x[2] >= topo.min_sub[q, 2]) & (x[2] < topo.max_sub[q, 2])] = c
    return cls


def moved_particles(topo, s, n, rng, far=0):
    """n particles of slab s displaced by up to 0.4 of a slab in z (periodic);
    `far` of them moved two slabs away."""
    lo, hi = topo.min_sub[s, 2], topo.max_sub[s, 2]
    L = topo.max_phys[2] - topo.min_phys[2]
    x = rng.random((3, n))
    x[2] = lo + x[2] * (hi - lo) + rng.uniform(-0.4, 0.4, n) * (hi - lo)
    x[2, :far] += 2 * (hi - lo)
    x[2] = np.mod(x[2] - topo.min_phys[2], L) + topo.min_phys[2]
    return np.asfortranarray(x)


def check_mapping(topo, before, after):
    """before/after {s: (xp, ids, u)} numpy; every particle ends in the slab
    that contains it, kept ones first in their order, then arrivals from
    below, then from above, each in the sender's order."""
    for s, (x, ids, u) in after.items():
        cls = route_rule(topo, s, x)
        assert (cls == 0).all()
        below, above = halo.neighbours(topo, s)
        xb, ib, ub = before[s]
        cb = route_rule(topo, s, xb)
        exp = [ib[0][cb == 0]]
        for q, c in ((below, 2), (above, 1)):
            xq, iq, _ = before[q]
            exp.append(iq[0][route_rule(topo, q, xq) == c])
        if below == above:  # two slabs: the neighbour's both groups come from one rank
            xq, iq, _ = before[below]
            cq = route_rule(topo, below, xq)
            exp = [ib[0][cb == 0], iq[0][cq == 1]]
        assert np.array_equal(ids[0], np.concatenate(exp)), s
        # positions and properties travel with their particle
        allx = np.concatenate([before[q][0] for q in before], axis=1)
        allu = np.concatenate([before[q][2] for q in before], axis=1)
        alli = np.concatenate([before[q][1] for q in before], axis=1)[0]
        pos = {int(i): k for k, i in enumerate(alli)}
        idx = [pos[int(i)] for i in ids[0]]
        assert np.array_equal(x, allx[:, idx]) and np.array_equal(u, allu[:, idx])


def _cpu_route(topo, s):
    def route(tid, mid, xp):
        cls = route_rule(topo, s, xp.numpy())
        perm = np.concatenate([np.nonzero(cls == c)[0] for c in range(4)]).astype(np.int32)
        return (-2 if (cls == 3).any() else 0), torch.from_numpy(perm), \
            [int((cls == c).sum()) for c in range(4)]
    return route


def _cpu_gather(src, perm, n):
    return src.t()[perm[:n].long()].t()


def _map_main(rank, world, port, out):
    from ppm_legacy_b200 import mapping
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = topo_for(3, 12, decomp=(1, 1, world))
        before = {}
        for s in range(world):
            rng = np.random.default_rng(500 + s)
            x = moved_particles(t, s, 300, rng)
            before[s] = (x, np.arange(s * 1000, s * 1000 + 300)[None, :],
                         np.asfortranarray(rng.standard_normal((2, 300))))
        x, i, u = before[rank]
        parts = {rank: (1, 1, torch.from_numpy(x), [torch.from_numpy(np.asfortranarray(i)),
                                                    torch.from_numpy(u)])}
        info, res = mapping.map_subs(parts, t, halo.DistComm(), route=_cpu_route(t, rank),
                                     gather=_cpu_gather)
        x2, (i2, u2) = res[rank]
        check_mapping(t, before, {rank: (x2.numpy(), i2.numpy(), u2.numpy())})
        assert info == 0
        dist.barrier()
        out.put((rank, "ok"))
    except Exception as e:  # reported to the parent, which fails the test
        import traceback
        out.put((rank, traceback.format_exc()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_particle_redistribution_over_gloo(world):
    """The size and particle-block exchange of ppm_map_part_partial over gloo
    (routing by a restatement of the rule on CPU; the device kernels are
    tested on the GPU)."""
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_map_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(v == "ok" for v in res.values()), res
