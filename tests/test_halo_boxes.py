"""The exchange of a cartesian decomposition (cuts along x, y and z) as the
library plans it (ppmg_halo_plan_boxes, the blocks of
ppm_map_field_ghost_init.f:234-447 for every neighbour and periodic shift),
applied here in numpy on CPU.

Each subdomain's field is built as the library's P2M on that subdomain leaves
it: the deposit of the subdomain's own particles (the oracle's periodic
deposit of those particles alone) over its ghost-extended box, whose nodes
are distinct modulo the mesh on every cut axis (so that the periodic view
equals the open deposit).  After the put every subdomain's real nodes must
hold the deposit of all particles; after the get its whole box must."""
import numpy as np
import pytest

from _util import random_particles, topo_for, unique_view
import _util as U  # noqa: E402
from oracle import oracle as O
from ppm_legacy_b200 import halo


def sub_of(t, xp):
    """0-based subdomain of every particle (closed-lower / open-upper boxes)."""
    own = np.full(xp.shape[1], -1)
    for s in range(t.nsubs):
        inside = np.ones(xp.shape[1], bool)
        for a in range(3):
            inside &= (xp[a] >= t.min_sub[s, a]) & (xp[a] < t.max_sub[s, a])
        own[inside & (own < 0)] = s
    assert (own >= 0).all()
    return own


def local_box(t, s, g):
    """Global 1-based node indices of the local nodes 1-g .. (last)+g per axis."""
    out = []
    for a in range(3):
        cut = int(t.nnodes[s, a]) != int(t.Nm[a])
        n = int(t.nnodes[s, a]) if cut else int(t.Nm[a])
        off = int(t.istart[s, a]) - 1 if cut else 0
        out.append(off + np.arange(1 - g[a], n + g[a] + 1))
    return out


def view(U, t, s, g):
    """The periodic values U(lda, Nc, Nc, Nc) at the local box of subdomain s."""
    idx = [(b - 1) % U.shape[1 + a] for a, b in enumerate(local_box(t, s, g))]
    return np.ascontiguousarray(U[np.ix_(range(U.shape[0]), *idx)])


def case(nc, decomp, kernel, g, lda, seed):
    rng = np.random.default_rng(seed)
    t = topo_for(3, nc, decomp=decomp)
    t1 = topo_for(3, nc)
    n = 2 * nc ** 3
    xp = random_particles(rng, 3, n)
    up = np.asfortranarray(rng.standard_normal((lda, n)))
    own = sub_of(t, xp)
    fa, lba, _ = O.p2m(t1, xp, up, kernel, [1, 1, 1])
    Ua = unique_view(fa, lba, [nc] * 3, 3)
    local, want = {}, {}
    for s in range(t.nsubs):
        sel = own == s
        fs, lbs, _ = O.p2m(t1, np.asfortranarray(xp[:, sel]), np.asfortranarray(up[:, sel]),
                           kernel, [1, 1, 1])
        local[s] = view(unique_view(fs, lbs, [nc] * 3, 3), t, s, g)
        want[s] = view(Ua, t, s, g)
    return t, local, want


def sl(lo, hi, g):
    """numpy slices of local nodes lo..hi (1-based) in an array whose first
    node is 1-g."""
    return (slice(None),) + tuple(slice(lo[a] - (1 - g[a]), hi[a] - (1 - g[a]) + 1)
                                  for a in range(3))


def apply(t, fields, g, put):
    """Every subdomain packs its sends, then applies its receives in order."""
    plans = {s: halo.plan_boxes(t, s, g, put) for s in fields}
    wire = {}
    for s, p in plans.items():
        for peer, tag, lo, hi in p["send"]:
            key = (s, peer, tag)
            assert key not in wire, key  # a tag names one block per pair
            wire[key] = fields[s][sl(lo, hi, g)].copy()
    for s, p in plans.items():
        for peer, tag, lo, hi in p["recv"]:
            blk = wire.pop((peer, s, tag))
            dst = fields[s][sl(lo, hi, g)]
            assert dst.shape == blk.shape, (s, peer, tag)
            if put:
                fields[s][sl(lo, hi, g)] = dst + blk
            else:
                fields[s][sl(lo, hi, g)] = blk
    assert not wire, sorted(wire)  # every send has its receive


def real(t, s, g):
    cut = [int(t.nnodes[s, a]) != int(t.Nm[a]) for a in range(3)]
    lo = [1 if cut[a] else 1 - g[a] for a in range(3)]
    hi = [int(t.nnodes[s, a]) if cut[a] else int(t.Nm[a]) + g[a] for a in range(3)]
    return sl(lo, hi, g)


@pytest.mark.parametrize("nc,decomp,kernel,g,lda", [
    (12, (2, 2, 2), 2, (2, 2, 2), 2),
    (12, (2, 2, 1), 2, (1, 2, 3), 1),
    (12, (1, 2, 2), 1, (1, 1, 1), 3),
    (12, (3, 2, 2), 2, (2, 1, 2), 1),
    (12, (2, 1, 3), 2, (1, 3, 2), 1),
    (12, (1, 1, 3), 2, (2, 2, 2), 1),
    (12, (4, 1, 1), 2, (2, 1, 1), 1)])
def test_put_then_get(nc, decomp, kernel, g, lda):
    t, local, want = case(nc, decomp, kernel, g, lda, seed=sum(decomp) + nc)
    scale = max(np.abs(w).max() for w in want.values())
    apply(t, local, g, put=True)
    for s in local:
        r = real(t, s, g)
        assert np.abs(local[s][r] - want[s][r]).max() <= 1e-13 * scale, s
    apply(t, local, g, put=False)
    for s in local:
        assert np.abs(local[s] - want[s]).max() <= 1e-13 * scale, s


@pytest.mark.parametrize("decomp,g", [((2, 2, 2), (2, 2, 2)), ((3, 2, 1), (3, 1, 2)),
                                       ((2, 2, 2), (6, 6, 6))])
def test_get_fills_each_ghost_node_once(decomp, g):
    """The get's boxes never touch a real node and cover every ghost node of a
    cut axis exactly once (so that one launch may copy them all)."""
    t = topo_for(3, 12, decomp=decomp)
    for s in range(t.nsubs):
        cut = [int(t.nnodes[s, a]) != int(t.Nm[a]) for a in range(3)]
        n = [int(t.nnodes[s, a]) if cut[a] else int(t.Nm[a]) for a in range(3)]
        hits = np.zeros(tuple(n[a] + 2 * g[a] for a in range(3)), int)
        for _, _, lo, hi in halo.plan_boxes(t, s, g, put=False)["recv"]:
            hits[sl(lo, hi, g)[1:]] += 1
        inner = tuple(slice(g[a], g[a] + n[a]) if cut[a] else slice(None) for a in range(3))
        want = np.ones_like(hits)
        want[inner] = 0
        assert np.array_equal(hits, want), s


def test_plan_is_refused_for_bad_geometry():
    t = topo_for(3, 12, decomp=(2, 2, 2))
    with pytest.raises(ValueError):
        halo.plan_boxes(t, 0, (7, 1, 1), put=True)  # wider than a subdomain
    bad = topo_for(3, 12, decomp=(2, 2, 2))
    bad.nnodes = bad.nnodes.copy()
    bad.nnodes[0, 0] = int(bad.Nm[0])  # spans x while the others are cut
    with pytest.raises(ValueError):
        halo.plan_boxes(bad, 1, (1, 1, 1), put=True)


# ---- the same exchange through ppm_legacy_b200.halo (torch tensors) --------

torch = pytest.importorskip("torch")


def fortran_fields(local):
    return {s: torch.from_numpy(np.asfortranarray(local[s][..., None])) for s in local}


@pytest.mark.parametrize("decomp,g", [((2, 2, 2), (2, 2, 2)), ((3, 1, 2), (1, 1, 2)),
                                       ((1, 2, 1), (1, 2, 1))])
def test_python_exchange_in_one_process(decomp, g):
    t, local, want = case(12, decomp, 2, g, 2, seed=31)
    scale = max(np.abs(w).max() for w in want.values())
    f = fortran_fields(local)
    lb = [1 - g[a] for a in range(3)]
    halo.put(f, t, list(g), lb, halo.LocalComm())
    for s in f:
        r = real(t, s, g)
        assert np.abs(f[s].numpy()[..., 0][r] - want[s][r]).max() <= 1e-13 * scale, s
    halo.get(f, t, list(g), lb, halo.LocalComm())
    for s in f:
        assert np.abs(f[s].numpy()[..., 0] - want[s]).max() <= 1e-13 * scale, s


@pytest.mark.parametrize("decomp,g", [((2, 2, 2), (2, 2, 2)), ((2, 1, 1), (2, 2, 2)),
                                       ((3, 1, 2), (1, 1, 2)), ((1, 2, 1), (1, 2, 1))])
def test_python_exchange_with_nccl_pairing(decomp, g):
    # the boxes of one neighbour and periodic shift: several messages between
    # the same two ranks, paired in posting order as NCCL pairs them
    t, local, want = case(12, decomp, 2, g, 2, seed=37)
    scale = max(np.abs(w).max() for w in want.values())
    f = fortran_fields(local)
    lb = [1 - g[a] for a in range(3)]
    halo.put(f, t, list(g), lb, U.PairOrderComm())
    for s in f:
        r = real(t, s, g)
        assert np.abs(f[s].numpy()[..., 0][r] - want[s][r]).max() <= 1e-13 * scale, s
    halo.get(f, t, list(g), lb, U.PairOrderComm())
    for s in f:
        assert np.abs(f[s].numpy()[..., 0] - want[s]).max() <= 1e-13 * scale, s


def _rank_main(rank, world, port, decomp, g, out):
    import os

    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, local, want = case(12, decomp, 2, g, 2, seed=5)
        scale = max(np.abs(w).max() for w in want.values())
        f = fortran_fields({rank: local[rank]})
        lb = [1 - g[a] for a in range(3)]
        halo.put(f, t, list(g), lb, halo.DistComm())
        r = real(t, rank, g)
        assert np.abs(f[rank].numpy()[..., 0][r] - want[rank][r]).max() <= 1e-13 * scale
        halo.get(f, t, list(g), lb, halo.DistComm())
        assert np.abs(f[rank].numpy()[..., 0] - want[rank]).max() <= 1e-13 * scale
        dist.barrier()
        out.put((rank, "ok"))
    except Exception as e:  # reported to the parent, which fails the test
        out.put((rank, repr(e)))
    finally:
        dist.destroy_process_group()


def test_python_exchange_over_gloo():
    """One subdomain per rank of a 2 x 2 x 1 cut (each neighbour is reached
    across two periodic shifts)."""
    import socket

    import torch.multiprocessing as mp
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    world, decomp, g = 4, (2, 2, 1), (2, 1, 1)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, decomp, g, out))
             for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(v == "ok" for v in res.values()), res
