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
