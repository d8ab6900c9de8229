"""The library's ghost-exchange plan between z-slab subdomains
(ppmg_halo_plan: which planes go where, host logic only) and the
torch.distributed mover of its transport (halo.DistMover), on CPU.

The plan-driven exchange (blocks moved by the mover, added or copied at the
plan's offsets as the library does on the device) must reproduce the Python
exchange (halo.put / halo.get) bit for bit, in one process and as world_size
2 and 3 gloo process groups.  Fields are built as the slab P2M leaves them
(tests/test_slab_exchange.py)."""
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
from ppm_legacy_b200 import halo  # noqa: E402
from test_slab_exchange import case, check_get, check_put  # noqa: E402


def plan_exchange(t, s, f, g, put, move):
    """One exchange of slab s's field f (numpy, F-order) through the library's
    plan; move(sends, recvs) moves (peer, tag, address, nbytes) blocks."""
    lb = [1 - g] * 3
    ub = [lb[a] + f.shape[1 + a] - 1 for a in range(3)]
    pl = halo.plan(t, s, f.shape[0], lb, ub, [g] * 3, put)
    flat = f.reshape(-1, order="F")  # a view: f is Fortran-contiguous
    n = pl["count"]
    if n == 0:
        return
    isz = flat.itemsize
    recv = [np.empty(n) for _ in range(2)]
    sends = [(p, tag, flat.ctypes.data + off * isz, n * isz) for p, tag, off in pl["send"]]
    recvs = [(p, tag, recv[b].ctypes.data, n * isz) for b, (p, tag, _) in enumerate(pl["recv"])]
    move(sends, recvs)
    for b, (_, _, off) in enumerate(pl["recv"]):
        if put:
            flat[off:off + n] += recv[b]
        else:
            flat[off:off + n] = recv[b]


@pytest.mark.parametrize("nc,nslab,kernel,g,lda", [
    (12, 2, 2, 2, 3), (12, 3, 2, 2, 1), (10, 2, 1, 1, 2), (16, 4, 2, 3, 1)])
def test_plan_matches_python_exchange(nc, nslab, kernel, g, lda):
    """Every slab exchanging from a thread of its own through halo.ThreadMover
    (host blocks), as the library's calls on several slab handles of one
    process do."""
    import threading
    t, local, want = case(nc, nslab, kernel, g, lda, seed=nc + nslab)
    ref = {s: torch.from_numpy(local[s].copy(order="F")) for s in local}
    mine = {s: local[s].copy(order="F") for s in local}
    mover = halo.ThreadMover(timeout=30)
    for put in (True, False):
        (halo.put if put else halo.get)(ref, t, [g] * 3, [1 - g] * 3, halo.LocalComm())
        errs = []

        def run(s):
            try:
                plan_exchange(t, s, mine[s], g, put,
                              lambda S, R: mover.exchange(s, S, R, False, None))
            except Exception as e:  # noqa: BLE001
                errs.append(repr(e))
        th = [threading.Thread(target=run, args=(s,)) for s in mine]
        for x in th:
            x.start()
        for x in th:
            x.join()
        assert not errs, errs
        for s in mine:
            assert np.array_equal(mine[s], ref[s].numpy())
    for s in mine:
        check_get(t, s, mine[s], want[s], g)


def test_plan_refuses_what_the_exchange_refuses():
    t, local, _ = case(12, 4, 2, 2, 1, seed=1)
    with pytest.raises(ValueError):  # nz = 3 < g = 4
        halo.plan(t, 0, 1, [-3] * 3, [17, 17, 8], [4] * 3, True)
    with pytest.raises(ValueError):  # field short of the upper ghost planes
        halo.plan(t, 0, 1, [-1] * 3, [15, 15, 5], [2] * 3, True)
    from _util import topo_for
    with pytest.raises(ValueError):  # not a cut along z
        halo.plan(topo_for(3, 12, decomp=(2, 1, 1)), 0, 1, [-1] * 3, [15] * 3, [2] * 3, True)


def _rank_main(rank, world, port, nc, g, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t, local, want = case(nc, world, 2, g, 3, seed=99)
        f = local[rank].copy(order="F")
        mover = halo.DistMover()

        def move(sends, recvs):
            mover.exchange(rank, sends, recvs, False, None)
        plan_exchange(t, rank, f, g, True, move)
        check_put(t, rank, f, want[rank], g)
        ref = {rank: torch.from_numpy(local[rank].copy(order="F"))}
        halo.put(ref, t, [g] * 3, [1 - g] * 3, halo.DistComm())
        assert np.array_equal(f, ref[rank].numpy())
        plan_exchange(t, rank, f, g, False, move)
        check_get(t, rank, f, want[rank], g)
        halo.get(ref, t, [g] * 3, [1 - g] * 3, halo.DistComm())
        assert np.array_equal(f, ref[rank].numpy())
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
def test_plan_exchange_over_gloo(world):
    """One slab per rank, the library's plan and halo.DistMover over gloo,
    equal to halo.DistComm's exchange and to the global deposit."""
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
