"""ppm_map_part_global between z-slab subdomains (mapping.map_global): every
particle goes to the slab that contains it, however far it moved; particles
in no slab are left out without an error (ppm_map_part_global.f:355-442).

CPU: the all-pairs size and block exchange over world_size 2 and 3 gloo
process groups, with the routing restated on CPU.  The device routing kernel
is checked against the same restatement in tests/test_gpu_map_global.py."""
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
from _util import topo_for  # noqa: E402
from ppm_legacy_b200 import halo  # noqa: E402


def global_rule(topo, x):
    """Destination of every particle: the slab whose [min_sub, max_sub) holds
    z (x, y inside the domain), testing the slabs from the last to the first;
    nsubs when none does."""
    ns = int(topo.nsubs)
    cls = np.full(x.shape[1], ns)
    inxy = np.all((x[:2] >= topo.min_phys[:2, None]) & (x[:2] < topo.max_phys[:2, None]), axis=0)
    for q in range(ns - 1, -1, -1):
        hit = inxy & (cls == ns) & (x[2] >= topo.min_sub[q, 2]) & (x[2] < topo.max_sub[q, 2])
        cls[hit] = q
    return cls


def scattered_particles(t, s, n, rng):
    """n particles of slab s after a large move: anywhere in the domain, a few
    outside it (they belong to no slab)."""
    x = rng.random((3, n))
    x[:, :5] = [[0.5, 0.5, 1.0, -0.1, 0.5], [0.5, 0.5, 0.5, 0.5, 1.5],
                [1.2, -0.01, 0.5, 0.5, 0.5]]
    return np.asfortranarray(x)


def cpu_route(topo):
    def route(tid, mid, xp, ns):
        cls = global_rule(topo, xp.numpy())
        perm = np.concatenate([np.nonzero(cls == c)[0] for c in range(ns + 1)]).astype(np.int32)
        return 0, torch.from_numpy(perm), [int((cls == c).sum()) for c in range(ns + 1)]
    return route


def cpu_gather(src, perm, n):
    return src.t()[perm[:n].long()].t()


def check(topo, before, after):
    """Every slab ends with exactly its particles: its own kept ones in their
    order, then the arrivals by ascending source slab, each in source order;
    positions and properties travel with their particle."""
    ns = int(topo.nsubs)
    for s, (x, ids, u) in after.items():
        exp = []
        for q in [s] + [q for q in range(ns) if q != s]:
            xq, iq, _ = before[q]
            exp.append(iq[0][global_rule(topo, xq) == s])
        assert np.array_equal(ids[0], np.concatenate(exp)), s
        allx = np.concatenate([before[q][0] for q in before], axis=1)
        allu = np.concatenate([before[q][2] for q in before], axis=1)
        alli = np.concatenate([before[q][1] for q in before], axis=1)[0]
        pos = {int(i): k for k, i in enumerate(alli)}
        idx = [pos[int(i)] for i in ids[0]]
        assert np.array_equal(x, allx[:, idx]) and np.array_equal(u, allu[:, idx])


def make_before(t, world, n=300):
    before = {}
    for s in range(world):
        rng = np.random.default_rng(700 + s)
        x = scattered_particles(t, s, n, rng)
        before[s] = (x, np.arange(s * 10 ** 6, s * 10 ** 6 + n)[None, :],  # unique ids
                     np.asfortranarray(rng.standard_normal((2, n))))
    return before


def test_all_slabs_in_one_process():
    from ppm_legacy_b200 import mapping
    t = topo_for(3, 12, decomp=(1, 1, 4))
    before = make_before(t, 4)
    parts = {s: (1, 1, torch.from_numpy(x), [torch.from_numpy(np.asfortranarray(i)),
                                             torch.from_numpy(u)])
             for s, (x, i, u) in before.items()}
    info, res = mapping.map_global(parts, t, halo.LocalComm(), route=cpu_route(t),
                                   gather=cpu_gather)
    assert info == 0
    check(t, before, {s: (x.numpy(), i.numpy(), u.numpy()) for s, (x, (i, u)) in res.items()})
    total = sum(r[0].shape[1] for r in res.values())
    lost = sum(int((global_rule(t, b[0]) == 4).sum()) for b in before.values())
    assert total + lost == 4 * 300 and lost > 0


def _main(rank, world, port, out):
    from ppm_legacy_b200 import mapping
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = topo_for(3, 12, decomp=(1, 1, world))
        before = make_before(t, world)
        x, i, u = before[rank]
        parts = {rank: (1, 1, torch.from_numpy(x), [torch.from_numpy(np.asfortranarray(i)),
                                                    torch.from_numpy(u)])}
        info, res = mapping.map_global(parts, t, halo.DistComm(), route=cpu_route(t),
                                       gather=cpu_gather)
        x2, (i2, u2) = res[rank]
        check(t, before, {rank: (x2.numpy(), i2.numpy(), u2.numpy())})
        assert info == 0
        dist.barrier()
        out.put((rank, "ok"))
    except Exception:  # reported to the parent, which fails the test
        import traceback
        out.put((rank, traceback.format_exc()))
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_global_mapping_over_gloo(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(v == "ok" for v in res.values()), res
