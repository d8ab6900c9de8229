"""Particle redistribution on cartesian cuts along several axes (mapping.map_subs
on a 2 x 2 x 2, 3 x 3 x 1 ... topology): ppm_map_part_partial over the
neighbour list (ppm_map_part_partial.f:288-420, 480-485), the neighbours of
ppmg_halo_neighbours.

CPU: the neighbour list against a restatement over the subdomain boxes, and
the exchange in one process (LocalComm) and over a world_size 4 gloo group,
with the routing restated on CPU.  The device routing kernel is checked
against the same restatement in tests/test_gpu_cuboid.py."""
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


def touching(t, s, q):
    """Whether the boxes of s and q share a face, an edge or a corner (the
    domain periodic): along every axis the real node ranges meet or overlap
    modulo the mesh."""
    for a in range(3):
        N = int(t.Nm[a]) - 1
        s0, s1 = int(t.istart[s, a]), int(t.istart[s, a]) + int(t.nnodes[s, a]) - 1
        q0, q1 = int(t.istart[q, a]), int(t.istart[q, a]) + int(t.nnodes[q, a]) - 1
        if not any(q0 + k * N <= s1 and s0 <= q1 + k * N for k in (-1, 0, 1)):
            return False
    return True


@pytest.mark.parametrize("decomp", [(2, 2, 2), (3, 3, 3), (4, 1, 1), (4, 4, 1), (1, 1, 3),
                                    (3, 2, 1)])
def test_neighbours_are_the_touching_boxes(decomp):
    t = topo_for(3, 12, decomp=decomp)
    for s in range(t.nsubs):
        want = [q for q in range(t.nsubs) if q != s and touching(t, s, q)]
        assert halo.cart_neighbours(t, s) == want, s
    if decomp == (3, 3, 3):
        assert all(len(halo.cart_neighbours(t, s)) == 26 for s in range(27))


def partial_rule(t, s, x):
    """Destination of every particle of subdomain s: the box among s and its
    neighbours that holds it (closed-lower / open-upper, tested from the last
    subdomain to the first), nsubs when none does."""
    ns = int(t.nsubs)
    reach = [s] + halo.cart_neighbours(t, s)
    cls = np.full(x.shape[1], ns)
    for q in sorted(reach, reverse=True):
        hit = cls == ns
        for a in range(3):
            hit &= (x[a] >= t.min_sub[q, a]) & (x[a] < t.max_sub[q, a])
        cls[hit] = q
    return cls


def cpu_route(t):
    def route(tid, mid, xp, ns):
        s = tid - 1  # the tests give subdomain s the topo id s + 1
        cls = partial_rule(t, s, xp.numpy())
        perm = np.concatenate([np.nonzero(cls == c)[0] for c in range(ns + 1)]).astype(np.int32)
        info = -2 if (cls == ns).any() else 0
        return info, torch.from_numpy(perm), [int((cls == c).sum()) for c in range(ns + 1)]
    return route


def cpu_gather(src, perm, n):
    return src.t()[perm[:n].long()].t()


def moved(t, s, n, rng, far):
    """n particles of subdomain s moved by up to half a subdomain along every
    axis (periodic); `far` of them moved across the domain's middle."""
    x = np.empty((3, n))
    for a in range(3):
        lo, hi = t.min_sub[s, a], t.max_sub[s, a]
        L = t.max_phys[a] - t.min_phys[a]
        x[a] = lo + rng.random(n) * (hi - lo) + rng.uniform(-0.5, 0.5, n) * (hi - lo)
        x[a, :far] += 0.5 * L
        x[a] = np.mod(x[a] - t.min_phys[a], L) + t.min_phys[a]
    return np.asfortranarray(x)


def make_before(t, n, far=0):
    before = {}
    for s in range(t.nsubs):
        rng = np.random.default_rng(900 + s)
        before[s] = (moved(t, s, n, rng, far), np.arange(s * 10 ** 6, s * 10 ** 6 + n)[None, :],
                     np.asfortranarray(rng.standard_normal((2, n))))
    return before


def check(t, before, after):
    """Every subdomain ends with exactly the particles it received: its kept
    ones in their order, then the arrivals by ascending source subdomain."""
    for s, (x, ids, u) in after.items():
        exp = [before[s][1][0][partial_rule(t, s, before[s][0]) == s]]
        for q in halo.cart_neighbours(t, s):
            exp.append(before[q][1][0][partial_rule(t, q, before[q][0]) == s])
        assert np.array_equal(ids[0], np.concatenate(exp)), s
        for a in range(3):
            assert ((x[a] >= t.min_sub[s, a]) & (x[a] < t.max_sub[s, a])).all()
        allu = np.concatenate([before[q][2] for q in before], axis=1)
        alli = np.concatenate([before[q][1] for q in before], axis=1)[0]
        pos = {int(i): k for k, i in enumerate(alli)}
        assert np.array_equal(u, allu[:, [pos[int(i)] for i in ids[0]]])


def parts_of(before, subs):
    return {s: (s + 1, 1, torch.from_numpy(before[s][0]),
                [torch.from_numpy(np.asfortranarray(before[s][1])),
                 torch.from_numpy(before[s][2])]) for s in subs}


@pytest.mark.parametrize("decomp,far", [((2, 2, 2), 0), ((3, 3, 1), 0), ((4, 4, 1), 7)])
def test_partial_mapping_in_one_process(decomp, far):
    from ppm_legacy_b200 import mapping
    t = topo_for(3, 12, decomp=decomp)
    before = make_before(t, 400, far)
    info, res = mapping.map_subs(parts_of(before, range(t.nsubs)), t, halo.LocalComm(),
                                 route=cpu_route(t), gather=cpu_gather)
    after = {s: (x.numpy(), i.numpy(), u.numpy()) for s, (x, (i, u)) in res.items()}
    check(t, before, after)
    lost = sum(int((partial_rule(t, s, b[0]) == t.nsubs).sum()) for s, b in before.items())
    assert info == (-2 if lost else 0)
    # on a 4 x 4 x 1 cut a move across half the domain lands two subdomains away
    assert (lost > 0) == (far > 0)
    assert sum(a[0].shape[1] for a in after.values()) + lost == 400 * t.nsubs


def _main(rank, world, port, out):
    from ppm_legacy_b200 import mapping
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = topo_for(3, 12, decomp=(2, 2, 1))
        before = make_before(t, 300)
        info, res = mapping.map_subs(parts_of(before, [rank]), t, halo.DistComm(),
                                     route=cpu_route(t), gather=cpu_gather)
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


def test_partial_mapping_over_gloo():
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    world = 4
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    procs = [ctx.Process(target=_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(out.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(v == "ok" for v in res.values()), res
